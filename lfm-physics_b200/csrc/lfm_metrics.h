// Layout of the float64 metrics reduction (metrics.cu, lfm_metrics_f64).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace lfm {

// Summed quantities; the partials rows then carry chi min and max.
enum MetricSum {
  kKinetic = 0,   // sum 1/2 (d psi/dt)^2
  kGradient,      // sum 1/2 c^2 |grad psi|^2
  kPotential,     // sum 1/2 chi^2 |psi|^2
  kPsiSq,         // sum |psi|^2
  kCount,         // interior cells
  kChiSum,        // sum (chi - chi_shift) over the interior
  kChiSq,         // sum (chi - chi_shift)^2 over the interior
  kWell,          // interior cells with chi < well
  kVoid,          // interior cells with chi > void
  kNonFinite,     // cells with a non-finite chi or |psi|^2
  kMetricSums
};
constexpr int kPartialStride = kMetricSums + 2;  // sums, chi min, chi max
constexpr int kMetricRows = 148 * 4;             // CTAs of the partial pass

struct MetricsArgs {
  int level;
  int N;
  const float* pr;
  const float* pr_prev;  // may be null: kinetic term 0
  const float* pi;
  const float* pi_prev;
  const float* chi;
  double dt;
  double c2;
  double radius;     // interior: dist <= radius
  double chi_shift;  // subtracted before the chi moments (conditioning)
  float well;
  float void_thr;
};

cudaError_t launch_metrics(const MetricsArgs& a, double* partials, int rows, double* out,
                           cudaStream_t stream);

}  // namespace lfm
