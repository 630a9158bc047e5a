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

// Defined in capi.cu: the shared argument checks and host finishing of the
// metrics entry points, and the thread's error detail.
int metrics_prepare(int level, const float* psi_r, const float* psi_r_prev, const float* psi_i,
                    const float* psi_i_prev, const float* chi, int N, double dt, double c,
                    double boundary_fraction, double well_threshold, double void_threshold,
                    double* out_host, MetricsArgs* out);
void metrics_finish(const double* sums, double chi_shift, double* out_host);
int abi_fail(int code, const char* detail);
int abi_cuda_fail(cudaError_t e, const char* what);

}  // namespace lfm
