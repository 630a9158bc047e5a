// On-device float64 metrics of a lattice state.
//
// Reproduces compute_metrics (lfm/analysis/metrics.py:29-111) apart from
// the cluster count:
//   energy_components (lfm/analysis/energy.py:26-113): per cell, in float64,
//     T = 1/2 sum_comp ((psi - psi_prev)/dt)^2
//     G = 1/2 c^2 sum_comp sum_axis g^2, g = np.gradient (central in the
//         interior, one-sided first differences at the two edges; NOT periodic)
//     V = 1/2 chi^2 sum_comp psi^2
//   chi_statistics / well_fraction / void_fraction over interior_mask
//   (lfm/analysis/structure.py:26-171): dist = sqrt((i-c)^2+(j-c)^2+(k-c)^2)
//   <= c*(1-boundary_fraction) with c = N/2, in float64.
// Each CTA reduces its cells to one row of partials in the scratch buffer; a
// second single-CTA kernel reduces the rows in a fixed order, so results are
// deterministic for a given grid.
#include <cstdio>
#include <mutex>

#include "lfm_b200.h"
#include "lfm_kernels.h"
#include "lfm_metrics.h"

namespace lfm {
namespace {

struct Acc {
  double s[kMetricSums];
  float mn, mx;
};

__device__ __forceinline__ double grad_axis(const float* f, int64_t x, int c, int N,
                                            int64_t stride) {
  if (c == 0) return (double)f[x + stride] - (double)f[x];
  if (c == N - 1) return (double)f[x] - (double)f[x - stride];
  return ((double)f[x + stride] - (double)f[x - stride]) / 2.0;
}

__device__ __forceinline__ void add_component(Acc& A, const float* p, const float* pp, int64_t x,
                                              int i, int j, int k, int N, double dt,
                                              double& psi_sq, double& kin, double& grad) {
  const double v = (double)p[x];
  if (pp) {
    const double d = (v - (double)pp[x]) / dt;  // (psi - psi_prev)/dt as energy.py:72
    kin += d * d;
  }
  const int64_t n2 = (int64_t)N * N;
  const double gx = grad_axis(p, x, i, N, n2);
  const double gy = grad_axis(p, x, j, N, N);
  const double gz = grad_axis(p, x, k, N, 1);
  grad += gx * gx;
  grad += gy * gy;
  grad += gz * gz;
  psi_sq += v * v;
  (void)A;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

template <int LEVEL>
__global__ void __launch_bounds__(256) metrics_partial_kernel(MetricsArgs a, double* partials) {
  const int N = a.N;
  const int64_t n3 = (int64_t)N * N * N;
  const double c = N / 2.0;
  Acc A;
#pragma unroll
  for (int q = 0; q < kMetricSums; ++q) A.s[q] = 0.0;
  A.mn = __int_as_float(0x7f800000);   // +inf
  A.mx = __int_as_float(0xff800000);   // -inf
  const int ncomp = (LEVEL == LFM_COLOR) ? 3 : 1;
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < n3;
       x += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(x % N);
    const int j = (int)((x / N) % N);
    const int i = (int)(x / ((int64_t)N * N));
    double psi_sq = 0.0, kin = 0.0, grad = 0.0;
    for (int comp = 0; comp < ncomp; ++comp) {
      const int64_t off = comp * n3;
      double kr = 0.0, gr = 0.0;
      add_component(A, a.pr + off, a.pr_prev ? a.pr_prev + off : nullptr, x, i, j, k, N,
                    a.dt, psi_sq, kr, gr);
      kin += kr;
      grad += gr;
      if (LEVEL != LFM_REAL) {
        double ki = 0.0, gi = 0.0;
        add_component(A, a.pi + off, a.pi_prev ? a.pi_prev + off : nullptr, x, i, j, k, N,
                      a.dt, psi_sq, ki, gi);
        kin += ki;
        grad += gi;
      }
    }
    const double chi = (double)a.chi[x];
    A.s[kKinetic] += 0.5 * kin;
    A.s[kGradient] += 0.5 * a.c2 * grad;
    A.s[kPotential] += 0.5 * (chi * chi) * psi_sq;
    A.s[kPsiSq] += psi_sq;
    // interior_mask: dist <= c*(1-bf) with c = N/2 (no half-cell shift)
    const double di = i - c, dj = j - c, dk = k - c;
    const double dist = sqrt(di * di + dj * dj + dk * dk);
    if (dist <= a.radius) {
      const float cf = a.chi[x];
      const double d = chi - a.chi_shift;
      A.s[kCount] += 1.0;
      A.s[kChiSum] += d;
      A.s[kChiSq] += d * d;
      A.s[kWell] += (cf < a.well) ? 1.0 : 0.0;
      A.s[kVoid] += (cf > a.void_thr) ? 1.0 : 0.0;
      A.mn = fminf(A.mn, cf);
      A.mx = fmaxf(A.mx, cf);
    }
    if (!isfinite(chi) || !isfinite(psi_sq)) A.s[kNonFinite] += 1.0;
  }
  // block reduction: warps -> shared -> row of partials
  __shared__ double sh[kMetricSums][8];
  __shared__ float shmn[8], shmx[8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int q = 0; q < kMetricSums; ++q) {
    const double v = warp_sum(A.s[q]);
    if (lane == 0) sh[q][w] = v;
  }
  const float mn = warp_min(A.mn), mx = warp_max(A.mx);
  if (lane == 0) {
    shmn[w] = mn;
    shmx[w] = mx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double* row = partials + (size_t)blockIdx.x * kPartialStride;
    for (int q = 0; q < kMetricSums; ++q) {
      double t = 0.0;
      for (int ww = 0; ww < nw; ++ww) t += sh[q][ww];
      row[q] = t;
    }
    float bmn = shmn[0], bmx = shmx[0];
    for (int ww = 1; ww < nw; ++ww) {
      bmn = fminf(bmn, shmn[ww]);
      bmx = fmaxf(bmx, shmx[ww]);
    }
    row[kMetricSums] = (double)bmn;
    row[kMetricSums + 1] = (double)bmx;
  }
}

// Sums the rows of partials in block order (one thread per quantity).
__global__ void metrics_finish_kernel(const double* partials, int rows, double* out) {
  const int q = threadIdx.x;
  if (q < kMetricSums) {
    double t = 0.0;
    for (int r = 0; r < rows; ++r) t += partials[(size_t)r * kPartialStride + q];
    out[q] = t;
  } else if (q == kMetricSums) {
    double m = partials[kMetricSums];
    for (int r = 1; r < rows; ++r) m = fmin(m, partials[(size_t)r * kPartialStride + q]);
    out[q] = m;
  } else if (q == kMetricSums + 1) {
    double m = partials[kMetricSums + 1];
    for (int r = 1; r < rows; ++r) m = fmax(m, partials[(size_t)r * kPartialStride + q]);
    out[q] = m;
  }
}

}  // namespace

cudaError_t launch_metrics(const MetricsArgs& a, double* partials, int rows, double* out,
                           cudaStream_t stream) {
  switch (a.level) {
    case LFM_REAL: metrics_partial_kernel<LFM_REAL><<<rows, 256, 0, stream>>>(a, partials); break;
    case LFM_COMPLEX:
      metrics_partial_kernel<LFM_COMPLEX><<<rows, 256, 0, stream>>>(a, partials);
      break;
    default: metrics_partial_kernel<LFM_COLOR><<<rows, 256, 0, stream>>>(a, partials); break;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  metrics_finish_kernel<<<1, 32, 0, stream>>>(partials, rows, out);
  return cudaGetLastError();
}

}  // namespace lfm

// ---------------------------------------------------------------------------
// Metrics without allocation (lfm_metrics_f64_noalloc).
//
// For callers that cannot allocate device memory: a process whose device
// memory is all held by another allocator (PyTorch's caching allocator can
// leave cudaMalloc failing while it keeps free blocks for itself), or a host
// program that allocates only at start-up and must not call cudaMalloc
// afterwards.  Such callers also hold no lfm_context, which is where
// lfm_metrics_f64 keeps its scratch.
//
// The per-CTA partials live in this file-scope device array instead.  Every
// GPU that loads the library holds it until the process ends:
// (kNoAllocRows + 1) rows x kPartialStride (12) doubles = 196,704 bytes
// (192 KiB).  One CTA reduces each 65536 cells, so a lattice may have at most
// kNoAllocRows * 65536 cells (N <= 512).  Host code must not pass the
// array's name to a kernel: on the host it only stands in for the symbol, and
// the device address comes from cudaGetSymbolAddress, taken once per device
// on the first call made with that device current.  That address belongs to
// the device's primary context (the one the CUDA runtime uses), so calls must
// be made with the primary context current.
// ---------------------------------------------------------------------------
namespace {

constexpr int kNoAllocRows = 2048;
constexpr long long kNoAllocCellsPerRow = 65536;

static __device__ __align__(256) double g_noalloc_partials[(kNoAllocRows + 1) *
                                                           lfm::kPartialStride];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_ptr[kNoAllocMaxDevices] = {nullptr};

int noalloc_scratch(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return lfm::abi_cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= kNoAllocMaxDevices)
    return lfm::abi_fail(LFM_ERR_UNSUPPORTED, "device index outside the scratch table");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    double* p = nullptr;
    e = cudaGetSymbolAddress((void**)&p, g_noalloc_partials);
    if (e != cudaSuccess) return lfm::abi_cuda_fail(e, "cudaGetSymbolAddress(metric scratch)");
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return LFM_OK;
}

}  // namespace

extern "C" int lfm_metrics_f64_noalloc(int level, const float* psi_r, const float* psi_r_prev,
                                       const float* psi_i, const float* psi_i_prev,
                                       const float* chi, int N, double dt, double c,
                                       double boundary_fraction, double well_threshold,
                                       double void_threshold, double* out_host, void* stream) {
  lfm::MetricsArgs a{};
  int rc = lfm::metrics_prepare(level, psi_r, psi_r_prev, psi_i, psi_i_prev, chi, N, dt, c,
                                boundary_fraction, well_threshold, void_threshold, out_host, &a);
  if (rc) return rc;
  const long long cells = (long long)N * N * N;
  const long long rows = (cells + kNoAllocCellsPerRow - 1) / kNoAllocCellsPerRow;
  if (rows > kNoAllocRows) {
    char msg[160];
    snprintf(msg, sizeof msg,
             "N=%d needs %lld partial rows; the static scratch holds %d (lattices up to 512^3)",
             N, rows, kNoAllocRows);
    return lfm::abi_fail(LFM_ERR_CAPACITY, msg);
  }
  double* scratch = nullptr;
  rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  // Every partial row and the final row are written before they are read,
  // so nothing left in the array by an earlier call needs clearing.
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* final_row = scratch + (size_t)kNoAllocRows * lfm::kPartialStride;
  cudaError_t e = lfm::launch_metrics(a, scratch, (int)rows, final_row, st);
  if (e != cudaSuccess) return lfm::abi_cuda_fail(e, "metrics launch");
  double r[lfm::kPartialStride];
  e = cudaMemcpyAsync(r, final_row, sizeof r, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return lfm::abi_cuda_fail(e, "metrics readback");
  lfm::metrics_finish(r, a.chi_shift, out_host);
  return LFM_OK;
}
