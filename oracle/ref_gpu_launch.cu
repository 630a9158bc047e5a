// Launchers for the reference's own CUDA step kernels.  TEST INFRASTRUCTURE
// ONLY: tests time them beside the fused kernels on the same GPU and check
// them against the oracle; the product never links them.
//
// The kernels themselves are the reference's CuPy RawKernel sources
// (lfm/core/backends/kernel_source.py: evolve_real :323-419, evolve_complex
// :424-540, evolve_gov01_gov02 :18-235).  build_ref_gpu.py copies them from
// the reference checkout into _ref/ref_kernels.cu at build time (that
// directory is not committed) and compiles this file against it.  The launch
// shape is the reference's (lfm/core/backends/cupy_backend.py:42-45): one
// thread per cell, 256-thread blocks, a 1-D grid.
#include <climits>
#include <cuda_runtime.h>

#include "ref_kernels.cu"

namespace {

// Blocks for one thread per cell; 0 when N^3 does not fit the kernels' int index.
unsigned blocks_for(int N, int colours) {
  if (N <= 0) return 0;
  const long long total = (long long)N * N * N;
  if (total * colours > INT_MAX) return 0;
  return (unsigned)((total + 255) / 256);
}

}  // namespace

extern "C" {

// Returns a cudaError_t code (0 = launched), or -1 for a size the kernels cannot index.
int ref_evolve_real(const float* E, const float* E_prev, const float* chi, const float* chi_prev,
                    const float* mask, float* E_next, float* E_prev_next, float* chi_next,
                    float* chi_prev_next, int N, float dt2, float kappa, float lam, float chi0,
                    float e0_sq, void* stream) {
  const unsigned blocks = blocks_for(N, 1);
  if (!blocks) return -1;
  evolve_real<<<blocks, 256, 0, (cudaStream_t)stream>>>(E, E_prev, chi, chi_prev, mask, E_next,
                                                         E_prev_next, chi_next, chi_prev_next, N,
                                                         dt2, kappa, lam, chi0, e0_sq);
  return (int)cudaGetLastError();
}

int ref_evolve_complex(const float* pr, const float* pr_prev, const float* pi,
                       const float* pi_prev, const float* chi, const float* chi_prev,
                       const float* mask, float* pr_next, float* pr_prev_next, float* pi_next,
                       float* pi_prev_next, float* chi_next, float* chi_prev_next, int N,
                       float dt2, float kappa, float lam, float chi0, float e0_sq, float eps_w,
                       void* stream) {
  const unsigned blocks = blocks_for(N, 1);
  if (!blocks) return -1;
  evolve_complex<<<blocks, 256, 0, (cudaStream_t)stream>>>(
      pr, pr_prev, pi, pi_prev, chi, chi_prev, mask, pr_next, pr_prev_next, pi_next,
      pi_prev_next, chi_next, chi_prev_next, N, dt2, kappa, lam, chi0, e0_sq, eps_w);
  return (int)cudaGetLastError();
}

// Psi fields are three colours packed [3 N^3]; sa: three S_a fields [3 N^3].
int ref_evolve_color(const float* pr, const float* pr_prev, const float* pi,
                     const float* pi_prev, const float* chi, const float* chi_prev,
                     const float* mask, float* pr_next, float* pr_prev_next, float* pi_next,
                     float* pi_prev_next, float* chi_next, float* chi_prev_next, int N,
                     float dt2, float kappa, float lam, float chi0, float e0_sq, float eps_w,
                     float kappa_c, float eps_cc, const float* sa, float kappa_string,
                     float kappa_tube, void* stream) {
  const unsigned blocks = blocks_for(N, 3);
  if (!blocks) return -1;
  evolve_gov01_gov02<<<blocks, 256, 0, (cudaStream_t)stream>>>(
      pr, pr_prev, pi, pi_prev, chi, chi_prev, mask, pr_next, pr_prev_next, pi_next,
      pi_prev_next, chi_next, chi_prev_next, N, dt2, kappa, lam, chi0, e0_sq, eps_w, kappa_c,
      eps_cc, sa, kappa_string, kappa_tube);
  return (int)cudaGetLastError();
}

}  // extern "C"
