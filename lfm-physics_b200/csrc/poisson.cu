// Poisson equilibration of chi (lfm/fields/equilibrium.py:26-121):
//
//   rhs = kappa (|Psi|^2 - e0^2)                       float32, NumPy's order
//   RHS = rfftn(rhs)                                   float32 transform (cuFFT R2C)
//   PHI = -RHS / k^2, PHI(0) = 0                       float64 (complex128 / float64)
//   dchi = irfftn(PHI) / N^3                           float64 transform (cuFFT Z2D)
//   chi = chi0 + float32(dchi), chi0 on the frozen shell (dist > N/2 (1 - bf))
//
// The FFTs are cuFFT's, so chi agrees with the reference to a float32 ulp or
// two rather than bit for bit; every other operation repeats NumPy's.
#include <cuda_runtime.h>

#include "lfm_kernels.h"
#include "lfm_math.cuh"

namespace lfm {
namespace {

// |Psi|^2 with NumPy's float32 order: psi_r^2 (+ psi_i^2); for three colours
// the axis-0 sums ((a0 + a1) + a2) of each part, then their sum.
__global__ void poisson_rhs_kernel(const float* __restrict__ pr, const float* __restrict__ pi,
                                   float* __restrict__ rhs, int64_t n3, int colours, float kappa,
                                   float e0_sq) {
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < n3;
       x += (int64_t)gridDim.x * blockDim.x) {
    float psi_sq;
    if (colours == 1) {
      psi_sq = fmul(pr[x], pr[x]);
      if (pi) psi_sq = fadd(psi_sq, fmul(pi[x], pi[x]));
    } else {
      float sr = fmul(pr[x], pr[x]);
      for (int a = 1; a < colours; ++a) sr = fadd(sr, fmul(pr[a * n3 + x], pr[a * n3 + x]));
      psi_sq = sr;
      if (pi) {
        float si = fmul(pi[x], pi[x]);
        for (int a = 1; a < colours; ++a) si = fadd(si, fmul(pi[a * n3 + x], pi[a * n3 + x]));
        psi_sq = fadd(sr, si);
      }
    }
    rhs[x] = fmul(kappa, fsub(psi_sq, e0_sq));
  }
}

// 2 pi m / N as numpy.fft.fftfreq(N) * 2 pi (m (1/N), then times 2 pi);
// the half axis counts 0 .. N/2 (rfftfreq).
__device__ __forceinline__ double angular_freq(int m, int n, bool half_axis) {
  const double val = 1.0 / (double)n;
  const int f = (!half_axis && m >= (n + 1) / 2) ? m - n : m;
  return __dmul_rn(__dmul_rn((double)f, val), 2.0 * 3.141592653589793);
}

__global__ void poisson_divide_kernel(const float2* __restrict__ in, double2* __restrict__ out,
                                      int N, int64_t count) {
  const int nz = N / 2 + 1;
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < count;
       x += (int64_t)gridDim.x * blockDim.x) {
    const int z = (int)(x % nz);
    const int y = (int)((x / nz) % N);
    const int xx = (int)(x / ((int64_t)nz * N));
    if (x == 0) {
      out[0] = make_double2(0.0, 0.0);
      continue;
    }
    const double kx = angular_freq(xx, N, false), ky = angular_freq(y, N, false),
                 kz = angular_freq(z, N, true);
    const double k2 =
        __dadd_rn(__dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky)), __dmul_rn(kz, kz));
    const float2 v = in[x];
    // -src / k2 with src widened to complex128 (Smith's division by k2 + 0i
    // reduces to a component-wise divide)
    out[x] = make_double2(__ddiv_rn(-(double)v.x, k2), __ddiv_rn(-(double)v.y, k2));
  }
}

__global__ void poisson_finish_kernel(const double* __restrict__ dchi, float* __restrict__ chi,
                                      int N, float chi0, double radius, int frozen) {
  const int64_t n3 = (int64_t)N * N * N;
  const double inv_n3 = 1.0 / (double)n3;
  const double c = N / 2.0;
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < n3;
       x += (int64_t)gridDim.x * blockDim.x) {
    float v = fadd(chi0, __double2float_rn(__dmul_rn(dchi[x], inv_n3)));
    if (frozen) {
      const int k = (int)(x % N), j = (int)((x / N) % N), i = (int)(x / ((int64_t)N * N));
      const double di = i - c, dj = j - c, dk = k - c;
      if (sqrt(di * di + dj * dj + dk * dk) > radius) v = chi0;
    }
    chi[x] = v;
  }
}

int grid_for(int64_t n) {
  int64_t b = (n + 255) / 256;
  return (int)(b > 148LL * 16 ? 148LL * 16 : b);
}

}  // namespace

cudaError_t launch_poisson_rhs(const float* pr, const float* pi, float* rhs, int N, int colours,
                               float kappa, float e0_sq, cudaStream_t stream) {
  const int64_t n3 = (int64_t)N * N * N;
  poisson_rhs_kernel<<<grid_for(n3), 256, 0, stream>>>(pr, pi, rhs, n3, colours, kappa, e0_sq);
  return cudaGetLastError();
}

cudaError_t launch_poisson_divide(const float2* in, double2* out, int N, cudaStream_t stream) {
  const int64_t count = (int64_t)N * N * (N / 2 + 1);
  poisson_divide_kernel<<<grid_for(count), 256, 0, stream>>>(in, out, N, count);
  return cudaGetLastError();
}

cudaError_t launch_poisson_finish(const double* dchi, float* chi, int N, float chi0,
                                  double radius, int frozen, cudaStream_t stream) {
  const int64_t n3 = (int64_t)N * N * N;
  poisson_finish_kernel<<<grid_for(n3), 256, 0, stream>>>(dchi, chi, N, chi0, radius, frozen);
  return cudaGetLastError();
}

}  // namespace lfm
