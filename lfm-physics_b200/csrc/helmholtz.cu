// Hand-written kernels around cuFFT for the S_a Helmholtz solve.
//
// S_a = IRFFT[ gamma/(gamma + D|k|^2) * RFFT(|Psi_a|^2) ]
// (lfm/core/backends/numpy_backend.py:341-356).  The filter is evaluated in
// float64 from k = 2*pi*fftfreq(N) exactly as NumPy builds it, divided by
// N^3 (cuFFT's inverse is unnormalised) and applied in float32.
#include "lfm_kernels.h"

namespace lfm {
namespace {

// |Psi_a|^2 = Pr*Pr + Pi*Pi for the three colours (numpy_backend.py:289).
__global__ void color_energy_kernel(const float4* __restrict__ pr, const float4* __restrict__ pi,
                                    float4* __restrict__ e, int64_t n4) {
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < n4;
       x += (int64_t)gridDim.x * blockDim.x) {
    const float4 r = __ldg(pr + x), i = __ldg(pi + x);
    float4 o;
    o.x = fadd(fmul(r.x, r.x), fmul(i.x, i.x));
    o.y = fadd(fmul(r.y, r.y), fmul(i.y, i.y));
    o.z = fadd(fmul(r.z, r.z), fmul(i.z, i.z));
    o.w = fadd(fmul(r.w, r.w), fmul(i.w, i.w));
    e[x] = o;
  }
}

__global__ void color_energy_scalar_kernel(const float* __restrict__ pr,
                                           const float* __restrict__ pi, float* __restrict__ e,
                                           int64_t n) {
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < n;
       x += (int64_t)gridDim.x * blockDim.x) {
    const float r = __ldg(pr + x), i = __ldg(pi + x);
    e[x] = fadd(fmul(r, r), fmul(i, i));
  }
}

// np.fft.fftfreq(n) * 2*pi: m * (1.0/n) for m < (n+1)/2, (m - n) * (1.0/n) otherwise.
__device__ __forceinline__ double wavenumber(int m, int n, bool half_axis) {
  const double val = 1.0 / (double)n;
  const int f = (!half_axis && m >= (n + 1) / 2) ? m - n : m;
  return __dmul_rn(__dmul_rn((double)f, val), 2.0 * 3.141592653589793);
}

// spec[a][x][y][z] *= (gamma/(gamma + D k^2)) / N^3 for the three colours,
// z over the N/2+1 half spectrum.
__global__ void helmholtz_multiply_kernel(float2* __restrict__ spec, int N, double gamma,
                                          double d, int64_t per_colour) {
  const int nz = N / 2 + 1;
  const double inv_n3 = 1.0 / ((double)N * N * N);
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < per_colour;
       x += (int64_t)gridDim.x * blockDim.x) {
    const int z = (int)(x % nz);
    const int y = (int)((x / nz) % N);
    const int xx = (int)(x / ((int64_t)nz * N));
    const double kx = wavenumber(xx, N, false), ky = wavenumber(y, N, false),
                 kz = wavenumber(z, N, true);
    const double k_sq = __dadd_rn(__dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky)),
                                  __dmul_rn(kz, kz));
    const double h = __ddiv_rn(gamma, __dadd_rn(gamma, __dmul_rn(d, k_sq)));
    const float scale = __double2float_rn(__dmul_rn(h, inv_n3));
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      float2 v = spec[a * per_colour + x];
      v.x = v.x * scale;
      v.y = v.y * scale;
      spec[a * per_colour + x] = v;
    }
  }
}

__global__ void clip_kernel(const float* __restrict__ in, float* __restrict__ out, int64_t n) {
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < n;
       x += (int64_t)gridDim.x * blockDim.x)
    out[x] = fmaxf(in[x], 0.0f);
}

int grid_for(int64_t n, int block) {
  int64_t b = (n + block - 1) / block;
  const int64_t cap = 148LL * 32;
  return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace

cudaError_t launch_color_energy(const float* pr, const float* pi, float* e, int N,
                                cudaStream_t stream) {
  const int64_t n = 3LL * N * N * N;
  const bool vec = ((reinterpret_cast<uintptr_t>(pr) | reinterpret_cast<uintptr_t>(pi) |
                     reinterpret_cast<uintptr_t>(e)) & 15) == 0 && n % 4 == 0;
  if (vec) {
    color_energy_kernel<<<grid_for(n / 4, 256), 256, 0, stream>>>(
        reinterpret_cast<const float4*>(pr), reinterpret_cast<const float4*>(pi),
        reinterpret_cast<float4*>(e), n / 4);
  } else {
    color_energy_scalar_kernel<<<grid_for(n, 256), 256, 0, stream>>>(pr, pi, e, n);
  }
  return cudaGetLastError();
}

cudaError_t launch_helmholtz_multiply_gd(float2* spec, int N, double gamma, double d,
                                         cudaStream_t stream) {
  const int64_t per_colour = (int64_t)N * N * (N / 2 + 1);
  helmholtz_multiply_kernel<<<grid_for(per_colour, 256), 256, 0, stream>>>(spec, N, gamma, d,
                                                                           per_colour);
  return cudaGetLastError();
}

cudaError_t launch_clip(const float* in, float* out, int64_t count, cudaStream_t stream) {
  clip_kernel<<<grid_for(count, 256), 256, 0, stream>>>(in, out, count);
  return cudaGetLastError();
}

}  // namespace lfm
