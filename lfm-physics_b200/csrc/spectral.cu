// S_a Helmholtz filter fused with the transforms along the slowest axis.
//
// The reference smooths each colour's |Psi_a|^2 as
//   S_a = IRFFT3[ gamma / (gamma + D |k|^2) * RFFT3(|Psi_a|^2) ]
// (lfm/core/backends/numpy_backend.py:341-356).  A 3-D transform is three 1-D
// passes, so the solve is split as
//   cuFFT 2-D R2C over (j, k) for every plane i and colour
//   -> this kernel: forward 1-D FFT along i, times the filter, inverse 1-D FFT
//   -> cuFFT 2-D C2R over (j, k).
// The kernel replaces three HBM round trips of the half spectrum (the forward
// pass along i, the filter multiply, the inverse pass along i) by one.
//
// Spectrum layout (cuFFT's R2C output): spec[a][x][w], w = y * (N/2+1) + z,
// so for a fixed x the columns w are contiguous.  A CTA owns TW consecutive
// columns of one colour and all N values of x in each.  The length-N FFT of a
// column is the four-step factorisation N = N1 * N2 (Bailey's "four-step FFT",
// also in Van Loan, Computational Frameworks for the FFT, 3.3): thread n1 of a
// column holds x[n1 + N1 m] (m < N2); a length-N2 DFT in registers, a twiddle
// w_N^(n1 k2), an exchange through shared memory, a length-N1 DFT in
// registers; the inverse retraces the steps with conjugate twiddles, so every
// thread ends with the elements it loaded.  The register DFTs are iterative
// radix-2 Cooley-Tukey (decimation in time).  Twiddles w_N^j = e^{-2 pi i j/N}
// come from tables computed on the host in double precision: the length-N
// table in shared memory for the twiddles between the two DFTs, and the
// length-32 table in constant memory for the register DFTs (M <= 32).
//
// The filter factor of each spectral point, gamma/(gamma + D k^2) / N^3
// rounded to float32 once, is read from a table over (|fx|, |fy|, fz) built by
// helmholtz_table_kernel with the float64 arithmetic of NumPy's filter
// (k = 2 pi fftfreq(N)); k^2 depends only on the magnitudes of the integer
// frequencies, so (N/2+1)^3 entries cover the spectrum.
#include "lfm_kernels.h"

#include <cmath>

namespace lfm {
namespace {

__host__ __device__ constexpr int bitrev(int i, int bits) {
  int r = 0;
  for (int b = 0; b < bits; ++b) r |= ((i >> b) & 1) << (bits - 1 - b);
  return r;
}
__host__ __device__ constexpr int log2i(int n) { return n <= 1 ? 0 : 1 + log2i(n / 2); }

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(__fmaf_rn(a.x, b.x, -__fmul_rn(a.y, b.y)),
                     __fmaf_rn(a.x, b.y, __fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }

// e^{-2 pi i t / 32}, t < 32: the twiddles of the register DFTs (M <= 32),
// w_M^u = c_w32[u * 32 / M].  The indices are compile-time constants, so each
// twiddle is an operand from the constant bank, not a shared-memory load.
// The values equal the pass's own table (e^{-2 pi i (u N / M) / N} has the same
// angle u / M in double).
__constant__ float2 c_w32[32];

// One radix-2 stage (butterflies of span LEN / 2) of an in-register DFT of
// size M; a[] is in bit-reversed order before the first stage.
template <int M, int LEN, bool INV>
__device__ __forceinline__ void dft_stage(float2 (&a)[M]) {
  static_assert(M <= 32, "register DFTs take their twiddles from c_w32");
  constexpr int half = LEN / 2, step = M / LEN;
#pragma unroll
  for (int i = 0; i < M; i += LEN) {
#pragma unroll
    for (int j = 0; j < half; ++j) {
      const int u = j * step;  // exponent in units of w_M
      float2 t = a[i + j + half];
      if (u == 0) {
      } else if (4 * u == M) {  // w_M^(M/4) = -i (forward), +i (inverse)
        t = INV ? make_float2(-t.y, t.x) : make_float2(t.y, -t.x);
      } else {
        const float2 w = c_w32[u * (32 / M)];
        t = cmul(t, INV ? conjf2(w) : w);
      }
      const float2 s = a[i + j];
      a[i + j] = make_float2(s.x + t.x, s.y + t.y);
      a[i + j + half] = make_float2(s.x - t.x, s.y - t.y);
    }
  }
  if constexpr (LEN < M) dft_stage<M, 2 * LEN, INV>(a);
}

// v[k] <- sum_j v[j] w_M^(s j k), s = -1 (forward, e^{-}) or +1 (inverse), in
// registers.
template <int M, bool INV>
__device__ __forceinline__ void dft_reg(float2 (&v)[M]) {
  constexpr int B = log2i(M);
  float2 a[M];
#pragma unroll
  for (int i = 0; i < M; ++i) a[bitrev(i, B)] = v[i];
  dft_stage<M, 2, INV>(a);
#pragma unroll
  for (int i = 0; i < M; ++i) v[i] = a[i];
}

// One CTA: TW columns w0 .. w0+TW-1 of colour a.  Thread (n1, c), n1 < N1,
// c < TW, tid = n1 * TW + c.  Shared exchange buffer S(c, n1, k2) at
// (k2 * N1 + n1) * TW + c: consecutive threads touch consecutive columns in
// every phase (two 8-byte wavefronts per warp, no further conflicts).
template <int N1, int N2, int TW>
__global__ void __launch_bounds__(N1* TW) helmholtz_xpass_kernel(float2* __restrict__ spec,
                                                                 const float* __restrict__ table,
                                                                 const float2* __restrict__ twg) {
  constexpr int N = N1 * N2;
  constexpr int H = N / 2 + 1;
  constexpr int64_t W = (int64_t)N * H;  // columns per colour
  constexpr int G = N2 / N1;             // k2 groups per thread after the exchange
  static_assert(N2 % N1 == 0, "N2 must be a multiple of N1");
  extern __shared__ float2 smem_x[];
  float2* tw = smem_x;      // N twiddles
  float2* S = smem_x + N;   // N * TW exchange buffer
  const int tid = threadIdx.x;
  const int n1 = tid / TW, c = tid % TW;
  for (int t = tid; t < N; t += N1 * TW) tw[t] = twg[t];
  const int64_t tiles_per_colour = W / TW;
  const int a = (int)(blockIdx.x / tiles_per_colour);
  const int64_t w = (blockIdx.x % tiles_per_colour) * TW + c;
  float2* col = spec + (int64_t)a * N * W + w;  // element x at col[x * W]
  const int y = (int)(w / H), z = (int)(w % H);
  const int fy = y <= N - y ? y : N - y;
  const float* trow = table + (int64_t)fy * H + z;  // + |fx| * H * H
  __syncthreads();  // twiddles

  // ---- forward along x -------------------------------------------------------
  float2 v[N2];
#pragma unroll
  for (int m = 0; m < N2; ++m) v[m] = col[(int64_t)(n1 + N1 * m) * W];
  dft_reg<N2, false>(v);  // v[k2] = Y[n1][k2]
#pragma unroll
  for (int k2 = 1; k2 < N2; ++k2) v[k2] = cmul(v[k2], tw[n1 * k2]);
#pragma unroll
  for (int k2 = 0; k2 < N2; ++k2) S[(k2 * N1 + n1) * TW + c] = v[k2];
  __syncthreads();
  float2 u[G][N1];  // group g: k2 = n1 + N1 g (this thread's k2 values)
#pragma unroll
  for (int g = 0; g < G; ++g) {
    const int k2 = n1 + N1 * g;
#pragma unroll
    for (int j = 0; j < N1; ++j) u[g][j] = S[(k2 * N1 + j) * TW + c];
    dft_reg<N1, false>(u[g]);  // u[g][k1] = X[k2 + N2 k1]
    // ---- the filter --------------------------------------------------------
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) {
      const int k = k2 + N2 * k1;
      const int fx = k <= N - k ? k : N - k;
      const float f = __ldg(trow + (int64_t)fx * H * H);
      u[g][k1] = make_float2(u[g][k1].x * f, u[g][k1].y * f);
    }
    // ---- inverse along x, first half ---------------------------------------
    dft_reg<N1, true>(u[g]);  // u[g][j] = sum_k1 X w_N1^(-k1 j)
#pragma unroll
    for (int j = 1; j < N1; ++j) u[g][j] = cmul(u[g][j], conjf2(tw[k2 * j]));
  }
  __syncthreads();  // every thread has read S
#pragma unroll
  for (int g = 0; g < G; ++g) {
    const int k2 = n1 + N1 * g;
#pragma unroll
    for (int j = 0; j < N1; ++j) S[(k2 * N1 + j) * TW + c] = u[g][j];
  }
  __syncthreads();
#pragma unroll
  for (int k2 = 0; k2 < N2; ++k2) v[k2] = S[(k2 * N1 + n1) * TW + c];
  dft_reg<N2, true>(v);  // v[m] = x[n1 + N1 m] (times N: unnormalised)
#pragma unroll
  for (int m = 0; m < N2; ++m) col[(int64_t)(n1 + N1 * m) * W] = v[m];
}

// np.fft.fftfreq(n) * 2*pi for the frequency magnitude f: f * (1.0/n) * 2*pi in
// float64 (the sign of f does not change k^2).
__device__ __forceinline__ double wave(int f, int n) {
  return __dmul_rn(__dmul_rn((double)f, 1.0 / (double)n), 2.0 * 3.141592653589793);
}

// table[(fx * H + fy) * H + fz] = float32(gamma / (gamma + D k^2) / N^3), the
// same float64 operations (and the same rounding) as a per-element filter.
__global__ void helmholtz_table_kernel(float* __restrict__ table, int N, double gamma,
                                       double d) {
  const int H = N / 2 + 1;
  const int64_t total = (int64_t)H * H * H;
  const double inv_n3 = 1.0 / ((double)N * N * N);
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int fz = (int)(t % H), fy = (int)((t / H) % H), fx = (int)(t / ((int64_t)H * H));
    const double kx = wave(fx, N), ky = wave(fy, N), kz = wave(fz, N);
    const double k_sq = __dadd_rn(__dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky)),
                                  __dmul_rn(kz, kz));
    const double h = __ddiv_rn(gamma, __dadd_rn(gamma, __dmul_rn(d, k_sq)));
    table[t] = __double2float_rn(__dmul_rn(h, inv_n3));
  }
}

template <int N1, int N2, int TW>
cudaError_t launch_xpass(float2* spec, const float* table, const float2* tw,
                         cudaStream_t stream) {
  constexpr int N = N1 * N2;
  constexpr int smem = (N + N * TW) * (int)sizeof(float2);
  static bool granted = false;  // the attribute is per function and process
  if (!granted) {
    cudaError_t e = cudaFuncSetAttribute(helmholtz_xpass_kernel<N1, N2, TW>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    granted = true;
  }
  const int64_t W = (int64_t)N * (N / 2 + 1);
  const int64_t tiles = 3 * (W / TW);
  helmholtz_xpass_kernel<N1, N2, TW><<<(unsigned)tiles, N1 * TW, smem, stream>>>(spec, table,
                                                                                  tw);
  return cudaGetLastError();
}

}  // namespace

cudaError_t upload_dft_twiddles() {
  float2 w[32];
  for (int t = 0; t < 32; ++t) {
    const double ang = -2.0 * 3.14159265358979323846 * (double)t / 32.0;
    w[t] = make_float2((float)std::cos(ang), (float)std::sin(ang));
  }
  return cudaMemcpyToSymbol(c_w32, w, sizeof(w));
}

bool helmholtz_xpass_supported(int N) {
  return N == 64 || N == 128 || N == 256 || N == 512 || N == 1024;
}

cudaError_t launch_helmholtz_table(float* table, int N, double gamma, double d,
                                   cudaStream_t stream) {
  const int64_t total = (int64_t)(N / 2 + 1) * (N / 2 + 1) * (N / 2 + 1);
  int64_t blocks = (total + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  helmholtz_table_kernel<<<(unsigned)blocks, 256, 0, stream>>>(table, N, gamma, d);
  return cudaGetLastError();
}

cudaError_t launch_helmholtz_xpass(float2* spec, const float* table, const float2* tw, int N,
                                   cudaStream_t stream) {
  switch (N) {
    case 64: return launch_xpass<8, 8, 32>(spec, table, tw, stream);
    case 128: return launch_xpass<8, 16, 32>(spec, table, tw, stream);
    case 256: return launch_xpass<16, 16, 16>(spec, table, tw, stream);
    case 512: return launch_xpass<16, 32, 16>(spec, table, tw, stream);
    case 1024: return launch_xpass<32, 32, 8>(spec, table, tw, stream);
    default: return cudaErrorNotSupported;
  }
}

}  // namespace lfm
