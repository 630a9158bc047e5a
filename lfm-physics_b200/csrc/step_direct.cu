// Direct step kernels: one thread per cell, neighbours read through L1.
//
// This is the general path: any N (odd sizes included), every level, both
// the protocol (out-of-place, reference A/B semantics) and the resident
// (in-place slot rotation) modes.  The fused 2.5D kernels in step_tma.cu
// take over when N is a multiple of 4.
#include "lfm_cells.cuh"
#include "lfm_index.cuh"
#include "lfm_kernels.h"

namespace lfm {
namespace {

__device__ __forceinline__ Faces faces_of(const S19& s) {
  Faces f;
  f.im = s.im; f.ip = s.ip; f.jm = s.jm; f.jp = s.jp; f.km = s.km; f.kp = s.kp;
  return f;
}

__device__ __forceinline__ float cell_mask(const StepArgs& a, int i, int j, int k, int64_t x) {
  if (a.mask) return __ldg(a.mask + x);
  return mask_from_q(a.lut, qterm(i + a.i_off, a.N) + qterm(j, a.N) + qterm(k, a.N));
}

// Previous-step value: slots written by the previous resident step hold the
// undamped field and get (1-mask) here, the same product the reference
// stored (numpy_backend.py:128).
__device__ __forceinline__ float prev_value(const StepArgs& a, const float* p, int64_t x,
                                            float absorb) {
  const float v = p[x];
  return a.damp_prev ? fmul(v, absorb) : v;
}

template <int LEVEL>
__global__ void __launch_bounds__(256) direct_step_kernel(const StepArgs a) {
  const int N = a.N;
  const int64_t n3 = (int64_t)N * N * N;
  // a slab updates planes [i_lo, i_hi) of its array and reads i_lo-1, i_hi
  const int64_t first = a.slab ? (int64_t)a.i_lo * N * N : 0;
  const int64_t count = a.slab ? (int64_t)(a.i_hi - a.i_lo) * N * N : n3;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t x = first + t;
    const int k = (int)(x % N);
    const int j = (int)((x / N) % N);
    const int i = (int)(x / ((int64_t)N * N));
    const Idx ix = a.slab ? neighbour_index_slab(i, j, k, N) : neighbour_index(i, j, k, N);
    const float mask = cell_mask(a, i, j, k, x);
    const float absorb = fsub(1.0f, mask);
    const S19 X = gather(a.chi, ix);
    const float chi_prev = a.chi_prev[x];
    if (LEVEL != LFM_COLOR && a.split) {
      // split chi: chi = chi0 + hi + lo (resident slots, previous Psi damped on read);
      // the offset's Laplacian is that of hi (lfm_cells.cuh, split chi)
      const float lapD = lap19_diff(X);
      const double d = split_value(X.c, a.chi_lo[x]);
      const double d_prev = split_value(chi_prev, a.chi_lo_prev[x]);
      SplitChi c;
      if (LEVEL == LFM_REAL) {
        const S19 E = gather(a.pr, ix);
        const RealSplit o = real_cell_split(lap19_fma(E), E.c, prev_value(a, a.pr_prev, x, absorb),
                                            lapD, d, d_prev, mask, absorb, a.c);
        a.pr_out[x] = o.psi;
        c = o.chi;
      } else {
        const S19 R = gather(a.pr, ix);
        const S19 I = gather(a.pi, ix);
        const ComplexSplit o = complex_cell_split(
            lap19_fma(R), R.c, prev_value(a, a.pr_prev, x, absorb), faces_of(R), lap19_fma(I),
            I.c, prev_value(a, a.pi_prev, x, absorb), faces_of(I), lapD, d, d_prev, mask, absorb,
            a.c);
        a.pr_out[x] = o.pr;
        a.pi_out[x] = o.pi;
        c = o.chi;
      }
      a.chi_out[x] = c.hi;
      a.chi_lo_out[x] = c.lo;
      continue;
    }
    if (LEVEL != LFM_COLOR && a.comp) {
      // compensated Delta form: *_prev hold the increments (updated in place)
      if (LEVEL == LFM_REAL) {
        const S19 E = gather(a.pr, ix);
        const RealComp o = real_cell_comp(lap19_fma(E), E.c, a.pr_prev[x], lap19_diff(X), X.c,
                                          chi_prev, mask, a.c);
        a.pr_out[x] = o.psi.v;
        a.pr_prev_out[x] = o.psi.d;
        a.chi_out[x] = o.chi.v;
        a.chi_prev_out[x] = o.chi.d;
      } else {
        const S19 R = gather(a.pr, ix);
        const S19 I = gather(a.pi, ix);
        const ComplexComp o = complex_cell_comp(lap19_fma(R), R.c, a.pr_prev[x], faces_of(R),
                                                lap19_fma(I), I.c, a.pi_prev[x], faces_of(I),
                                                lap19_diff(X), X.c, chi_prev, mask, a.c);
        a.pr_out[x] = o.pr.v;
        a.pr_prev_out[x] = o.pr.d;
        a.pi_out[x] = o.pi.v;
        a.pi_prev_out[x] = o.pi.d;
        a.chi_out[x] = o.chi.v;
        a.chi_prev_out[x] = o.chi.d;
      }
      continue;
    }
    if (LEVEL == LFM_REAL) {
      const S19 E = gather(a.pr, ix);
      const RealOut o =
          real_cell(lap19(E), E.c, prev_value(a, a.pr_prev, x, absorb), lap19(X), X.c, chi_prev,
                    mask, a.c);
      a.pr_out[x] = o.psi;
      a.chi_out[x] = o.chi;
      if (a.pr_prev_out) a.pr_prev_out[x] = o.psi_prev;
      if (a.chi_prev_out) a.chi_prev_out[x] = o.chi_prev;
    } else if (LEVEL == LFM_COMPLEX) {
      const S19 R = gather(a.pr, ix);
      const S19 I = gather(a.pi, ix);
      const ComplexOut o = complex_cell(
          lap19(R), R.c, prev_value(a, a.pr_prev, x, absorb), faces_of(R), lap19(I), I.c,
          prev_value(a, a.pi_prev, x, absorb), faces_of(I), lap19(X), X.c, chi_prev, mask, a.c);
      a.pr_out[x] = o.pr;
      a.pi_out[x] = o.pi;
      a.chi_out[x] = o.chi;
      if (a.pr_prev_out) a.pr_prev_out[x] = o.pr_prev;
      if (a.pi_prev_out) a.pi_prev_out[x] = o.pi_prev;
      if (a.chi_prev_out) a.chi_prev_out[x] = o.chi_prev;
    } else {
      float pr_c[3], pi_c[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        pr_c[c] = __ldg(a.pr + c * n3 + x);
        pi_c[c] = __ldg(a.pi + c * n3 + x);
      }
      ColorAcc A;
      color_begin(A, X.c, mask, pr_c, pi_c, a.c);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const S19 R = gather(a.pr + c * n3, ix);
        const S19 I = gather(a.pi + c * n3, ix);
        const ColorCompOut o = color_component(
            A, c, lap19(R), R.c, prev_value(a, a.pr_prev + c * n3, x, absorb), faces_of(R),
            lap19(I), I.c, prev_value(a, a.pi_prev + c * n3, x, absorb), faces_of(I), a.c);
        a.pr_out[c * n3 + x] = o.pr;
        a.pi_out[c * n3 + x] = o.pi;
        if (a.energy_out) a.energy_out[c * n3 + x] = fadd(fmul(o.pr, o.pr), fmul(o.pi, o.pi));
        if (a.pr_prev_out) a.pr_prev_out[c * n3 + x] = o.pr_prev;
        if (a.pi_prev_out) a.pi_prev_out[c * n3 + x] = o.pi_prev;
      }
      float sa[3] = {0.0f, 0.0f, 0.0f};
      if (a.sa) {
#pragma unroll
        for (int c = 0; c < 3; ++c) sa[c] = __ldg(a.sa + c * n3 + x);
        if (a.sa_clip_out) {
#pragma unroll
          for (int c = 0; c < 3; ++c) a.sa_clip_out[c * n3 + x] = fmaxf(sa[c], 0.0f);
        }
      }
      a.chi_out[x] = color_finish(A, lap19(X), chi_prev, a.sa != nullptr, sa, a.c);
      if (a.chi_prev_out) a.chi_prev_out[x] = X.c;
    }
  }
}

}  // namespace

cudaError_t launch_direct_step(const StepArgs& a, cudaStream_t stream) {
  const int64_t n3 = a.slab ? (int64_t)(a.i_hi - a.i_lo) * a.N * a.N : (int64_t)a.N * a.N * a.N;
  const int block = 256;
  int64_t blocks = (n3 + block - 1) / block;
  const int64_t cap = 148LL * 16;  // grid-stride beyond 16 waves of CTAs
  if (blocks > cap) blocks = cap;
  switch (a.level) {
    case LFM_REAL: direct_step_kernel<LFM_REAL><<<(int)blocks, block, 0, stream>>>(a); break;
    case LFM_COMPLEX: direct_step_kernel<LFM_COMPLEX><<<(int)blocks, block, 0, stream>>>(a); break;
    default: direct_step_kernel<LFM_COLOR><<<(int)blocks, block, 0, stream>>>(a); break;
  }
  return cudaGetLastError();
}

}  // namespace lfm
