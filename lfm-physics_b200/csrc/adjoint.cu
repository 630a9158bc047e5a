// Adjoint (reverse-mode) leapfrog step for the REAL and COMPLEX levels.
//
// The forward step (lfm/core/backends/numpy_backend.py:80-205), per cell with
// absorb a = 1 - mask, K = kappa/chi0, L the periodic 19-point Laplacian and
// D_ax f = f[x+e_ax] - f[x-e_ax]:
//
//   P'   = a (2P - P_prev + dt2 (L P - X^2 P))        for P = Pr, Pi
//   P_prev' = a P
//   j    = 1/2 sum_ax (Pr D_ax Pi - Pi D_ax Pr)
//   Q    = Pr^2 + Pi^2 + eps_w j - e0^2               (REAL: E^2 - e0^2)
//   acc  = L X - K X Q - [lambda > 0] 4 lambda X (X^2 - chi0^2)
//   Xn   = 2X - X_prev + dt2 acc,  X' = mask chi0 + a max(Xn, -chi0)
//   X_prev' = X
//
// Given the adjoints of (P', P_prev', X', X_prev') this kernel returns the
// adjoints of (P, P_prev, X, X_prev).  L is symmetric and D_ax is
// antisymmetric, so the transposed stencils are L and -D_ax.  With
// u = a gP', gXn = a gX' [Xn not clamped], gQ = -dt2 gXn K X and
// w = eps_w gQ / 2:
//
//   gP_prev = -u                  gX_prev = -gXn
//   gPr = a gPr_prev' + 2u_r + dt2 L u_r - dt2 X^2 u_r + 2 Pr gQ + w sum D Pi + sum D (w Pi)
//   gPi = a gPi_prev' + 2u_i + dt2 L u_i - dt2 X^2 u_i + 2 Pi gQ - w sum D Pr - sum D (w Pr)
//   gX  = gX_prev' + 2 gXn + dt2 L gXn - dt2 gXn (H'(X) + K Q) - 2 dt2 X (Pr u_r + Pi u_i)
//
// with H'(X) = 4 lambda (3 X^2 - chi0^2).  The clamp test needs Xn, which
// depends on the cell's whole stencil; it is read back from the step's output
// instead: a cell was clamped exactly when X' equals mask chi0 + a (-chi0) in
// the forward's float32 arithmetic (a == 0 cells carry no gradient anyway).
//
// Arithmetic is plain float32 (contractions allowed): the adjoint is not tied
// to the reference bit for bit; its accuracy is checked against float64
// autograd and central differences.
#include "lfm_b200.h"
#include "lfm_index.cuh"
#include "lfm_kernels.h"

namespace lfm {
namespace {

struct AdjArgs {
  int level, N;
  const float *pr, *pi, *chi, *chi_next;
  MaskLut lut;
  const float *g_pr, *g_prp, *g_pi, *g_pip, *g_chi, *g_chip;
  float *o_pr, *o_prp, *o_pi, *o_pip, *o_chi, *o_chip;
  float dt2, K, eps_w, e0_sq, four_lambda, chi0, chi0_sq, neg_chi0;
  int use_lambda;
};

// ---- tiled kernel ----------------------------------------------------------
// A CTA owns a TI x TJ x TK block of cells.  Phase 1 evaluates, once per
// point of the block and its one-cell halo, everything the transposed
// stencils need from a neighbour (a*gP', a*gX'*[not clamped], and at the
// COMPLEX level Pr, Pi, w*Pr, w*Pi), into shared memory.  Phase 2 applies
// the stencils from shared memory.  Threads run along k (coalesced loads,
// conflict-free shared-memory rows).
constexpr int TI = 4, TJ = 8, TK = 32;
constexpr int HI = TI + 2, HJ = TJ + 2, HK = TK + 2;
constexpr int HALO = HI * HJ * HK;
constexpr int kThreads = TJ * TK;  // 256: one (j, k) column of TI cells each

template <int LEVEL>
struct TileSmem {
  static constexpr int NF = (LEVEL == LFM_COMPLEX) ? 7 : 2;
  float f[NF][HALO];  // ur, gx [, ui, pr, pi, wpr, wpi]
};

__device__ __forceinline__ int wrapmod(int x, int N) {
  x %= N;
  return x < 0 ? x + N : x;
}

template <int LEVEL>
__global__ void __launch_bounds__(kThreads) adjoint_tile_kernel(const AdjArgs A) {
  extern __shared__ __align__(16) float sm_raw[];
  TileSmem<LEVEL>& S = *reinterpret_cast<TileSmem<LEVEL>*>(sm_raw);
  const int N = A.N;
  const int tiles_k = (N + TK - 1) / TK, tiles_j = (N + TJ - 1) / TJ;
  int t = blockIdx.x;
  const int k0 = (t % tiles_k) * TK;
  t /= tiles_k;
  const int j0 = (t % tiles_j) * TJ;
  const int i0 = (t / tiles_j) * TI;
  const float c_w = -0.5f * A.eps_w * A.K * A.dt2;  // w(y) = c_w X(y) gXn(y)

  // phase 1: point terms of the block and its halo
  for (int h = threadIdx.x; h < HALO; h += kThreads) {
    const int hk = h % HK, hj = (h / HK) % HJ, hi = h / (HK * HJ);
    const int gi = wrapmod(i0 + hi - 1, N), gj = wrapmod(j0 + hj - 1, N),
              gk = wrapmod(k0 + hk - 1, N);
    const int64_t y = ((int64_t)gi * N + gj) * N + gk;
    const float m = mask_from_q_flat(A.lut, qterm(gi, N) + qterm(gj, N) + qterm(gk, N));
    const float a = fsub(1.0f, m);
    // the clamp value the forward writes: mask*chi0 + a*(-chi0)
    const float clamped = fadd(fmul(m, A.chi0), fmul(a, A.neg_chi0));
    const float gx = (__ldg(A.chi_next + y) != clamped) ? a * __ldg(A.g_chi + y) : 0.0f;
    S.f[0][h] = a * __ldg(A.g_pr + y);
    S.f[1][h] = gx;
    if constexpr (LEVEL == LFM_COMPLEX) {
      const float pr = __ldg(A.pr + y), pi = __ldg(A.pi + y);
      const float w = c_w * __ldg(A.chi + y) * gx;
      S.f[2][h] = a * __ldg(A.g_pi + y);
      S.f[3][h] = pr;
      S.f[4][h] = pi;
      S.f[5][h] = w * pr;
      S.f[6][h] = w * pi;
    }
  }
  __syncthreads();

  // phase 2: one (j, k) column of TI cells per thread
  const int tk = threadIdx.x % TK, tj = threadIdx.x / TK;
  const int gj = j0 + tj, gk = k0 + tk;
  if (gj >= N || gk >= N) return;
  constexpr int DI = HJ * HK, DJ = HK;
  const float third = 1.0f / 3.0f, sixth = 1.0f / 6.0f;
#pragma unroll
  for (int ti = 0; ti < TI; ++ti) {
    const int gi = i0 + ti;
    if (gi >= N) break;
    const int64_t x = ((int64_t)gi * N + gj) * N + gk;
    const int c = ((ti + 1) * HJ + (tj + 1)) * HK + (tk + 1);
    // transposed (= the) Laplacian of a shared-memory field at the centre
    auto lap = [&](const float* f) {
      const float faces = f[c - DI] + f[c + DI] + f[c - DJ] + f[c + DJ] + f[c - 1] + f[c + 1];
      const float edges = f[c - DI - DJ] + f[c - DI + DJ] + f[c + DI - DJ] + f[c + DI + DJ] +
                          f[c - DI - 1] + f[c - DI + 1] + f[c + DI - 1] + f[c + DI + 1] +
                          f[c - DJ - 1] + f[c - DJ + 1] + f[c + DJ - 1] + f[c + DJ + 1];
      return third * faces + sixth * edges - 4.0f * f[c];
    };
    // sum over the axes of f[x + e] - f[x - e]
    auto dsum = [&](const float* f) {
      return (f[c + DI] - f[c - DI]) + (f[c + DJ] - f[c - DJ]) + (f[c + 1] - f[c - 1]);
    };
    const float ur = S.f[0][c], gx = S.f[1][c];
    const float lapR = lap(S.f[0]), lapX = lap(S.f[1]);
    const float m0 = mask_from_q_flat(A.lut, qterm(gi, N) + qterm(gj, N) + qterm(gk, N));
    const float a0 = fsub(1.0f, m0);
    const float X = __ldg(A.chi + x);
    const float X2 = X * X;
    const float gacc = A.dt2 * gx;
    const float gQ = -gacc * A.K * X;
    const float hp = A.use_lambda ? A.four_lambda * (3.0f * X2 - A.chi0_sq) : 0.0f;
    if constexpr (LEVEL == LFM_COMPLEX) {
      const float ui = S.f[2][c], Pr = S.f[3][c], Pi = S.f[4][c];
      const float lapI = lap(S.f[2]);
      const float dPr = dsum(S.f[3]), dPi = dsum(S.f[4]);
      const float dwPr = dsum(S.f[5]), dwPi = dsum(S.f[6]);
      const float jt = 0.5f * (Pr * dPi - Pi * dPr);
      const float Q = Pr * Pr + Pi * Pi + A.eps_w * jt - A.e0_sq;
      const float w0 = 0.5f * A.eps_w * gQ;
      A.o_pr[x] = a0 * __ldg(A.g_prp + x) + 2.0f * ur + A.dt2 * lapR - A.dt2 * X2 * ur +
                  2.0f * Pr * gQ + w0 * dPi + dwPi;
      A.o_pi[x] = a0 * __ldg(A.g_pip + x) + 2.0f * ui + A.dt2 * lapI - A.dt2 * X2 * ui +
                  2.0f * Pi * gQ - w0 * dPr - dwPr;
      A.o_prp[x] = -ur;
      A.o_pip[x] = -ui;
      A.o_chi[x] = __ldg(A.g_chip + x) + 2.0f * gx + A.dt2 * lapX - gacc * (hp + A.K * Q) -
                   2.0f * A.dt2 * X * (Pr * ur + Pi * ui);
    } else {
      const float E = __ldg(A.pr + x);
      const float Q = E * E - A.e0_sq;
      A.o_pr[x] = a0 * __ldg(A.g_prp + x) + 2.0f * ur + A.dt2 * lapR - A.dt2 * X2 * ur +
                  2.0f * E * gQ;
      A.o_prp[x] = -ur;
      A.o_chi[x] = __ldg(A.g_chip + x) + 2.0f * gx + A.dt2 * lapX - gacc * (hp + A.K * Q) -
                   2.0f * A.dt2 * X * E * ur;
    }
    A.o_chip[x] = -gx;
  }
}

}  // namespace

cudaError_t launch_adjoint_step(int level, int N, const float* pr, const float* pi,
                                const float* chi, const float* chi_next, const MaskLut& lut,
                                const float* const g_out[6], float* const g_in[6],
                                const StepConsts& c, cudaStream_t stream) {
  AdjArgs A{};
  A.level = level;
  A.N = N;
  A.pr = pr;
  A.pi = pi;
  A.chi = chi;
  A.chi_next = chi_next;
  A.lut = lut;
  A.g_pr = g_out[0]; A.g_prp = g_out[1]; A.g_pi = g_out[2]; A.g_pip = g_out[3];
  A.g_chi = g_out[4]; A.g_chip = g_out[5];
  A.o_pr = g_in[0]; A.o_prp = g_in[1]; A.o_pi = g_in[2]; A.o_pip = g_in[3];
  A.o_chi = g_in[4]; A.o_chip = g_in[5];
  A.dt2 = c.dt2;
  A.K = c.k_over_chi0;
  A.eps_w = c.eps_w;
  A.e0_sq = c.e0_sq;
  A.four_lambda = c.four_lambda;
  A.chi0 = c.chi0;
  A.chi0_sq = c.chi0_sq;
  A.neg_chi0 = c.neg_chi0;
  A.use_lambda = c.use_lambda;
  const int tiles = ((N + TK - 1) / TK) * ((N + TJ - 1) / TJ) * ((N + TI - 1) / TI);
  if (level == LFM_REAL) {
    const int smem = (int)sizeof(TileSmem<LFM_REAL>);
    adjoint_tile_kernel<LFM_REAL><<<tiles, kThreads, smem, stream>>>(A);
  } else {
    const int smem = (int)sizeof(TileSmem<LFM_COMPLEX>);
    static bool granted = false;  // 57 KB: above the 48 KB default
    if (!granted) {
      cudaError_t e = cudaFuncSetAttribute(adjoint_tile_kernel<LFM_COMPLEX>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
      if (e != cudaSuccess) return e;
      granted = true;
    }
    adjoint_tile_kernel<LFM_COMPLEX><<<tiles, kThreads, smem, stream>>>(A);
  }
  return cudaGetLastError();
}

}  // namespace lfm
