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

struct Nb {
  int di, dj, dk;
  float w;   // Laplacian weight
  int axis;  // face neighbours: 0, 1, 2; edges: -1
  float sign;
};

// The 18 neighbours: 6 faces (1/3) then 12 edges (1/6).
__constant__ Nb kNb[18] = {
    {-1, 0, 0, 1.0f / 3.0f, 0, -1.0f}, {1, 0, 0, 1.0f / 3.0f, 0, 1.0f},
    {0, -1, 0, 1.0f / 3.0f, 1, -1.0f}, {0, 1, 0, 1.0f / 3.0f, 1, 1.0f},
    {0, 0, -1, 1.0f / 3.0f, 2, -1.0f}, {0, 0, 1, 1.0f / 3.0f, 2, 1.0f},
    {-1, -1, 0, 1.0f / 6.0f, -1, 0.0f}, {-1, 1, 0, 1.0f / 6.0f, -1, 0.0f},
    {1, -1, 0, 1.0f / 6.0f, -1, 0.0f},  {1, 1, 0, 1.0f / 6.0f, -1, 0.0f},
    {-1, 0, -1, 1.0f / 6.0f, -1, 0.0f}, {-1, 0, 1, 1.0f / 6.0f, -1, 0.0f},
    {1, 0, -1, 1.0f / 6.0f, -1, 0.0f},  {1, 0, 1, 1.0f / 6.0f, -1, 0.0f},
    {0, -1, -1, 1.0f / 6.0f, -1, 0.0f}, {0, -1, 1, 1.0f / 6.0f, -1, 0.0f},
    {0, 1, -1, 1.0f / 6.0f, -1, 0.0f},  {0, 1, 1, 1.0f / 6.0f, -1, 0.0f},
};

__device__ __forceinline__ int wrap(int x, int N) { return x < 0 ? x + N : (x >= N ? x - N : x); }

// a, u_r, u_i and gXn of cell (i, j, k).
struct Point {
  float a, ur, ui, gx;
};

template <int LEVEL>
__device__ __forceinline__ Point point(const AdjArgs& A, int i, int j, int k, int64_t y) {
  const float m = mask_from_q_flat(A.lut, qterm(i, A.N) + qterm(j, A.N) + qterm(k, A.N));
  Point p;
  p.a = fsub(1.0f, m);
  // the clamp value the forward writes: mask*chi0 + a*(-chi0)
  const float clamped = fadd(fmul(m, A.chi0), fmul(p.a, A.neg_chi0));
  const bool live = __ldg(A.chi_next + y) != clamped;
  p.gx = live ? p.a * __ldg(A.g_chi + y) : 0.0f;
  p.ur = p.a * __ldg(A.g_pr + y);
  p.ui = (LEVEL == LFM_COMPLEX) ? p.a * __ldg(A.g_pi + y) : 0.0f;
  return p;
}

template <int LEVEL>
__global__ void __launch_bounds__(256) adjoint_step_kernel(const AdjArgs A) {
  const int N = A.N;
  const int64_t n3 = (int64_t)N * N * N;
  const float c_w = -0.5f * A.eps_w * A.K * A.dt2;  // w(y) = c_w X(y) gXn(y)
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < n3;
       x += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(x % N);
    const int j = (int)((x / N) % N);
    const int i = (int)(x / ((int64_t)N * N));
    const Point p0 = point<LEVEL>(A, i, j, k, x);
    float lapR = -4.0f * p0.ur, lapI = -4.0f * p0.ui, lapX = -4.0f * p0.gx;
    float dPr = 0.0f, dPi = 0.0f, dwPr = 0.0f, dwPi = 0.0f;
#pragma unroll
    for (int q = 0; q < 18; ++q) {
      const Nb nb = kNb[q];
      const int yi = wrap(i + nb.di, N), yj = wrap(j + nb.dj, N), yk = wrap(k + nb.dk, N);
      const int64_t y = ((int64_t)yi * N + yj) * N + yk;
      const Point p = point<LEVEL>(A, yi, yj, yk, y);
      lapR += nb.w * p.ur;
      lapX += nb.w * p.gx;
      if (LEVEL == LFM_COMPLEX) lapI += nb.w * p.ui;
      if (q < 6 && LEVEL == LFM_COMPLEX) {
        const float pr = __ldg(A.pr + y), pi = __ldg(A.pi + y);
        const float wy = c_w * __ldg(A.chi + y) * p.gx;
        dPr += nb.sign * pr;
        dPi += nb.sign * pi;
        dwPr += nb.sign * wy * pr;
        dwPi += nb.sign * wy * pi;
      }
    }
    const float X = __ldg(A.chi + x);
    const float Pr = __ldg(A.pr + x);
    const float Pi = (LEVEL == LFM_COMPLEX) ? __ldg(A.pi + x) : 0.0f;
    float Q;
    if (LEVEL == LFM_COMPLEX) {
      const float jt = 0.5f * (Pr * dPi - Pi * dPr);
      Q = Pr * Pr + Pi * Pi + A.eps_w * jt - A.e0_sq;
    } else {
      Q = Pr * Pr - A.e0_sq;
    }
    const float gacc = A.dt2 * p0.gx;
    const float gQ = -gacc * A.K * X;
    const float X2 = X * X;
    A.o_pr[x] = p0.a * __ldg(A.g_prp + x) + 2.0f * p0.ur + A.dt2 * lapR - A.dt2 * X2 * p0.ur +
                2.0f * Pr * gQ +
                ((LEVEL == LFM_COMPLEX) ? (0.5f * A.eps_w * gQ) * dPi + dwPi : 0.0f);
    A.o_prp[x] = -p0.ur;
    if (LEVEL == LFM_COMPLEX) {
      A.o_pi[x] = p0.a * __ldg(A.g_pip + x) + 2.0f * p0.ui + A.dt2 * lapI - A.dt2 * X2 * p0.ui +
                  2.0f * Pi * gQ - (0.5f * A.eps_w * gQ) * dPr - dwPr;
      A.o_pip[x] = -p0.ui;
    }
    const float hp = A.use_lambda ? A.four_lambda * (3.0f * X2 - A.chi0_sq) : 0.0f;
    A.o_chi[x] = __ldg(A.g_chip + x) + 2.0f * p0.gx + A.dt2 * lapX - gacc * (hp + A.K * Q) -
                 2.0f * A.dt2 * X * (Pr * p0.ur + Pi * p0.ui);
    A.o_chip[x] = -p0.gx;
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
  const int64_t n3 = (int64_t)N * N * N;
  const int block = 256;
  int64_t blocks = (n3 + block - 1) / block;
  if (blocks > 148LL * 16) blocks = 148LL * 16;
  if (level == LFM_REAL)
    adjoint_step_kernel<LFM_REAL><<<(int)blocks, block, 0, stream>>>(A);
  else
    adjoint_step_kernel<LFM_COMPLEX><<<(int)blocks, block, 0, stream>>>(A);
  return cudaGetLastError();
}

}  // namespace lfm
