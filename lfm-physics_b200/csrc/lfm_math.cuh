// Per-cell arithmetic of the leapfrog step, shared by every kernel.
//
// Each helper restates one expression of the reference's NumPy backend
// (lfm/core/backends/numpy_backend.py:80-382) with the same operation
// order and one float32 rounding per operation.  The explicit __fadd_rn /
// __fsub_rn / __fmul_rn intrinsics are never contracted into fused
// multiply-adds, so a kernel built from these helpers reproduces NumPy's
// float32 results bit for bit whatever the compiler flags.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "lfm_b200.h"

namespace lfm {

__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }

// Scalar parameters rounded to float32 on the host the way NumPy rounds a
// Python float that meets a float32 array (NEP 50 "weak" scalars).  Compound
// constants (kappa/chi0, 4*lambda, dt2*eps_cc ...) are formed in double first,
// as Python evaluates them before they meet an array.
struct StepConsts {
  float dt2;
  float k_over_chi0;   // kappa / chi0
  float four_lambda;   // 4.0 * lambda_self
  float chi0_sq;       // chi0 * chi0
  float chi0;
  float neg_chi0;
  float e0_sq;
  float eps_w;
  float kc_over_chi0;  // kappa_c / chi0
  float dt2_eps_cc;    // dt2 * epsilon_cc
  float kappa_string;
  float kappa_tube;
  int use_lambda;      // lambda_self > 0   (numpy_backend.py:113)
  int use_cc;          // epsilon_cc > 0    (numpy_backend.py:254)
  int use_fc;          // kappa_c > 0       (numpy_backend.py:314)
  int use_ccv;         // kappa_string > 0  (numpy_backend.py:249)
};

inline StepConsts make_step_consts(double dt2, double kappa, double lambda_self, double chi0,
                                   double e0_sq, double eps_w, double kappa_c, double eps_cc,
                                   double kappa_string, double kappa_tube) {
  StepConsts c;
  c.dt2 = (float)dt2;
  c.k_over_chi0 = (float)(kappa / chi0);
  c.four_lambda = (float)(4.0 * lambda_self);
  c.chi0_sq = (float)(chi0 * chi0);
  c.chi0 = (float)chi0;
  c.neg_chi0 = (float)(-chi0);
  c.e0_sq = (float)e0_sq;
  c.eps_w = (float)eps_w;
  c.kc_over_chi0 = (float)(kappa_c / chi0);
  c.dt2_eps_cc = (float)(dt2 * eps_cc);
  c.kappa_string = (float)kappa_string;
  c.kappa_tube = (float)kappa_tube;
  c.use_lambda = lambda_self > 0.0;
  c.use_cc = eps_cc > 0.0;
  c.use_fc = kappa_c > 0.0;
  c.use_ccv = kappa_string > 0.0;
  return c;
}

// The 19 values a cell's Laplacian reads, named by offset from the cell.
struct S19 {
  float c, im, ip, jm, jp, km, kp;
  float imjm, imjp, ipjm, ipjp, imkm, imkp, ipkm, ipkp, jmkm, jmkp, jpkm, jpkp;
};

// laplacian_19pt (lfm/core/stencils.py:43-71): faces summed in the order the
// np.roll terms appear (roll(+1) = the x-1 neighbour), then the 12 edges,
// then (1/3)*faces + (1/6)*edges + (-4)*centre.
__device__ __forceinline__ float lap19(const S19& f) {
  float faces = fadd(f.im, f.ip);
  faces = fadd(faces, f.jm);
  faces = fadd(faces, f.jp);
  faces = fadd(faces, f.km);
  faces = fadd(faces, f.kp);
  float edges = fadd(f.imjm, f.imjp);
  edges = fadd(edges, f.ipjm);
  edges = fadd(edges, f.ipjp);
  edges = fadd(edges, f.imkm);
  edges = fadd(edges, f.imkp);
  edges = fadd(edges, f.ipkm);
  edges = fadd(edges, f.ipkp);
  edges = fadd(edges, f.jmkm);
  edges = fadd(edges, f.jmkp);
  edges = fadd(edges, f.jpkm);
  edges = fadd(edges, f.jpkp);
  const float face_w = (float)(1.0 / 3.0);  // STENCIL_FACE_WEIGHT rounded to float32
  const float edge_w = (float)(1.0 / 6.0);  // STENCIL_EDGE_WEIGHT rounded to float32
  return fadd(fadd(fmul(face_w, faces), fmul(edge_w, edges)), fmul(-4.0f, f.c));
}

// GOV-01: 2.0*P - P_prev + dt2*(lap - chi_sq*P)   (numpy_backend.py:108)
__device__ __forceinline__ float gov01(float p, float p_prev, float lap, float chi_sq,
                                       const StepConsts& s) {
  return fadd(fsub(fmul(2.0f, p), p_prev), fmul(s.dt2, fsub(lap, fmul(chi_sq, p))));
}

// chi_accel -= 4*lambda*chi*(chi^2 - chi0^2) when lambda > 0 (numpy_backend.py:113-114)
__device__ __forceinline__ float mexican_hat(float acc, float chi, float chi_sq,
                                             const StepConsts& s) {
  if (!s.use_lambda) return acc;
  return fsub(acc, fmul(fmul(s.four_lambda, chi), fsub(chi_sq, s.chi0_sq)));
}

// 2.0*chi - chi_prev + dt2*accel, clamp at -chi0, sponge blend
// mask*chi0 + (1-mask)*chi_new   (numpy_backend.py:115-124)
__device__ __forceinline__ float gov02_finish(float chi, float chi_prev, float acc, float mask,
                                              float absorb, const StepConsts& s) {
  float chi_new = fadd(fsub(fmul(2.0f, chi), chi_prev), fmul(s.dt2, acc));
  if (chi_new < s.neg_chi0) chi_new = s.neg_chi0;
  return fadd(fmul(mask, s.chi0), fmul(absorb, chi_new));
}

// One axis of the momentum current: Pr*(Pi[+] - Pi[-]) - Pi*(Pr[+] - Pr[-])
// (numpy_backend.py:174-182, with np.roll(-1) the + neighbour).
__device__ __forceinline__ float current_axis(float pr, float pi, float pr_p, float pr_m,
                                              float pi_p, float pi_m) {
  return fsub(fmul(pr, fsub(pi_p, pi_m)), fmul(pi, fsub(pr_p, pr_m)));
}

// Mask value from the radial lookup table (see lfm_mask_lut in lfm_b200.h).
struct MaskLut {
  const float* table;
  int32_t shift, q_lo, q_hi;
  int32_t count;  // entries in `table`
};

__device__ __forceinline__ float mask_from_q(const MaskLut& m, int32_t q) {
  if (q < m.q_lo) return 0.0f;
  if (q > m.q_hi) return 1.0f;
  return __ldg(m.table + ((q - m.q_lo) >> m.shift));
}

// Branch-free variant: the table load is predicated on the band test, so a
// warp does not diverge around it.
__device__ __forceinline__ float mask_from_q_flat(const MaskLut& m, int32_t q) {
  const bool in_band = (q >= m.q_lo) & (q <= m.q_hi);
  float t = 0.0f;
  if (in_band) t = __ldg(m.table + ((q - m.q_lo) >> m.shift));
  return in_band ? t : (q < m.q_lo ? 0.0f : 1.0f);
}

// Squared doubled offset from the lattice centre: (2x - N + 1)^2.
__device__ __forceinline__ int32_t qterm(int x, int N) {
  const int32_t d = 2 * x - N + 1;
  return d * d;
}

}  // namespace lfm
