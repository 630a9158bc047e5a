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
#include <cstring>
#include <cuda_runtime.h>

#include "lfm_b200.h"

namespace lfm {

__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }

// Two cells' values in one 64-bit register pair.  Additions and
// subtractions run as Blackwell's packed FADD2 (each lane rounded on its own,
// exactly as the scalar operation rounds it).  Multiplications stay two scalar
// __fmul_rn: a packed FMUL2 feeding a packed FADD2 was measured to come out
// fused (one rounding, about half of all results an ulp off), written with
// the __fmul2_rn intrinsic (also under -fmad=false) or as mul.rn.f32x2 PTX,
// while the scalar _rn operations are never contracted.
struct F2 {
  float2 v;
};
__device__ __forceinline__ F2 pk(float a, float b) { return F2{make_float2(a, b)}; }
__device__ __forceinline__ F2 fadd(F2 a, F2 b) { return F2{__fadd2_rn(a.v, b.v)}; }
#ifdef LFM_PACKED_MUL_FMA
// a*b as fma(a, b, -0): one rounding of the exact product (a -0 addend leaves
// every product, signed zeros included, unchanged).
__device__ __forceinline__ F2 fmul(F2 a, F2 b) {
  unsigned long long ra, rb, rd;
  const unsigned long long nz = 0x8000000080000000ull;
  memcpy(&ra, &a.v, 8);
  memcpy(&rb, &b.v, 8);
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(rd) : "l"(ra), "l"(rb), "l"(nz));
  F2 d;
  memcpy(&d.v, &rd, 8);
  return d;
}
#else
__device__ __forceinline__ F2 fmul(F2 a, F2 b) {
  return pk(__fmul_rn(a.v.x, b.v.x), __fmul_rn(a.v.y, b.v.y));
}
#endif
__device__ __forceinline__ F2 fsub(F2 a, F2 b) {
  unsigned long long ra, rb, rd;
  memcpy(&ra, &a.v, 8);
  memcpy(&rb, &b.v, 8);
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(rd) : "l"(ra), "l"(rb));
  F2 d;
  memcpy(&d.v, &rd, 8);
  return d;
}

// A product whose every consumer is a multiplication or a store, never an
// addition: then nothing can contract it, and two cells take one packed
// FMUL2.  (fmul above stays scalar because its products do feed additions.)
__device__ __forceinline__ float pmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ F2 pmul(F2 a, F2 b) {
  unsigned long long ra, rb, rd;
  memcpy(&ra, &a.v, 8);
  memcpy(&rb, &b.v, 8);
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(rd) : "l"(ra), "l"(rb));
  F2 d;
  memcpy(&d.v, &rd, 8);
  return d;
}

// A float constant as the value type T (broadcast to both lanes for F2).
template <class T>
__device__ __forceinline__ T cst(float a);
template <>
__device__ __forceinline__ float cst<float>(float a) { return a; }
template <>
__device__ __forceinline__ F2 cst<F2>(float a) { return pk(a, a); }

// x < lo ? lo : x per lane (a NaN stays NaN, as NumPy's boolean-mask clamp
// keeps it), as one max.NaN: for a number lo it returns lo below lo, x from
// lo up, and NaN for a NaN x.
__device__ __forceinline__ float clamp_below(float x, float lo) {
  float d;
  asm("max.NaN.f32 %0, %1, %2;" : "=f"(d) : "f"(x), "f"(lo));
  return d;
}
__device__ __forceinline__ F2 clamp_below(F2 x, float lo) {
  return pk(clamp_below(x.v.x, lo), clamp_below(x.v.y, lo));
}

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
  // The same parameters unrounded, for the split-chi steps, which evaluate
  // the accelerations in float64 (lfm_cells.cuh, "split chi").
  double dt2_d, k_over_chi0_d, four_lambda_d, chi0_d, chi0_sq_d, e0_sq_d, eps_w_d;
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
  c.dt2_d = dt2;
  c.k_over_chi0_d = kappa / chi0;
  c.four_lambda_d = 4.0 * lambda_self;
  c.chi0_d = chi0;
  c.chi0_sq_d = chi0 * chi0;
  c.e0_sq_d = e0_sq;
  c.eps_w_d = eps_w;
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

// The pointwise helpers below take T = float (one cell) or F2 (two cells,
// packed); both evaluate the same operations in the same order per cell.

// 2.0*x, as x + x: doubling is exact in binary floating point (x + x and
// 2*x give the same bits for every x, zeros, infinities and NaN included),
// and for two cells the addition is one packed FADD2.
template <class T>
__device__ __forceinline__ T twice(T x) {
  return fadd(x, x);
}

// GOV-01: 2.0*P - P_prev + dt2*(lap - chi_sq*P)   (numpy_backend.py:108)
template <class T>
__device__ __forceinline__ T gov01(T p, T p_prev, T lap, T chi_sq, const StepConsts& s) {
  return fadd(fsub(twice(p), p_prev), fmul(cst<T>(s.dt2), fsub(lap, fmul(chi_sq, p))));
}

// chi_accel -= 4*lambda*chi*(chi^2 - chi0^2) when lambda > 0 (numpy_backend.py:113-114)
template <class T>
__device__ __forceinline__ T mexican_hat(T acc, T chi, T chi_sq, const StepConsts& s) {
  if (!s.use_lambda) return acc;
  return fsub(acc, fmul(fmul(cst<T>(s.four_lambda), chi), fsub(chi_sq, cst<T>(s.chi0_sq))));
}

// 2.0*chi - chi_prev + dt2*accel, clamp at -chi0, sponge blend
// mask*chi0 + (1-mask)*chi_new   (numpy_backend.py:115-124)
template <class T>
__device__ __forceinline__ T gov02_finish(T chi, T chi_prev, T acc, T mask, T absorb,
                                          const StepConsts& s) {
  T chi_new = fadd(fsub(twice(chi), chi_prev), fmul(cst<T>(s.dt2), acc));
  chi_new = clamp_below(chi_new, s.neg_chi0);
  return fadd(fmul(mask, cst<T>(s.chi0)), fmul(absorb, chi_new));
}

// One axis of the momentum current: Pr*(Pi[+] - Pi[-]) - Pi*(Pr[+] - Pr[-])
// (numpy_backend.py:174-182, with np.roll(-1) the + neighbour).
template <class T>
__device__ __forceinline__ T current_axis(T pr, T pi, T pr_p, T pr_m, T pi_p, T pi_m) {
  return fsub(fmul(pr, fsub(pi_p, pi_m)), fmul(pi, fsub(pr_p, pr_m)));
}

// lap19 of two cells at once.  The neighbours in i and j sit at the same
// vector position as the cells, so those sums run packed; the k-neighbours
// (k-1, k+1) are the next cell over, so those adds run per lane.  The order
// of every cell's additions is the one lap19 uses.
__device__ __forceinline__ F2 lap19_pair(const S19& a, const S19& b) {
  F2 faces = fadd(pk(a.im, b.im), pk(a.ip, b.ip));
  faces = fadd(faces, pk(a.jm, b.jm));
  faces = fadd(faces, pk(a.jp, b.jp));
  float fa = fadd(faces.v.x, a.km), fb = fadd(faces.v.y, b.km);
  fa = fadd(fa, a.kp);
  fb = fadd(fb, b.kp);
  F2 edges = fadd(pk(a.imjm, b.imjm), pk(a.imjp, b.imjp));
  edges = fadd(edges, pk(a.ipjm, b.ipjm));
  edges = fadd(edges, pk(a.ipjp, b.ipjp));
  float ea = edges.v.x, eb = edges.v.y;
  ea = fadd(ea, a.imkm); eb = fadd(eb, b.imkm);
  ea = fadd(ea, a.imkp); eb = fadd(eb, b.imkp);
  ea = fadd(ea, a.ipkm); eb = fadd(eb, b.ipkm);
  ea = fadd(ea, a.ipkp); eb = fadd(eb, b.ipkp);
  ea = fadd(ea, a.jmkm); eb = fadd(eb, b.jmkm);
  ea = fadd(ea, a.jmkp); eb = fadd(eb, b.jmkp);
  ea = fadd(ea, a.jpkm); eb = fadd(eb, b.jpkm);
  ea = fadd(ea, a.jpkp); eb = fadd(eb, b.jpkp);
  const float face_w = (float)(1.0 / 3.0);
  const float edge_w = (float)(1.0 / 6.0);
  return fadd(fadd(fmul(cst<F2>(face_w), pk(fa, fb)), fmul(cst<F2>(edge_w), pk(ea, eb))),
              fmul(cst<F2>(-4.0f), pk(a.c, b.c)));
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
