// Per-cell updates of the three field levels, built from lfm_math.cuh.
//
// A kernel gathers the stencil values of a cell (S19) and the previous-step
// values, then calls one of these.  The order of operations follows
// lfm/core/backends/numpy_backend.py:80-382 line by line, so results are
// bit-identical to the reference's NumPy float32 path.
#pragma once

#include "lfm_math.cuh"

namespace lfm {

// ---- REAL (numpy_backend.py:80-130) ---------------------------------------
// T = float for one cell, F2 for two cells packed (same operations per cell).
template <class T>
struct RealOutT {
  T psi, psi_prev, chi, chi_prev;
};
using RealOut = RealOutT<float>;

// absorb = 1 - mask, passed in by kernels that also damp the stored
// previous field with it (one subtraction per cell instead of two).
template <class T>
__device__ __forceinline__ RealOutT<T> real_cell_ab(T lapE, T e, T e_prev, T lapX, T chi,
                                                    T chi_prev, T mask, T absorb,
                                                    const StepConsts& s) {
  const T chi_sq = fmul(chi, chi);
  const T E_new = gov01(e, e_prev, lapE, chi_sq, s);
  // chi_source = (kappa/chi0)*chi*(E*E - e0_sq)
  const T src = fmul(pmul(cst<T>(s.k_over_chi0), chi), fsub(fmul(e, e), cst<T>(s.e0_sq)));
  T acc = fsub(lapX, src);
  acc = mexican_hat(acc, chi, chi_sq, s);
  RealOutT<T> o;
  o.psi = pmul(E_new, absorb);  // stored
  o.psi_prev = pmul(e, absorb);
  o.chi = gov02_finish(chi, chi_prev, acc, mask, absorb, s);
  o.chi_prev = chi;
  return o;
}

template <class T>
__device__ __forceinline__ RealOutT<T> real_cell(T lapE, T e, T e_prev, T lapX, T chi,
                                                 T chi_prev, T mask, const StepConsts& s) {
  return real_cell_ab(lapE, e, e_prev, lapX, chi, chi_prev, mask, fsub(cst<T>(1.0f), mask), s);
}

// ---- COMPLEX (numpy_backend.py:132-205) -----------------------------------
template <class T>
struct ComplexOutT {
  T pr, pr_prev, pi, pi_prev, chi, chi_prev;
};
using ComplexOut = ComplexOutT<float>;

// Face neighbours of one field, for the momentum current.
template <class T>
struct FacesT {
  T im, ip, jm, jp, km, kp;
};
using Faces = FacesT<float>;

__device__ __forceinline__ FacesT<F2> pk_faces(const Faces& a, const Faces& b) {
  FacesT<F2> f;
  f.im = pk(a.im, b.im); f.ip = pk(a.ip, b.ip);
  f.jm = pk(a.jm, b.jm); f.jp = pk(a.jp, b.jp);
  f.km = pk(a.km, b.km); f.kp = pk(a.kp, b.kp);
  return f;
}

template <class T>
__device__ __forceinline__ T momentum_current(T pr, T pi, const FacesT<T>& R,
                                              const FacesT<T>& I) {
  const T jx = current_axis(pr, pi, R.ip, R.im, I.ip, I.im);
  const T jy = current_axis(pr, pi, R.jp, R.jm, I.jp, I.jm);
  const T jz = current_axis(pr, pi, R.kp, R.km, I.kp, I.km);
  return pmul(cst<T>(0.5f), fadd(fadd(jx, jy), jz));  // j_total = 0.5*(j_x + j_y + j_z)
}

template <class T>
__device__ __forceinline__ ComplexOutT<T> complex_cell_ab(T lapR, T pr, T pr_prev,
                                                          const FacesT<T>& R, T lapI, T pi,
                                                          T pi_prev, const FacesT<T>& I, T lapX,
                                                          T chi, T chi_prev, T mask, T absorb,
                                                          const StepConsts& s) {
  const T chi_sq = fmul(chi, chi);
  const T Pr_new = gov01(pr, pr_prev, lapR, chi_sq, s);
  const T Pi_new = gov01(pi, pi_prev, lapI, chi_sq, s);
  const T psi_sq = fadd(fmul(pr, pr), fmul(pi, pi));
  const T jt = momentum_current(pr, pi, R, I);
  // (kappa/chi0)*chi*(psi_sq + eps_w*j - e0_sq)
  const T src = fmul(pmul(cst<T>(s.k_over_chi0), chi),
                     fsub(fadd(psi_sq, fmul(cst<T>(s.eps_w), jt)), cst<T>(s.e0_sq)));
  T acc = fsub(lapX, src);
  acc = mexican_hat(acc, chi, chi_sq, s);
  ComplexOutT<T> o;
  o.pr = pmul(Pr_new, absorb);  // stored
  o.pi = pmul(Pi_new, absorb);
  o.pr_prev = pmul(pr, absorb);
  o.pi_prev = pmul(pi, absorb);
  o.chi = gov02_finish(chi, chi_prev, acc, mask, absorb, s);
  o.chi_prev = chi;
  return o;
}

template <class T>
__device__ __forceinline__ ComplexOutT<T> complex_cell(T lapR, T pr, T pr_prev,
                                                       const FacesT<T>& R, T lapI, T pi,
                                                       T pi_prev, const FacesT<T>& I, T lapX,
                                                       T chi, T chi_prev, T mask,
                                                       const StepConsts& s) {
  return complex_cell_ab(lapR, pr, pr_prev, R, lapI, pi, pi_prev, I, lapX, chi, chi_prev, mask,
                         fsub(cst<T>(1.0f), mask), s);
}

// ---- COLOR (numpy_backend.py:207-382), three colours ----------------------
// The colour step is split so a kernel can stream one colour at a time:
// color_begin -> color_component (a = 0, 1, 2) -> color_finish.  T = float
// for one cell or F2 for two cells packed; the operations that have no
// packed form (the division by 3, the float64 step of f_c, the S_a clip)
// run per lane.
template <class T>
struct ColorAccT {
  T chi, chi_sq, mask, absorb;
  T pr_avg, pi_avg;
  T psi_sq_total, j_total;
  T ea[3];
  T jd[3][3];  // per colour, per axis current (for CCV)
};
using ColorAcc = ColorAccT<float>;

__device__ __forceinline__ float div3(float x) { return __fdiv_rn(x, 3.0f); }
__device__ __forceinline__ F2 div3(F2 x) { return pk(div3(x.v.x), div3(x.v.y)); }

// np.clip(sa, 0, None) as the kernels have always evaluated it
__device__ __forceinline__ float clip0(float x) { return fmaxf(x, 0.0f); }
__device__ __forceinline__ F2 clip0(F2 x) { return pk(clip0(x.v.x), clip0(x.v.y)); }

// f_c = sum_sq / total_sq - 1/3 where total_sq > 1e-30, else 0: a float32
// quotient, then "- 1/3" in float64 (the float64 out array of np.divide),
// rounded back to float32.
__device__ __forceinline__ float fc_value(float ssq, float tsq) {
  const bool safe = tsq > (float)1e-30;
  const double ratio = safe ? (double)__fdiv_rn(ssq, tsq) : 0.0;
  return __double2float_rn(__dmul_rn(__dsub_rn(ratio, 1.0 / 3.0), safe ? 1.0 : 0.0));
}
__device__ __forceinline__ F2 fc_value(F2 ssq, F2 tsq) {
  return pk(fc_value(ssq.v.x, tsq.v.x), fc_value(ssq.v.y, tsq.v.y));
}

template <class T>
__device__ __forceinline__ void color_begin(ColorAccT<T>& A, T chi, T mask, const T pr_c[3],
                                            const T pi_c[3], const StepConsts& s) {
  A.chi = chi;
  A.chi_sq = fmul(chi, chi);
  A.mask = mask;
  A.absorb = fsub(cst<T>(1.0f), mask);
  A.pr_avg = cst<T>(0.0f);
  A.pi_avg = cst<T>(0.0f);
  if (s.use_cc) {  // Pr_avg = (0 + Pr_0 + Pr_1 + Pr_2) / 3   (numpy_backend.py:254-262)
    T r = cst<T>(0.0f), i = cst<T>(0.0f);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      r = fadd(r, pr_c[a]);
      i = fadd(i, pi_c[a]);
    }
    A.pr_avg = div3(r);
    A.pi_avg = div3(i);
  }
  A.psi_sq_total = cst<T>(0.0f);
  A.j_total = cst<T>(0.0f);
}

template <class T>
struct ColorCompOutT {
  T pr, pr_prev, pi, pi_prev;
};
using ColorCompOut = ColorCompOutT<float>;

// numpy_backend.py:268-310 for colour a.
template <class T>
__device__ __forceinline__ ColorCompOutT<T> color_component(ColorAccT<T>& A, int a, T lapR, T pr,
                                                            T pr_prev, const FacesT<T>& R, T lapI,
                                                            T pi, T pi_prev, const FacesT<T>& I,
                                                            const StepConsts& s) {
  T Pr_new = gov01(pr, pr_prev, lapR, A.chi_sq, s);
  T Pi_new = gov01(pi, pi_prev, lapI, A.chi_sq, s);
  if (s.use_cc) {  // -= dt2*eps_cc*chi^2*(Psi_a - Psi_bar)
    const T t = pmul(cst<T>(s.dt2_eps_cc), A.chi_sq);  // feeds only the products below
    Pr_new = fsub(Pr_new, fmul(t, fsub(pr, A.pr_avg)));
    Pi_new = fsub(Pi_new, fmul(t, fsub(pi, A.pi_avg)));
  }
  const T e = fadd(fmul(pr, pr), fmul(pi, pi));
  A.ea[a] = e;
  A.psi_sq_total = fadd(A.psi_sq_total, e);
  const T jx = current_axis(pr, pi, R.ip, R.im, I.ip, I.im);
  const T jy = current_axis(pr, pi, R.jp, R.jm, I.jp, I.jm);
  const T jz = current_axis(pr, pi, R.kp, R.km, I.kp, I.km);
  A.j_total = fadd(A.j_total, fmul(cst<T>(0.5f), fadd(fadd(jx, jy), jz)));
  A.jd[a][0] = jx;
  A.jd[a][1] = jy;
  A.jd[a][2] = jz;
  ColorCompOutT<T> o;  // stored values only
  o.pr = pmul(Pr_new, A.absorb);
  o.pi = pmul(Pi_new, A.absorb);
  o.pr_prev = pmul(pr, A.absorb);
  o.pi_prev = pmul(pi, A.absorb);
  return o;
}

// f_c, CCV, SCV and GOV-02 (numpy_backend.py:312-370).  sa_raw holds the
// unclipped S_a values of the cell (clipped here) or is ignored when
// has_sa is false.  Returns the new chi.
template <class T>
__device__ __forceinline__ T color_finish(const ColorAccT<T>& A, T lapX, T chi_prev, bool has_sa,
                                          const T sa_raw[3], const StepConsts& s) {
  const float third = (float)(1.0 / 3.0);
  T color_var = cst<T>(0.0f);
  if (s.use_fc) {
    T ssq = fadd(fmul(A.ea[0], A.ea[0]), fmul(A.ea[1], A.ea[1]));
    ssq = fadd(ssq, fmul(A.ea[2], A.ea[2]));
    const T tsq = pmul(A.psi_sq_total, A.psi_sq_total);  // feeds only the comparison and quotient
    const T fc = fc_value(ssq, tsq);
    color_var = fmul(pmul(pmul(cst<T>(s.kc_over_chi0), A.chi), fc), A.psi_sq_total);
  }
  T ccv = cst<T>(0.0f);
  if (s.use_ccv) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      T sq = fadd(fmul(A.jd[0][d], A.jd[0][d]), fmul(A.jd[1][d], A.jd[1][d]));
      sq = fadd(sq, fmul(A.jd[2][d], A.jd[2][d]));
      T sm = fadd(A.jd[0][d], A.jd[1][d]);
      sm = fadd(sm, A.jd[2][d]);
      ccv = fadd(ccv, fsub(sq, fmul(cst<T>(third), pmul(sm, sm))));
    }
  }
  T scv = cst<T>(0.0f);
  if (has_sa) {
    T ssum = cst<T>(0.0f), ssq = cst<T>(0.0f);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const T v = clip0(sa_raw[a]);
      ssum = fadd(ssum, v);
      ssq = fadd(ssq, fmul(v, v));
    }
    scv = fsub(ssq, fmul(cst<T>(third), pmul(ssum, ssum)));
  }
  const T src = fmul(pmul(cst<T>(s.k_over_chi0), A.chi),
                     fsub(fadd(A.psi_sq_total, fmul(cst<T>(s.eps_w), A.j_total)), cst<T>(s.e0_sq)));
  T acc = fsub(lapX, src);
  acc = fsub(acc, color_var);
  acc = fsub(acc, fmul(cst<T>(s.kappa_string), ccv));
  acc = fsub(acc, fmul(cst<T>(s.kappa_tube), scv));
  acc = mexican_hat(acc, A.chi, A.chi_sq, s);
  return gov02_finish(A.chi, chi_prev, acc, A.mask, A.absorb, s);
}

}  // namespace lfm

// ---- compensated float32 (Delta form) ----------------------------------------
//
// State per field: the value P and the increment D = P - P_prev, where
// P_prev is the previous value as the reference stores it ((1-mask)*P for
// Psi, undamped for chi).  The leapfrog with the sponge becomes
//   Psi:  D' = (1-m)(D + dt2*acc),          Psi' = Psi - m*Psi + D'
//   chi:  r  = D + dt2*acc  (clamped so that chi + r >= -chi0),
//         D' = r + m*(chi0 - chi - r),      chi' = chi + D'
// which is the reference update in exact arithmetic.  The new value is
// formed with error-free transformations (two-sum, FMA two-product); its
// rounding error is added to the stored increment, so the bits lost when
// the small increment meets the large value come back in the next step
// (compensated summation).  FMA is used freely: this path is measured
// against the float64 oracle, not against the float32 reference bits.
namespace lfm {

// Rounding error of s = a + b (Knuth's two-sum): a + b == s + err exactly.
__device__ __forceinline__ float two_sum_err(float a, float b, float s) {
  const float bb = __fsub_rn(s, a);
  return __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}

// FMA-form Laplacian (same neighbours; sums then two fused weightings).
__device__ __forceinline__ float lap19_fma(const S19& f) {
  float faces = f.im + f.ip;
  faces += f.jm;
  faces += f.jp;
  faces += f.km;
  faces += f.kp;
  float edges = f.imjm + f.imjp;
  edges += f.ipjm;
  edges += f.ipjp;
  edges += f.imkm;
  edges += f.imkp;
  edges += f.ipkm;
  edges += f.ipkp;
  edges += f.jmkm;
  edges += f.jmkp;
  edges += f.jpkm;
  edges += f.jpkp;
  return fmaf((float)(1.0 / 3.0), faces, fmaf((float)(1.0 / 6.0), edges, -4.0f * f.c));
}

// Laplacian as weighted sums of neighbour - centre differences: the same
// value in exact arithmetic (the weights sum to 4), but each difference of
// two nearby values is exact in float32 (Sterbenz), so a smooth field keeps
// its full precision -- chi ~ 19 loses nothing to the large neighbour sums.
__device__ __forceinline__ float lap19_diff(const S19& f) {
  const float c = f.c;
  float faces = (f.im - c) + (f.ip - c);
  faces += (f.jm - c) + (f.jp - c);
  faces += (f.km - c) + (f.kp - c);
  float edges = (f.imjm - c) + (f.imjp - c);
  edges += (f.ipjm - c) + (f.ipjp - c);
  edges += (f.imkm - c) + (f.imkp - c);
  edges += (f.ipkm - c) + (f.ipkp - c);
  edges += (f.jmkm - c) + (f.jmkp - c);
  edges += (f.jpkm - c) + (f.jpkp - c);
  return fmaf((float)(1.0 / 3.0), faces, (float)(1.0 / 6.0) * edges);
}

// lap - chi^2 * p with the rounding errors of chi^2 and of the product folded
// back in (FMA two-products): the mass term is the largest one in GOV-01.
__device__ __forceinline__ float accel_mass(float lap, float chi, float p) {
  const float sq = __fmul_rn(chi, chi);
  const float e_sq = fmaf(chi, chi, -sq);  // chi^2 == sq + e_sq
  const float q = __fmul_rn(sq, p);
  const float e_q = fmaf(sq, p, -q);       // sq*p == q + e_q
  return (lap - q) - fmaf(e_sq, p, e_q);
}

struct CompVal {
  float v, d;  // new value, new stored increment
};

// Psi update with the sponge: D' = (1-m)t, t = D + dt2*acc; Psi' = Psi - m*Psi + D'.
__device__ __forceinline__ CompVal comp_psi(float psi, float d, float acc, float m,
                                            const StepConsts& s) {
  // The operations inside the error-free transformations are pinned with
  // _rn intrinsics so that the compiler cannot fuse them.
  const float t = fmaf(s.dt2, acc, d);
  const float dn = fmaf(-m, t, t);            // (1-m)*t, one rounding
  const float p = __fmul_rn(m, psi);
  const float ep = fmaf(m, psi, -p);          // m*psi == p + ep
  const float inc = __fsub_rn(dn, p);
  const float e2 = two_sum_err(dn, -p, inc);  // dn - p == inc + e2
  const float v = __fadd_rn(psi, inc);
  const float e3 = two_sum_err(psi, inc, v);  // psi + inc == v + e3
  CompVal o;
  o.v = v;
  o.d = dn + ((e3 + e2) - ep);                // Psi'_exact - v folded into D'
  return o;
}

// chi update: clamp at -chi0 and the sponge blend m*chi0 + (1-m)*chi_raw in
// increment form.
__device__ __forceinline__ CompVal comp_chi(float chi, float d, float acc, float m,
                                            const StepConsts& s) {
  float r = fmaf(s.dt2, acc, d);
  if (chi + r < s.neg_chi0) r = s.neg_chi0 - chi;
  const float inc = fmaf(m, (s.chi0 - chi) - r, r);
  const float v = __fadd_rn(chi, inc);
  CompVal o;
  o.v = v;
  o.d = inc + two_sum_err(chi, inc, v);
  return o;
}

__device__ __forceinline__ float comp_mexican_hat(float acc, float chi, float chi_sq,
                                                  const StepConsts& s) {
  if (!s.use_lambda) return acc;
  return fmaf(-s.four_lambda * chi, chi_sq - s.chi0_sq, acc);
}

struct RealComp {
  CompVal psi, chi;
};

__device__ __forceinline__ RealComp real_cell_comp(float lapE, float e, float de, float lapX,
                                                   float chi, float dchi, float mask,
                                                   const StepConsts& s) {
  const float chi_sq = chi * chi;
  const float accE = accel_mass(lapE, chi, e);
  const float src = s.k_over_chi0 * chi * fmaf(e, e, -s.e0_sq);
  float accX = lapX - src;
  accX = comp_mexican_hat(accX, chi, chi_sq, s);
  RealComp o;
  o.psi = comp_psi(e, de, accE, mask, s);
  o.chi = comp_chi(chi, dchi, accX, mask, s);
  return o;
}

struct ComplexComp {
  CompVal pr, pi, chi;
};

__device__ __forceinline__ ComplexComp complex_cell_comp(float lapR, float pr, float dr,
                                                         const Faces& R, float lapI, float pi,
                                                         float di, const Faces& I, float lapX,
                                                         float chi, float dchi, float mask,
                                                         const StepConsts& s) {
  const float chi_sq = chi * chi;
  const float accR = accel_mass(lapR, chi, pr);
  const float accI = accel_mass(lapI, chi, pi);
  const float psi_sq = fmaf(pr, pr, pi * pi);
  const float jx = pr * (I.ip - I.im) - pi * (R.ip - R.im);
  const float jy = pr * (I.jp - I.jm) - pi * (R.jp - R.jm);
  const float jz = pr * (I.kp - I.km) - pi * (R.kp - R.km);
  const float jt = 0.5f * (jx + jy + jz);
  const float src = s.k_over_chi0 * chi * (fmaf(s.eps_w, jt, psi_sq) - s.e0_sq);
  float accX = lapX - src;
  accX = comp_mexican_hat(accX, chi, chi_sq, s);
  ComplexComp o;
  o.pr = comp_psi(pr, dr, accR, mask, s);
  o.pi = comp_psi(pi, di, accI, mask, s);
  o.chi = comp_chi(chi, dchi, accX, mask, s);
  return o;
}

}  // namespace lfm

// ---- split chi (two-float offset from chi0) -----------------------------------
//
// chi is held as chi0 + hi + lo with hi, lo float32 and lo the part of the
// offset below one ulp of hi (about 48 significant bits in all).  Psi stays
// one float32 per value.  Float32 storage of chi itself is what limits the
// plain path's accuracy against float64: chi ~ 19 keeps only ~2e-6 of
// absolute precision, its per-step increments are rounded away, and Psi's
// frequency follows chi.  Here the chi update and every acceleration term that
// involves chi run in float64; the Laplacians stay float32, and the offset's
// is that of hi alone, by neighbour-minus-centre differences (exact for nearby
// values).  lo is below half an ulp of hi, so its 19-point Laplacian moves the
// offset by at most about dt2 * 12 ulp(hi) per step: 0.005 ulp at dt = 0.02.
// An emulation of the 64^3 REAL workload over 1000 steps against float64 gave
// max-relative errors E 3.5e-6, chi 4.5e-8 without it and 4.0e-6, 6.8e-8 with
// it, so lo is a point field of the step.  The update is the reference's
// (numpy_backend.py:80-205) in exact arithmetic:
//   Psi' = (1-m)(2 Psi - Psi_prev + dt2 (lap Psi - chi^2 Psi))
//   d'   = (1-m) max(2 d - d_prev + dt2 acc_chi, -2 chi0),   d = chi - chi0
// (the sponge blend m chi0 + (1-m) chi_new and the clamp chi >= -chi0 in
// offset form).  Every operation is an explicit _rn intrinsic, so the fused
// and the direct kernels give the same bits.
namespace lfm {

__device__ __forceinline__ double split_value(float hi, float lo) {
  return __dadd_rn((double)hi, (double)lo);
}


// One Psi component: the acceleration lap - chi^2 p in float64, rounded once,
// then p_new = dt2 * acc + (2p - p_prev) in float32 (not yet absorbed).
__device__ __forceinline__ float split_psi(float lap, float p, float p_prev, double chi_sq,
                                           const StepConsts& s) {
  const float acc = __double2float_rn(__fma_rn(-chi_sq, (double)p, (double)lap));
  return __fmaf_rn(s.dt2, acc, __fmaf_rn(2.0f, p, -p_prev));
}

struct SplitChi {
  float hi, lo;
};

// chi offset update in float64 from its acceleration; split back into two floats.
__device__ __forceinline__ SplitChi split_chi(double d, double d_prev, double acc, float mask,
                                              const StepConsts& s) {
  double dn = __fma_rn(s.dt2_d, acc, __dsub_rn(__dadd_rn(d, d), d_prev));
  const double lim = -2.0 * s.chi0_d;
  dn = dn < lim ? lim : dn;  // chi >= -chi0; a NaN stays NaN
  dn = __dmul_rn(__dsub_rn(1.0, (double)mask), dn);
  SplitChi o;
  o.hi = __double2float_rn(dn);
  o.lo = __double2float_rn(__dsub_rn(dn, (double)o.hi));
  return o;
}

// Mexican-hat term of the chi acceleration, float64.
__device__ __forceinline__ double split_hat(double acc, double chi, double chi_sq,
                                            const StepConsts& s) {
  if (!s.use_lambda) return acc;
  return __fma_rn(-__dmul_rn(s.four_lambda_d, chi), __dsub_rn(chi_sq, s.chi0_sq_d), acc);
}

struct RealSplit {
  float psi;  // new E, absorbed (stored)
  SplitChi chi;
};

// REAL: lapE = lap19_fma(E), lapD = lap19_diff(H); e_prev as the reference
// reads it (absorbed); d, d_prev the chi offsets (split_value).
__device__ __forceinline__ RealSplit real_cell_split(float lapE, float e, float e_prev, float lapD,
                                                     double d, double d_prev, float mask,
                                                     float absorb, const StepConsts& s) {
  const double chi = __dadd_rn(s.chi0_d, d);
  const double chi_sq = __dmul_rn(chi, chi);
  const float e_new = split_psi(lapE, e, e_prev, chi_sq, s);
  const double ed = (double)e;
  const double src =
      __dmul_rn(__dmul_rn(s.k_over_chi0_d, chi), __fma_rn(ed, ed, -s.e0_sq_d));
  const double acc = split_hat(__dsub_rn((double)lapD, src), chi, chi_sq, s);
  RealSplit o;
  o.psi = __fmul_rn(e_new, absorb);
  o.chi = split_chi(d, d_prev, acc, mask, s);
  return o;
}

struct ComplexSplit {
  float pr, pi;  // absorbed (stored)
  SplitChi chi;
};

// COMPLEX: the momentum current from float32 neighbour differences (exact for
// nearby values), its products and sums in float64.
__device__ __forceinline__ ComplexSplit complex_cell_split(float lapR, float pr, float pr_prev,
                                                           const Faces& R, float lapI, float pi,
                                                           float pi_prev, const Faces& I,
                                                           float lapD, double d, double d_prev,
                                                           float mask, float absorb,
                                                           const StepConsts& s) {
  const double chi = __dadd_rn(s.chi0_d, d);
  const double chi_sq = __dmul_rn(chi, chi);
  const float r_new = split_psi(lapR, pr, pr_prev, chi_sq, s);
  const float i_new = split_psi(lapI, pi, pi_prev, chi_sq, s);
  const double prd = (double)pr, pid = (double)pi;
  const double psi_sq = __fma_rn(prd, prd, __dmul_rn(pid, pid));
  auto axis = [&](float rp, float rm, float ip, float im) {
    return __fma_rn(prd, (double)__fsub_rn(ip, im), -__dmul_rn(pid, (double)__fsub_rn(rp, rm)));
  };
  const double jt = __dmul_rn(0.5, __dadd_rn(__dadd_rn(axis(R.ip, R.im, I.ip, I.im),
                                                       axis(R.jp, R.jm, I.jp, I.jm)),
                                             axis(R.kp, R.km, I.kp, I.km)));
  const double q = __dsub_rn(__fma_rn(s.eps_w_d, jt, psi_sq), s.e0_sq_d);
  const double src = __dmul_rn(__dmul_rn(s.k_over_chi0_d, chi), q);
  const double acc = split_hat(__dsub_rn((double)lapD, src), chi, chi_sq, s);
  ComplexSplit o;
  o.pr = __fmul_rn(r_new, absorb);
  o.pi = __fmul_rn(i_new, absorb);
  o.chi = split_chi(d, d_prev, acc, mask, s);
  return o;
}

}  // namespace lfm
