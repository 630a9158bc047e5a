// CPU oracle for the lfm-physics leapfrog step.  TEST INFRASTRUCTURE ONLY.
//
// This file restates the reference's NumPy backend
// (lfm/core/backends/numpy_backend.py:80-382) and its 19-point Laplacian
// (lfm/core/stencils.py:26-71) as plain loops.  Only the tests, the smoke
// check and the CPU-baseline leg of the benchmark load it; the product
// path never does.
//
// The float32 instantiation reproduces NumPy's float32 arithmetic exactly:
//  * every Python float constant meets a float32 array as a "weak" scalar,
//    so it is rounded to float32 first (NumPy 2 / NEP 50).  Compound
//    constants such as kappa/chi0 are formed in double (Python float
//    arithmetic) and rounded once;
//  * each NumPy expression is evaluated as Python parses it, left to right,
//    one rounding per operation, with no fused multiply-add (build with
//    -ffp-contract=off);
//  * the colour variance f_c divides in float32 (NumPy chooses the ufunc
//    loop from the float32 inputs), then subtracts 1/3 in float64 because
//    the quotient lands in a float64 out array (numpy_backend.py:318-325).
// The float64 instantiation is the same algorithm carried out entirely in
// double: the FP64 oracle the error reports are measured against.
//
// The Helmholtz S_a solve (numpy_backend.py:341-356) needs an FFT and stays
// in NumPy (oracle/oracle.py); the colour step here takes the clipped S_a
// fields as an input.

#include <algorithm>
#include <cstdint>
#include <cmath>
#include <thread>
#include <vector>

namespace {

int g_threads = 1;
// Planes [g_i0, g_i1) of the slowest axis are stepped (default: all).  The
// CPU baseline uses this to time a bounded slab of a large lattice.
int g_i0 = 0, g_i1 = -1;

// Runs body(i) for i in [0, n) on g_threads std::threads, split into
// contiguous slabs of the slowest axis.
template <typename F>
void parallel_for(int n, F body) {
  const int a = std::max(0, std::min(g_i0, n));
  const int b = (g_i1 < 0) ? n : std::max(a, std::min(g_i1, n));
  const int m = b - a;
  const int t = std::max(1, std::min(g_threads, m));
  if (t == 1) {
    for (int i = a; i < b; ++i) body(i);
    return;
  }
  std::vector<std::thread> pool;
  pool.reserve(t);
  for (int w = 0; w < t; ++w) {
    const int lo = a + (int)((int64_t)m * w / t), hi = a + (int)((int64_t)m * (w + 1) / t);
    pool.emplace_back([=, &body] { for (int i = lo; i < hi; ++i) body(i); });
  }
  for (auto& th : pool) th.join();
}

template <typename T>
struct Consts {
  T dt2, two, half, third, face_w, edge_w, center_w;
  T k_over_chi0, four_lambda, chi0_sq, chi0, neg_chi0, e0_sq, eps_w;
  T kc_over_chi0, dt2_eps_cc, kappa_string, kappa_tube, ncolors;
  bool use_lambda;
  double one_third_d;
};

// Python-float constants rounded to T as NumPy rounds a weak scalar.
template <typename T>
Consts<T> make_consts(double dt2, double kappa, double lambda_self, double chi0,
                      double e0_sq, double eps_w, double kappa_c, double eps_cc,
                      double kappa_string, double kappa_tube) {
  Consts<T> c;
  c.dt2 = (T)dt2;
  c.two = (T)2.0;
  c.half = (T)0.5;
  c.third = (T)(1.0 / 3.0);
  c.face_w = (T)(1.0 / 3.0);   // STENCIL_FACE_WEIGHT (lfm/constants.py:135)
  c.edge_w = (T)(1.0 / 6.0);   // STENCIL_EDGE_WEIGHT (lfm/constants.py:138)
  c.center_w = (T)(-4.0);      // STENCIL_CENTER_WEIGHT (lfm/constants.py:141)
  c.k_over_chi0 = (T)(kappa / chi0);
  c.four_lambda = (T)(4.0 * lambda_self);
  c.chi0_sq = (T)(chi0 * chi0);
  c.chi0 = (T)chi0;
  c.neg_chi0 = (T)(-chi0);
  c.e0_sq = (T)e0_sq;
  c.eps_w = (T)eps_w;
  c.kc_over_chi0 = (T)(kappa_c / chi0);
  c.dt2_eps_cc = (T)(dt2 * eps_cc);
  c.kappa_string = (T)kappa_string;
  c.kappa_tube = (T)kappa_tube;
  c.ncolors = (T)3.0;
  c.use_lambda = lambda_self > 0.0;
  c.one_third_d = 1.0 / 3.0;
  return c;
}

struct Nbr {
  int64_t c, im, ip, jm, jp, km, kp;
  int64_t imjm, imjp, ipjm, ipjp, imkm, imkp, ipkm, ipkp, jmkm, jmkp, jpkm, jpkp;
};

// Periodic neighbour offsets of cell (i, j, k) in C order, idx = (i*N + j)*N + k.
inline Nbr neighbours(int i, int j, int k, int N) {
  const int64_t n = N;
  const int64_t I[3] = {(i + N - 1) % N, i, (i + 1) % N};
  const int64_t J[3] = {(j + N - 1) % N, j, (j + 1) % N};
  const int64_t K[3] = {(k + N - 1) % N, k, (k + 1) % N};
  auto at = [&](int a, int b, int d) { return (I[a] * n + J[b]) * n + K[d]; };
  Nbr r;
  r.c = at(1, 1, 1);
  r.im = at(0, 1, 1); r.ip = at(2, 1, 1);
  r.jm = at(1, 0, 1); r.jp = at(1, 2, 1);
  r.km = at(1, 1, 0); r.kp = at(1, 1, 2);
  r.imjm = at(0, 0, 1); r.imjp = at(0, 2, 1); r.ipjm = at(2, 0, 1); r.ipjp = at(2, 2, 1);
  r.imkm = at(0, 1, 0); r.imkp = at(0, 1, 2); r.ipkm = at(2, 1, 0); r.ipkp = at(2, 1, 2);
  r.jmkm = at(1, 0, 0); r.jmkp = at(1, 0, 2); r.jpkm = at(1, 2, 0); r.jpkp = at(1, 2, 2);
  return r;
}

// laplacian_19pt (stencils.py:43-71): np.roll(f, 1, axis) is f[x-1].
template <typename T>
inline T lap19(const T* f, const Nbr& n, const Consts<T>& c) {
  T faces = f[n.im] + f[n.ip];
  faces = faces + f[n.jm];
  faces = faces + f[n.jp];
  faces = faces + f[n.km];
  faces = faces + f[n.kp];
  T edges = f[n.imjm] + f[n.imjp];
  edges = edges + f[n.ipjm];
  edges = edges + f[n.ipjp];
  edges = edges + f[n.imkm];
  edges = edges + f[n.imkp];
  edges = edges + f[n.ipkm];
  edges = edges + f[n.ipkp];
  edges = edges + f[n.jmkm];
  edges = edges + f[n.jmkp];
  edges = edges + f[n.jpkm];
  edges = edges + f[n.jpkp];
  T a = c.face_w * faces;
  T b = c.edge_w * edges;
  T s = a + b;
  T d = c.center_w * f[n.c];
  return s + d;
}

// GOV-02 tail shared by all levels: clamp at -chi0 (numpy_backend.py:118),
// then the sponge blend (numpy_backend.py:122-124).
template <typename T>
inline T chi_finish(T chi_new, T mask, T absorb, const Consts<T>& c) {
  if (chi_new < c.neg_chi0) chi_new = c.neg_chi0;
  T a = mask * c.chi0;
  T b = absorb * chi_new;
  return a + b;
}

template <typename T>
inline T mexican_hat(T chi_accel, T chi, T chi_sq, const Consts<T>& c) {
  if (!c.use_lambda) return chi_accel;
  T t = c.four_lambda * chi;
  T u = chi_sq - c.chi0_sq;
  return chi_accel - t * u;
}

// GOV-01 update: 2.0*P - P_prev + dt2*(lap - chi_sq*P).
template <typename T>
inline T gov01(T p, T p_prev, T lap, T chi_sq, const Consts<T>& c) {
  T a = c.two * p;
  T b = a - p_prev;
  T m = chi_sq * p;
  T d = lap - m;
  T e = c.dt2 * d;
  return b + e;
}

template <typename T>
void step_real(const T* E, const T* Ep, const T* chi, const T* chip, const T* mask,
               T* E_out, T* Ep_out, T* chi_out, T* chip_out, int N, const Consts<T>& c) {
  parallel_for(N, [&](int i) {
    for (int j = 0; j < N; ++j)
      for (int k = 0; k < N; ++k) {
        const Nbr n = neighbours(i, j, k, N);
        const int64_t x = n.c;
        T lapE = lap19(E, n, c);
        T lapC = lap19(chi, n, c);
        T ch = chi[x];
        T chi_sq = ch * ch;
        T e = E[x];
        T E_new = gov01(e, Ep[x], lapE, chi_sq, c);
        // chi_source = (kappa/chi0)*chi*(E*E - e0_sq)   (numpy_backend.py:111)
        T s1 = c.k_over_chi0 * ch;
        T s2 = e * e;
        T s3 = s2 - c.e0_sq;
        T src = s1 * s3;
        T acc = lapC - src;
        acc = mexican_hat(acc, ch, chi_sq, c);
        T a2 = c.two * ch;
        T b2 = a2 - chip[x];
        T e2 = c.dt2 * acc;
        T chi_new = b2 + e2;
        T m = mask[x];
        T absorb = (T)1.0 - m;
        E_out[x] = E_new * absorb;
        Ep_out[x] = e * absorb;
        chi_out[x] = chi_finish(chi_new, m, absorb, c);
        chip_out[x] = ch;
      }
  });
}

// Central-difference current along one axis: P_r*(P_i[+]-P_i[-]) - P_i*(P_r[+]-P_r[-]).
template <typename T>
inline T current(const T* Pr, const T* Pi, int64_t x, int64_t plus, int64_t minus) {
  T dPi = Pi[plus] - Pi[minus];
  T dPr = Pr[plus] - Pr[minus];
  T a = Pr[x] * dPi;
  T b = Pi[x] * dPr;
  return a - b;
}

template <typename T>
void step_complex(const T* Pr, const T* Prp, const T* Pi, const T* Pip, const T* chi,
                  const T* chip, const T* mask, T* Pr_out, T* Prp_out, T* Pi_out,
                  T* Pip_out, T* chi_out, T* chip_out, int N, const Consts<T>& c) {
  parallel_for(N, [&](int i) {
    for (int j = 0; j < N; ++j)
      for (int k = 0; k < N; ++k) {
        const Nbr n = neighbours(i, j, k, N);
        const int64_t x = n.c;
        T ch = chi[x];
        T chi_sq = ch * ch;
        T lapR = lap19(Pr, n, c);
        T lapI = lap19(Pi, n, c);
        T lapC = lap19(chi, n, c);
        T pr = Pr[x], pi = Pi[x];
        T Pr_new = gov01(pr, Prp[x], lapR, chi_sq, c);
        T Pi_new = gov01(pi, Pip[x], lapI, chi_sq, c);
        T psi_sq = pr * pr + pi * pi;  // two products, then one sum
        T jx = current(Pr, Pi, x, n.ip, n.im);
        T jy = current(Pr, Pi, x, n.jp, n.jm);
        T jz = current(Pr, Pi, x, n.kp, n.km);
        T jsum = jx + jy;
        jsum = jsum + jz;
        T jt = c.half * jsum;
        // (kappa/chi0)*chi*(psi_sq + eps_w*j - e0_sq)   (numpy_backend.py:186)
        T s1 = c.k_over_chi0 * ch;
        T w = c.eps_w * jt;
        T s2 = psi_sq + w;
        T s3 = s2 - c.e0_sq;
        T src = s1 * s3;
        T acc = lapC - src;
        acc = mexican_hat(acc, ch, chi_sq, c);
        T chi_new = (c.two * ch - chip[x]) + c.dt2 * acc;
        T m = mask[x];
        T absorb = (T)1.0 - m;
        Pr_out[x] = Pr_new * absorb;
        Pi_out[x] = Pi_new * absorb;
        Prp_out[x] = pr * absorb;
        Pip_out[x] = pi * absorb;
        chi_out[x] = chi_finish(chi_new, m, absorb, c);
        chip_out[x] = ch;
      }
  });
}

// step_color (numpy_backend.py:207-382), three colours, [colour][i][j][k] layout.
// sa: the clipped S_a fields (3*N^3) or nullptr when the SCV term is off.
template <typename T>
void step_color(const T* Pr, const T* Prp, const T* Pi, const T* Pip, const T* chi,
                const T* chip, const T* mask, T* Pr_out, T* Prp_out, T* Pi_out,
                T* Pip_out, T* chi_out, T* chip_out, int N, const Consts<T>& c,
                double kappa_c, double eps_cc, double kappa_string, const T* sa) {
  const int64_t total = (int64_t)N * N * N;
  const bool use_cc = eps_cc > 0.0;
  const bool use_fc = kappa_c > 0.0;
  const bool use_ccv = kappa_string > 0.0;
  parallel_for(N, [&](int i) {
    for (int j = 0; j < N; ++j)
      for (int k = 0; k < N; ++k) {
        const Nbr n = neighbours(i, j, k, N);
        const int64_t x = n.c;
        T ch = chi[x];
        T chi_sq = ch * ch;
        T pr_avg = (T)0, pi_avg = (T)0;
        if (use_cc) {
          for (int a = 0; a < 3; ++a) {
            pr_avg = pr_avg + Pr[a * total + x];
            pi_avg = pi_avg + Pi[a * total + x];
          }
          pr_avg = pr_avg / c.ncolors;  // Pr_avg /= n_colors
          pi_avg = pi_avg / c.ncolors;
        }
        T psi_sq_total = (T)0, j_total = (T)0;
        T ea[3], jd[3][3];
        T m = mask[x];
        T absorb = (T)1.0 - m;
        for (int a = 0; a < 3; ++a) {
          const T* R = Pr + a * total;
          const T* I = Pi + a * total;
          T pr = R[x], pi = I[x];
          T lapR = lap19(R, n, c);
          T lapI = lap19(I, n, c);
          T Pr_new = gov01(pr, Prp[a * total + x], lapR, chi_sq, c);
          T Pi_new = gov01(pi, Pip[a * total + x], lapI, chi_sq, c);
          if (use_cc) {  // Pr_new -= dt2*eps_cc*chi_sq*(Pr - Pr_avg)
            T t = c.dt2_eps_cc * chi_sq;
            Pr_new = Pr_new - t * (pr - pr_avg);
            Pi_new = Pi_new - t * (pi - pi_avg);
          }
          Pr_out[a * total + x] = Pr_new * absorb;
          Pi_out[a * total + x] = Pi_new * absorb;
          Prp_out[a * total + x] = pr * absorb;
          Pip_out[a * total + x] = pi * absorb;
          T e = pr * pr + pi * pi;
          ea[a] = e;
          psi_sq_total = psi_sq_total + e;
          T jx = current(R, I, x, n.ip, n.im);
          T jy = current(R, I, x, n.jp, n.jm);
          T jz = current(R, I, x, n.kp, n.km);
          T js = jx + jy;
          js = js + jz;
          j_total = j_total + c.half * js;
          jd[a][0] = jx; jd[a][1] = jy; jd[a][2] = jz;
        }
        T color_var = (T)0;
        if (use_fc) {
          // sum over colours of e_a^2 in colour order; ratio in float64.
          T ssq = ea[0] * ea[0] + ea[1] * ea[1];
          ssq = ssq + ea[2] * ea[2];
          T tsq = psi_sq_total * psi_sq_total;
          bool safe = tsq > (T)1e-30;
          // np.divide picks its float32 loop from the inputs; the float64
          // out array only receives the rounded quotient.
          double ratio = safe ? (double)(T)(ssq / tsq) : 0.0;
          double fc_d = (ratio - c.one_third_d) * (safe ? 1.0 : 0.0);
          T fc = (T)fc_d;
          T t1 = c.kc_over_chi0 * ch;
          T t2 = t1 * fc;
          color_var = t2 * psi_sq_total;
        }
        T ccv = (T)0;
        if (use_ccv) {
          for (int d = 0; d < 3; ++d) {
            T sq = jd[0][d] * jd[0][d] + jd[1][d] * jd[1][d];
            sq = sq + jd[2][d] * jd[2][d];
            T s = jd[0][d] + jd[1][d];
            s = s + jd[2][d];
            T s2 = s * s;
            ccv = ccv + (sq - c.third * s2);
          }
        }
        T scv = (T)0;
        if (sa) {
          T ssum = (T)0, ssq = (T)0;
          for (int a = 0; a < 3; ++a) {
            T v = sa[a * total + x];
            ssum = ssum + v;
            ssq = ssq + v * v;
          }
          T s2 = ssum * ssum;
          scv = ssq - c.third * s2;
        }
        T lapC = lap19(chi, n, c);
        T s1 = c.k_over_chi0 * ch;
        T w = c.eps_w * j_total;
        T s2 = psi_sq_total + w;
        T s3 = s2 - c.e0_sq;
        T src = s1 * s3;
        T acc = lapC - src;
        acc = acc - color_var;
        acc = acc - c.kappa_string * ccv;
        acc = acc - c.kappa_tube * scv;
        acc = mexican_hat(acc, ch, chi_sq, c);
        T chi_new = (c.two * ch - chip[x]) + c.dt2 * acc;
        chi_out[x] = chi_finish(chi_new, m, absorb, c);
        chip_out[x] = ch;
      }
  });
}

}  // namespace

extern "C" {

void oracle_set_threads(int n) { g_threads = n > 0 ? n : 1; }
void oracle_set_plane_range(int i0, int i1) {
  g_i0 = i0;
  g_i1 = i1;
}
int oracle_max_threads(void) {
  unsigned h = std::thread::hardware_concurrency();
  return h ? (int)h : 1;
}

#define ORACLE_LAPLACIAN(T, NAME)                                                         \
  void NAME(const T* f, T* out, int N) {                                                  \
    auto c = make_consts<T>(0, 0, 0, 1, 0, 0, 0, 0, 0, 0);                                 \
    parallel_for(N, [&](int i) {                                                          \
      for (int j = 0; j < N; ++j)                                                         \
        for (int k = 0; k < N; ++k) {                                                     \
          const Nbr n = neighbours(i, j, k, N);                                           \
          out[n.c] = lap19(f, n, c);                                                      \
        }                                                                                 \
    });                                                                                   \
  }
ORACLE_LAPLACIAN(float, oracle_laplacian_f32)
ORACLE_LAPLACIAN(double, oracle_laplacian_f64)

#define ORACLE_REAL(T, NAME)                                                              \
  void NAME(const T* E, const T* Ep, const T* chi, const T* chip, const T* mask, T* Eo,    \
            T* Epo, T* co, T* cpo, int N, double dt2, double kappa, double lambda_self,    \
            double chi0, double e0_sq) {                                                  \
    auto c = make_consts<T>(dt2, kappa, lambda_self, chi0, e0_sq, 0, 0, 0, 0, 0);          \
    step_real<T>(E, Ep, chi, chip, mask, Eo, Epo, co, cpo, N, c);                          \
  }
ORACLE_REAL(float, oracle_step_real_f32)
ORACLE_REAL(double, oracle_step_real_f64)

#define ORACLE_COMPLEX(T, NAME)                                                           \
  void NAME(const T* Pr, const T* Prp, const T* Pi, const T* Pip, const T* chi,            \
            const T* chip, const T* mask, T* Pro, T* Prpo, T* Pio, T* Pipo, T* co, T* cpo, \
            int N, double dt2, double kappa, double lambda_self, double chi0,             \
            double e0_sq, double eps_w) {                                                 \
    auto c = make_consts<T>(dt2, kappa, lambda_self, chi0, e0_sq, eps_w, 0, 0, 0, 0);      \
    step_complex<T>(Pr, Prp, Pi, Pip, chi, chip, mask, Pro, Prpo, Pio, Pipo, co, cpo, N, c); \
  }
ORACLE_COMPLEX(float, oracle_step_complex_f32)
ORACLE_COMPLEX(double, oracle_step_complex_f64)

#define ORACLE_COLOR(T, NAME)                                                             \
  void NAME(const T* Pr, const T* Prp, const T* Pi, const T* Pip, const T* chi,            \
            const T* chip, const T* mask, T* Pro, T* Prpo, T* Pio, T* Pipo, T* co, T* cpo, \
            int N, double dt2, double kappa, double lambda_self, double chi0,             \
            double e0_sq, double eps_w, double kappa_c, double eps_cc,                    \
            double kappa_string, double kappa_tube, const T* sa) {                        \
    auto c = make_consts<T>(dt2, kappa, lambda_self, chi0, e0_sq, eps_w, kappa_c, eps_cc, \
                            kappa_string, kappa_tube);                                    \
    step_color<T>(Pr, Prp, Pi, Pip, chi, chip, mask, Pro, Prpo, Pio, Pipo, co, cpo, N, c,  \
                  kappa_c, eps_cc, kappa_string, sa);                                     \
  }
ORACLE_COLOR(float, oracle_step_color_f32)
ORACLE_COLOR(double, oracle_step_color_f64)

}  // extern "C"
