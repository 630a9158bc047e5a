/*
 * lfm_b200.h -- C ABI of the B200 (sm_100a) leapfrog library liblfm_b200.so.
 *
 * One call advances one lattice by one leapfrog step of GOV-01 (Psi) and
 * GOV-02 (chi) over the periodic 19-point Laplacian, with the cos^2 sponge,
 * the chi >= -chi0 clamp and, at the COLOR level, the cross-colour, f_c,
 * CCV and SCV terms.  All pointers are device pointers unless a parameter
 * name ends in _host.  Arrays are flat float32 in C order,
 * idx = (i*N + j)*N + k; colour arrays are [colour][i][j][k] with 3 colours.
 * Every entry point returns 0 (LFM_OK) or an LFM_ERR_* code; lfm_strerror()
 * names it and lfm_last_error_detail() gives the message of the calling
 * thread's last failure.  Launches are asynchronous on `stream` (a
 * cudaStream_t passed as void*; NULL = legacy default stream).
 *
 * Scalar parameters are the reference's Python floats (double).  They are
 * rounded to float32 inside the library exactly as NumPy rounds a Python
 * float meeting a float32 array, so the plain float32 steps reproduce the
 * reference's NumPy float32 path bit for bit.
 */
#ifndef LFM_B200_H
#define LFM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LFM_B200_ABI_VERSION 1

enum lfm_status {
  LFM_OK = 0,
  LFM_ERR_INVALID_ARG = 1,   /* bad size, null pointer, overlapping buffers */
  LFM_ERR_ALIGNMENT = 2,     /* a device pointer is not 16-byte aligned */
  LFM_ERR_UNSUPPORTED = 3,   /* combination this build does not provide */
  LFM_ERR_CUDA = 4,          /* a CUDA runtime call failed */
  LFM_ERR_CUFFT = 5,         /* a cuFFT call failed */
  LFM_ERR_MASK = 6,          /* mask is not a function of the radial key q */
  LFM_ERR_DEVICE_TIMEOUT = 7,/* a bounded device-side wait gave up */
  LFM_ERR_NONFINITE = 8,     /* a reduction met NaN/Inf */
  LFM_ERR_CAPACITY = 9       /* output table or scratch too small */
};

/* Field levels, as lfm.config.FieldLevel (lfm/config.py:36-46). */
enum lfm_level { LFM_REAL = 0, LFM_COMPLEX = 1, LFM_COLOR = 2 };

const char* lfm_strerror(int status);
const char* lfm_last_error_detail(void);
int lfm_abi_version(void);

/* ------------------------------------------------------------------------
 * Sponge mask lookup table.
 *
 * The reference's mask (lfm/core/backends/numpy_backend.py:49-69) is a pure
 * function of the integer key q = (2i-N+1)^2 + (2j-N+1)^2 + (2k-N+1)^2
 * (4*R^2 in the reference's float32 coordinates, exact for N <= 2048).
 * lfm_mask_lut_build scans the host copy of the N^3 mask and stores, for the
 * band q_lo <= q <= q_hi where the mask is neither 0 nor 1, one float32 per
 * key step of 2^shift.  The step kernels then read 4 bytes per cell from an
 * L1-resident table instead of streaming the N^3 mask.  The values are the
 * host mask's own float32 values, so the table is bit-exact.  Returns
 * LFM_ERR_MASK if two cells with the same q hold different values.
 * ------------------------------------------------------------------------ */
typedef struct lfm_mask_lut {
  int32_t N;      /* lattice edge */
  int32_t shift;  /* table index = (q - q_lo) >> shift; 3 for even N, 2 for odd N */
  int32_t q_lo;   /* q < q_lo: mask 0 */
  int32_t q_hi;   /* q > q_hi: mask 1 */
  int32_t count;  /* table entries used */
} lfm_mask_lut;

int lfm_mask_lut_build(int N, const float* mask_host, float* table_host, int capacity,
                       lfm_mask_lut* out);

/* ------------------------------------------------------------------------
 * Protocol steps: the reference Backend's step_* calls, one for one.
 *
 * Replace lfm/core/backends/cupy_backend.py:127-169 (step_real),
 * :171-222 (step_complex) and :224-317 (step_color), whose kernels are
 * evolve_real / evolve_complex / evolve_gov01_gov02 in
 * lfm/core/backends/kernel_source.py:323-419, :424-540, :18-235.  Inputs
 * and outputs are separate buffers (the reference's A/B double buffer):
 * psi_out = damped new field, psi_prev_out = damped current field,
 * chi_out = new chi, chi_prev_out = current chi.  boundary_mask is the
 * device copy of the N^3 mask.
 * ------------------------------------------------------------------------ */
int lfm_step_real_f32(const float* psi_in, const float* psi_prev_in, const float* chi_in,
                      const float* chi_prev_in, const float* boundary_mask, float* psi_out,
                      float* psi_prev_out, float* chi_out, float* chi_prev_out, int N,
                      double dt2, double kappa, double lambda_self, double chi0,
                      double e0_sq, void* stream);

int lfm_step_complex_f32(const float* psi_r_in, const float* psi_r_prev_in,
                         const float* psi_i_in, const float* psi_i_prev_in,
                         const float* chi_in, const float* chi_prev_in,
                         const float* boundary_mask, float* psi_r_out, float* psi_r_prev_out,
                         float* psi_i_out, float* psi_i_prev_out, float* chi_out,
                         float* chi_prev_out, int N, double dt2, double kappa,
                         double lambda_self, double chi0, double e0_sq, double epsilon_w,
                         void* stream);

/* sa_fields_out (3*N^3, may be NULL) receives the clipped S_a fields when
 * kappa_tube > 0, as numpy_backend.py:341-356; sa_fields_in is accepted for
 * signature parity and, like the reference, not read when kappa_tube > 0.
 * The S_a solve needs cuFFT plans and spectrum scratch, held in `ctx`
 * (see lfm_context_create); ctx may be NULL when kappa_tube == 0. */
typedef struct lfm_context lfm_context;

int lfm_step_color_f32(lfm_context* ctx, const float* psi_r_in, const float* psi_r_prev_in,
                       const float* psi_i_in, const float* psi_i_prev_in,
                       const float* chi_in, const float* chi_prev_in,
                       const float* boundary_mask, float* psi_r_out, float* psi_r_prev_out,
                       float* psi_i_out, float* psi_i_prev_out, float* chi_out,
                       float* chi_prev_out, int N, double dt2, double kappa,
                       double lambda_self, double chi0, double e0_sq, double epsilon_w,
                       double kappa_c, double epsilon_cc, double kappa_string,
                       double kappa_tube, const float* sa_fields_in, float* sa_fields_out,
                       double sa_gamma, double sa_d, double dt, void* stream);

/* ------------------------------------------------------------------------
 * Library context: cuFFT plans and spectrum scratch for the S_a solve,
 * keyed by lattice edge, on the device that is current at creation.
 * Replaces the per-step plan/filter rebuild of cupy_backend.py:261-279.
 * ------------------------------------------------------------------------ */
int lfm_context_create(lfm_context** out);
int lfm_context_destroy(lfm_context* ctx);

/* ------------------------------------------------------------------------
 * Resident-lattice steps (the fast path behind lfm_b200.Evolver).
 *
 * Same arithmetic as the protocol steps, but each field keeps two slots and
 * the step writes the new values into the slot that held the previous ones:
 * psi_prev_io is read at each cell and then overwritten with the new psi,
 * chi_prev_io likewise with the new chi.  The caller then swaps the roles of
 * the slots.  Because the reference stores psi_prev' = (1-mask)*psi, a slot
 * that was written by the previous call holds the undamped field; pass
 * damp_prev = 1 to apply (1-mask) on read (the same single float32 product,
 * so the result is unchanged bit for bit), or 0 when the host wrote the
 * previous field itself.  chi's previous field is never damped.
 * The mask comes from the lookup table (table = device copy of the table
 * built by lfm_mask_lut_build).  Moves 24 B/cell (REAL), 36 B (COMPLEX).
 * ------------------------------------------------------------------------ */
int lfm_leapfrog_real_f32(const float* psi, float* psi_prev_io, const float* chi,
                          float* chi_prev_io, const float* mask_table,
                          const lfm_mask_lut* lut, int damp_prev, int N, double dt2,
                          double kappa, double lambda_self, double chi0, double e0_sq,
                          void* stream);

int lfm_leapfrog_complex_f32(const float* psi_r, float* psi_r_prev_io, const float* psi_i,
                             float* psi_i_prev_io, const float* chi, float* chi_prev_io,
                             const float* mask_table, const lfm_mask_lut* lut, int damp_prev,
                             int N, double dt2, double kappa, double lambda_self,
                             double chi0, double e0_sq, double epsilon_w, void* stream);

/* sa: raw (unclipped) S_a fields from lfm_helmholtz_sa_f32 of this step's
 * psi, or NULL when kappa_tube == 0; the kernel clips them at 0 on read. */
int lfm_leapfrog_color_f32(const float* psi_r, float* psi_r_prev_io, const float* psi_i,
                           float* psi_i_prev_io, const float* chi, float* chi_prev_io,
                           const float* mask_table, const lfm_mask_lut* lut, int damp_prev,
                           int N, double dt2, double kappa, double lambda_self, double chi0,
                           double e0_sq, double epsilon_w, double kappa_c, double epsilon_cc,
                           double kappa_string, double kappa_tube, const float* sa,
                           void* stream);

/* lfm_leapfrog_color_f32 that also writes |Psi_a|^2 = Pr_a^2 + Pi_a^2 of the
 * new fields (as stored) to energy_out (3 N^3 floats, distinct from every
 * other buffer; NULL: not written), in the step kernel's epilogue.  The next
 * step's S_a solve then starts from it (lfm_helmholtz_sa_from_energy_f32)
 * instead of reading all six Psi arrays again: the same bits as the
 * |Psi_a|^2 lfm_helmholtz_sa_f32 forms (numpy_backend.py:289). */
int lfm_leapfrog_color_energy_f32(const float* psi_r, float* psi_r_prev_io, const float* psi_i,
                                  float* psi_i_prev_io, const float* chi, float* chi_prev_io,
                                  const float* mask_table, const lfm_mask_lut* lut,
                                  int damp_prev, int N, double dt2, double kappa,
                                  double lambda_self, double chi0, double e0_sq,
                                  double epsilon_w, double kappa_c, double epsilon_cc,
                                  double kappa_string, double kappa_tube, const float* sa,
                                  float* energy_out, void* stream);

/* ------------------------------------------------------------------------
 * Compensated float32 steps (Delta form).  No counterpart kernel in the
 * reference; they advance the same equations as lfm_leapfrog_real_f32 /
 * _complex_f32 (numpy_backend.py:80-205) with more accuracy.
 *
 * State per field: the value (psi, chi) and the increment
 * d = value - previous value as the reference stores it ((1-mask)*psi_prev
 * for Psi, chi_prev for chi).  A step reads the values (stencil) and the
 * increments, writes the new values to *_next (distinct buffers) and the
 * new increments over the old ones.  The new value's rounding error is
 * folded into its increment (two-sum), so the sub-ulp part of each update is
 * carried forward instead of lost.  Moves 32 B/cell (REAL), 48 B (COMPLEX).
 * ------------------------------------------------------------------------ */
int lfm_leapfrog_real_comp_f32(const float* psi, float* psi_next, float* dpsi_io,
                               const float* chi, float* chi_next, float* dchi_io,
                               const float* mask_table, const lfm_mask_lut* lut, int N,
                               double dt2, double kappa, double lambda_self, double chi0,
                               double e0_sq, void* stream);

int lfm_leapfrog_complex_comp_f32(const float* psi_r, float* psi_r_next, float* dpsi_r_io,
                                  const float* psi_i, float* psi_i_next, float* dpsi_i_io,
                                  const float* chi, float* chi_next, float* dchi_io,
                                  const float* mask_table, const lfm_mask_lut* lut, int N,
                                  double dt2, double kappa, double lambda_self, double chi0,
                                  double e0_sq, double epsilon_w, void* stream);

/* ------------------------------------------------------------------------
 * Split-chi steps.  No counterpart kernel in the reference; they advance the
 * equations of lfm_leapfrog_real_f32 / _complex_f32 (numpy_backend.py:80-205)
 * close to float64 accuracy.
 *
 * chi is held as chi0 + hi + lo, two float32 slots per time level (hi, and lo
 * the part below one ulp of hi); Psi as in the plain resident step.  The chi
 * update and every acceleration term involving chi run in float64, the
 * Laplacians in float32 (chi's is hi's, from neighbour differences; lo enters
 * the step at the cell only).  The slots rotate
 * as in lfm_leapfrog_real_f32: each call reads (cur, prev) of every field and
 * writes the new values over prev; damp_prev as there (Psi's previous slot is
 * multiplied by (1 - mask) on read).  chi's previous slots are undamped.
 * Moves 36 B/cell (REAL), 48 B (COMPLEX).  Lattices with N % 4 != 0 take the
 * direct kernel, with the same results.
 * ------------------------------------------------------------------------ */
int lfm_leapfrog_real_split_f32(const float* psi, float* psi_prev_io, const float* chi_hi,
                                float* chi_hi_prev_io, const float* chi_lo, float* chi_lo_prev_io,
                                const float* mask_table, const lfm_mask_lut* lut, int damp_prev,
                                int N, double dt2, double kappa, double lambda_self, double chi0,
                                double e0_sq, void* stream);

int lfm_leapfrog_complex_split_f32(const float* psi_r, float* psi_r_prev_io, const float* psi_i,
                                   float* psi_i_prev_io, const float* chi_hi,
                                   float* chi_hi_prev_io, const float* chi_lo,
                                   float* chi_lo_prev_io, const float* mask_table,
                                   const lfm_mask_lut* lut, int damp_prev, int N, double dt2,
                                   double kappa, double lambda_self, double chi0, double e0_sq,
                                   double epsilon_w, void* stream);

/* One split-chi step out of place, as lfm_advance_f32 for the plain step: reads
 * (cur, prev) of every field, writes the new state to the *_out buffers (the
 * adjoint's recomputed segments).  damp_prev as in the resident call. */
int lfm_advance_split_f32(int level, const float* psi_r, const float* psi_r_prev,
                          float* psi_r_out, const float* psi_i, const float* psi_i_prev,
                          float* psi_i_out, const float* chi_hi, const float* chi_hi_prev,
                          float* chi_hi_out, const float* chi_lo, const float* chi_lo_prev,
                          float* chi_lo_out, const float* mask_table, const lfm_mask_lut* lut,
                          int damp_prev, int N, double dt2, double kappa, double lambda_self,
                          double chi0, double e0_sq, double epsilon_w, void* stream);

/* ------------------------------------------------------------------------
 * Poisson equilibration of chi (lfm/fields/equilibrium.py:26-121, as
 * Simulation.equilibrate calls it, lfm/simulation.py:877-963):
 * chi = chi0 + dchi with  laplacian(dchi) = kappa (|Psi|^2 - e0_sq)  solved
 * by FFT on the periodic lattice (DC of dchi = 0); with frozen != 0, chi0 on
 * the shell dist > N/2 (1 - boundary_fraction) (~interior_mask).  |Psi|^2
 * sums psi_r^2 (+ psi_i^2), over three colours at the COLOR level (3 N^3
 * inputs); psi_i may be NULL at the REAL level.  The forward transform is a
 * float32 cuFFT R2C, the -1/k^2 divide and the inverse are float64 (as NumPy
 * evaluates them), so chi agrees with the reference to a float32 ulp or two.
 * cuFFT plans and scratch live in ctx.
 * ------------------------------------------------------------------------ */
int lfm_poisson_chi_f32(lfm_context* ctx, int level, const float* psi_r, const float* psi_i,
                        int N, double chi0, double kappa, double e0_sq,
                        double boundary_fraction, int frozen, float* chi_out, void* stream);

/* ------------------------------------------------------------------------
 * One slab of a lattice split along i across GPUs (the natural sharding of a
 * single large lattice; the reference steps the whole lattice on one device,
 * lfm/core/backends/numpy_backend.py:80-205).  Level LFM_REAL or LFM_COMPLEX.
 * Every array holds n_local + 2 planes of N x N: plane 0 and plane
 * n_local + 1 are ghost copies of global planes i_first - 1 and
 * i_first + n_local (mod N), planes 1 .. n_local are global planes
 * i_first .. i_first + n_local - 1.  The step is the resident step of
 * lfm_leapfrog_*_f32 restricted to planes 1 .. n_local: it reads the ghost
 * planes of psi / chi as they are and writes the new fields over the
 * previous ones.  The caller refreshes the ghost planes of the new fields
 * (from the neighbouring slabs) before the next step.  The results are the
 * whole-lattice step's bits on those planes.  psi_i* are ignored (may be
 * NULL) at the REAL level.
 * ------------------------------------------------------------------------ */
int lfm_slab_step_f32(int level, const float* psi_r, float* psi_r_prev_io, const float* psi_i,
                      float* psi_i_prev_io, const float* chi, float* chi_prev_io,
                      const float* mask_table, const lfm_mask_lut* lut, int damp_prev, int N,
                      int n_local, int i_first, double dt2, double kappa, double lambda_self,
                      double chi0, double e0_sq, double epsilon_w, void* stream);

/* The slab step restricted to the slab's planes [plane_lo, plane_hi), 1 <=
 * plane_lo < plane_hi <= n_local + 1 (lfm_slab_step_f32 is the range
 * [1, n_local + 1)).  It lets a caller step the two boundary planes first,
 * start their exchange with the neighbouring slabs, and step the interior
 * planes while the exchange is in flight: the interior reads no ghost plane
 * and writes none, and the new boundary planes are final once their range has
 * run.  Each plane's bits are those of the whole-lattice step. */
int lfm_slab_step_planes_f32(int level, const float* psi_r, float* psi_r_prev_io,
                             const float* psi_i, float* psi_i_prev_io, const float* chi,
                             float* chi_prev_io, const float* mask_table, const lfm_mask_lut* lut,
                             int damp_prev, int N, int n_local, int i_first, int plane_lo,
                             int plane_hi, double dt2, double kappa, double lambda_self,
                             double chi0, double e0_sq, double epsilon_w, void* stream);

/* Out-of-place form of lfm_leapfrog_real_f32 / lfm_leapfrog_complex_f32
 * (level LFM_REAL or LFM_COMPLEX): the same step and the same bits, with the
 * new fields written to *_out instead of over the previous ones, which stay
 * read-only.  The outputs must not overlap any input.  psi_i* are ignored
 * (may be NULL) at the REAL level. */
int lfm_advance_f32(int level, const float* psi_r, const float* psi_r_prev, float* psi_r_out,
                    const float* psi_i, const float* psi_i_prev, float* psi_i_out,
                    const float* chi, const float* chi_prev, float* chi_out,
                    const float* mask_table, const lfm_mask_lut* lut, int damp_prev, int N,
                    double dt2, double kappa, double lambda_self, double chi0, double e0_sq,
                    double epsilon_w, void* stream);

/* ------------------------------------------------------------------------
 * Adjoint (reverse-mode) step, REAL and COMPLEX.  New: the reference has no
 * adjoint; this differentiates its step (lfm/core/backends/numpy_backend.py:
 * 80-205) as written, in the reference representation of the state (A/B
 * buffers, P_prev' = (1-mask) P).  Inputs: the state the step read (psi_r,
 * psi_i, chi), chi after the step (chi_next, for the clamp at -chi0) and
 * g_out[6], the adjoints of the step's outputs in the order (psi_r,
 * psi_r_prev, psi_i, psi_i_prev, chi, chi_prev).  Writes g_in[6], the
 * adjoints of its inputs in the same order (entries 2 and 3 unused, may be
 * NULL, at the REAL level).  g_in must not overlap any input.  float32
 * arithmetic; kappa etc. as in lfm_leapfrog_*_f32.
 * ------------------------------------------------------------------------ */
int lfm_adjoint_step_f32(int level, const float* psi_r, const float* psi_i, const float* chi,
                         const float* chi_next, const float* mask_table, const lfm_mask_lut* lut,
                         const float* const* g_out, float* const* g_in, int N, double dt2,
                         double kappa, double lambda_self, double chi0, double e0_sq,
                         double epsilon_w, void* stream);

/* ------------------------------------------------------------------------
 * Batches of independent lattices (the runs lfm/sweep.py:14-157 makes one
 * Simulation at a time), stepped together: one launch per step, persistent
 * CTAs taking (lattice, row tile, plane chunk) items from a work list sorted
 * by cost (all REAL items, then all COMPLEX ones), each item marched like the
 * fused single-lattice kernel.  REAL and
 * COMPLEX lattices, N a multiple of 4, any mix of sizes and parameters.  Each
 * lattice keeps two slots per field in the resident layout of
 * lfm_leapfrog_*_f32: at parity p, slot p holds the current fields and slot
 * 1-p the previous ones, which the step overwrites with the new fields.
 * damp_prev as in lfm_leapfrog_*_f32.  Results are bit-identical to stepping
 * each lattice alone.  The batch owns two device counters, so launches of one
 * batch must be ordered (one stream).
 * ------------------------------------------------------------------------ */
typedef struct lfm_lattice_desc {
  int32_t N;
  int32_t level;          /* LFM_REAL or LFM_COMPLEX */
  float* psi_r[2];        /* slots of Psi (real part) */
  float* psi_i[2];        /* slots of the imaginary part; NULL at the REAL level */
  float* chi[2];          /* slots of chi */
  const float* mask_table;
  lfm_mask_lut lut;
  double dt2, kappa, lambda_self, chi0, e0_sq, epsilon_w;
} lfm_lattice_desc;

typedef struct lfm_batch_tuning {
  int32_t threads;      /* cap on the CTA size (multiple of 32, <= 512); 0 = 256 */
  int32_t stages;       /* shared-memory stages, 3..6; 0 = 5 */
  int32_t item_cells;   /* target cells per work item; 0 = 131072 */
  int32_t ctas_per_sm;  /* persistent CTAs per SM; 0 = as many as fit */
} lfm_batch_tuning;

typedef struct lfm_batch lfm_batch;

/* Plans the work lists and uploads the descriptors (device memory owned by
 * the batch).  tuning may be NULL.  The buffers stay owned by the caller. */
int lfm_batch_create(const lfm_lattice_desc* lattices, int count,
                     const lfm_batch_tuning* tuning, lfm_batch** out);
/* One step of every lattice (one kernel launch). */
int lfm_batch_step(lfm_batch* batch, int parity, int damp_prev, void* stream);
/* Launch shape: work items, CTA size, persistent CTAs, dynamic shared memory. */
int lfm_batch_info(const lfm_batch* batch, int* items, int* threads, int* grid, int* smem);
int lfm_batch_destroy(lfm_batch* batch);
/* The plan lfm_batch_create would make, on the host only (no device needed;
 * 128 registers per thread and `sms` SMs assumed, 148 when sms <= 0).
 * items_out: 6 int32 per item (level, lattice, j0, j1, i0, i1) in the order
 * CTAs take them (grouped by lattice shape, the REAL shapes first, largest
 * items first within a shape); launch_out: (threads, smem, grid).
 * Either may be NULL;
 * nitems_out gets the item count. */
int lfm_batch_plan(const lfm_lattice_desc* lattices, int count, const lfm_batch_tuning* tuning,
                   int sms, int32_t* items_out, int max_items, int* nitems_out,
                   int32_t* launch_out);

/* ------------------------------------------------------------------------
 * S_a Helmholtz solve (numpy_backend.py:341-356, cupy_backend.py:261-279):
 * sa_raw[a] = IRFFT[ gamma/(gamma + D|k|^2) * RFFT(|Psi_a|^2) ] for a = 0..2,
 * k = 2*pi*fftfreq(N), computed in float32.  N in {64, 128, 256, 512, 1024}:
 * cuFFT 2-D R2C over (j, k) per plane, one hand-written pass along i (forward
 * FFT, the filter with 1/N^3 folded in, inverse FFT), cuFFT 2-D C2R; other N:
 * cuFFT 3-D R2C, a hand-written k-space multiply, 3-D C2R
 * (lfm_set_sa_transform).  sa_raw is NOT clipped; consumers clip at 0
 * (lfm_sa_clip_f32 for a host-visible copy).
 * ------------------------------------------------------------------------ */
int lfm_helmholtz_sa_f32(lfm_context* ctx, const float* psi_r, const float* psi_i,
                         float* sa_raw, int N, double sa_gamma, double sa_d, void* stream);
int lfm_sa_clip_f32(const float* sa_raw, float* sa_out, int64_t count, void* stream);

/* The S_a solve of lfm_helmholtz_sa_f32 from |Psi_a|^2 already at hand
 * (energy: 3 N^3 floats, e.g. from lfm_leapfrog_color_energy_f32), skipping
 * the pass that forms it from psi_r and psi_i.  The energy array is consumed:
 * its contents are undefined afterwards. */
int lfm_helmholtz_sa_from_energy_f32(lfm_context* ctx, const float* energy, float* sa_raw,
                                     int N, double sa_gamma, double sa_d, void* stream);

/* ------------------------------------------------------------------------
 * Float64 metrics of a state, reduced on the device (replaces the host
 * compute_metrics of lfm/analysis/metrics.py:29-111 except the cluster
 * count; energy terms as lfm/analysis/energy.py:26-113 with np.gradient's
 * non-periodic edges; chi statistics over interior_mask,
 * lfm/analysis/structure.py:148-171).  psi_*_prev may be NULL (kinetic 0);
 * psi_i* are NULL at the REAL level; colour arrays hold 3 components.
 * out_host[LFM_METRICS_COUNT] receives, in order: energy_kinetic,
 * energy_gradient, energy_potential, energy_total, chi_min, chi_max,
 * chi_mean, chi_std, well_fraction, void_fraction, psi_sq_total,
 * interior_cells, nonfinite_cells.  Synchronises `stream`.  Scratch for the
 * per-CTA partials lives in `ctx`.
 * ------------------------------------------------------------------------ */
#define LFM_METRICS_COUNT 13
int lfm_metrics_f64(lfm_context* ctx, int level, const float* psi_r, const float* psi_r_prev,
                    const float* psi_i, const float* psi_i_prev, const float* chi, int N,
                    double dt, double c, double boundary_fraction, double well_threshold,
                    double void_threshold, double* out_host, void* stream);

/* The metrics of lfm_metrics_f64 without any device allocation.  No
 * counterpart in the reference.  For callers that cannot call cudaMalloc --
 * a process whose device memory is held by another allocator (a caching
 * allocator such as PyTorch's can keep the free memory to itself), or a
 * program that must not allocate after start-up -- and that therefore hold
 * no lfm_context.  The per-CTA partials go to a static device array of
 * 196,704 bytes (192 KiB: 2049 rows of 12 doubles) that every GPU loading
 * the library keeps until the process ends; lattices up to 512^3 cells fit,
 * larger ones return LFM_ERR_CAPACITY.  The first call on each device looks
 * up the array's device address and should come before any stream capture on
 * that device; the address is the device's primary context's, so calls must
 * run with the primary context current (the CUDA runtime's default).  All
 * calls share the array: calls that overlap on the GPU (two streams, two
 * threads) race; serialise them.  Outputs come in the same order as
 * lfm_metrics_f64's: chi min/max and the cell counts are identical, and the
 * sums agree to rounding (the partial sums are grouped differently). */
int lfm_metrics_f64_noalloc(int level, const float* psi_r, const float* psi_r_prev,
                            const float* psi_i, const float* psi_i_prev, const float* chi, int N,
                            double dt, double c, double boundary_fraction,
                            double well_threshold, double void_threshold, double* out_host,
                            void* stream);

/* Transform of the S_a solve (no counterpart in the reference, which always
 * runs 3-D FFTs): 1 = split (default): 2-D cuFFT transforms over (j, k) and
 * one hand-written pass along i that does the forward FFT, the Helmholtz
 * filter and the inverse FFT (N in {64, 128, 256, 512, 1024}; other N use the
 * 3-D path); 0 = 3-D cuFFT transforms with a separate filter pass.  Both
 * follow numpy_backend.py:341-356 and agree to float32 rounding.
 * Process-wide; for tests and tuning. */
int lfm_set_sa_transform(int mode);

/* Kernel path for the step calls: 0 = automatic (fused 2.5D kernel where
 * it applies, the direct kernel otherwise), 1 = direct kernel only,
 * 2 = fused kernel only (calls it cannot serve return LFM_ERR_UNSUPPORTED).
 * Process-wide; for tests and tuning. */
int lfm_set_step_path(int path);

/* Tile configuration of the fused kernel for (level, N): cells per thread
 * along k (vec: 2 or 4 at REAL and COMPLEX, 1 or 2 at COLOR, 0 = automatic;
 * the fused kernel refuses other widths, like any tile it cannot run), rows per tile,
 * shared-memory stages and planes per chunk (ic 0 = automatic).  tj <= 0
 * removes the entry and restores the built-in choice.  lfm_tune_get reports
 * the configuration the last fused step of that (level, N) ran with. */
int lfm_tune_set(int level, int N, int vec, int tj, int stages, int ic);
int lfm_tune_get(int level, int N, int* vec, int* tj, int* stages, int* ic, int* threads,
                 int* smem);

/* Reads (and optionally clears) the device status word that bounded
 * device-side waits set on timeout.  It first synchronises the current
 * device (cudaDeviceSynchronize), so every kernel launched before the call,
 * on any stream, has finished; with clear, only the bits it read are cleared
 * (atomically on the device).  A step whose wait gave up has returned with
 * its outputs partly written, so a non-zero word means the state is not
 * usable.  The Python layer (Evolver.get_*, synchronize, BatchedLattices and
 * SlabEvolver reads) calls this and raises LfmError on a non-zero word. */
int lfm_device_status(int* status_out, int clear);

/* Failure-detection test: launches, on `stream`, one CTA that waits through
 * the step kernels' bounded wait on an mbarrier nothing completes.  The wait
 * gives up after limit_ns (1 us .. 1 s), ORs LFM_ERR_DEVICE_TIMEOUT into the
 * device status word and returns; the context stays usable. */
int lfm_selftest_device_timeout(unsigned long long limit_ns, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LFM_B200_H */
