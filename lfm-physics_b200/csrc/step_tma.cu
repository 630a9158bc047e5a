// Fused 2.5D step kernels for sm_100a (N % 4 == 0).
//
// Layout: fields are C-order [i][j][k], k contiguous.  A CTA owns a tile of
// TJ whole rows (j0 .. j0+TJ-1, every k) and marches along i over a chunk
// of planes [i0, i1).  For each plane p the TMA engine copies, with 1-D bulk
// copies (cp.async.bulk) completing on an mbarrier:
//   * every stencil field (Psi components and chi): the TJ tile rows plus
//     the two periodic halo rows j0-1 and j0+TJ -> TJ+2 rows of N floats;
//   * in the register-queue kernels (REAL, COMPLEX, the batch), every point
//     field (previous-step fields, the protocol mask): the TJ tile rows
// into one stage of an S-deep shared-memory ring.  The barrier kernel
// (COLOR, below) stages only its seven stencil fields and reads the point
// fields (previous-step fields, mask, S_a) once per cell from global memory.
// There, computing plane i reads the stages of planes i-1, i, i+1; after a
// CTA barrier the stage of i-1 is refilled with plane i-1+S, so S-3 planes
// stream in while one is computed.
// Periodic wrap in i and j is folded into the copy addresses; wrap in k is
// resolved when reading shared memory.  Each thread updates V consecutive
// cells of one row with vector loads/stores; its k-1 / k+V neighbours come
// from the adjacent lanes by warp shuffle (shared memory at row ends and
// warp edges).  Arithmetic: lfm_cells.cuh, bit-identical to the reference.
//
// Every mbarrier wait is bounded by wall time (%globaltimer); on timeout the
// CTA records LFM_ERR_DEVICE_TIMEOUT in the status word, waits (bounded)
// for its own copies in flight and returns.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <mutex>

#include "lfm_cells.cuh"
#include "lfm_batch.h"
#include "lfm_kernels.h"
#include "lfm_tune.h"

namespace lfm {
namespace {

constexpr int kMaxStencil = 7;
// Step forms of the register-queue kernel: the reference's float32 step
// (bit-exact), the compensated Delta form, and split chi (chi0 + hi + lo).
constexpr int kPlain = 0, kComp = 1, kSplit = 2;
constexpr int kMaxPoint = 11;
constexpr int kMaxStages = 6;
constexpr uint64_t kWaitLimitNs = 1000000000ull;  // 1 s per wait
constexpr uint64_t kDrainLimitNs = 100000000ull;  // 0.1 s per stage when draining

struct TmaParams {
  StepArgs a;
  const float* sf[kMaxStencil];  // stencil fields (base of each component)
  const float* pf[kMaxPoint];    // point fields
  int ns, np;                    // counts
  int pf_mask;                   // index of the mask point field, -1 = lookup table
  int pf_sa;                     // index of S_a colour 0, -1 = none
  int N, TJ, IC, S, JT;
  int TJL;  // rows of the stage layout: TJ, or a batch lattice's largest tile for a shorter one
  int stage_floats;
  int tab_off;  // float offset of the shared-memory sponge table's tab[0], -1 = read through L1
};

// ---- PTX helpers -------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Raises the barrier's expected transaction bytes without arriving.
__device__ __forceinline__ void mbar_add_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_copy_g2s(float* dst, const float* src, uint32_t bytes,
                                              uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint32_t atom_add_acq_rel_cta(uint32_t* p, uint32_t v) {
  uint32_t old;
  asm volatile("atom.acq_rel.cta.shared::cta.add.u32 %0, [%1], %2;"
               : "=r"(old)
               : "r"(smem_addr(p)), "r"(v)
               : "memory");
  return old;
}

// Orders generic-proxy shared-memory accesses made before it (this thread's,
// and the other warps' ones acquired through the counter) before the
// async-proxy (TMA) writes issued after it.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ uint64_t now_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// try_wait that may suspend the thread for up to hint_ns until the phase
// completes (it resumes as soon as it does), so a waiting warp sleeps instead
// of spinning on the issue slots of the warps that have their data.
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t* bar, uint32_t parity,
                                                    uint32_t hint_ns) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0;
}

constexpr uint32_t kSleepHintNs = 2000;

// SLEEP: retry with mbar_try_wait_sleep.  Measured on the long single-lattice
// marches: +0.4-0.8% (300 ns to 20 us alike); on the batch kernel's short
// items: -5.6%, so there the retries spin.
template <bool SLEEP = false>
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = now_ns();
  while (true) {
    if (SLEEP ? mbar_try_wait_sleep(bar, parity, kSleepHintNs) : mbar_try_wait(bar, parity))
      return true;
    if (now_ns() - t0 > limit_ns) return false;
  }
}

// ---- vector helpers ------------------------------------------------------------
template <int V>
struct Vec {
  float v[V];
};

template <int V>
__device__ __forceinline__ Vec<V> lds(const float* smem, int off) {
  Vec<V> r;
  if constexpr (V == 4) {
    const float4 t = *reinterpret_cast<const float4*>(smem + off);
    r.v[0] = t.x; r.v[1] = t.y; r.v[2] = t.z; r.v[3] = t.w;
  } else if constexpr (V == 2) {
    const float2 t = *reinterpret_cast<const float2*>(smem + off);
    r.v[0] = t.x; r.v[1] = t.y;
  } else {
    r.v[0] = smem[off];
  }
  return r;
}

template <int V>
__device__ __forceinline__ void stg(float* p, const float (&x)[V]) {
  if constexpr (V == 4) {
    *reinterpret_cast<float4*>(p) = make_float4(x[0], x[1], x[2], x[3]);
  } else if constexpr (V == 2) {
    *reinterpret_cast<float2*>(p) = make_float2(x[0], x[1]);
  } else {
    *p = x[0];
  }
}

// Coherent vector load from global memory (the point fields of the
// barrier kernel; in the resident layout a thread reads its own prev cells
// and then overwrites them, so the read-only path is not used).
template <int V>
__device__ __forceinline__ Vec<V> ldgv(const float* p) {
  Vec<V> r;
  if constexpr (V == 4) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    r.v[0] = t.x; r.v[1] = t.y; r.v[2] = t.z; r.v[3] = t.w;
  } else if constexpr (V == 2) {
    const float2 t = *reinterpret_cast<const float2*>(p);
    r.v[0] = t.x; r.v[1] = t.y;
  } else {
    r.v[0] = *p;
  }
  return r;
}

// Per-thread geometry inside the tile.
struct Lane {
  int r;        // tile row (0..TJ-1)
  int k0;       // first k of the thread's V cells
  int km1, kpv; // periodic k0-1 and k0+V
  bool fix_l, fix_r;  // neighbour not in the adjacent lane: read shared memory
};

__device__ __forceinline__ float left_nb(float mine_last, const float* smem, int row_off,
                                         const Lane& L) {
  float v = __shfl_up_sync(0xffffffffu, mine_last, 1);
  if (L.fix_l) v = smem[row_off + L.km1];
  return v;
}

__device__ __forceinline__ float right_nb(float mine_first, const float* smem, int row_off,
                                          const Lane& L) {
  float v = __shfl_down_sync(0xffffffffu, mine_first, 1);
  if (L.fix_r) v = smem[row_off + L.kpv];
  return v;
}

// The 19-point stencil of one field for the thread's V cells.  fm/f0/fp are
// the offsets of this field's TJ+2 rows in the stages of planes i-1, i, i+1
// (row 0 = tile row -1).  Returns the Laplacian and centre per cell and, with
// FACES, the six face neighbours (for the momentum current).
template <int V, bool FACES>
__device__ __forceinline__ void field_stencil(const float* smem, int fm, int f0, int fp, int N,
                                              const Lane& L, float (&lap)[V], float (&ctr)[V],
                                              Faces (&faces)[V]) {
  const int rm = (L.r) * N, r0 = (L.r + 1) * N, rp = (L.r + 2) * N;
  const Vec<V> A_m = lds<V>(smem, f0 + rm + L.k0);
  const Vec<V> A_0 = lds<V>(smem, f0 + r0 + L.k0);
  const Vec<V> A_p = lds<V>(smem, f0 + rp + L.k0);
  const Vec<V> M_m = lds<V>(smem, fm + rm + L.k0);
  const Vec<V> M_0 = lds<V>(smem, fm + r0 + L.k0);
  const Vec<V> M_p = lds<V>(smem, fm + rp + L.k0);
  const Vec<V> P_m = lds<V>(smem, fp + rm + L.k0);
  const Vec<V> P_0 = lds<V>(smem, fp + r0 + L.k0);
  const Vec<V> P_p = lds<V>(smem, fp + rp + L.k0);
  // k0-1 and k0+V: with two cells per lane, the second and first value of the
  // aligned neighbouring pairs (periodic in k); otherwise the adjacent lanes'
  // values by shuffle, from shared memory at row ends and warp edges.
  float A_m_l, A_m_r, A_0_l, A_0_r, A_p_l, A_p_r, M_0_l, M_0_r, P_0_l, P_0_r;
  if constexpr (V == 2) {
    const int kl = L.km1 - 1, kr = L.kpv;
    A_m_l = lds<2>(smem, f0 + rm + kl).v[1];
    A_m_r = lds<2>(smem, f0 + rm + kr).v[0];
    A_0_l = lds<2>(smem, f0 + r0 + kl).v[1];
    A_0_r = lds<2>(smem, f0 + r0 + kr).v[0];
    A_p_l = lds<2>(smem, f0 + rp + kl).v[1];
    A_p_r = lds<2>(smem, f0 + rp + kr).v[0];
    M_0_l = lds<2>(smem, fm + r0 + kl).v[1];
    M_0_r = lds<2>(smem, fm + r0 + kr).v[0];
    P_0_l = lds<2>(smem, fp + r0 + kl).v[1];
    P_0_r = lds<2>(smem, fp + r0 + kr).v[0];
  } else {
    A_m_l = left_nb(A_m.v[V - 1], smem, f0 + rm, L);
    A_m_r = right_nb(A_m.v[0], smem, f0 + rm, L);
    A_0_l = left_nb(A_0.v[V - 1], smem, f0 + r0, L);
    A_0_r = right_nb(A_0.v[0], smem, f0 + r0, L);
    A_p_l = left_nb(A_p.v[V - 1], smem, f0 + rp, L);
    A_p_r = right_nb(A_p.v[0], smem, f0 + rp, L);
    M_0_l = left_nb(M_0.v[V - 1], smem, fm + r0, L);
    M_0_r = right_nb(M_0.v[0], smem, fm + r0, L);
    P_0_l = left_nb(P_0.v[V - 1], smem, fp + r0, L);
    P_0_r = right_nb(P_0.v[0], smem, fp + r0, L);
  }
  S19 st[V];
#pragma unroll
  for (int e = 0; e < V; ++e) {
    S19& s = st[e];
    s.c = A_0.v[e];
    s.im = M_0.v[e];
    s.ip = P_0.v[e];
    s.jm = A_m.v[e];
    s.jp = A_p.v[e];
    s.km = e > 0 ? A_0.v[e - 1] : A_0_l;
    s.kp = e < V - 1 ? A_0.v[e + 1] : A_0_r;
    s.imjm = M_m.v[e];
    s.imjp = M_p.v[e];
    s.ipjm = P_m.v[e];
    s.ipjp = P_p.v[e];
    s.imkm = e > 0 ? M_0.v[e - 1] : M_0_l;
    s.imkp = e < V - 1 ? M_0.v[e + 1] : M_0_r;
    s.ipkm = e > 0 ? P_0.v[e - 1] : P_0_l;
    s.ipkp = e < V - 1 ? P_0.v[e + 1] : P_0_r;
    s.jmkm = e > 0 ? A_m.v[e - 1] : A_m_l;
    s.jmkp = e < V - 1 ? A_m.v[e + 1] : A_m_r;
    s.jpkm = e > 0 ? A_p.v[e - 1] : A_p_l;
    s.jpkp = e < V - 1 ? A_p.v[e + 1] : A_p_r;
    if constexpr (V != 2) lap[e] = lap19(s);
    ctr[e] = s.c;
    if (FACES) {
      faces[e].im = s.im; faces[e].ip = s.ip;
      faces[e].jm = s.jm; faces[e].jp = s.jp;
      faces[e].km = s.km; faces[e].kp = s.kp;
    }
  }
  if constexpr (V == 2) {  // i/j sums of both cells as packed additions
    const F2 l = lap19_pair(st[0], st[1]);
    lap[0] = l.v.x;
    lap[1] = l.v.y;
  }
}

// One output plane of the COLOR step: seven 19-point stencils from the
// ring, the point fields from global memory, lfm_cells.cuh's colour update.
template <int V>
__device__ __forceinline__ void color_plane(const TmaParams& P, const float* smem, int sm, int s0,
                                            int sp, int i, const Lane& L, int j) {
  const StepArgs& a = P.a;
  const int N = P.N, TJ = P.TJ;
  const int field_rows = (TJ + 2) * N;
  const int64_t gofs = ((int64_t)i * N + j) * N + L.k0;

  // sponge factor per cell
  float mask[V], absorb[V];
  if (P.pf_mask >= 0) {
    const Vec<V> m = ldgv<V>(P.pf[P.pf_mask] + gofs);
#pragma unroll
    for (int e = 0; e < V; ++e) mask[e] = m.v[e];
  } else {
    const int32_t qij = qterm(i, N) + qterm(j, N);
#pragma unroll
    for (int e = 0; e < V; ++e) mask[e] = mask_from_q(a.lut, qij + qterm(L.k0 + e, N));
  }
#pragma unroll
  for (int e = 0; e < V; ++e) absorb[e] = fsub(1.0f, mask[e]);

  // Point fields (previous values, mask, S_a) are read once per cell, from
  // global memory; only the stencil fields go through the shared-memory ring.
  auto prev = [&](int g, float (&out)[V]) {
    const Vec<V> p = ldgv<V>(P.pf[g] + gofs);
#pragma unroll
    for (int e = 0; e < V; ++e) out[e] = a.damp_prev ? fmul(p.v[e], absorb[e]) : p.v[e];
  };
  auto plain = [&](int g, float (&out)[V]) {
    const Vec<V> p = ldgv<V>(P.pf[g] + gofs);
#pragma unroll
    for (int e = 0; e < V; ++e) out[e] = p.v[e];
  };

  Faces nofaces[V];
  const int64_t n3 = (int64_t)N * N * N;
  // stencil fields: R0 R1 R2 I0 I1 I2 chi ; point fields: Rp0..2 Ip0..2 chip [mask] [S0..2]
  // the point loads first: their latency runs under the stencil arithmetic
  float lapX[V], cX[V], xp[V], rpc[3][V], ipc[3][V], sac[3][V];
  plain(6, xp);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    prev(c, rpc[c]);
    prev(3 + c, ipc[c]);
  }
  const bool has_sa = P.pf_sa >= 0;
  if (has_sa) {
#pragma unroll
    for (int c = 0; c < 3; ++c) plain(P.pf_sa + c, sac[c]);
  }
  field_stencil<V, false>(smem, sm + 6 * field_rows, s0 + 6 * field_rows, sp + 6 * field_rows,
                          N, L, lapX, cX, nofaces);
  Vec<V> cr[3], ci[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    cr[c] = lds<V>(smem, s0 + c * field_rows + (L.r + 1) * N + L.k0);
    ci[c] = lds<V>(smem, s0 + (3 + c) * field_rows + (L.r + 1) * N + L.k0);
  }
  if constexpr (V == 2) {
    // both cells of the lane at once: packed additions, per lane where needed
    const F2 prc[3] = {pk(cr[0].v[0], cr[0].v[1]), pk(cr[1].v[0], cr[1].v[1]),
                       pk(cr[2].v[0], cr[2].v[1])};
    const F2 pic[3] = {pk(ci[0].v[0], ci[0].v[1]), pk(ci[1].v[0], ci[1].v[1]),
                       pk(ci[2].v[0], ci[2].v[1])};
    ColorAccT<F2> A;
    color_begin(A, pk(cX[0], cX[1]), pk(mask[0], mask[1]), prc, pic, a.c);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float lapR[V], cR[V], lapI[V], cI[V];
      Faces fR[V], fI[V];
      field_stencil<V, true>(smem, sm + c * field_rows, s0 + c * field_rows,
                             sp + c * field_rows, N, L, lapR, cR, fR);
      field_stencil<V, true>(smem, sm + (3 + c) * field_rows, s0 + (3 + c) * field_rows,
                             sp + (3 + c) * field_rows, N, L, lapI, cI, fI);
      const ColorCompOutT<F2> o = color_component(
          A, c, pk(lapR[0], lapR[1]), pk(cR[0], cR[1]), pk(rpc[c][0], rpc[c][1]),
          pk_faces(fR[0], fR[1]), pk(lapI[0], lapI[1]), pk(cI[0], cI[1]),
          pk(ipc[c][0], ipc[c][1]), pk_faces(fI[0], fI[1]), a.c);
      const float o_r[V] = {o.pr.v.x, o.pr.v.y}, o_i[V] = {o.pi.v.x, o.pi.v.y};
      stg<V>(a.pr_out + c * n3 + gofs, o_r);
      stg<V>(a.pi_out + c * n3 + gofs, o_i);
      if (a.energy_out) {  // |Psi_a|^2 of the stored values, for the next S_a solve
        const F2 en = fadd(fmul(o.pr, o.pr), fmul(o.pi, o.pi));
        const float o_e[V] = {en.v.x, en.v.y};
        stg<V>(a.energy_out + c * n3 + gofs, o_e);
      }
      if (a.pr_prev_out) {
        const float o_rp[V] = {o.pr_prev.v.x, o.pr_prev.v.y};
        stg<V>(a.pr_prev_out + c * n3 + gofs, o_rp);
      }
      if (a.pi_prev_out) {
        const float o_ip[V] = {o.pi_prev.v.x, o.pi_prev.v.y};
        stg<V>(a.pi_prev_out + c * n3 + gofs, o_ip);
      }
    }
    F2 saf[3];
    if (has_sa) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        saf[c] = pk(sac[c][0], sac[c][1]);
        if (a.sa_clip_out) {
          const float t[V] = {fmaxf(sac[c][0], 0.0f), fmaxf(sac[c][1], 0.0f)};
          stg<V>(a.sa_clip_out + c * n3 + gofs, t);
        }
      }
    }
    const F2 oc = color_finish(A, pk(lapX[0], lapX[1]), pk(xp[0], xp[1]), has_sa, saf, a.c);
    const float o_c[V] = {oc.v.x, oc.v.y};
    stg<V>(a.chi_out + gofs, o_c);
    if (a.chi_prev_out) stg<V>(a.chi_prev_out + gofs, cX);
  } else {  // one cell per lane
    ColorAcc A[V];
    {
#pragma unroll
      for (int e = 0; e < V; ++e) {
        const float prc[3] = {cr[0].v[e], cr[1].v[e], cr[2].v[e]};
        const float pic[3] = {ci[0].v[e], ci[1].v[e], ci[2].v[e]};
        color_begin(A[e], cX[e], mask[e], prc, pic, a.c);
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float lapR[V], cR[V], lapI[V], cI[V];
      Faces fR[V], fI[V];
      field_stencil<V, true>(smem, sm + c * field_rows, s0 + c * field_rows, sp + c * field_rows,
                             N, L, lapR, cR, fR);
      field_stencil<V, true>(smem, sm + (3 + c) * field_rows, s0 + (3 + c) * field_rows,
                             sp + (3 + c) * field_rows, N, L, lapI, cI, fI);
      float o_r[V], o_i[V], o_rp[V], o_ip[V];
#pragma unroll
      for (int e = 0; e < V; ++e) {
        const ColorCompOut o =
            color_component(A[e], c, lapR[e], cR[e], rpc[c][e], fR[e], lapI[e], cI[e], ipc[c][e],
                            fI[e], a.c);
        o_r[e] = o.pr; o_i[e] = o.pi; o_rp[e] = o.pr_prev; o_ip[e] = o.pi_prev;
      }
      stg<V>(a.pr_out + c * n3 + gofs, o_r);
      stg<V>(a.pi_out + c * n3 + gofs, o_i);
      if (a.energy_out) {
        float o_e[V];
#pragma unroll
        for (int e = 0; e < V; ++e) o_e[e] = fadd(fmul(o_r[e], o_r[e]), fmul(o_i[e], o_i[e]));
        stg<V>(a.energy_out + c * n3 + gofs, o_e);
      }
      if (a.pr_prev_out) stg<V>(a.pr_prev_out + c * n3 + gofs, o_rp);
      if (a.pi_prev_out) stg<V>(a.pi_prev_out + c * n3 + gofs, o_ip);
    }
    float sa[V][3];
    if (has_sa) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float t[V];
#pragma unroll
        for (int e = 0; e < V; ++e) t[e] = sac[c][e];
#pragma unroll
        for (int e = 0; e < V; ++e) sa[e][c] = t[e];
        if (a.sa_clip_out) {
#pragma unroll
          for (int e = 0; e < V; ++e) t[e] = fmaxf(t[e], 0.0f);
          stg<V>(a.sa_clip_out + c * n3 + gofs, t);
        }
      }
    }
    float o_c[V];
#pragma unroll
    for (int e = 0; e < V; ++e) o_c[e] = color_finish(A[e], lapX[e], xp[e], has_sa, sa[e], a.c);
    stg<V>(a.chi_out + gofs, o_c);
    if (a.chi_prev_out) stg<V>(a.chi_prev_out + gofs, cX);
  }
}

// Copies plane (i0 - 1 + u) into stage u % S: the stencil fields' tile rows
// and halo rows, and with PT the point fields' tile rows (the register-queue
// kernels read them from the stage; the barrier kernel reads them from global
// memory).  ONE: away from the wrap in j, a stencil field's rows j0-1 ..
// j0+TJ are contiguous and go as one copy instead of the tile rows and two
// one-row halo copies.  Measured with identical bits: COMPLEX +4 % at 256^3
// and 512^3, the compensated REAL step +1.5 %; the plain REAL step -0.5 % and
// the COLOR stencil -3.6 %, so those keep the separate halo copies.
// The stage layout has room for TJL tile rows (TJL >= TJ: a batch item shorter
// than its lattice's largest tile leaves the last rows of each field unused).
template <bool SLAB = true, bool PT = true, bool ONE = false>
__device__ __forceinline__ void issue_plane(const TmaParams& P, float* smem, uint64_t* bars,
                                            int u, int i0, int i1, int j0) {
  const int N = P.N, TJ = P.TJ, TJL = P.TJL;
  const int p = i0 - 1 + u;
  const int pw = (SLAB && P.a.slab) ? p : (p % N + N) % N;  // slabs read their ghost planes
  const int s = u % P.S;
  float* st = smem + (size_t)s * P.stage_floats;
  const bool point = PT && (p >= i0) && (p < i1);
  const uint32_t row_bytes = 4u * (uint32_t)N;
  const uint32_t bytes =
      row_bytes * (uint32_t)(P.ns * (TJ + 2) + (point ? P.np * TJ : 0));
  mbar_expect_tx(&bars[s], bytes);
  const int jm = (j0 == 0) ? N - 1 : j0 - 1;
  const int jp = (j0 + TJ == N) ? 0 : j0 + TJ;
  const int64_t plane = (int64_t)pw * N;
  const bool contiguous = ONE && j0 > 0 && j0 + TJ < N;
  for (int f = 0; f < P.ns; ++f) {
    float* d = st + (size_t)f * (TJL + 2) * N;
    const float* g = P.sf[f];
    if (contiguous) {
      bulk_copy_g2s(d, g + (plane + j0 - 1) * N, row_bytes * (TJ + 2), &bars[s]);
    } else {
      bulk_copy_g2s(d + N, g + (plane + j0) * N, row_bytes * TJ, &bars[s]);
      bulk_copy_g2s(d, g + (plane + jm) * N, row_bytes, &bars[s]);
      bulk_copy_g2s(d + (size_t)(TJ + 1) * N, g + (plane + jp) * N, row_bytes, &bars[s]);
    }
  }
  if (point) {
    float* base = st + (size_t)P.ns * (TJL + 2) * N;
    for (int g = 0; g < P.np; ++g)
      bulk_copy_g2s(base + (size_t)g * TJL * N, P.pf[g] + (plane + j0) * N, row_bytes * TJ,
                    &bars[s]);
  }
}

// The register-queue kernels that copy a stencil field's rows as one (above).
template <int LEVEL, int MODE>
constexpr bool kOneCopy = LEVEL == LFM_COMPLEX || MODE != kPlain;

template <int LEVEL, int V>
__global__ void __launch_bounds__(512) tma_step_kernel(const __grid_constant__ TmaParams P) {
  static_assert(LEVEL == LFM_COLOR, "REAL and COMPLEX run on the register-queue kernel");
  extern __shared__ __align__(128) float smem[];
  __shared__ __align__(8) uint64_t bars[kMaxStages];
  __shared__ int abort_flag;

  const int N = P.N, TJ = P.TJ, S = P.S;
  const int jt = blockIdx.x % P.JT, ch = blockIdx.x / P.JT;
  const int j0 = jt * TJ;
  const int i0 = ch * P.IC;
  const int i1 = min(i0 + P.IC, N);
  const int nplanes = (i1 - i0) + 2;
  const int tid = threadIdx.x, lane = tid & 31;
  const int tpr = N / V;

  Lane L;
  L.r = tid / tpr;
  const int kv = tid % tpr;
  L.k0 = kv * V;
  L.km1 = (L.k0 == 0) ? N - 1 : L.k0 - 1;
  L.kpv = (L.k0 + V == N) ? 0 : L.k0 + V;
  L.fix_l = (lane == 0) || (kv == 0);
  L.fix_r = (lane == 31) || (kv == tpr - 1);
  const int j = j0 + L.r;

  if (tid == 0) {
    for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
    abort_flag = 0;
    mbar_init_fence();
  }
  __syncthreads();
  int issued = 0;
  if (tid == 0) {
    for (; issued < min(S, nplanes); ++issued)
      issue_plane<true, false>(P, smem, bars, issued, i0, i1, j0);
  }

  int waited = 0;
  for (int c = 0; c < i1 - i0; ++c) {
    bool ok = true;
    while (waited <= c + 2) {
      ok = ok && mbar_wait_bounded(&bars[waited % S], (uint32_t)((waited / S) & 1), kWaitLimitNs);
      ++waited;
    }
    if (!ok) {
      abort_flag = 1;
      atomicOr(P.a.status, LFM_ERR_DEVICE_TIMEOUT);
    } else {
      const int sf = P.stage_floats;
      color_plane<V>(P, smem, (c % S) * sf, ((c + 1) % S) * sf, ((c + 2) % S) * sf,
                              i0 + c, L, j);
    }
    __syncthreads();
    if (abort_flag) break;
    if (tid == 0 && c + S < nplanes) {
      issue_plane<true, false>(P, smem, bars, c + S, i0, i1, j0);
      issued = c + S + 1;
    }
  }
  if (abort_flag && tid == 0) {
    // Let the copies this CTA started finish before its shared memory goes away.
    for (int u = max(waited, issued - S); u < issued; ++u)
      mbar_wait_bounded(&bars[u % S], (uint32_t)((u / S) & 1), kDrainLimitNs);
  }
}

// ---- register-queue kernel (REAL, COMPLEX) -------------------------------------
//
// Same tiles and copy ring as tma_step_kernel, but each plane of a stencil
// field is read from shared memory once: the thread keeps, for the planes
// i-1, i, i+1, the rows j-1, j, j+1 of its V cells in registers and rotates
// them as it marches (the loop is unrolled by three so the rotation is a
// renaming).  Neighbours k0-1 and k0+V are plain scalar loads.  A stage is
// dead once its plane has been the centre plane, so it is refilled one plane
// earlier than in tma_step_kernel: S stages keep S-2 planes in flight.
template <int V>
struct QPlane {
  Vec<V> m, z, p;        // rows j-1, j, j+1
  float zl, zr;          // row j at k0-1, k0+V
  float ml, mr, pl, pr;  // rows j-1, j+1 at k0-1, k0+V (loaded when centre)
};

struct QLane {
  int j, k0;                               // the thread's row and first cell
  int o_m, o_z, o_p;                       // row offsets at k0 in a field block
  int o_zl, o_zr, o_ml, o_mr, o_pl, o_pr;  // neighbour offsets
  int o_pt;                                // point rows at k0 (from the stage base)
};

// Radial keys of a thread's cells.  A cell's key q = qterm(i) + qterm(j) +
// qterm(k0 + e) is 3 mod 8 for even N (each term an odd square, 1 mod 8) and
// 0 mod 4 for odd N (even squares); the table steps by 2^shift, shift 3 or 2.
// Then q >> shift = (qterm(i) >> shift) + (qterm(j) >> shift) +
// (qterm(k) >> shift) exactly, so a table offset is a sum of three per-axis
// terms: offset = min_relu(4*(qterm(i) >> shift) + aj4 + ak4[e], cap4).
template <int V>
struct QKeys {
  int32_t qj;  // qterm(j)
  int32_t aj4, cap4;
  int32_t ak4[V];  // 4 * (qterm(k0 + e) >> shift)
};

__device__ __forceinline__ int key_shift(int N) { return (N & 1) ? 2 : 3; }

// max(min(a, b), 0) in one instruction.
__device__ __forceinline__ int32_t min_relu(int32_t a, int32_t b) {
  int32_t d;
  asm("min.relu.s32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}

// The sponge table in shared memory:
//   tab[0] = 0, tab[1 + t] = lut.table[t] (t < count), tab[count + 1] = 1,
// with tab[1] on a 16-byte boundary so the copy engine can fill it.
// A cell's entry is t = (q >> shift) - (q_lo >> shift) + 1 clamped to
// [0, count + 1]: keys below the band land on the 0, keys above it on the 1,
// so the lookup needs no band test and no select.  q_lo is capped at 3 N^2
// (above every key) for the all-zero mask (q_lo = INT32_MAX): every offset
// clamps to 0 then; the all-one mask (q_lo = 0, count = 0) clamps to 1.
template <int V>
__device__ __forceinline__ void sponge_key(QKeys<V>& K, const MaskLut& lut, int j, int k0,
                                           int N) {
  const int sh = key_shift(N);
  const int32_t key_lo = min(lut.q_lo, 3 * N * N) >> sh;
  K.qj = qterm(j, N);
  K.aj4 = 4 * ((K.qj >> sh) + 1 - key_lo);
  K.cap4 = 4 * (lut.count + 1);
#pragma unroll
  for (int e = 0; e < V; ++e) K.ak4[e] = 4 * (qterm(k0 + e, N) >> sh);
}

// Mask values of a thread's cells from the shared-memory table (sponge_key).
template <int V>
__device__ __forceinline__ void tab_mask(const float* tab, int32_t qi, int N, const QKeys<V>& K,
                                         float (&mask)[V]) {
  const int32_t b4 = 4 * (qi >> key_shift(N)) + K.aj4;
  const char* t = reinterpret_cast<const char*>(tab);
#pragma unroll
  for (int e = 0; e < V; ++e)
    mask[e] = *reinterpret_cast<const float*>(t + min_relu(b4 + K.ak4[e], K.cap4));
}

// Mask values through L1 from the global table, for lattices whose table does
// not fit beside the ring.  The table load is predicated on the band test
// (mask_from_q_flat); qterm(k) comes back from ak4: 2 * ak4 + 1 for even N
// (8a + 1 = 2 * 4a + 1), ak4 itself for odd N (4b).
template <int V>
__device__ __forceinline__ void q_mask(const MaskLut& lut, int32_t qi, int N, const QKeys<V>& K,
                                       float (&mask)[V]) {
  const int32_t qij = qi + K.qj;
  const bool even = !(N & 1);
#pragma unroll
  for (int e = 0; e < V; ++e)
    mask[e] = mask_from_q_flat(lut, qij + (even ? 2 * K.ak4[e] + 1 : K.ak4[e]));
}

template <int V>
__device__ __forceinline__ void q_load(QPlane<V>& q, const float* smem, int base, const QLane& L) {
  q.m = lds<V>(smem, base + L.o_m);
  q.z = lds<V>(smem, base + L.o_z);
  q.p = lds<V>(smem, base + L.o_p);
  q.zl = smem[base + L.o_zl];
  q.zr = smem[base + L.o_zr];
}

template <int V>
__device__ __forceinline__ void q_centre(QPlane<V>& q, const float* smem, int base,
                                         const QLane& L) {
  q.ml = smem[base + L.o_ml];
  q.mr = smem[base + L.o_mr];
  q.pl = smem[base + L.o_pl];
  q.pr = smem[base + L.o_pr];
}

template <int V>
__device__ __forceinline__ S19 q_s19(const QPlane<V>& M, const QPlane<V>& A, const QPlane<V>& P,
                                     int e) {
  S19 s;
  s.c = A.z.v[e];
  s.im = M.z.v[e];
  s.ip = P.z.v[e];
  s.jm = A.m.v[e];
  s.jp = A.p.v[e];
  s.km = e > 0 ? A.z.v[e - 1] : A.zl;
  s.kp = e < V - 1 ? A.z.v[e + 1] : A.zr;
  s.imjm = M.m.v[e];
  s.imjp = M.p.v[e];
  s.ipjm = P.m.v[e];
  s.ipjp = P.p.v[e];
  s.imkm = e > 0 ? M.z.v[e - 1] : M.zl;
  s.imkp = e < V - 1 ? M.z.v[e + 1] : M.zr;
  s.ipkm = e > 0 ? P.z.v[e - 1] : P.zl;
  s.ipkp = e < V - 1 ? P.z.v[e + 1] : P.zr;
  s.jmkm = e > 0 ? A.m.v[e - 1] : A.ml;
  s.jmkp = e < V - 1 ? A.m.v[e + 1] : A.mr;
  s.jpkm = e > 0 ? A.p.v[e - 1] : A.pl;
  s.jpkp = e < V - 1 ? A.p.v[e + 1] : A.pr;
  return s;
}

__device__ __forceinline__ Faces faces_of(const S19& s) {
  Faces f;
  f.im = s.im; f.ip = s.ip; f.jm = s.jm; f.jp = s.jp; f.km = s.km; f.kp = s.kp;
  return f;
}

// Stencil and point fields of the march: Psi components and chi (split chi:
// its hi part) in the stencil, their previous values (and split chi's lo and
// lo_prev) as point fields.
template <int LEVEL, int MODE = kPlain>
struct QFields {
  static constexpr int ns = (LEVEL == LFM_REAL) ? 2 : 3;     // Psi components, chi (hi)
  static constexpr int np = ns + (MODE == kSplit ? 2 : 0);  // their previous; split: lo, lo_prev
};

// Tile geometry of a march.  GeomRT reads it from the parameters (any
// lattice, any tile); GeomCT<N, TJ, NS> fixes it at compile time for the
// headline tiles (3 stages, resident point fields), so every shared-memory
// offset of a plane folds into an immediate beside one per-thread base.
// TABM: where the sponge table is read: 0 = as P.tab_off says at run time,
// 1 = shared memory (P.tab_off), -1 = through L1.
template <int TABM>
struct GeomRTT {
  static constexpr bool kFixed = false;
  static constexpr bool kSlab = true;  // may step a slab (plane range, ghost planes)
  static constexpr int kStages = 0;    // stage count known at run time only
  static constexpr int TAB = -1;       // the sponge table's place comes with the parameters
  static constexpr int kTabMode = TABM;
  int N, TJ, S, SF;  // TJ: the stage layout's rows
  __device__ __forceinline__ explicit GeomRTT(const TmaParams& P)
      : N(P.N), TJ(P.TJL), S(P.S), SF(P.stage_floats) {}
};
using GeomRT = GeomRTT<0>;

// A batch lattice shape fixed at compile time: row length N and the layout's
// TJ rows (the lattice's largest tile; its shorter tiles leave rows unused),
// so every shared-memory offset of a plane but the stage base is an
// immediate.  The ring depth stays a run-time value.
template <int N_, int TJ_, int NS_, int TABM>
struct GeomBT {
  static constexpr bool kFixed = false;
  static constexpr bool kSlab = false;
  static constexpr int kStages = 0;
  static constexpr int TAB = -1;
  static constexpr int kTabMode = TABM;
  static constexpr int N = N_, TJ = TJ_, SF = N_ * (NS_ * (TJ_ + 2) + NS_ * TJ_);
  int S;
  __device__ __forceinline__ explicit GeomBT(const TmaParams& P) : S(P.S) {}
};

// SLAB_: the tile may step a slab of planes (one rank's part of a lattice
// split along i, with its ghost planes); otherwise whole lattices only.
template <int N_, int TJ_, int NS_, int S_ = 3, bool SLAB_ = false, int NP_ = NS_>
struct GeomCT {
  static_assert(N_ % 2 == 0, "the sponge keys of the compile-time tiles assume even N");
  static constexpr bool kFixed = true;
  static constexpr bool kSlab = SLAB_;
  static constexpr int kStages = S_;
  static constexpr int N = N_, TJ = TJ_, S = S_, SF = N_ * (NS_ * (TJ_ + 2) + NP_ * TJ_);
  static constexpr int TAB = S * SF + 3;  // float offset of the sponge table's tab[0]
  static constexpr int kTabMode = 1;
  __device__ __forceinline__ explicit GeomCT(const TmaParams&) {}
};

// Shared bookkeeping of the barrier-free march.
struct QShared {
  uint32_t done[kMaxStages];  // warps finished with the stage's current plane
  int issued;                 // planes handed to the copy engine so far
  int abort_flag;
};

// One plane of the march with the roles (prev, cur, next) = (PA, PB, PC) of
// the register queue.  Warps do not wait for each other: each one releases
// the centre plane's stage when it is done with it, and the last warp to do
// so refills the stage with the plane S further on.  Returns false when the
// CTA must stop (a bounded wait gave up).
// SCUR / SNXT: the stages of the centre and the next plane when the
// geometry fixes them (3 stages, the loop unrolled by 3), else -1.
template <int LEVEL, int V, int MODE, bool PARTIAL, int PA, int PB, int PC, class G = GeomRT,
          int SCUR = -1, int SNXT = -1>
__device__ __forceinline__ bool q_plane(const TmaParams& P, float* smem, uint64_t* bars,
                                        QShared& sh, QPlane<V> (&Q)[QFields<LEVEL, MODE>::ns][3],
                                        const QLane& L, int c, int i0, int i1, int j0,
                                        int nplanes, int nwarps, int& s_cur_rt, int& s_nxt_rt,
                                        uint32_t& ph_nxt, const QKeys<V>& K,
                                        bool lane_active) {
  // PARTIAL: the CTA may be wider than the tile (batch kernel)
  const bool active = !PARTIAL || lane_active;
  constexpr int NS = QFields<LEVEL, MODE>::ns;
  const StepArgs& a = P.a;
  const G g(P);
  const int N = g.N, TJ = g.TJ;
  const int FB = (TJ + 2) * N;
  const int PTS = TJ * N;  // point-field stride
  const int SF = g.SF;
  const int s_cur = SCUR >= 0 ? SCUR : s_cur_rt;
  const int s_nxt = SNXT >= 0 ? SNXT : s_nxt_rt;
  // packed two-cell arithmetic in the compile-time tiles (V even)
  constexpr bool PK = (V % 2 == 0);
  // another warp gave up on a wait: stop (looked at once per unrolled round
  // of three planes; a plane's own wait is bounded anyway)
  if (PA == 0 && *(volatile int*)&sh.abort_flag) return false;
  if (!mbar_wait_bounded<G::kFixed>(&bars[s_nxt], ph_nxt, kWaitLimitNs)) {
    *(volatile int*)&sh.abort_flag = 1;
    atomicOr(a.status, LFM_ERR_DEVICE_TIMEOUT);
    return false;
  }
  const int bn = s_nxt * SF, bc = s_cur * SF;
  // Threads beyond the tile's rows (a batch tile narrower than the CTA) only
  // take part in the waits and the stage release.
  if (active) {
#pragma unroll
  for (int f = 0; f < NS; ++f) {
    q_load<V>(Q[f][PC], smem, bn + f * FB, L);
    q_centre<V>(Q[f][PB], smem, bc + f * FB, L);
  }
  const int i = i0 + c;
  const int j = L.j, k0 = L.k0;
  float mask[V], absorb[V];
  if constexpr (G::kFixed) {
    // the compile-time tiles never stream the mask; their table sits at TAB
    tab_mask<V>(smem + G::TAB, qterm(i + (G::kSlab ? a.i_off : 0), N), N, K, mask);
  } else if (P.pf_mask >= 0) {  // the streamed mask, from the centre plane's stage
    const Vec<V> m = lds<V>(smem, bc + L.o_pt + P.pf_mask * PTS);
#pragma unroll
    for (int e = 0; e < V; ++e) mask[e] = m.v[e];
  } else {
    const int32_t qi = qterm(i + (G::kSlab ? a.i_off : 0), N);  // a slab's global plane
    if (G::kTabMode > 0 || (G::kTabMode == 0 && P.tab_off >= 0))
      tab_mask<V>(smem + P.tab_off, qi, N, K, mask);
    else
      q_mask<V>(a.lut, qi, N, K, mask);
  }
#pragma unroll
  for (int e = 0; e < V; ++e) absorb[e] = fsub(1.0f, mask[e]);
  const int64_t gofs = ((int64_t)i * N + j) * N + k0;
  if constexpr (MODE == kSplit) {
    // Split chi: stencil fields Psi (Psi_r, Psi_i), hi; point fields their
    // previous slots in the same order, then lo and lo_prev.  New values go
    // over the previous slots.
    if constexpr (LEVEL == LFM_REAL) {
      const Vec<V> ep = lds<V>(smem, bc + L.o_pt);
      const Vec<V> hp = lds<V>(smem, bc + L.o_pt + PTS);
      const Vec<V> lc = lds<V>(smem, bc + L.o_pt + 2 * PTS);
      const Vec<V> lp = lds<V>(smem, bc + L.o_pt + 3 * PTS);
      float o_e[V], o_h[V], o_l[V];
#pragma unroll
      for (int e = 0; e < V; ++e) {
        const S19 E = q_s19<V>(Q[0][PA], Q[0][PB], Q[0][PC], e);
        const S19 H = q_s19<V>(Q[1][PA], Q[1][PB], Q[1][PC], e);
        const float epv = a.damp_prev ? fmul(ep.v[e], absorb[e]) : ep.v[e];
        const RealSplit o =
            real_cell_split(lap19_fma(E), E.c, epv, lap19_diff(H), split_value(H.c, lc.v[e]),
                            split_value(hp.v[e], lp.v[e]), mask[e], absorb[e], a.c);
        o_e[e] = o.psi; o_h[e] = o.chi.hi; o_l[e] = o.chi.lo;
      }
      stg<V>(a.pr_out + gofs, o_e);
      stg<V>(a.chi_out + gofs, o_h);
      stg<V>(a.chi_lo_out + gofs, o_l);
    } else {
      const Vec<V> rp = lds<V>(smem, bc + L.o_pt);
      const Vec<V> ip = lds<V>(smem, bc + L.o_pt + PTS);
      const Vec<V> hp = lds<V>(smem, bc + L.o_pt + 2 * PTS);
      const Vec<V> lc = lds<V>(smem, bc + L.o_pt + 3 * PTS);
      const Vec<V> lp = lds<V>(smem, bc + L.o_pt + 4 * PTS);
      float o_r[V], o_i[V], o_h[V], o_l[V];
#pragma unroll
      for (int e = 0; e < V; ++e) {
        const S19 R = q_s19<V>(Q[0][PA], Q[0][PB], Q[0][PC], e);
        const S19 I = q_s19<V>(Q[1][PA], Q[1][PB], Q[1][PC], e);
        const S19 H = q_s19<V>(Q[2][PA], Q[2][PB], Q[2][PC], e);
        const float rpv = a.damp_prev ? fmul(rp.v[e], absorb[e]) : rp.v[e];
        const float ipv = a.damp_prev ? fmul(ip.v[e], absorb[e]) : ip.v[e];
        const ComplexSplit o = complex_cell_split(
            lap19_fma(R), R.c, rpv, faces_of(R), lap19_fma(I), I.c, ipv, faces_of(I),
            lap19_diff(H), split_value(H.c, lc.v[e]), split_value(hp.v[e], lp.v[e]), mask[e],
            absorb[e], a.c);
        o_r[e] = o.pr; o_i[e] = o.pi; o_h[e] = o.chi.hi; o_l[e] = o.chi.lo;
      }
      stg<V>(a.pr_out + gofs, o_r);
      stg<V>(a.pi_out + gofs, o_i);
      stg<V>(a.chi_out + gofs, o_h);
      stg<V>(a.chi_lo_out + gofs, o_l);
    }
  } else if constexpr (MODE == kComp) {
    // Delta form: point fields hold the increments; new values go to the
    // *_out buffers, new increments over the increments (*_prev_out).
    if constexpr (LEVEL == LFM_REAL) {
      const Vec<V> de = lds<V>(smem, bc + L.o_pt);
      const Vec<V> dx = lds<V>(smem, bc + L.o_pt + PTS);
      float o_e[V], o_de[V], o_x[V], o_dx[V];
#pragma unroll
      for (int e = 0; e < V; ++e) {
        const S19 E = q_s19<V>(Q[0][PA], Q[0][PB], Q[0][PC], e);
        const S19 X = q_s19<V>(Q[1][PA], Q[1][PB], Q[1][PC], e);
        const RealComp o =
            real_cell_comp(lap19_fma(E), E.c, de.v[e], lap19_diff(X), X.c, dx.v[e], mask[e], a.c);
        o_e[e] = o.psi.v; o_de[e] = o.psi.d; o_x[e] = o.chi.v; o_dx[e] = o.chi.d;
      }
      stg<V>(a.pr_out + gofs, o_e);
      stg<V>(a.pr_prev_out + gofs, o_de);
      stg<V>(a.chi_out + gofs, o_x);
      stg<V>(a.chi_prev_out + gofs, o_dx);
    } else {
      const Vec<V> dr = lds<V>(smem, bc + L.o_pt);
      const Vec<V> di = lds<V>(smem, bc + L.o_pt + PTS);
      const Vec<V> dx = lds<V>(smem, bc + L.o_pt + 2 * PTS);
      float o_r[V], o_dr[V], o_i[V], o_di[V], o_x[V], o_dx[V];
#pragma unroll
      for (int e = 0; e < V; ++e) {
        const S19 R = q_s19<V>(Q[0][PA], Q[0][PB], Q[0][PC], e);
        const S19 I = q_s19<V>(Q[1][PA], Q[1][PB], Q[1][PC], e);
        const S19 X = q_s19<V>(Q[2][PA], Q[2][PB], Q[2][PC], e);
        const ComplexComp o = complex_cell_comp(lap19_fma(R), R.c, dr.v[e], faces_of(R),
                                                lap19_fma(I), I.c, di.v[e], faces_of(I),
                                                lap19_diff(X), X.c, dx.v[e], mask[e], a.c);
        o_r[e] = o.pr.v; o_dr[e] = o.pr.d; o_i[e] = o.pi.v; o_di[e] = o.pi.d;
        o_x[e] = o.chi.v; o_dx[e] = o.chi.d;
      }
      stg<V>(a.pr_out + gofs, o_r);
      stg<V>(a.pr_prev_out + gofs, o_dr);
      stg<V>(a.pi_out + gofs, o_i);
      stg<V>(a.pi_prev_out + gofs, o_di);
      stg<V>(a.chi_out + gofs, o_x);
      stg<V>(a.chi_prev_out + gofs, o_dx);
    }
  } else if constexpr (LEVEL == LFM_REAL) {
    const Vec<V> ep = lds<V>(smem, bc + L.o_pt);
    const Vec<V> xp = lds<V>(smem, bc + L.o_pt + PTS);
    float o_psi[V], o_chi[V], o_pp[V], o_cp[V];
    if constexpr (PK) {
      // two cells per packed FADD2 / FMUL2
#pragma unroll
      for (int e = 0; e < V; e += 2) {
        const S19 E0 = q_s19<V>(Q[0][PA], Q[0][PB], Q[0][PC], e);
        const S19 E1 = q_s19<V>(Q[0][PA], Q[0][PB], Q[0][PC], e + 1);
        const S19 X0 = q_s19<V>(Q[1][PA], Q[1][PB], Q[1][PC], e);
        const S19 X1 = q_s19<V>(Q[1][PA], Q[1][PB], Q[1][PC], e + 1);
        const F2 mk = pk(mask[e], mask[e + 1]);
        const F2 ab = fsub(cst<F2>(1.0f), mk);
        F2 epv = pk(ep.v[e], ep.v[e + 1]);
        if (a.damp_prev) epv = fmul(epv, ab);
        const RealOutT<F2> o =
            real_cell_ab(lap19_pair(E0, E1), pk(E0.c, E1.c), epv, lap19_pair(X0, X1),
                         pk(X0.c, X1.c), pk(xp.v[e], xp.v[e + 1]), mk, ab, a.c);
        o_psi[e] = o.psi.v.x; o_psi[e + 1] = o.psi.v.y;
        o_chi[e] = o.chi.v.x; o_chi[e + 1] = o.chi.v.y;
        o_pp[e] = o.psi_prev.v.x; o_pp[e + 1] = o.psi_prev.v.y;
        o_cp[e] = o.chi_prev.v.x; o_cp[e + 1] = o.chi_prev.v.y;
      }
    } else {
#pragma unroll
    for (int e = 0; e < V; ++e) {
      const S19 E = q_s19<V>(Q[0][PA], Q[0][PB], Q[0][PC], e);
      const S19 X = q_s19<V>(Q[1][PA], Q[1][PB], Q[1][PC], e);
      const float epv = a.damp_prev ? fmul(ep.v[e], absorb[e]) : ep.v[e];
      const RealOut o = real_cell(lap19(E), E.c, epv, lap19(X), X.c, xp.v[e], mask[e], a.c);
      o_psi[e] = o.psi; o_chi[e] = o.chi; o_pp[e] = o.psi_prev; o_cp[e] = o.chi_prev;
    }
    }
    stg<V>(a.pr_out + gofs, o_psi);
    stg<V>(a.chi_out + gofs, o_chi);
    if (a.pr_prev_out) stg<V>(a.pr_prev_out + gofs, o_pp);
    if (a.chi_prev_out) stg<V>(a.chi_prev_out + gofs, o_cp);
  } else {
    const Vec<V> rp = lds<V>(smem, bc + L.o_pt);
    const Vec<V> ip = lds<V>(smem, bc + L.o_pt + PTS);
    const Vec<V> xp = lds<V>(smem, bc + L.o_pt + 2 * PTS);
    float o_r[V], o_i[V], o_c[V], o_rp[V], o_ip[V], o_cp[V];
    if constexpr (PK) {
#pragma unroll
      for (int e = 0; e < V; e += 2) {
        const S19 R0 = q_s19<V>(Q[0][PA], Q[0][PB], Q[0][PC], e);
        const S19 R1 = q_s19<V>(Q[0][PA], Q[0][PB], Q[0][PC], e + 1);
        const S19 I0 = q_s19<V>(Q[1][PA], Q[1][PB], Q[1][PC], e);
        const S19 I1 = q_s19<V>(Q[1][PA], Q[1][PB], Q[1][PC], e + 1);
        const S19 X0 = q_s19<V>(Q[2][PA], Q[2][PB], Q[2][PC], e);
        const S19 X1 = q_s19<V>(Q[2][PA], Q[2][PB], Q[2][PC], e + 1);
        const F2 mk = pk(mask[e], mask[e + 1]);
        const F2 ab = fsub(cst<F2>(1.0f), mk);
        F2 rpv = pk(rp.v[e], rp.v[e + 1]), ipv = pk(ip.v[e], ip.v[e + 1]);
        if (a.damp_prev) {
          rpv = fmul(rpv, ab);
          ipv = fmul(ipv, ab);
        }
        const ComplexOutT<F2> o = complex_cell_ab(
            lap19_pair(R0, R1), pk(R0.c, R1.c), rpv, pk_faces(faces_of(R0), faces_of(R1)),
            lap19_pair(I0, I1), pk(I0.c, I1.c), ipv, pk_faces(faces_of(I0), faces_of(I1)),
            lap19_pair(X0, X1), pk(X0.c, X1.c), pk(xp.v[e], xp.v[e + 1]), mk, ab, a.c);
        o_r[e] = o.pr.v.x; o_r[e + 1] = o.pr.v.y;
        o_i[e] = o.pi.v.x; o_i[e + 1] = o.pi.v.y;
        o_c[e] = o.chi.v.x; o_c[e + 1] = o.chi.v.y;
        o_rp[e] = o.pr_prev.v.x; o_rp[e + 1] = o.pr_prev.v.y;
        o_ip[e] = o.pi_prev.v.x; o_ip[e + 1] = o.pi_prev.v.y;
        o_cp[e] = o.chi_prev.v.x; o_cp[e + 1] = o.chi_prev.v.y;
      }
    } else {
#pragma unroll
    for (int e = 0; e < V; ++e) {
      const S19 R = q_s19<V>(Q[0][PA], Q[0][PB], Q[0][PC], e);
      const S19 I = q_s19<V>(Q[1][PA], Q[1][PB], Q[1][PC], e);
      const S19 X = q_s19<V>(Q[2][PA], Q[2][PB], Q[2][PC], e);
      const float rpv = a.damp_prev ? fmul(rp.v[e], absorb[e]) : rp.v[e];
      const float ipv = a.damp_prev ? fmul(ip.v[e], absorb[e]) : ip.v[e];
      const ComplexOut o = complex_cell(lap19(R), R.c, rpv, faces_of(R), lap19(I), I.c, ipv,
                                        faces_of(I), lap19(X), X.c, xp.v[e], mask[e], a.c);
      o_r[e] = o.pr; o_i[e] = o.pi; o_c[e] = o.chi;
      o_rp[e] = o.pr_prev; o_ip[e] = o.pi_prev; o_cp[e] = o.chi_prev;
    }
    }
    stg<V>(a.pr_out + gofs, o_r);
    stg<V>(a.pi_out + gofs, o_i);
    stg<V>(a.chi_out + gofs, o_c);
    if (a.pr_prev_out) stg<V>(a.pr_prev_out + gofs, o_rp);
    if (a.pi_prev_out) stg<V>(a.pi_prev_out + gofs, o_ip);
    if (a.chi_prev_out) stg<V>(a.chi_prev_out + gofs, o_cp);
  }
  }  // active
  // Release the centre plane's stage (u = c+1); the last warp refills it
  // with u = c+1+S.
  __syncwarp();
  if ((threadIdx.x & 31) == 0) {
    const uint32_t before = atom_add_acq_rel_cta(&sh.done[s_cur], 1u);
    if (before == (uint32_t)(nwarps - 1)) {
      sh.done[s_cur] = 0u;
      fence_proxy_async_smem();
      if (c + 1 + g.S < nplanes) {
        issue_plane<G::kSlab, true, kOneCopy<LEVEL, MODE>>(P, smem, bars, c + 1 + g.S, i0, i1, j0);
        atomicMax(&sh.issued, c + 2 + g.S);
      }
    }
  }
  __syncwarp();
  if constexpr (SNXT >= 0) {
    if (SNXT == 2) ph_nxt ^= 1u;  // the next plane's stage wraps to 0
  } else {
    s_cur_rt = s_nxt_rt;
    s_nxt_rt = (s_nxt_rt + 1 == g.S) ? 0 : s_nxt_rt + 1;
    if (s_nxt_rt == 0) ph_nxt ^= 1u;
  }
  return true;
}

// The march of one tile: rows j0 .. j0+rows-1 (all k), planes [i0, i1).
// Initialises the stage barriers and the bookkeeping itself, so a CTA may
// run several marches one after another (the batch kernel).
template <int LEVEL, int V, int MODE, bool PARTIAL, class G = GeomRT>
__device__ __forceinline__ void q_march(const TmaParams& P, float* smem, uint64_t* bars,
                                        QShared& sh, int j0, int i0, int i1, int rows) {
  constexpr int NS = QFields<LEVEL, MODE>::ns;
  const G g(P);
  const int N = g.N, TJ = g.TJ, S = g.S;
  const int n = i1 - i0;
  const int nplanes = n + 2;
  const int tid = threadIdx.x;
  const int nwarps = blockDim.x >> 5;
  const int tpr = N / V;
  const bool active = !PARTIAL || tid < rows * tpr;
  const int r = active ? tid / tpr : 0;
  const int k0 = active ? (tid % tpr) * V : 0;
  const int km1 = (k0 == 0) ? N - 1 : k0 - 1;
  const int kpv = (k0 + V == N) ? 0 : k0 + V;
  QLane L;
  L.j = j0 + r;
  L.k0 = k0;
  L.o_m = r * N + k0;
  L.o_z = (r + 1) * N + k0;
  L.o_p = (r + 2) * N + k0;
  L.o_zl = (r + 1) * N + km1;
  L.o_zr = (r + 1) * N + kpv;
  L.o_ml = r * N + km1;
  L.o_mr = r * N + kpv;
  L.o_pl = (r + 2) * N + km1;
  L.o_pr = (r + 2) * N + kpv;
  L.o_pt = NS * (TJ + 2) * N + r * N + k0;
  QKeys<V> K;
  sponge_key<V>(K, P.a.lut, j0 + r, k0, N);

  __syncthreads();  // a previous march in this CTA is over in every warp
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&bars[s], 1);
      sh.done[s] = 0u;
    }
    sh.abort_flag = 0;
    sh.issued = 0;
    mbar_init_fence();
  }
  __syncthreads();
  // The sponge table in shared memory (tab_at = offset of tab[0], < 0 when it
  // is read through L1): the copy engine moves the whole 16-byte groups of a
  // 16-byte aligned table, completing on stage 0's barrier together with
  // plane i0-1; threads store the rest and the two guards.  The barrier
  // before the march orders them before the first lookup.
  const int tab_at = G::kFixed ? G::TAB : (G::kTabMode < 0 ? -1 : P.tab_off);
  int tab_bulk = 0;
  if (tab_at >= 0 && (reinterpret_cast<uintptr_t>(P.a.lut.table) & 15u) == 0)
    tab_bulk = P.a.lut.count & ~3;
  if (tid == 0) {
    // a previous march of this CTA read this shared memory (generic proxy)
    fence_proxy_async_smem();
    if (tab_bulk > 0) {
      mbar_add_tx(&bars[0], 4u * (uint32_t)tab_bulk);
      bulk_copy_g2s(smem + tab_at + 1, P.a.lut.table, 4u * (uint32_t)tab_bulk, &bars[0]);
    }
    const int first = min(S, nplanes);
    for (int u = 0; u < first; ++u)
      issue_plane<G::kSlab, true, kOneCopy<LEVEL, MODE>>(P, smem, bars, u, i0, i1, j0);
    sh.issued = first;
  }
  if (tab_at >= 0) {
    float* tab = smem + tab_at;
    const int cnt = P.a.lut.count;
    for (int t = tab_bulk + tid; t < cnt; t += blockDim.x) tab[1 + t] = __ldg(P.a.lut.table + t);
    if (tid == 0) {
      tab[0] = 0.0f;
      tab[cnt + 1] = 1.0f;
    }
  }
  QPlane<V> Q[NS][3];
  // planes i0-1 (u = 0, stage 0) and i0 (u = 1, stage 1): both first uses, parity 0
  bool ok = mbar_wait_bounded(&bars[0], 0u, kWaitLimitNs);
  ok = mbar_wait_bounded(&bars[1 % S], 0u, kWaitLimitNs) && ok;
  if (!ok) {
    sh.abort_flag = 1;
    atomicOr(P.a.status, LFM_ERR_DEVICE_TIMEOUT);
  } else if (active) {
#pragma unroll
    for (int f = 0; f < NS; ++f) {
      q_load<V>(Q[f][0], smem, 0 * g.SF + f * (TJ + 2) * N, L);
      q_load<V>(Q[f][1], smem, (1 % S) * g.SF + f * (TJ + 2) * N, L);
    }
  }
  __syncthreads();
  if (!sh.abort_flag) {
    // stage 0 (plane i0-1) is dead: refill it with u = S
    if (tid == 0 && S < nplanes) {
      fence_proxy_async_smem();
      issue_plane<G::kSlab, true, kOneCopy<LEVEL, MODE>>(P, smem, bars, S, i0, i1, j0);
      sh.issued = S + 1;
    }
    int s_cur = 1 % S, s_nxt = 2 % S;
    uint32_t ph_nxt = (uint32_t)((2 / S) & 1);
    int c = 0;
    // With a fixed 3-stage geometry, unrolled position p of the loop always
    // has its centre plane in stage (p + 1) % 3 and the next in (p + 2) % 3.
    constexpr bool F = G::kStages == 3;
    while (true) {
      if (c >= n || !q_plane<LEVEL, V, MODE, PARTIAL, 0, 1, 2, G, F ? 1 : -1, F ? 2 : -1>(
                        P, smem, bars, sh, Q, L, c, i0, i1, j0, nplanes, nwarps, s_cur, s_nxt,
                        ph_nxt, K, active))
        break;
      if (++c >= n || !q_plane<LEVEL, V, MODE, PARTIAL, 1, 2, 0, G, F ? 2 : -1, F ? 0 : -1>(
                          P, smem, bars, sh, Q, L, c, i0, i1, j0, nplanes, nwarps, s_cur, s_nxt,
                          ph_nxt, K, active))
        break;
      if (++c >= n || !q_plane<LEVEL, V, MODE, PARTIAL, 2, 0, 1, G, F ? 0 : -1, F ? 1 : -1>(
                          P, smem, bars, sh, Q, L, c, i0, i1, j0, nplanes, nwarps, s_cur, s_nxt,
                          ph_nxt, K, active))
        break;
      ++c;
    }
  }
  if (*(volatile int*)&sh.abort_flag && (tid & 31) == 0) {
    // The last use of each stage is the only one that can still be in flight;
    // let it land before this CTA's shared memory is reused or released.
    const int issued = *(volatile int*)&sh.issued;
    for (int u = max(0, issued - S); u < issued; ++u)
      mbar_wait_bounded(&bars[u % S], (uint32_t)((u / S) & 1), kDrainLimitNs);
  }
}

template <int LEVEL, int V, int MODE, class G = GeomRT>
__global__ void __launch_bounds__(512) tma_queue_kernel(const __grid_constant__ TmaParams P) {
  extern __shared__ __align__(128) float smem[];
  __shared__ __align__(8) uint64_t bars[kMaxStages];
  __shared__ QShared sh;
  const G g(P);
  const int jt = blockIdx.x % P.JT, ch = blockIdx.x / P.JT;
  const bool slab = G::kSlab && P.a.slab;
  const int lo = slab ? P.a.i_lo : 0, hi = slab ? P.a.i_hi : g.N;
  const int i0 = lo + ch * P.IC;
  q_march<LEVEL, V, MODE, false, G>(P, smem, bars, sh, jt * g.TJ, i0, min(i0 + P.IC, hi), g.TJ);
}

// ---- batch kernel: many lattices, one launch per step -------------------------
//
// Persistent CTAs take (lattice, row tile, plane chunk) items from a work list
// sorted by cost, through a device counter (largest first, next free CTA takes
// the next item), and run the same barrier-free march on each.  REAL and
// COMPLEX items share the launch.  The per-item parameters (slot pointers for
// this step's parity, constants, mask table, tile shape) are built in shared
// memory from the lattice descriptor.  The last CTA to retire rewinds the
// counters for the next launch on the stream.
// rows: the item's tile rows (the lattice's TJ or one fewer)
template <int LEVEL>
__device__ __forceinline__ void batch_params(TmaParams& P, const BatchLattice& L,
                                             const BatchParams& B, int rows) {
  const int cur = B.parity, nxt = 1 - B.parity;
  StepArgs a{};
  a.level = LEVEL;
  a.N = L.N;
  a.c = L.c;
  a.pr = L.pr[cur];
  a.pr_prev = L.pr[nxt];
  a.pr_out = L.pr[nxt];
  a.chi = L.chi[cur];
  a.chi_prev = L.chi[nxt];
  a.chi_out = L.chi[nxt];
  if (LEVEL == LFM_COMPLEX) {
    a.pi = L.pi[cur];
    a.pi_prev = L.pi[nxt];
    a.pi_out = L.pi[nxt];
  }
  a.lut = L.lut;
  a.damp_prev = B.damp_prev;
  a.status = B.status;
  P.a = a;
  if (LEVEL == LFM_REAL) {
    P.ns = 2;
    P.sf[0] = a.pr; P.sf[1] = a.chi;
    P.np = 2;
    P.pf[0] = a.pr_prev; P.pf[1] = a.chi_prev;
  } else {
    P.ns = 3;
    P.sf[0] = a.pr; P.sf[1] = a.pi; P.sf[2] = a.chi;
    P.np = 3;
    P.pf[0] = a.pr_prev; P.pf[1] = a.pi_prev; P.pf[2] = a.chi_prev;
  }
  P.pf_mask = -1;
  P.pf_sa = -1;
  P.N = L.N;
  P.TJ = rows;
  P.TJL = L.TJ;  // a shorter tile keeps the lattice's stage layout
  P.IC = L.IC;
  P.S = B.stages;
  P.JT = (L.N + L.TJ - 1) / L.TJ;
  P.stage_floats = L.stage_floats;
  P.tab_off = B.tab_off;  // after the largest ring of the batch, or -1
}

// The item loop of one shape class: CTAs take the class's items through its
// counter and march each with the class's geometry G.
template <int LEVEL, int V, class G>
__device__ __forceinline__ void batch_class(const BatchParams& B, const BatchItem* items,
                                            int nitems, int* next_item, float* smem,
                                            uint64_t* bars, QShared& sh, TmaParams& P,
                                            int& s_item) {
  while (true) {
    __syncthreads();  // every warp is done with the previous item
    if (threadIdx.x == 0) s_item = atomicAdd(next_item, 1);
    __syncthreads();
    const int w = s_item;
    if (w >= nitems) break;
    const BatchItem it = items[w];
    if (threadIdx.x == 0) {
      const BatchLattice& L = B.lattices[it.lattice];
      batch_params<LEVEL>(P, L, B, it.j1 - it.j0);
    }
    __syncthreads();  // P is visible to every thread
    q_march<LEVEL, V, kPlain, true, G>(P, smem, bars, sh, it.j0, it.i0, it.i1, P.TJ);
    __syncthreads();  // every wait of the march is over
    if (sh.abort_flag) break;  // same value in every thread
    if (threadIdx.x == 0)
      for (int s = 0; s < B.stages; ++s) mbar_inval(&bars[s]);  // the next march re-initialises
  }
}

template <int C, int TABM>
__device__ __forceinline__ void batch_run_class(const BatchParams& B, float* smem,
                                                uint64_t* bars, QShared& sh, TmaParams& P,
                                                int& s_item) {
  constexpr BatchShape K = kBatchShapes[C];
  constexpr int V = K.level == LFM_REAL ? 4 : 2;
  // (the GeomBT arguments of a run-time class are placeholders: that branch is not taken)
  using G = std::conditional_t<K.N == 0, GeomRTT<TABM>,
                               GeomBT<(K.N ? K.N : 4), (K.TJ ? K.TJ : 1),
                                      QFields<K.level>::ns, TABM>>;
  __syncthreads();
  if (!sh.abort_flag && B.class_n[C] > 0)
    batch_class<K.level, V, G>(B, B.items + B.class_off[C], B.class_n[C], B.next_item + C,
                               smem, bars, sh, P, s_item);
  if constexpr (C + 1 < kBatchClasses) batch_run_class<C + 1, TABM>(B, smem, bars, sh, P, s_item);
}

// Every CTA drains the shape classes (kBatchShapes) in order, each through
// its own loop with its own geometry: a CTA done with one class starts on
// the next at once, so the launch has a single tail (the smallest COMPLEX
// items).  The class loops run one after the other, so their register
// demands do not add up.  TABM: the sponge tables in shared memory
// (1, B.tab_off >= 0) or through L1 (-1).  The explicit one block per SM in
// the launch bounds keeps ptxas at 128 registers: without it, for a kernel
// this size, it allocated 64 and spilled kilobytes per thread.
template <int TABM>
__global__ void __launch_bounds__(512, 1) tma_batch_kernel(const __grid_constant__ BatchParams B) {
  extern __shared__ __align__(128) float smem[];
  __shared__ __align__(8) uint64_t bars[kMaxStages];
  __shared__ QShared sh;
  __shared__ TmaParams P;
  __shared__ int s_item;
  sh.abort_flag = 0;
  batch_run_class<0, TABM>(B, smem, bars, sh, P, s_item);
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(B.retired, 1) == (int)gridDim.x - 1) {
      // every CTA has taken its last item: rewind for the next launch
      for (int c = 0; c < kBatchClasses; ++c) atomicExch(B.next_item + c, 0);
      atomicExch(B.retired, 0);
    }
  }
}

// ---- host side -------------------------------------------------------------------
struct Choice {
  int TJ = 0, S = 0, IC = 0, threads = 0, smem = 0;
};

// Dynamic shared memory a configuration may use: the 227 KB opt-in limit
// less 1 KB for the kernel's static shared memory (mbarriers, abort flag).
constexpr int kSmemLimit = 226 * 1024;

int stage_bytes(int N, int TJ, int ns, int np) { return 4 * N * (ns * (TJ + 2) + np * TJ); }

// Shared-memory carveouts an SM can be configured with (KB); the rest of the
// 256 KB L1/shared array is L1 cache, which holds the sponge lookup table.
int carveout_kb(int bytes) {
  static const int kCarve[] = {0, 8, 16, 32, 64, 100, 132, 164, 196, 228};
  for (int c : kCarve)
    if (bytes <= c * 1024) return c;
  return 228;
}

// extra_smem: bytes of shared memory beyond the stage ring (the mask table
// when it is staged there); l1_table_bytes: a table read through L1 that the
// carveout must leave room for (0 when none).
Choice choose(int level, int N, int V, int ns, int np, bool queue, int max_threads,
              int regs, const TileConfig* forced, int extra_smem, int l1_table_bytes,
              int planes = 0) {
  if (planes <= 0) planes = N;  // planes the march covers (a slab's own planes)
  Choice best;
  double best_score = -1.0;
  const int tpr = N / V;
  const int min_s = queue ? 3 : 4;  // stages live at once: 2 (queue) or 3
  for (int TJ = 1; TJ <= N; ++TJ) {
    if (N % TJ) continue;
    const int threads = TJ * tpr;
    if (threads % 32 || threads < 64 || threads > max_threads) continue;
    for (int S = min_s; S <= kMaxStages; ++S) {
      const int smem = S * stage_bytes(N, TJ, ns, np) + extra_smem;
      if (smem > kSmemLimit) continue;
      if (forced && (forced->tj != TJ || forced->stages != S)) continue;
      const int cta_by_smem = (228 * 1024) / (smem + 1024);
      const int cta_by_thr = 2048 / threads;
      const int cta_by_reg = 65536 / std::max(1, regs * threads);
      const int ctas = std::max(1, std::min(std::min(cta_by_smem, cta_by_thr), cta_by_reg));
      const double warps = std::min(ctas * threads / 32, 48);
      const double halo = (double)TJ / (TJ + 2);  // useful fraction of stencil rows
      // planes streamed ahead; the register-queue kernels measured no gain
      // from a second plane in flight (3 vs 4 stages at 256^3 and 512^3), so
      // their bonus stops at one and the smaller ring wins the tie
      const double depth = std::min(S - (min_s - 1), queue ? 1 : 2) / 2.0;
      // L1 left beside the shared-memory carveout must hold the mask table
      const int l1_kb = 256 - carveout_kb(ctas * (smem + 1024));
      // (measured at 512^3: a 60-92 KB L1 beside the 67 KB table runs 10-15% slower)
      const bool table_fits = l1_table_bytes == 0 || l1_kb * 1024 >= l1_table_bytes + 48 * 1024;
      // The barrier kernel (COLOR) waits for the whole CTA once per plane; a
      // second CTA on the SM computes meanwhile.  Measured at COLOR 256^3 with
      // S_a: 2 rows x 4 stages, two 256-thread CTAs per SM, 1.082 ms per step
      // against 1.112 for 4 rows x 5 stages (one 512-thread CTA); at 128^3
      // and 64^3 the two shapes were within noise.
      const double overlap = (!queue && ctas >= 2) ? 0.3 : 0.0;
      const double score =
          warps / 48.0 + 0.6 * halo + 0.25 * depth + (table_fits ? 0.5 : 0.0) + overlap;
      if (score > best_score) {
        best_score = score;
        best.TJ = TJ;
        best.S = S;
        best.threads = threads;
        best.smem = smem;
      }
    }
  }
  if (!best.TJ) return best;
  const int JT = N / best.TJ;
  const int ctas = std::max(1, std::min(std::min((228 * 1024) / (best.smem + 1024),
                                                 2048 / best.threads),
                                        65536 / std::max(1, regs * best.threads)));
  if (forced && forced->ic > 0) {
    best.IC = std::min(forced->ic, planes);
  } else {
    // Planes per chunk: minimise waves x (pipeline fill + (IC + 2) planes).
    // A CTA streams one plane of TJ x N cells in t_plane, no faster than the
    // ring's S - 2 planes in flight allow; per-SM rates measured at 512^3
    // (REAL, 0.97 kcell/us) and 256^3 (COMPLEX, 0.46).  Large lattices end up
    // balancing their last wave, small ones (latency-bound) take short
    // chunks and many CTAs.
    const double slots = 148.0 * ctas;
    const double r_sm = (level == LFM_REAL) ? 0.97e3 : (level == LFM_COMPLEX ? 0.46e3 : 0.2e3);
    const double t_fill = 2.0, t_lat = 1.5;  // us
    const double t_plane = std::max((double)best.TJ * N * ctas / r_sm,
                                    t_lat / std::max(1, best.S - (min_s - 1)));
    double best_t = 1e300;
    for (int chunks = 1; chunks <= std::max(1, planes / 2); ++chunks) {
      const int ic = (planes + chunks - 1) / chunks;
      const double waves = std::ceil((double)JT * chunks / slots);
      const double t = waves * (t_fill + (ic + 2) * t_plane);
      if (t < best_t * (1.0 - 1e-9)) {
        best_t = t;
        best.IC = ic;
      }
    }
  }
  return best;
}

template <typename K>
cudaError_t kernel_regs(K kernel, int* regs) {
  cudaFuncAttributes fa{};
  cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
  *regs = fa.numRegs;
  return e;
}

// Raises the kernel's dynamic shared-memory limit to what the launch needs
// (within the device's opt-in limit less its static shared memory) and launches.
template <typename K>
cudaError_t launch_kernel(K kernel, int* granted, std::mutex* mu, const TmaParams& P,
                          const Choice& ch, cudaStream_t stream) {
  {
    std::lock_guard<std::mutex> lk(*mu);
    if (ch.smem > *granted) {
      int dev = 0, optin = 0;
      cudaError_t e = cudaGetDevice(&dev);
      if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
      cudaFuncAttributes fa{};
      if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, kernel);
      if (e != cudaSuccess) return e;
      if (ch.smem + (int)fa.sharedSizeBytes > optin) return cudaErrorNotSupported;
      e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, ch.smem);
      if (e != cudaSuccess) return e;
      *granted = ch.smem;
    }
  }
  const int JT = P.N / P.TJ;
  const int planes = P.a.slab ? P.a.i_hi - P.a.i_lo : P.N;
  const int chunks = (planes + P.IC - 1) / P.IC;
  kernel<<<JT * chunks, ch.threads, ch.smem, stream>>>(P);
  return cudaGetLastError();
}

template <int LEVEL, int V, bool QUEUE, int MODE>
struct KernelSlot {
  static std::mutex mu;
  static int granted;
  static auto fn() {
    if constexpr (QUEUE)
      return tma_queue_kernel<LEVEL, V, MODE>;
    else
      return tma_step_kernel<LEVEL, V>;
  }
};
template <int LEVEL, int V, bool QUEUE, int MODE>
std::mutex KernelSlot<LEVEL, V, QUEUE, MODE>::mu;
template <int LEVEL, int V, bool QUEUE, int MODE>
int KernelSlot<LEVEL, V, QUEUE, MODE>::granted = 0;

// Compile-time tiles for the headline sizes (resident layout); MODE kComp:
// the compensated (Delta-form) step on the same tile.
template <int LEVEL, int V, int N, int TJ, int S, int MODE = kPlain, bool SLAB = false>
struct FixedSlot {
  static std::mutex mu;
  static int granted;
  static auto fn() {
    using F = QFields<LEVEL, MODE>;
    return tma_queue_kernel<LEVEL, V, MODE, GeomCT<N, TJ, F::ns, S, SLAB, F::np>>;
  }
};
template <int LEVEL, int V, int N, int TJ, int S, int MODE, bool SLAB>
std::mutex FixedSlot<LEVEL, V, N, TJ, S, MODE, SLAB>::mu;
template <int LEVEL, int V, int N, int TJ, int S, int MODE, bool SLAB>
int FixedSlot<LEVEL, V, N, TJ, S, MODE, SLAB>::granted = 0;

// The compile-time tiles: step form, level, cells per lane, N, rows, stages.
// The compensated step has one at the throughput size; split chi at 256^3 and
// 512^3, two cells per lane (its ring adds chi's lo and lo_prev as point fields).
struct FixedTile {
  int mode, level, V, N, TJ, S;
};
constexpr FixedTile kFixedTiles[] = {
    {kPlain, LFM_REAL, 4, 512, 4, 3},    {kPlain, LFM_REAL, 4, 256, 8, 3},
    {kPlain, LFM_COMPLEX, 2, 512, 2, 3}, {kPlain, LFM_COMPLEX, 2, 256, 4, 3},
    {kPlain, LFM_REAL, 4, 128, 8, 3},    {kPlain, LFM_COMPLEX, 2, 128, 4, 3},
    {kComp, LFM_REAL, 4, 512, 4, 3},     {kSplit, LFM_REAL, 2, 512, 2, 3},
    {kSplit, LFM_REAL, 2, 256, 4, 3},    {kSplit, LFM_COMPLEX, 2, 512, 2, 3},
    {kSplit, LFM_COMPLEX, 2, 256, 4, 3}};

// The stage count of the compile-time tile (mode, level, V, N, TJ); 0 if none.
constexpr int fixed_stages(int mode, int level, int V, int N, int TJ) {
  for (const FixedTile& t : kFixedTiles)
    if (t.mode == mode && t.level == level && t.V == V && t.N == N && t.TJ == TJ) return t.S;
  return 0;
}

// The fixed tile for (mode, level, V, N), if any.
const FixedTile* fixed_tile(int mode, int level, int V, int N) {
  for (const FixedTile& t : kFixedTiles)
    if (t.mode == mode && t.level == level && t.V == V && t.N == N) return &t;
  return nullptr;
}

template <int LEVEL, int V, int N, int TJ, int MODE = kPlain, bool SLAB = false>
cudaError_t launch_fixed(TmaParams& P, const Choice& ch, cudaStream_t stream) {
  using Slot = FixedSlot<LEVEL, V, N, TJ, fixed_stages(MODE, LEVEL, V, N, TJ), MODE, SLAB>;
  return launch_kernel(Slot::fn(), &Slot::granted, &Slot::mu, P, ch, stream);
}

// Shared memory of the sponge table of the compile-time tiles: count entries
// between a 0 and a 1, after 3 floats of padding that put the first entry on a
// 16-byte boundary, rounded up to 16 bytes.
int sponge_table_bytes(int count) { return (4 * (count + 5) + 15) / 16 * 16; }

// Launches the compile-time variant when the chosen tile is one of
// kFixedTiles (no streamed mask or S_a) and its ring plus the sponge table fit
// in shared memory (ch.smem includes the table then); false if not.
template <int LEVEL, int V, int MODE = kPlain>
bool try_fixed(TmaParams& P, const Choice& ch, cudaStream_t stream, cudaError_t* err) {
  if (P.np != QFields<LEVEL, MODE>::np || P.ns != QFields<LEVEL, MODE>::ns || P.pf_mask >= 0 ||
      P.pf_sa >= 0)
    return false;
  const FixedTile* t = fixed_tile(MODE, LEVEL, V, P.N);
  if (!t || t->TJ != ch.TJ || t->S != ch.S) return false;
  if (ch.smem != t->S * stage_bytes(P.N, ch.TJ, P.ns, P.np) + sponge_table_bytes(P.a.lut.count))
    return false;
  if (P.a.slab) {
    // a rank's slab of a lattice split along i: the plain 512^3 tiles
    if constexpr (MODE == kPlain && LEVEL == LFM_REAL && V == 4) {
      if (P.N == 512) { *err = launch_fixed<LEVEL, V, 512, 4, kPlain, true>(P, ch, stream); return true; }
    } else if constexpr (MODE == kPlain && LEVEL == LFM_COMPLEX && V == 2) {
      if (P.N == 512) { *err = launch_fixed<LEVEL, V, 512, 2, kPlain, true>(P, ch, stream); return true; }
    }
    return false;
  }
  if constexpr (MODE == kSplit) {
    if constexpr (V == 2) {
      if (P.N == 512) { *err = launch_fixed<LEVEL, V, 512, 2, kSplit>(P, ch, stream); return true; }
      if (P.N == 256) { *err = launch_fixed<LEVEL, V, 256, 4, kSplit>(P, ch, stream); return true; }
    }
    return false;
  } else if constexpr (MODE == kComp) {
    if constexpr (LEVEL == LFM_REAL && V == 4) {
      *err = launch_fixed<LEVEL, V, 512, 4, kComp>(P, ch, stream);
      return true;
    }
    return false;
  } else if constexpr (LEVEL == LFM_REAL && V == 4) {
    if (P.N == 512) { *err = launch_fixed<LEVEL, V, 512, 4>(P, ch, stream); return true; }
    if (P.N == 256) { *err = launch_fixed<LEVEL, V, 256, 8>(P, ch, stream); return true; }
    if (P.N == 128) { *err = launch_fixed<LEVEL, V, 128, 8>(P, ch, stream); return true; }
  } else if constexpr (LEVEL == LFM_COMPLEX && V == 2) {
    if (P.N == 512) { *err = launch_fixed<LEVEL, V, 512, 2>(P, ch, stream); return true; }
    if (P.N == 256) { *err = launch_fixed<LEVEL, V, 256, 4>(P, ch, stream); return true; }
    if (P.N == 128) { *err = launch_fixed<LEVEL, V, 128, 4>(P, ch, stream); return true; }
  }
  return false;
}

template <int LEVEL, int V, bool QUEUE, int MODE = kPlain>
cudaError_t plan_and_launch(TmaParams& P, const TileConfig* forced, cudaStream_t stream) {
  using Slot = KernelSlot<LEVEL, V, QUEUE, MODE>;
  int regs = 0;
  cudaError_t e = kernel_regs(Slot::fn(), &regs);
  if (e != cudaSuccess) return e;
  // threads per CTA the register file can hold (at least one CTA per SM)
  const int max_threads = std::min(512, (65536 / std::max(regs, 1)) / 32 * 32);
  // The register-queue kernels keep the sponge table in shared memory after
  // the ring when it fits (tab_smem); otherwise they read it through L1, and
  // the carveout must leave L1 room for it (table_bytes).
  const int count = (P.pf_mask >= 0) ? 0 : P.a.lut.count;
  const int table_bytes = 4 * count;
  const bool want_tab = QUEUE && P.pf_mask < 0;
  const int tab_smem = want_tab ? sponge_table_bytes(count) : 0;
  // Without a forced tile, the sizes with a compile-time variant take its
  // tile (TJ rows, S stages) when its ring and the sponge table fit in shared
  // memory; the planner still picks the plane chunk.
  TileConfig fixed_cfg;
  const bool slab_tile = !P.a.slab || (MODE == kPlain && P.N == 512);  // slab variants: 512^3
  const bool resident = P.ns == QFields<LEVEL, MODE>::ns && P.np == QFields<LEVEL, MODE>::np;
  const FixedTile* ft = (QUEUE && P.pf_mask < 0 && P.pf_sa < 0 && resident && slab_tile)
                            ? fixed_tile(MODE, LEVEL, V, P.N) : nullptr;
  if (ft && ft->S * stage_bytes(P.N, ft->TJ, P.ns, P.np) + tab_smem > kSmemLimit) ft = nullptr;
  if (!forced && ft) {
    fixed_cfg = TileConfig{ft->TJ, ft->S, 0, 0, 0, V};
    forced = &fixed_cfg;
  }
  const int planes = P.a.slab ? P.a.i_hi - P.a.i_lo : P.N;
  bool tab_in_smem = want_tab;
  const int np_staged = QUEUE ? P.np : 0;  // the barrier kernel reads point fields from global
  Choice ch = choose(LEVEL, P.N, V, P.ns, np_staged, QUEUE, max_threads, regs, forced, tab_smem,
                     0, planes);
  if (!ch.TJ && want_tab) {  // the table does not fit beside any ring: through L1
    tab_in_smem = false;
    ch = choose(LEVEL, P.N, V, P.ns, np_staged, QUEUE, max_threads, regs, forced, 0,
                table_bytes, planes);
  }
  if (!ch.TJ) return cudaErrorNotSupported;
  P.TJ = ch.TJ;
  P.TJL = ch.TJ;
  P.S = ch.S;
  P.IC = ch.IC;
  P.JT = P.N / ch.TJ;
  P.stage_floats = stage_bytes(P.N, ch.TJ, P.ns, np_staged) / 4;
  // tab[1] lands on a 16-byte boundary: stage_floats is a multiple of N, N of 4
  P.tab_off = tab_in_smem ? ch.S * P.stage_floats + 3 : -1;
  TileConfig used{ch.TJ, ch.S, ch.IC, ch.threads, ch.smem, V};
  tune_record(LEVEL, P.N, used);
  if constexpr (QUEUE) {
    cudaError_t fe = cudaSuccess;
    if (try_fixed<LEVEL, V, MODE>(P, ch, stream, &fe)) return fe;
  }
  return launch_kernel(Slot::fn(), &Slot::granted, &Slot::mu, P, ch, stream);
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace

namespace {

// One CTA waits on an mbarrier that nothing arrives at, through the bounded
// wait of the step kernels: the wait gives up after limit_ns and records
// LFM_ERR_DEVICE_TIMEOUT in the status word, and the kernel returns.
__global__ void wait_selftest_kernel(int* status, uint64_t limit_ns) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_init_fence();
  }
  __syncthreads();
  if (!mbar_wait_bounded(&bar, 0u, limit_ns)) atomicOr(status, LFM_ERR_DEVICE_TIMEOUT);
}

}  // namespace

cudaError_t launch_wait_selftest(int* status, uint64_t limit_ns, cudaStream_t stream) {
  wait_selftest_kernel<<<1, 32, 0, stream>>>(status, limit_ns);
  return cudaGetLastError();
}

cudaError_t launch_tma_step(const StepArgs& a, cudaStream_t stream) {
  const int N = a.N;
  if (N % 4 != 0 || N < 8) return cudaErrorNotSupported;
  TmaParams P{};
  P.a = a;
  P.N = N;
  P.pf_mask = -1;
  P.tab_off = -1;  // set by the planner when the table goes to shared memory
  P.pf_sa = -1;
  const int64_t n3 = (int64_t)N * N * N;
  if (a.split) {
    // split chi: stencil fields Psi..., hi; point fields their previous slots,
    // then lo and lo_prev
    if (a.level == LFM_COLOR || a.comp || a.mask || !a.chi_lo || !a.chi_lo_prev ||
        !a.chi_lo_out)
      return cudaErrorNotSupported;
    int f = 0;
    P.sf[f] = a.pr; P.pf[f++] = a.pr_prev;
    if (a.level == LFM_COMPLEX) { P.sf[f] = a.pi; P.pf[f++] = a.pi_prev; }
    P.sf[f] = a.chi; P.pf[f++] = a.chi_prev;
    P.ns = f;
    P.pf[f++] = a.chi_lo;
    P.pf[f++] = a.chi_lo_prev;
    P.np = f;
  } else if (a.level == LFM_REAL) {
    P.ns = 2;
    P.sf[0] = a.pr; P.sf[1] = a.chi;
    P.pf[0] = a.pr_prev; P.pf[1] = a.chi_prev;
    P.np = 2;
  } else if (a.level == LFM_COMPLEX) {
    P.ns = 3;
    P.sf[0] = a.pr; P.sf[1] = a.pi; P.sf[2] = a.chi;
    P.pf[0] = a.pr_prev; P.pf[1] = a.pi_prev; P.pf[2] = a.chi_prev;
    P.np = 3;
  } else {
    P.ns = 7;
    for (int c = 0; c < 3; ++c) {
      P.sf[c] = a.pr + c * n3;
      P.sf[3 + c] = a.pi + c * n3;
      P.pf[c] = a.pr_prev + c * n3;
      P.pf[3 + c] = a.pi_prev + c * n3;
    }
    P.sf[6] = a.chi;
    P.pf[6] = a.chi_prev;
    P.np = 7;
  }
  if (a.mask) {
    P.pf_mask = P.np;
    P.pf[P.np++] = a.mask;
  }
  if (a.level == LFM_COLOR && a.sa) {
    P.pf_sa = P.np;
    for (int c = 0; c < 3; ++c) P.pf[P.np++] = a.sa + c * n3;
  }
  // every copy source and every vector store needs 16-byte alignment
  const void* ptrs[] = {a.pr, a.pi, a.chi, a.pr_prev, a.pi_prev, a.chi_prev, a.pr_out, a.pi_out,
                        a.chi_out, a.pr_prev_out, a.pi_prev_out, a.chi_prev_out, a.mask, a.sa,
                        a.sa_clip_out, a.chi_lo, a.chi_lo_prev, a.chi_lo_out, a.energy_out};
  for (const void* p : ptrs)
    if (p && !aligned16(p)) return cudaErrorNotSupported;

  TileConfig forced_cfg;
  const bool have_forced = tune_lookup(a.level, N, &forced_cfg);
  const TileConfig* forced = have_forced ? &forced_cfg : nullptr;
  if (a.split) {
    // split chi: two cells per lane (three or four stencil fields, like COMPLEX)
    if (N % 2) return cudaErrorNotSupported;
    // (a tuning recorded for the plain step's tile does not apply)
    return a.level == LFM_REAL ? plan_and_launch<LFM_REAL, 2, true, kSplit>(P, nullptr, stream)
                               : plan_and_launch<LFM_COMPLEX, 2, true, kSplit>(P, nullptr, stream);
  }
  if (a.comp) {
    // compensated Delta form: REAL and COMPLEX, register-queue kernel only
    if (a.level == LFM_REAL)
      return (N % 4) ? cudaErrorNotSupported
                     : plan_and_launch<LFM_REAL, 4, true, kComp>(P, forced, stream);
    if (a.level == LFM_COMPLEX)
      return (N % 2) ? cudaErrorNotSupported
                     : plan_and_launch<LFM_COMPLEX, 2, true, kComp>(P, forced, stream);
    return cudaErrorNotSupported;
  }
  if (a.level == LFM_REAL) {
    const int v = (have_forced && forced_cfg.vec) ? forced_cfg.vec : 4;
    if ((v != 2 && v != 4) || N % v) return cudaErrorNotSupported;
    return v == 2 ? plan_and_launch<LFM_REAL, 2, true>(P, forced, stream)
                  : plan_and_launch<LFM_REAL, 4, true>(P, forced, stream);
  }
  if (a.level == LFM_COMPLEX) {
    const int v = (have_forced && forced_cfg.vec) ? forced_cfg.vec : 2;
    if ((v != 2 && v != 4) || N % v) return cudaErrorNotSupported;
    return v == 4 ? plan_and_launch<LFM_COMPLEX, 4, true>(P, forced, stream)
                  : plan_and_launch<LFM_COMPLEX, 2, true>(P, forced, stream);
  }
  // COLOR: two cells per lane, or one when a tuning asks for it (twice the
  // warps on the same ring, each with half the independent arithmetic)
  const int vc = (have_forced && forced_cfg.vec) ? forced_cfg.vec : 2;
  if (vc != 1 && vc != 2) return cudaErrorNotSupported;
  return vc == 1 ? plan_and_launch<LFM_COLOR, 1, false>(P, forced, stream)
                 : plan_and_launch<LFM_COLOR, 2, false>(P, forced, stream);
}


// ---- batch launcher -------------------------------------------------------------
namespace {
std::mutex g_batch_mu;
int g_batch_granted[2] = {0, 0};  // dynamic shared memory granted to the two batch kernels

template <typename K>
cudaError_t grant_smem(K kernel, int smem, int* granted) {
  std::lock_guard<std::mutex> lk(g_batch_mu);
  if (smem <= *granted) return cudaSuccess;
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess)
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa{};
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, kernel);
  if (e != cudaSuccess) return e;
  if (smem + (int)fa.sharedSizeBytes > optin) return cudaErrorNotSupported;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e == cudaSuccess) *granted = smem;
  return e;
}
}  // namespace

cudaError_t batch_kernel_regs(int* regs) {
  // the larger of the two variants' demands
  cudaFuncAttributes fa{}, fb{};
  cudaError_t e = cudaFuncGetAttributes(&fa, tma_batch_kernel<1>);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fb, tma_batch_kernel<-1>);
  if (e == cudaSuccess) *regs = std::max(fa.numRegs, fb.numRegs);
  return e;
}

cudaError_t launch_batch_step(const BatchParams& B, int threads, int smem, int grid,
                              cudaStream_t stream) {
  if (B.nitems == 0) return cudaSuccess;
  const bool tab = B.tab_off >= 0;
  auto kernel = tab ? tma_batch_kernel<1> : tma_batch_kernel<-1>;
  cudaError_t e = grant_smem(kernel, smem, &g_batch_granted[tab ? 1 : 0]);
  if (e != cudaSuccess) return e;
  kernel<<<grid, threads, smem, stream>>>(B);
  return cudaGetLastError();
}

}  // namespace lfm
