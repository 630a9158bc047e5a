// C ABI of liblfm_b200.so (declared in include/lfm_b200.h): argument
// checks, kernel-path choice, the sponge lookup table, and the library
// context that owns the cuFFT plans and scratch of the S_a solve.
#include <cufft.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "lfm_b200.h"
#include "lfm_batch.h"
#include "lfm_kernels.h"
#include "lfm_metrics.h"

// Device status word: bounded device-side waits OR an LFM_ERR_* code into
// it when they give up (read back with lfm_device_status).
__device__ int g_lfm_status;

namespace {
__global__ void status_clear_kernel(int bits) { atomicAnd(&g_lfm_status, ~bits); }
}  // namespace

namespace lfm {
cudaError_t launch_status_clear(int bits) {
  status_clear_kernel<<<1, 1>>>(bits);
  return cudaGetLastError();
}
}  // namespace lfm

namespace {

thread_local std::string t_detail;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  t_detail = buf;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  return fail(LFM_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// Kernel path: 0 = choose (fused 2.5D kernel when it applies), 1 = direct
// kernel only, 2 = fused kernel only (LFM_ERR_UNSUPPORTED when it cannot run).
std::atomic<int> g_path{0};
// S_a transform: 1 = split (2-D cuFFT + fused pass along i) where N allows it,
// 0 = 3-D cuFFT with a separate filter pass.  Process-wide; for tests.
std::atomic<int> g_sa_split{1};

constexpr int kMaxDevices = 64;
std::mutex g_status_mu;
int* g_status_ptr[kMaxDevices] = {nullptr};

int status_word(int** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return fail(LFM_ERR_UNSUPPORTED, "device %d", dev);
  std::lock_guard<std::mutex> lk(g_status_mu);
  if (!g_status_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_lfm_status);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_lfm_status)");
    g_status_ptr[dev] = static_cast<int*>(p);
  }
  *out = g_status_ptr[dev];
  return LFM_OK;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int check_n(int N) {
  if (N < 2 || N > 2048) return fail(LFM_ERR_INVALID_ARG, "N=%d outside [2, 2048]", N);
  return LFM_OK;
}

struct Span {
  const void* p;
  size_t bytes;
};

bool overlaps(Span a, Span b) {
  if (!a.p || !b.p) return false;
  const char* a0 = static_cast<const char*>(a.p);
  const char* b0 = static_cast<const char*>(b.p);
  return a0 < b0 + b.bytes && b0 < a0 + a.bytes;
}

int check_disjoint(const std::vector<Span>& ins, const std::vector<Span>& outs) {
  for (size_t o = 0; o < outs.size(); ++o) {
    for (const Span& i : ins)
      if (overlaps(outs[o], i))
        return fail(LFM_ERR_INVALID_ARG, "output buffer %zu overlaps an input buffer", o);
    for (size_t o2 = o + 1; o2 < outs.size(); ++o2)
      if (overlaps(outs[o], outs[o2]))
        return fail(LFM_ERR_INVALID_ARG, "output buffers %zu and %zu overlap", o, o2);
  }
  return LFM_OK;
}

int run_step(lfm::StepArgs& a, cudaStream_t stream) {
  int rc = status_word(&a.status);
  if (rc) return rc;
  const int path = g_path.load();
  cudaError_t e = cudaErrorNotSupported;
  if (path != 1) {
    e = lfm::launch_tma_step(a, stream);
    if (e != cudaSuccess && e != cudaErrorNotSupported) return cuda_fail(e, "fused step launch");
    if (e == cudaErrorNotSupported && path == 2)
      return fail(LFM_ERR_UNSUPPORTED, "no fused-kernel configuration for N=%d level=%d", a.N,
                  a.level);
  }
  if (e == cudaErrorNotSupported) {
    e = lfm::launch_direct_step(a, stream);
    if (e != cudaSuccess) return cuda_fail(e, "direct step launch");
  }
  return LFM_OK;
}

lfm::MaskLut device_lut(const float* table, const lfm_mask_lut* lut) {
  lfm::MaskLut m;
  m.table = table;
  m.shift = lut->shift;
  m.q_lo = lut->q_lo;
  m.q_hi = lut->q_hi;
  m.count = lut->count;
  return m;
}

int check_lut(const float* table, const lfm_mask_lut* lut, int N) {
  if (!lut) return fail(LFM_ERR_INVALID_ARG, "mask lookup table descriptor is null");
  if (lut->N != N)
    return fail(LFM_ERR_INVALID_ARG, "lookup table is for N=%d, step N=%d", lut->N, N);
  if (lut->count > 0 && !table) return fail(LFM_ERR_INVALID_ARG, "mask table pointer is null");
  if (lut->shift != (N % 2 == 0 ? 3 : 2))
    return fail(LFM_ERR_INVALID_ARG, "mask table shift %d does not match N=%d", lut->shift, N);
  const int64_t want = lut->q_hi >= lut->q_lo
                           ? (((int64_t)lut->q_hi - lut->q_lo) >> lut->shift) + 1 : 0;
  if (lut->count != want)
    return fail(LFM_ERR_INVALID_ARG, "mask table count %d, its key band holds %lld", lut->count,
                (long long)want);
  return LFM_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// library context: cuFFT plans + spectrum scratch per lattice edge
// ---------------------------------------------------------------------------
struct FftSlot {
  cufftHandle r2c = 0, c2r = 0;
  float2* spec = nullptr;   // 3 * N * N * (N/2+1) complex
  float* sa_raw = nullptr;  // 3 * N^3, for protocol colour steps
  // Split transform (power-of-two N, spectral.cu): 2-D transforms over (j, k)
  // for every plane and colour, the pass along i fused with the filter.
  cufftHandle r2c_2d = 0, c2r_2d = 0;
  float2* twiddles = nullptr;                              // e^{-2 pi i t / N}, t < N
  std::map<std::pair<double, double>, float*> tables;      // filter per (gamma, D)
};

// Poisson equilibration scratch per lattice edge: float32 R2C of the
// right-hand side, float64 Z2D of the divided spectrum.
struct PoissonSlot {
  cufftHandle r2c = 0, z2d = 0;
  float* rhs = nullptr;       // N^3
  float2* spec_f = nullptr;   // N * N * (N/2+1)
  double2* spec_d = nullptr;  // N * N * (N/2+1)
  double* out = nullptr;      // N^3
};

struct lfm_context {
  int device = 0;
  std::mutex mu;
  std::map<int, FftSlot> slots;
  std::map<int, PoissonSlot> poisson;
  double* metric_partials = nullptr;  // kMetricRows x kPartialStride, then the final row
};

namespace {

int fft_slot(lfm_context* ctx, int N, bool need_sa_raw, FftSlot** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev != ctx->device)
    return fail(LFM_ERR_INVALID_ARG, "context belongs to device %d, current device is %d",
                ctx->device, dev);
  FftSlot& s = ctx->slots[N];
  if (!s.spec) {
    int n[3] = {N, N, N};
    const int real_dist = N * N * N, cplx_dist = N * N * (N / 2 + 1);
    if (cufftPlanMany(&s.r2c, 3, n, nullptr, 1, real_dist, nullptr, 1, cplx_dist, CUFFT_R2C, 3) !=
        CUFFT_SUCCESS)
      return fail(LFM_ERR_CUFFT, "cufftPlanMany R2C N=%d", N);
    if (cufftPlanMany(&s.c2r, 3, n, nullptr, 1, cplx_dist, nullptr, 1, real_dist, CUFFT_C2R, 3) !=
        CUFFT_SUCCESS)
      return fail(LFM_ERR_CUFFT, "cufftPlanMany C2R N=%d", N);
    e = cudaMalloc(&s.spec, sizeof(float2) * 3 * (size_t)cplx_dist);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc spectrum");
  }
  if (need_sa_raw && !s.sa_raw) {
    e = cudaMalloc(&s.sa_raw, sizeof(float) * 3 * (size_t)N * N * N);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc S_a scratch");
  }
  *out = &s;
  return LFM_OK;
}

int poisson_slot(lfm_context* ctx, int N, PoissonSlot** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev != ctx->device)
    return fail(LFM_ERR_INVALID_ARG, "context belongs to device %d, current device is %d",
                ctx->device, dev);
  PoissonSlot& s = ctx->poisson[N];
  if (!s.out) {
    const size_t n3 = (size_t)N * N * N, nc = (size_t)N * N * (N / 2 + 1);
    if (cufftPlan3d(&s.r2c, N, N, N, CUFFT_R2C) != CUFFT_SUCCESS)
      return fail(LFM_ERR_CUFFT, "cufftPlan3d R2C N=%d", N);
    if (cufftPlan3d(&s.z2d, N, N, N, CUFFT_Z2D) != CUFFT_SUCCESS)
      return fail(LFM_ERR_CUFFT, "cufftPlan3d Z2D N=%d", N);
    e = cudaMalloc(&s.rhs, sizeof(float) * n3);
    if (e == cudaSuccess) e = cudaMalloc(&s.spec_f, sizeof(float2) * nc);
    if (e == cudaSuccess) e = cudaMalloc(&s.spec_d, sizeof(double2) * nc);
    if (e == cudaSuccess) e = cudaMalloc(&s.out, sizeof(double) * n3);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc Poisson scratch");
  }
  *out = &s;
  return LFM_OK;
}

// The split transform's plans, twiddles and the filter table for (gamma, D),
// created on first use (outside stream capture: they allocate and upload).
int split_transform(FftSlot* s, int N, double gamma, double d, cudaStream_t stream,
                    float** table) {
  const std::pair<double, double> key(gamma, d);
  auto it = s->tables.find(key);
  if (s->r2c_2d && it != s->tables.end()) {
    *table = it->second;
    return LFM_OK;
  }
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaError_t e = cudaStreamIsCapturing(stream, &cap);
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamIsCapturing");
  if (cap != cudaStreamCaptureStatusNone)
    return fail(LFM_ERR_UNSUPPORTED,
                "the first S_a solve for N=%d, gamma=%g, D=%g must run outside stream capture",
                N, gamma, d);
  const int nz = N / 2 + 1;
  if (!s->r2c_2d) {
    int n[2] = {N, N}, inr[2] = {N, N}, inc[2] = {N, nz};
    if (cufftPlanMany(&s->r2c_2d, 2, n, inr, 1, N * N, inc, 1, N * nz, CUFFT_R2C, 3 * N) !=
        CUFFT_SUCCESS)
      return fail(LFM_ERR_CUFFT, "cufftPlanMany 2-D R2C N=%d", N);
    if (cufftPlanMany(&s->c2r_2d, 2, n, inc, 1, N * nz, inr, 1, N * N, CUFFT_C2R, 3 * N) !=
        CUFFT_SUCCESS)
      return fail(LFM_ERR_CUFFT, "cufftPlanMany 2-D C2R N=%d", N);
    std::vector<float2> tw(N);
    for (int t = 0; t < N; ++t) {
      const double ang = -2.0 * 3.14159265358979323846 * (double)t / (double)N;
      tw[t] = make_float2((float)std::cos(ang), (float)std::sin(ang));
    }
    e = cudaMalloc(&s->twiddles, sizeof(float2) * N);
    if (e == cudaSuccess)
      e = cudaMemcpy(s->twiddles, tw.data(), sizeof(float2) * N, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = lfm::upload_dft_twiddles();  // this context's device
    if (e != cudaSuccess) return cuda_fail(e, "twiddle table");
  }
  float* t = nullptr;
  e = cudaMalloc(&t, sizeof(float) * (size_t)nz * nz * nz);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc filter table");
  e = lfm::launch_helmholtz_table(t, N, gamma, d, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) {
    cudaFree(t);
    return cuda_fail(e, "filter table");
  }
  s->tables[key] = t;
  *table = t;
  return LFM_OK;
}

// S_a from |Psi_a|^2: from pr, pi (the energy is formed first, into the
// output buffer), or from a given energy array (pr == pi == nullptr).
int helmholtz(lfm_context* ctx, const float* pr, const float* pi, float* sa_raw, int N,
              double gamma, double d, cudaStream_t stream, bool use_ctx_scratch,
              float** sa_used, const float* energy = nullptr) {
  std::lock_guard<std::mutex> lk(ctx->mu);
  FftSlot* s = nullptr;
  int rc = fft_slot(ctx, N, use_ctx_scratch, &s);
  if (rc) return rc;
  float* dst = use_ctx_scratch ? s->sa_raw : sa_raw;
  cudaError_t e;
  const float* src = energy;
  if (!src) {
    e = lfm::launch_color_energy(pr, pi, dst, N, stream);
    if (e != cudaSuccess) return cuda_fail(e, "|Psi_a|^2 launch");
    src = dst;
  }
  if (lfm::helmholtz_xpass_supported(N) && g_sa_split.load()) {
    float* table = nullptr;
    rc = split_transform(s, N, gamma, d, stream, &table);
    if (rc) return rc;
    if (cufftSetStream(s->r2c_2d, stream) != CUFFT_SUCCESS ||
        cufftExecR2C(s->r2c_2d, const_cast<float*>(src),
                     reinterpret_cast<cufftComplex*>(s->spec)) != CUFFT_SUCCESS)
      return fail(LFM_ERR_CUFFT, "cufftExecR2C 2-D N=%d", N);
    e = lfm::launch_helmholtz_xpass(s->spec, table, s->twiddles, N, stream);
    if (e != cudaSuccess) return cuda_fail(e, "Helmholtz pass along i");
    if (cufftSetStream(s->c2r_2d, stream) != CUFFT_SUCCESS ||
        cufftExecC2R(s->c2r_2d, reinterpret_cast<cufftComplex*>(s->spec), dst) != CUFFT_SUCCESS)
      return fail(LFM_ERR_CUFFT, "cufftExecC2R 2-D N=%d", N);
    if (sa_used) *sa_used = dst;
    return LFM_OK;
  }
  if (cufftSetStream(s->r2c, stream) != CUFFT_SUCCESS ||
      cufftExecR2C(s->r2c, const_cast<float*>(src),
                   reinterpret_cast<cufftComplex*>(s->spec)) != CUFFT_SUCCESS)
    return fail(LFM_ERR_CUFFT, "cufftExecR2C N=%d", N);
  e = lfm::launch_helmholtz_multiply_gd(s->spec, N, gamma, d, stream);
  if (e != cudaSuccess) return cuda_fail(e, "Helmholtz multiply launch");
  if (cufftSetStream(s->c2r, stream) != CUFFT_SUCCESS ||
      cufftExecC2R(s->c2r, reinterpret_cast<cufftComplex*>(s->spec), dst) != CUFFT_SUCCESS)
    return fail(LFM_ERR_CUFFT, "cufftExecC2R N=%d", N);
  if (sa_used) *sa_used = dst;
  return LFM_OK;
}

}  // namespace

extern "C" {

const char* lfm_strerror(int status) {
  switch (status) {
    case LFM_OK: return "ok";
    case LFM_ERR_INVALID_ARG: return "invalid argument";
    case LFM_ERR_ALIGNMENT: return "device pointer not 16-byte aligned";
    case LFM_ERR_UNSUPPORTED: return "unsupported configuration";
    case LFM_ERR_CUDA: return "CUDA error";
    case LFM_ERR_CUFFT: return "cuFFT error";
    case LFM_ERR_MASK: return "mask is not a function of the radial key";
    case LFM_ERR_DEVICE_TIMEOUT: return "device-side wait timed out";
    case LFM_ERR_NONFINITE: return "non-finite value";
    case LFM_ERR_CAPACITY: return "capacity exceeded";
    default: return "unknown status";
  }
}

const char* lfm_last_error_detail(void) { return t_detail.c_str(); }

int lfm_abi_version(void) { return LFM_B200_ABI_VERSION; }

int lfm_set_sa_transform(int mode) {
  if (mode < 0 || mode > 1) return fail(LFM_ERR_INVALID_ARG, "mode %d not in {0,1}", mode);
  g_sa_split.store(mode);
  return LFM_OK;
}

int lfm_set_step_path(int path) {
  if (path < 0 || path > 2) return fail(LFM_ERR_INVALID_ARG, "path %d not in {0,1,2}", path);
  g_path.store(path);
  return LFM_OK;
}

int lfm_mask_lut_build(int N, const float* mask_host, float* table_host, int capacity,
                       lfm_mask_lut* out) {
  int rc = check_n(N);
  if (rc) return rc;
  if (!mask_host || !out) return fail(LFM_ERR_INVALID_ARG, "null mask or descriptor");
  const int shift = (N % 2 == 0) ? 3 : 2;
  int32_t q_lo = INT32_MAX, q_hi = INT32_MIN;
  // Pass 1: the band of keys whose mask is neither exactly 0 nor exactly 1.
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j)
      for (int k = 0; k < N; ++k) {
        const int32_t di = 2 * i - N + 1, dj = 2 * j - N + 1, dk = 2 * k - N + 1;
        const int32_t q = di * di + dj * dj + dk * dk;
        const float m = mask_host[((int64_t)i * N + j) * N + k];
        if (m != 0.0f) q_lo = std::min(q_lo, q);
        if (m != 1.0f) q_hi = std::max(q_hi, q);
      }
  lfm_mask_lut d;
  d.N = N;
  d.shift = shift;
  if (q_lo == INT32_MAX) {  // mask identically 0: every key below the (empty) band
    d.q_lo = INT32_MAX;
    d.q_hi = INT32_MAX - 1;
    d.count = 0;
  } else if (q_hi == INT32_MIN) {  // mask identically 1
    d.q_lo = 0;
    d.q_hi = -1;
    d.count = 0;
  } else {
    d.q_lo = q_lo;
    d.q_hi = q_hi;
    d.count = q_hi >= q_lo ? ((q_hi - q_lo) >> shift) + 1 : 0;
  }
  if (d.count > capacity || (d.count > 0 && !table_host))
    return fail(LFM_ERR_CAPACITY, "mask table needs %d entries, capacity %d", d.count, capacity);
  // Pass 2: fill the band and check that equal keys carry equal values.
  std::vector<uint8_t> seen(d.count, 0);
  for (int i = 0; i < d.count; ++i) table_host[i] = 0.0f;
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j)
      for (int k = 0; k < N; ++k) {
        const int32_t di = 2 * i - N + 1, dj = 2 * j - N + 1, dk = 2 * k - N + 1;
        const int32_t q = di * di + dj * dj + dk * dk;
        const float m = mask_host[((int64_t)i * N + j) * N + k];
        if (q < d.q_lo || q > d.q_hi) {
          const float want = q < d.q_lo ? 0.0f : 1.0f;
          if (memcmp(&m, &want, sizeof m) != 0)
            return fail(LFM_ERR_MASK, "cell (%d,%d,%d) outside the band has mask %g", i, j, k, m);
          continue;
        }
        if ((q - d.q_lo) & ((1 << shift) - 1))
          return fail(LFM_ERR_MASK, "key %d off the 2^%d lattice", q, shift);
        const int idx = (q - d.q_lo) >> shift;
        if (seen[idx]) {
          if (memcmp(&table_host[idx], &m, sizeof m) != 0)
            return fail(LFM_ERR_MASK, "key %d has two mask values", q);
        } else {
          table_host[idx] = m;
          seen[idx] = 1;
        }
      }
  *out = d;
  return LFM_OK;
}

int lfm_step_real_f32(const float* psi_in, const float* psi_prev_in, const float* chi_in,
                      const float* chi_prev_in, const float* boundary_mask, float* psi_out,
                      float* psi_prev_out, float* chi_out, float* chi_prev_out, int N,
                      double dt2, double kappa, double lambda_self, double chi0, double e0_sq,
                      void* stream) {
  int rc = check_n(N);
  if (rc) return rc;
  if (!psi_in || !psi_prev_in || !chi_in || !chi_prev_in || !boundary_mask || !psi_out ||
      !psi_prev_out || !chi_out || !chi_prev_out)
    return fail(LFM_ERR_INVALID_ARG, "null buffer");
  const size_t b = sizeof(float) * (size_t)N * N * N;
  rc = check_disjoint({{psi_in, b}, {psi_prev_in, b}, {chi_in, b}, {chi_prev_in, b},
                       {boundary_mask, b}},
                      {{psi_out, b}, {psi_prev_out, b}, {chi_out, b}, {chi_prev_out, b}});
  if (rc) return rc;
  lfm::StepArgs a{};
  a.level = LFM_REAL;
  a.N = N;
  a.c = lfm::make_step_consts(dt2, kappa, lambda_self, chi0, e0_sq, 0, 0, 0, 0, 0);
  a.pr = psi_in; a.pr_prev = psi_prev_in; a.chi = chi_in; a.chi_prev = chi_prev_in;
  a.pr_out = psi_out; a.pr_prev_out = psi_prev_out;
  a.chi_out = chi_out; a.chi_prev_out = chi_prev_out;
  a.mask = boundary_mask;
  return run_step(a, static_cast<cudaStream_t>(stream));
}

int lfm_step_complex_f32(const float* psi_r_in, const float* psi_r_prev_in,
                         const float* psi_i_in, const float* psi_i_prev_in, const float* chi_in,
                         const float* chi_prev_in, const float* boundary_mask,
                         float* psi_r_out, float* psi_r_prev_out, float* psi_i_out,
                         float* psi_i_prev_out, float* chi_out, float* chi_prev_out, int N,
                         double dt2, double kappa, double lambda_self, double chi0,
                         double e0_sq, double epsilon_w, void* stream) {
  int rc = check_n(N);
  if (rc) return rc;
  if (!psi_r_in || !psi_r_prev_in || !psi_i_in || !psi_i_prev_in || !chi_in || !chi_prev_in ||
      !boundary_mask || !psi_r_out || !psi_r_prev_out || !psi_i_out || !psi_i_prev_out ||
      !chi_out || !chi_prev_out)
    return fail(LFM_ERR_INVALID_ARG, "null buffer");
  const size_t b = sizeof(float) * (size_t)N * N * N;
  rc = check_disjoint({{psi_r_in, b}, {psi_r_prev_in, b}, {psi_i_in, b}, {psi_i_prev_in, b},
                       {chi_in, b}, {chi_prev_in, b}, {boundary_mask, b}},
                      {{psi_r_out, b}, {psi_r_prev_out, b}, {psi_i_out, b}, {psi_i_prev_out, b},
                       {chi_out, b}, {chi_prev_out, b}});
  if (rc) return rc;
  lfm::StepArgs a{};
  a.level = LFM_COMPLEX;
  a.N = N;
  a.c = lfm::make_step_consts(dt2, kappa, lambda_self, chi0, e0_sq, epsilon_w, 0, 0, 0, 0);
  a.pr = psi_r_in; a.pr_prev = psi_r_prev_in; a.pi = psi_i_in; a.pi_prev = psi_i_prev_in;
  a.chi = chi_in; a.chi_prev = chi_prev_in;
  a.pr_out = psi_r_out; a.pr_prev_out = psi_r_prev_out;
  a.pi_out = psi_i_out; a.pi_prev_out = psi_i_prev_out;
  a.chi_out = chi_out; a.chi_prev_out = chi_prev_out;
  a.mask = boundary_mask;
  return run_step(a, static_cast<cudaStream_t>(stream));
}

int lfm_step_color_f32(lfm_context* ctx, const float* psi_r_in, const float* psi_r_prev_in,
                       const float* psi_i_in, const float* psi_i_prev_in, const float* chi_in,
                       const float* chi_prev_in, const float* boundary_mask, float* psi_r_out,
                       float* psi_r_prev_out, float* psi_i_out, float* psi_i_prev_out,
                       float* chi_out, float* chi_prev_out, int N, double dt2, double kappa,
                       double lambda_self, double chi0, double e0_sq, double epsilon_w,
                       double kappa_c, double epsilon_cc, double kappa_string,
                       double kappa_tube, const float* sa_fields_in, float* sa_fields_out,
                       double sa_gamma, double sa_d, double dt, void* stream) {
  (void)sa_fields_in;  // recomputed from psi when used (numpy_backend.py:341-356)
  (void)dt;
  int rc = check_n(N);
  if (rc) return rc;
  if (!psi_r_in || !psi_r_prev_in || !psi_i_in || !psi_i_prev_in || !chi_in || !chi_prev_in ||
      !boundary_mask || !psi_r_out || !psi_r_prev_out || !psi_i_out || !psi_i_prev_out ||
      !chi_out || !chi_prev_out)
    return fail(LFM_ERR_INVALID_ARG, "null buffer");
  const size_t b = sizeof(float) * (size_t)N * N * N, b3 = 3 * b;
  const bool use_sa = kappa_tube > 0.0 && sa_fields_out != nullptr;
  rc = check_disjoint({{psi_r_in, b3}, {psi_r_prev_in, b3}, {psi_i_in, b3}, {psi_i_prev_in, b3},
                       {chi_in, b}, {chi_prev_in, b}, {boundary_mask, b}},
                      {{psi_r_out, b3}, {psi_r_prev_out, b3}, {psi_i_out, b3},
                       {psi_i_prev_out, b3}, {chi_out, b}, {chi_prev_out, b},
                       {use_sa ? sa_fields_out : nullptr, b3}});
  if (rc) return rc;
  lfm::StepArgs a{};
  a.level = LFM_COLOR;
  a.N = N;
  a.c = lfm::make_step_consts(dt2, kappa, lambda_self, chi0, e0_sq, epsilon_w, kappa_c,
                              epsilon_cc, kappa_string, kappa_tube);
  a.pr = psi_r_in; a.pr_prev = psi_r_prev_in; a.pi = psi_i_in; a.pi_prev = psi_i_prev_in;
  a.chi = chi_in; a.chi_prev = chi_prev_in;
  a.pr_out = psi_r_out; a.pr_prev_out = psi_r_prev_out;
  a.pi_out = psi_i_out; a.pi_prev_out = psi_i_prev_out;
  a.chi_out = chi_out; a.chi_prev_out = chi_prev_out;
  a.mask = boundary_mask;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (use_sa) {
    if (!ctx) return fail(LFM_ERR_INVALID_ARG, "kappa_tube > 0 needs a library context");
    float* sa_raw = nullptr;
    rc = helmholtz(ctx, psi_r_in, psi_i_in, nullptr, N, sa_gamma, sa_d, st, true, &sa_raw);
    if (rc) return rc;
    a.sa = sa_raw;
    a.sa_clip_out = sa_fields_out;
  }
  return run_step(a, st);
}

int lfm_context_create(lfm_context** out) {
  if (!out) return fail(LFM_ERR_INVALID_ARG, "null output");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  lfm_context* c = new lfm_context;
  c->device = dev;
  *out = c;
  return LFM_OK;
}

int lfm_context_destroy(lfm_context* ctx) {
  if (!ctx) return LFM_OK;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(ctx->device);
  for (auto& kv : ctx->slots) {
    if (kv.second.r2c) cufftDestroy(kv.second.r2c);
    if (kv.second.c2r) cufftDestroy(kv.second.c2r);
    if (kv.second.r2c_2d) cufftDestroy(kv.second.r2c_2d);
    if (kv.second.c2r_2d) cufftDestroy(kv.second.c2r_2d);
    if (kv.second.spec) cudaFree(kv.second.spec);
    if (kv.second.sa_raw) cudaFree(kv.second.sa_raw);
    if (kv.second.twiddles) cudaFree(kv.second.twiddles);
    for (auto& t : kv.second.tables) cudaFree(t.second);
  }
  for (auto& kv : ctx->poisson) {
    PoissonSlot& p = kv.second;
    if (p.r2c) cufftDestroy(p.r2c);
    if (p.z2d) cufftDestroy(p.z2d);
    if (p.rhs) cudaFree(p.rhs);
    if (p.spec_f) cudaFree(p.spec_f);
    if (p.spec_d) cudaFree(p.spec_d);
    if (p.out) cudaFree(p.out);
  }
  if (ctx->metric_partials) cudaFree(ctx->metric_partials);
  cudaSetDevice(prev);
  delete ctx;
  return LFM_OK;
}

int lfm_leapfrog_real_f32(const float* psi, float* psi_prev_io, const float* chi,
                          float* chi_prev_io, const float* mask_table, const lfm_mask_lut* lut,
                          int damp_prev, int N, double dt2, double kappa, double lambda_self,
                          double chi0, double e0_sq, void* stream) {
  int rc = check_n(N);
  if (rc) return rc;
  if (!psi || !psi_prev_io || !chi || !chi_prev_io) return fail(LFM_ERR_INVALID_ARG, "null buffer");
  rc = check_lut(mask_table, lut, N);
  if (rc) return rc;
  const size_t b = sizeof(float) * (size_t)N * N * N;
  rc = check_disjoint({{psi, b}, {chi, b}}, {{psi_prev_io, b}, {chi_prev_io, b}});
  if (rc) return rc;
  lfm::StepArgs a{};
  a.level = LFM_REAL;
  a.N = N;
  a.c = lfm::make_step_consts(dt2, kappa, lambda_self, chi0, e0_sq, 0, 0, 0, 0, 0);
  a.pr = psi; a.pr_prev = psi_prev_io; a.pr_out = psi_prev_io;
  a.chi = chi; a.chi_prev = chi_prev_io; a.chi_out = chi_prev_io;
  a.lut = device_lut(mask_table, lut);
  a.damp_prev = damp_prev ? 1 : 0;
  return run_step(a, static_cast<cudaStream_t>(stream));
}

int lfm_leapfrog_complex_f32(const float* psi_r, float* psi_r_prev_io, const float* psi_i,
                             float* psi_i_prev_io, const float* chi, float* chi_prev_io,
                             const float* mask_table, const lfm_mask_lut* lut, int damp_prev,
                             int N, double dt2, double kappa, double lambda_self, double chi0,
                             double e0_sq, double epsilon_w, void* stream) {
  int rc = check_n(N);
  if (rc) return rc;
  if (!psi_r || !psi_r_prev_io || !psi_i || !psi_i_prev_io || !chi || !chi_prev_io)
    return fail(LFM_ERR_INVALID_ARG, "null buffer");
  rc = check_lut(mask_table, lut, N);
  if (rc) return rc;
  const size_t b = sizeof(float) * (size_t)N * N * N;
  rc = check_disjoint({{psi_r, b}, {psi_i, b}, {chi, b}},
                      {{psi_r_prev_io, b}, {psi_i_prev_io, b}, {chi_prev_io, b}});
  if (rc) return rc;
  lfm::StepArgs a{};
  a.level = LFM_COMPLEX;
  a.N = N;
  a.c = lfm::make_step_consts(dt2, kappa, lambda_self, chi0, e0_sq, epsilon_w, 0, 0, 0, 0);
  a.pr = psi_r; a.pr_prev = psi_r_prev_io; a.pr_out = psi_r_prev_io;
  a.pi = psi_i; a.pi_prev = psi_i_prev_io; a.pi_out = psi_i_prev_io;
  a.chi = chi; a.chi_prev = chi_prev_io; a.chi_out = chi_prev_io;
  a.lut = device_lut(mask_table, lut);
  a.damp_prev = damp_prev ? 1 : 0;
  return run_step(a, static_cast<cudaStream_t>(stream));
}

int lfm_poisson_chi_f32(lfm_context* ctx, int level, const float* psi_r, const float* psi_i,
                        int N, double chi0, double kappa, double e0_sq,
                        double boundary_fraction, int frozen, float* chi_out, void* stream) {
  if (!ctx) return fail(LFM_ERR_INVALID_ARG, "null context");
  int rc = check_n(N);
  if (rc) return rc;
  if (level < LFM_REAL || level > LFM_COLOR) return fail(LFM_ERR_INVALID_ARG, "level %d", level);
  if (!psi_r || !chi_out || (level != LFM_REAL && !psi_i))
    return fail(LFM_ERR_INVALID_ARG, "null buffer");
  if (frozen && !(boundary_fraction > 0.0 && boundary_fraction < 1.0))
    return fail(LFM_ERR_INVALID_ARG, "boundary_fraction %g", boundary_fraction);
  const int colours = level == LFM_COLOR ? 3 : 1;
  const size_t b = sizeof(float) * (size_t)N * N * N;
  rc = check_disjoint({{psi_r, colours * b}, {psi_i, psi_i ? colours * b : 0}}, {{chi_out, b}});
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(ctx->mu);
  PoissonSlot* s = nullptr;
  rc = poisson_slot(ctx, N, &s);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = lfm::launch_poisson_rhs(psi_r, level == LFM_REAL ? nullptr : psi_i, s->rhs, N,
                                          colours, (float)kappa, (float)e0_sq, st);
  if (e != cudaSuccess) return cuda_fail(e, "Poisson rhs launch");
  if (cufftSetStream(s->r2c, st) != CUFFT_SUCCESS ||
      cufftExecR2C(s->r2c, s->rhs, reinterpret_cast<cufftComplex*>(s->spec_f)) != CUFFT_SUCCESS)
    return fail(LFM_ERR_CUFFT, "cufftExecR2C N=%d", N);
  e = lfm::launch_poisson_divide(s->spec_f, s->spec_d, N, st);
  if (e != cudaSuccess) return cuda_fail(e, "Poisson divide launch");
  if (cufftSetStream(s->z2d, st) != CUFFT_SUCCESS ||
      cufftExecZ2D(s->z2d, reinterpret_cast<cufftDoubleComplex*>(s->spec_d), s->out) !=
          CUFFT_SUCCESS)
    return fail(LFM_ERR_CUFFT, "cufftExecZ2D N=%d", N);
  e = lfm::launch_poisson_finish(s->out, chi_out, N, (float)chi0,
                                 N / 2.0 * (1.0 - boundary_fraction), frozen ? 1 : 0, st);
  if (e != cudaSuccess) return cuda_fail(e, "Poisson finish launch");
  return LFM_OK;
}

int lfm_slab_step_f32(int level, const float* psi_r, float* psi_r_prev_io, const float* psi_i,
                      float* psi_i_prev_io, const float* chi, float* chi_prev_io,
                      const float* mask_table, const lfm_mask_lut* lut, int damp_prev, int N,
                      int n_local, int i_first, double dt2, double kappa, double lambda_self,
                      double chi0, double e0_sq, double epsilon_w, void* stream) {
  return lfm_slab_step_planes_f32(level, psi_r, psi_r_prev_io, psi_i, psi_i_prev_io, chi,
                                  chi_prev_io, mask_table, lut, damp_prev, N, n_local, i_first,
                                  1, n_local + 1, dt2, kappa, lambda_self, chi0, e0_sq, epsilon_w,
                                  stream);
}

int lfm_slab_step_planes_f32(int level, const float* psi_r, float* psi_r_prev_io,
                             const float* psi_i, float* psi_i_prev_io, const float* chi,
                             float* chi_prev_io, const float* mask_table, const lfm_mask_lut* lut,
                             int damp_prev, int N, int n_local, int i_first, int plane_lo,
                             int plane_hi, double dt2, double kappa, double lambda_self,
                             double chi0, double e0_sq, double epsilon_w, void* stream) {
  if (level != LFM_REAL && level != LFM_COMPLEX)
    return fail(LFM_ERR_UNSUPPORTED, "slab step: level %d (REAL and COMPLEX only)", level);
  int rc = check_n(N);
  if (rc) return rc;
  if (n_local < 1 || i_first < 0 || i_first + n_local > N)
    return fail(LFM_ERR_INVALID_ARG, "slab planes [%d, %d) outside [0, %d)", i_first,
                i_first + n_local, N);
  if (plane_lo < 1 || plane_hi > n_local + 1 || plane_lo >= plane_hi)
    return fail(LFM_ERR_INVALID_ARG, "slab plane range [%d, %d) outside [1, %d]", plane_lo,
                plane_hi, n_local + 1);
  const bool cx = level == LFM_COMPLEX;
  if (!psi_r || !psi_r_prev_io || !chi || !chi_prev_io || (cx && (!psi_i || !psi_i_prev_io)))
    return fail(LFM_ERR_INVALID_ARG, "null buffer");
  rc = check_lut(mask_table, lut, N);
  if (rc) return rc;
  const size_t b = sizeof(float) * (size_t)(n_local + 2) * N * N;
  std::vector<Span> ins = {{psi_r, b}, {chi, b}};
  std::vector<Span> outs = {{psi_r_prev_io, b}, {chi_prev_io, b}};
  if (cx) {
    ins.push_back({psi_i, b});
    outs.push_back({psi_i_prev_io, b});
  }
  rc = check_disjoint(ins, outs);
  if (rc) return rc;
  lfm::StepArgs a{};
  a.level = level;
  a.N = N;
  a.c = lfm::make_step_consts(dt2, kappa, lambda_self, chi0, e0_sq, cx ? epsilon_w : 0.0, 0, 0,
                              0, 0);
  a.pr = psi_r; a.pr_prev = psi_r_prev_io; a.pr_out = psi_r_prev_io;
  if (cx) {
    a.pi = psi_i; a.pi_prev = psi_i_prev_io; a.pi_out = psi_i_prev_io;
  }
  a.chi = chi; a.chi_prev = chi_prev_io; a.chi_out = chi_prev_io;
  a.lut = device_lut(mask_table, lut);
  a.damp_prev = damp_prev ? 1 : 0;
  a.slab = 1;
  a.ni = n_local + 2;
  a.i_lo = plane_lo;
  a.i_hi = plane_hi;
  a.i_off = i_first - 1;
  return run_step(a, static_cast<cudaStream_t>(stream));
}

int lfm_advance_f32(int level, const float* psi_r, const float* psi_r_prev, float* psi_r_out,
                    const float* psi_i, const float* psi_i_prev, float* psi_i_out,
                    const float* chi, const float* chi_prev, float* chi_out,
                    const float* mask_table, const lfm_mask_lut* lut, int damp_prev, int N,
                    double dt2, double kappa, double lambda_self, double chi0, double e0_sq,
                    double epsilon_w, void* stream) {
  if (level != LFM_REAL && level != LFM_COMPLEX)
    return fail(LFM_ERR_UNSUPPORTED, "advance: level %d (REAL and COMPLEX only)", level);
  int rc = check_n(N);
  if (rc) return rc;
  const bool cx = level == LFM_COMPLEX;
  if (!psi_r || !psi_r_prev || !psi_r_out || !chi || !chi_prev || !chi_out ||
      (cx && (!psi_i || !psi_i_prev || !psi_i_out)))
    return fail(LFM_ERR_INVALID_ARG, "null buffer");
  rc = check_lut(mask_table, lut, N);
  if (rc) return rc;
  const size_t b = sizeof(float) * (size_t)N * N * N;
  std::vector<Span> ins = {{psi_r, b}, {psi_r_prev, b}, {chi, b}, {chi_prev, b}};
  std::vector<Span> outs = {{psi_r_out, b}, {chi_out, b}};
  if (cx) {
    ins.push_back({psi_i, b});
    ins.push_back({psi_i_prev, b});
    outs.push_back({psi_i_out, b});
  }
  rc = check_disjoint(ins, outs);
  if (rc) return rc;
  lfm::StepArgs a{};
  a.level = level;
  a.N = N;
  a.c = lfm::make_step_consts(dt2, kappa, lambda_self, chi0, e0_sq, cx ? epsilon_w : 0.0, 0, 0,
                              0, 0);
  a.pr = psi_r; a.pr_prev = psi_r_prev; a.pr_out = psi_r_out;
  if (cx) {
    a.pi = psi_i; a.pi_prev = psi_i_prev; a.pi_out = psi_i_out;
  }
  a.chi = chi; a.chi_prev = chi_prev; a.chi_out = chi_out;
  a.lut = device_lut(mask_table, lut);
  a.damp_prev = damp_prev ? 1 : 0;
  return run_step(a, static_cast<cudaStream_t>(stream));
}

int lfm_adjoint_step_f32(int level, const float* psi_r, const float* psi_i, const float* chi,
                         const float* chi_next, const float* mask_table, const lfm_mask_lut* lut,
                         const float* const* g_out, float* const* g_in, int N, double dt2,
                         double kappa, double lambda_self, double chi0, double e0_sq,
                         double epsilon_w, void* stream) {
  if (level != LFM_REAL && level != LFM_COMPLEX)
    return fail(LFM_ERR_UNSUPPORTED, "adjoint step: level %d (REAL and COMPLEX only)", level);
  int rc = check_n(N);
  if (rc) return rc;
  const bool cx = level == LFM_COMPLEX;
  if (!psi_r || !chi || !chi_next || !g_out || !g_in || (cx && !psi_i))
    return fail(LFM_ERR_INVALID_ARG, "null buffer");
  for (int f = 0; f < 6; ++f) {
    const bool need = cx || (f != 2 && f != 3);
    if (need && (!g_out[f] || !g_in[f]))
      return fail(LFM_ERR_INVALID_ARG, "adjoint buffer %d is null", f);
  }
  rc = check_lut(mask_table, lut, N);
  if (rc) return rc;
  const size_t b = sizeof(float) * (size_t)N * N * N;
  std::vector<Span> ins = {{psi_r, b}, {chi, b}, {chi_next, b}};
  std::vector<Span> outs;
  if (cx) ins.push_back({psi_i, b});
  for (int f = 0; f < 6; ++f) {
    if (!cx && (f == 2 || f == 3)) continue;
    ins.push_back({g_out[f], b});
    outs.push_back({g_in[f], b});
  }
  rc = check_disjoint(ins, outs);
  if (rc) return rc;
  const lfm::StepConsts c =
      lfm::make_step_consts(dt2, kappa, lambda_self, chi0, e0_sq, epsilon_w, 0, 0, 0, 0);
  cudaError_t e = lfm::launch_adjoint_step(level, N, psi_r, psi_i, chi, chi_next,
                                           device_lut(mask_table, lut), g_out, g_in, c,
                                           static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "adjoint step launch");
  return LFM_OK;
}

int lfm_leapfrog_color_f32(const float* psi_r, float* psi_r_prev_io, const float* psi_i,
                           float* psi_i_prev_io, const float* chi, float* chi_prev_io,
                           const float* mask_table, const lfm_mask_lut* lut, int damp_prev,
                           int N, double dt2, double kappa, double lambda_self, double chi0,
                           double e0_sq, double epsilon_w, double kappa_c, double epsilon_cc,
                           double kappa_string, double kappa_tube, const float* sa,
                           void* stream) {
  return lfm_leapfrog_color_energy_f32(psi_r, psi_r_prev_io, psi_i, psi_i_prev_io, chi,
                                       chi_prev_io, mask_table, lut, damp_prev, N, dt2, kappa,
                                       lambda_self, chi0, e0_sq, epsilon_w, kappa_c, epsilon_cc,
                                       kappa_string, kappa_tube, sa, nullptr, stream);
}

int lfm_leapfrog_color_energy_f32(const float* psi_r, float* psi_r_prev_io, const float* psi_i,
                                  float* psi_i_prev_io, const float* chi, float* chi_prev_io,
                                  const float* mask_table, const lfm_mask_lut* lut,
                                  int damp_prev, int N, double dt2, double kappa,
                                  double lambda_self, double chi0, double e0_sq,
                                  double epsilon_w, double kappa_c, double epsilon_cc,
                                  double kappa_string, double kappa_tube, const float* sa,
                                  float* energy_out, void* stream) {
  int rc = check_n(N);
  if (rc) return rc;
  if (!psi_r || !psi_r_prev_io || !psi_i || !psi_i_prev_io || !chi || !chi_prev_io)
    return fail(LFM_ERR_INVALID_ARG, "null buffer");
  rc = check_lut(mask_table, lut, N);
  if (rc) return rc;
  const size_t b = sizeof(float) * (size_t)N * N * N, b3 = 3 * b;
  rc = check_disjoint({{psi_r, b3}, {psi_i, b3}, {chi, b}, {sa, sa ? b3 : 0}},
                      {{psi_r_prev_io, b3}, {psi_i_prev_io, b3}, {chi_prev_io, b},
                       {energy_out, energy_out ? b3 : 0}});
  if (rc) return rc;
  lfm::StepArgs a{};
  a.level = LFM_COLOR;
  a.N = N;
  a.c = lfm::make_step_consts(dt2, kappa, lambda_self, chi0, e0_sq, epsilon_w, kappa_c,
                              epsilon_cc, kappa_string, kappa_tube);
  a.pr = psi_r; a.pr_prev = psi_r_prev_io; a.pr_out = psi_r_prev_io;
  a.pi = psi_i; a.pi_prev = psi_i_prev_io; a.pi_out = psi_i_prev_io;
  a.chi = chi; a.chi_prev = chi_prev_io; a.chi_out = chi_prev_io;
  a.lut = device_lut(mask_table, lut);
  a.damp_prev = damp_prev ? 1 : 0;
  a.sa = (kappa_tube > 0.0) ? sa : nullptr;
  a.energy_out = energy_out;
  return run_step(a, static_cast<cudaStream_t>(stream));
}

int lfm_leapfrog_real_comp_f32(const float* psi, float* psi_next, float* dpsi_io,
                               const float* chi, float* chi_next, float* dchi_io,
                               const float* mask_table, const lfm_mask_lut* lut, int N,
                               double dt2, double kappa, double lambda_self, double chi0,
                               double e0_sq, void* stream) {
  int rc = check_n(N);
  if (rc) return rc;
  if (!psi || !psi_next || !dpsi_io || !chi || !chi_next || !dchi_io)
    return fail(LFM_ERR_INVALID_ARG, "null buffer");
  rc = check_lut(mask_table, lut, N);
  if (rc) return rc;
  const size_t b = sizeof(float) * (size_t)N * N * N;
  rc = check_disjoint({{psi, b}, {chi, b}},
                      {{psi_next, b}, {dpsi_io, b}, {chi_next, b}, {dchi_io, b}});
  if (rc) return rc;
  lfm::StepArgs a{};
  a.level = LFM_REAL;
  a.N = N;
  a.comp = 1;
  a.c = lfm::make_step_consts(dt2, kappa, lambda_self, chi0, e0_sq, 0, 0, 0, 0, 0);
  a.pr = psi; a.pr_prev = dpsi_io; a.pr_out = psi_next; a.pr_prev_out = dpsi_io;
  a.chi = chi; a.chi_prev = dchi_io; a.chi_out = chi_next; a.chi_prev_out = dchi_io;
  a.lut = device_lut(mask_table, lut);
  return run_step(a, static_cast<cudaStream_t>(stream));
}

int lfm_leapfrog_complex_comp_f32(const float* psi_r, float* psi_r_next, float* dpsi_r_io,
                                  const float* psi_i, float* psi_i_next, float* dpsi_i_io,
                                  const float* chi, float* chi_next, float* dchi_io,
                                  const float* mask_table, const lfm_mask_lut* lut, int N,
                                  double dt2, double kappa, double lambda_self, double chi0,
                                  double e0_sq, double epsilon_w, void* stream) {
  int rc = check_n(N);
  if (rc) return rc;
  if (!psi_r || !psi_r_next || !dpsi_r_io || !psi_i || !psi_i_next || !dpsi_i_io || !chi ||
      !chi_next || !dchi_io)
    return fail(LFM_ERR_INVALID_ARG, "null buffer");
  rc = check_lut(mask_table, lut, N);
  if (rc) return rc;
  const size_t b = sizeof(float) * (size_t)N * N * N;
  rc = check_disjoint({{psi_r, b}, {psi_i, b}, {chi, b}},
                      {{psi_r_next, b}, {dpsi_r_io, b}, {psi_i_next, b}, {dpsi_i_io, b},
                       {chi_next, b}, {dchi_io, b}});
  if (rc) return rc;
  lfm::StepArgs a{};
  a.level = LFM_COMPLEX;
  a.N = N;
  a.comp = 1;
  a.c = lfm::make_step_consts(dt2, kappa, lambda_self, chi0, e0_sq, epsilon_w, 0, 0, 0, 0);
  a.pr = psi_r; a.pr_prev = dpsi_r_io; a.pr_out = psi_r_next; a.pr_prev_out = dpsi_r_io;
  a.pi = psi_i; a.pi_prev = dpsi_i_io; a.pi_out = psi_i_next; a.pi_prev_out = dpsi_i_io;
  a.chi = chi; a.chi_prev = dchi_io; a.chi_out = chi_next; a.chi_prev_out = dchi_io;
  a.lut = device_lut(mask_table, lut);
  return run_step(a, static_cast<cudaStream_t>(stream));
}

int lfm_leapfrog_real_split_f32(const float* psi, float* psi_prev_io, const float* chi_hi,
                                float* chi_hi_prev_io, const float* chi_lo, float* chi_lo_prev_io,
                                const float* mask_table, const lfm_mask_lut* lut, int damp_prev,
                                int N, double dt2, double kappa, double lambda_self, double chi0,
                                double e0_sq, void* stream) {
  int rc = check_n(N);
  if (rc) return rc;
  if (!psi || !psi_prev_io || !chi_hi || !chi_hi_prev_io || !chi_lo || !chi_lo_prev_io)
    return fail(LFM_ERR_INVALID_ARG, "null buffer");
  rc = check_lut(mask_table, lut, N);
  if (rc) return rc;
  const size_t b = sizeof(float) * (size_t)N * N * N;
  rc = check_disjoint({{psi, b}, {chi_hi, b}, {chi_lo, b}},
                      {{psi_prev_io, b}, {chi_hi_prev_io, b}, {chi_lo_prev_io, b}});
  if (rc) return rc;
  lfm::StepArgs a{};
  a.level = LFM_REAL;
  a.N = N;
  a.split = 1;
  a.c = lfm::make_step_consts(dt2, kappa, lambda_self, chi0, e0_sq, 0, 0, 0, 0, 0);
  a.pr = psi; a.pr_prev = psi_prev_io; a.pr_out = psi_prev_io;
  a.chi = chi_hi; a.chi_prev = chi_hi_prev_io; a.chi_out = chi_hi_prev_io;
  a.chi_lo = chi_lo; a.chi_lo_prev = chi_lo_prev_io; a.chi_lo_out = chi_lo_prev_io;
  a.lut = device_lut(mask_table, lut);
  a.damp_prev = damp_prev ? 1 : 0;
  return run_step(a, static_cast<cudaStream_t>(stream));
}

int lfm_leapfrog_complex_split_f32(const float* psi_r, float* psi_r_prev_io, const float* psi_i,
                                   float* psi_i_prev_io, const float* chi_hi,
                                   float* chi_hi_prev_io, const float* chi_lo,
                                   float* chi_lo_prev_io, const float* mask_table,
                                   const lfm_mask_lut* lut, int damp_prev, int N, double dt2,
                                   double kappa, double lambda_self, double chi0, double e0_sq,
                                   double epsilon_w, void* stream) {
  int rc = check_n(N);
  if (rc) return rc;
  if (!psi_r || !psi_r_prev_io || !psi_i || !psi_i_prev_io || !chi_hi || !chi_hi_prev_io ||
      !chi_lo || !chi_lo_prev_io)
    return fail(LFM_ERR_INVALID_ARG, "null buffer");
  rc = check_lut(mask_table, lut, N);
  if (rc) return rc;
  const size_t b = sizeof(float) * (size_t)N * N * N;
  rc = check_disjoint({{psi_r, b}, {psi_i, b}, {chi_hi, b}, {chi_lo, b}},
                      {{psi_r_prev_io, b}, {psi_i_prev_io, b}, {chi_hi_prev_io, b},
                       {chi_lo_prev_io, b}});
  if (rc) return rc;
  lfm::StepArgs a{};
  a.level = LFM_COMPLEX;
  a.N = N;
  a.split = 1;
  a.c = lfm::make_step_consts(dt2, kappa, lambda_self, chi0, e0_sq, epsilon_w, 0, 0, 0, 0);
  a.pr = psi_r; a.pr_prev = psi_r_prev_io; a.pr_out = psi_r_prev_io;
  a.pi = psi_i; a.pi_prev = psi_i_prev_io; a.pi_out = psi_i_prev_io;
  a.chi = chi_hi; a.chi_prev = chi_hi_prev_io; a.chi_out = chi_hi_prev_io;
  a.chi_lo = chi_lo; a.chi_lo_prev = chi_lo_prev_io; a.chi_lo_out = chi_lo_prev_io;
  a.lut = device_lut(mask_table, lut);
  a.damp_prev = damp_prev ? 1 : 0;
  return run_step(a, static_cast<cudaStream_t>(stream));
}

int lfm_advance_split_f32(int level, const float* psi_r, const float* psi_r_prev,
                          float* psi_r_out, const float* psi_i, const float* psi_i_prev,
                          float* psi_i_out, const float* chi_hi, const float* chi_hi_prev,
                          float* chi_hi_out, const float* chi_lo, const float* chi_lo_prev,
                          float* chi_lo_out, const float* mask_table, const lfm_mask_lut* lut,
                          int damp_prev, int N, double dt2, double kappa, double lambda_self,
                          double chi0, double e0_sq, double epsilon_w, void* stream) {
  if (level != LFM_REAL && level != LFM_COMPLEX)
    return fail(LFM_ERR_UNSUPPORTED, "advance: level %d (REAL and COMPLEX only)", level);
  int rc = check_n(N);
  if (rc) return rc;
  const bool cx = level == LFM_COMPLEX;
  if (!psi_r || !psi_r_prev || !psi_r_out || !chi_hi || !chi_hi_prev || !chi_hi_out ||
      !chi_lo || !chi_lo_prev || !chi_lo_out || (cx && (!psi_i || !psi_i_prev || !psi_i_out)))
    return fail(LFM_ERR_INVALID_ARG, "null buffer");
  rc = check_lut(mask_table, lut, N);
  if (rc) return rc;
  const size_t b = sizeof(float) * (size_t)N * N * N;
  std::vector<Span> ins = {{psi_r, b}, {psi_r_prev, b}, {chi_hi, b},
                           {chi_hi_prev, b}, {chi_lo, b}, {chi_lo_prev, b}};
  std::vector<Span> outs = {{psi_r_out, b}, {chi_hi_out, b}, {chi_lo_out, b}};
  if (cx) {
    ins.push_back({psi_i, b});
    ins.push_back({psi_i_prev, b});
    outs.push_back({psi_i_out, b});
  }
  rc = check_disjoint(ins, outs);
  if (rc) return rc;
  lfm::StepArgs a{};
  a.level = level;
  a.N = N;
  a.split = 1;
  a.c = lfm::make_step_consts(dt2, kappa, lambda_self, chi0, e0_sq, cx ? epsilon_w : 0.0, 0, 0,
                              0, 0);
  a.pr = psi_r; a.pr_prev = psi_r_prev; a.pr_out = psi_r_out;
  if (cx) {
    a.pi = psi_i; a.pi_prev = psi_i_prev; a.pi_out = psi_i_out;
  }
  a.chi = chi_hi; a.chi_prev = chi_hi_prev; a.chi_out = chi_hi_out;
  a.chi_lo = chi_lo; a.chi_lo_prev = chi_lo_prev; a.chi_lo_out = chi_lo_out;
  a.lut = device_lut(mask_table, lut);
  a.damp_prev = damp_prev ? 1 : 0;
  return run_step(a, static_cast<cudaStream_t>(stream));
}

int lfm_helmholtz_sa_f32(lfm_context* ctx, const float* psi_r, const float* psi_i,
                         float* sa_raw, int N, double sa_gamma, double sa_d, void* stream) {
  int rc = check_n(N);
  if (rc) return rc;
  if (!ctx || !psi_r || !psi_i || !sa_raw) return fail(LFM_ERR_INVALID_ARG, "null argument");
  const size_t b3 = 3 * sizeof(float) * (size_t)N * N * N;
  rc = check_disjoint({{psi_r, b3}, {psi_i, b3}}, {{sa_raw, b3}});
  if (rc) return rc;
  return helmholtz(ctx, psi_r, psi_i, sa_raw, N, sa_gamma, sa_d,
                   static_cast<cudaStream_t>(stream), false, nullptr);
}

int lfm_helmholtz_sa_from_energy_f32(lfm_context* ctx, const float* energy, float* sa_raw,
                                     int N, double sa_gamma, double sa_d, void* stream) {
  int rc = check_n(N);
  if (rc) return rc;
  if (!ctx || !energy || !sa_raw) return fail(LFM_ERR_INVALID_ARG, "null argument");
  const size_t b3 = 3 * sizeof(float) * (size_t)N * N * N;
  rc = check_disjoint({{energy, b3}}, {{sa_raw, b3}});
  if (rc) return rc;
  return helmholtz(ctx, nullptr, nullptr, sa_raw, N, sa_gamma, sa_d,
                   static_cast<cudaStream_t>(stream), false, nullptr, energy);
}

int lfm_sa_clip_f32(const float* sa_raw, float* sa_out, int64_t count, void* stream) {
  if (!sa_raw || !sa_out || count < 0) return fail(LFM_ERR_INVALID_ARG, "bad argument");
  if (count == 0) return LFM_OK;
  cudaError_t e = lfm::launch_clip(sa_raw, sa_out, count, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "clip launch");
  return LFM_OK;
}

}  // extern "C"

namespace {

// Turns the reduced sums into the metrics of lfm_metrics_f64.
void finish_metrics(const double* r, double chi_shift, double* out) {
  const double count = r[lfm::kCount];
  out[0] = r[lfm::kKinetic];
  out[1] = r[lfm::kGradient];
  out[2] = r[lfm::kPotential];
  out[3] = out[0] + out[1] + out[2];
  if (count > 0) {
    const double mean_d = r[lfm::kChiSum] / count;
    double var = r[lfm::kChiSq] / count - mean_d * mean_d;
    if (var < 0) var = 0;
    out[4] = r[lfm::kMetricSums];
    out[5] = r[lfm::kMetricSums + 1];
    out[6] = chi_shift + mean_d;
    out[7] = sqrt(var);
    out[8] = r[lfm::kWell] / count;
    out[9] = r[lfm::kVoid] / count;
  } else {
    for (int q = 4; q < 10; ++q) out[q] = 0.0;
  }
  out[10] = r[lfm::kPsiSq];
  out[11] = count;
  out[12] = r[lfm::kNonFinite];
}

int check_metrics_args(int level, const float* psi_r, const float* psi_i, const float* chi, int N,
                       double dt, double boundary_fraction, double* out_host) {
  int rc = check_n(N);
  if (rc) return rc;
  if (level < 0 || level > 2) return fail(LFM_ERR_INVALID_ARG, "level %d", level);
  if (!psi_r || !chi || !out_host || (level > 0 && !psi_i))
    return fail(LFM_ERR_INVALID_ARG, "null buffer");
  if (!(dt > 0)) return fail(LFM_ERR_INVALID_ARG, "dt must be positive");
  if (!(boundary_fraction >= 0 && boundary_fraction <= 1))
    return fail(LFM_ERR_INVALID_ARG, "boundary_fraction %g outside [0, 1]", boundary_fraction);
  return LFM_OK;
}

lfm::MetricsArgs metrics_args(int level, const float* psi_r, const float* psi_r_prev,
                              const float* psi_i, const float* psi_i_prev, const float* chi,
                              int N, double dt, double c, double boundary_fraction,
                              double well_threshold, double void_threshold) {
  lfm::MetricsArgs a{};
  a.level = level;
  a.N = N;
  a.pr = psi_r;
  a.pr_prev = psi_r_prev;
  a.pi = level > 0 ? psi_i : nullptr;
  a.pi_prev = level > 0 ? psi_i_prev : nullptr;
  a.chi = chi;
  a.dt = dt;
  a.c2 = c * c;
  a.radius = (N / 2.0) * (1.0 - boundary_fraction);
  a.chi_shift = 19.0;
  a.well = (float)well_threshold;
  a.void_thr = (float)void_threshold;
  return a;
}

}  // namespace

namespace lfm {

// Argument checks, kernel arguments and host finishing of the metrics, for
// entry points defined in other files (lfm_metrics_f64_noalloc).
int metrics_prepare(int level, const float* psi_r, const float* psi_r_prev, const float* psi_i,
                    const float* psi_i_prev, const float* chi, int N, double dt, double c,
                    double boundary_fraction, double well_threshold, double void_threshold,
                    double* out_host, MetricsArgs* out) {
  const int rc = check_metrics_args(level, psi_r, psi_i, chi, N, dt, boundary_fraction, out_host);
  if (rc) return rc;
  *out = metrics_args(level, psi_r, psi_r_prev, psi_i, psi_i_prev, chi, N, dt, c,
                      boundary_fraction, well_threshold, void_threshold);
  return LFM_OK;
}

void metrics_finish(const double* sums, double chi_shift, double* out_host) {
  finish_metrics(sums, chi_shift, out_host);
}

int abi_fail(int code, const char* detail) { return fail(code, "%s", detail); }

int abi_cuda_fail(cudaError_t e, const char* what) { return cuda_fail(e, what); }

}  // namespace lfm

extern "C" {

int lfm_metrics_f64(lfm_context* ctx, int level, const float* psi_r, const float* psi_r_prev,
                    const float* psi_i, const float* psi_i_prev, const float* chi, int N,
                    double dt, double c, double boundary_fraction, double well_threshold,
                    double void_threshold, double* out_host, void* stream) {
  if (!ctx) return fail(LFM_ERR_INVALID_ARG, "null context");
  int rc = check_metrics_args(level, psi_r, psi_i, chi, N, dt, boundary_fraction, out_host);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(ctx->mu);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev != ctx->device)
    return fail(LFM_ERR_INVALID_ARG, "context belongs to device %d, current device is %d",
                ctx->device, dev);
  if (!ctx->metric_partials) {
    e = cudaMalloc(&ctx->metric_partials,
                   sizeof(double) * (lfm::kMetricRows + 1) * lfm::kPartialStride);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc metric partials");
  }
  const lfm::MetricsArgs a = metrics_args(level, psi_r, psi_r_prev, psi_i, psi_i_prev, chi, N,
                                          dt, c, boundary_fraction, well_threshold,
                                          void_threshold);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* final_row = ctx->metric_partials + (size_t)lfm::kMetricRows * lfm::kPartialStride;
  e = lfm::launch_metrics(a, ctx->metric_partials, lfm::kMetricRows, final_row, st);
  if (e != cudaSuccess) return cuda_fail(e, "metrics launch");
  double r[lfm::kPartialStride];
  e = cudaMemcpyAsync(r, final_row, sizeof r, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "metrics readback");
  finish_metrics(r, a.chi_shift, out_host);
  return LFM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// batches of lattices
// ---------------------------------------------------------------------------
namespace {

// Host-side plan of a batch: tile shape per lattice, one work list (REAL
// and COMPLEX items together) and the launch shape.  Pure host arithmetic
// (lfm_batch_plan exposes it without a device).
struct BatchPlan {
  std::vector<lfm::BatchItem> items;  // by shape class (REAL ones first), each largest first
  int real_items = 0;
  int class_off[lfm::kBatchClasses] = {}, class_n[lfm::kBatchClasses] = {};
  int threads = 0, smem = 0, grid = 0;
  int tab_off = -1;  // float offset of the shared-memory sponge table, -1 = through L1
  std::vector<int> TJ, IC, stage_floats;
};

constexpr int kBatchSmemLimit = 226 * 1024;

// Defaults: the autotuner's pick on the 256-lattice sweep (256 threads, 5
// stages, 128 k cells per item: 93.7 GCell/s against 85.5 with 3 stages).
int validate_batch_tuning(const lfm_batch_tuning* in, lfm_batch_tuning* t) {
  *t = lfm_batch_tuning{256, 5, 131072, 0};
  if (in) {
    if (in->threads) t->threads = in->threads;
    if (in->stages) t->stages = in->stages;
    if (in->item_cells) t->item_cells = in->item_cells;
    t->ctas_per_sm = in->ctas_per_sm;
  }
  if (t->threads < 32 || t->threads > 512 || t->threads % 32)
    return fail(LFM_ERR_INVALID_ARG, "threads %d not a multiple of 32 in [32, 512]", t->threads);
  if (t->stages < 3 || t->stages > 6)
    return fail(LFM_ERR_INVALID_ARG, "stages %d not in [3, 6]", t->stages);
  if (t->item_cells < 1024) return fail(LFM_ERR_INVALID_ARG, "item_cells %d < 1024", t->item_cells);
  if (t->ctas_per_sm < 0) return fail(LFM_ERR_INVALID_ARG, "ctas_per_sm %d", t->ctas_per_sm);
  return LFM_OK;
}

int check_lattice_shape(const lfm_lattice_desc& d, int l) {
  int rc = check_n(d.N);
  if (rc) return rc;
  if (d.level != LFM_REAL && d.level != LFM_COMPLEX)
    return fail(LFM_ERR_UNSUPPORTED, "lattice %d: level %d (batches hold REAL and COMPLEX)", l,
                d.level);
  if (d.N % 4 || d.N < 8)
    return fail(LFM_ERR_UNSUPPORTED, "lattice %d: N=%d is not a multiple of 4 >= 8", l, d.N);
  return LFM_OK;
}

// Bytes a cell moves per step (the sort key's weight): REAL 6 fields x 4 B,
// COMPLEX 9.
inline long item_cost(const lfm::BatchItem& it, int N) {
  return (long)(it.j1 - it.j0) * N * (it.i1 - it.i0) * (it.level == LFM_REAL ? 24 : 36);
}

// regs: registers per thread of the batch kernel; sms: SM count.
int plan_batch(const lfm_lattice_desc* L, int count, const lfm_batch_tuning& t, int regs,
               int sms, BatchPlan* plan) {
  plan->TJ.assign(count, 0);
  plan->IC.assign(count, 0);
  plan->stage_floats.assign(count, 0);
  plan->items.clear();
  int threads = 32, max_stage = 0;
  for (int l = 0; l < count; ++l) {
    const int level = L[l].level;
    const int V = (level == LFM_REAL) ? 4 : 2;
    const int ns = (level == LFM_REAL) ? 2 : 3;
    const int N = L[l].N;
    const int tpr = N / V;
    if (tpr > t.threads)
      return fail(LFM_ERR_UNSUPPORTED, "lattice %d: a row of N=%d needs %d threads > %d", l, N,
                  tpr, t.threads);
    // As few row tiles as the CTA allows, their rows as even as possible
    // (N / tiles or one more; they need not divide N), so that about all of
    // the CTA's threads have cells (N = 96 REAL at 512 threads: 5 tiles of
    // 20, 19, 19, 19, 19 rows and 90 % of the lanes, against 6 x 16 rows and
    // 75 % with a divisor of N).  TJ is the largest tile.
    const int tj_max = t.threads / tpr;
    const int tiles = (N + tj_max - 1) / tj_max;
    const int base = N / tiles, rem = N % tiles;
    const int TJ = base + (rem > 0 ? 1 : 0);
    // chunks of about item_cells cells, the planes split as evenly as possible
    const double cells = (double)TJ * N * N;
    const int chunks = std::max(1, std::min(N / 2, (int)(cells / t.item_cells + 0.5)));
    const int IC = (N + chunks - 1) / chunks;
    plan->TJ[l] = TJ;
    plan->IC[l] = IC;
    // ns halo-extended fields + ns point fields (the previous-step values)
    plan->stage_floats[l] = N * (ns * (TJ + 2) + ns * TJ);
    max_stage = std::max(max_stage, plan->stage_floats[l]);
    threads = std::max(threads, ((TJ * tpr + 31) / 32) * 32);
    for (int k = 0, j0 = 0; k < tiles; ++k) {
      const int j1 = j0 + base + (k < rem ? 1 : 0);
      for (int i0 = 0; i0 < N; i0 += IC)
        plan->items.push_back({l, level, j0, j1, i0, std::min(N, i0 + IC)});
      j0 = j1;
    }
  }
  // By shape class (the REAL classes first), largest first within a class:
  // each free CTA takes the next item of the class it is on
  // (longest-processing-time order within the class).
  std::vector<int> cls(count);
  for (int l = 0; l < count; ++l) cls[l] = lfm::batch_class_of(L[l].level, L[l].N, plan->TJ[l]);
  std::stable_sort(plan->items.begin(), plan->items.end(),
                   [&](const lfm::BatchItem& a, const lfm::BatchItem& b) {
                     if (cls[a.lattice] != cls[b.lattice]) return cls[a.lattice] < cls[b.lattice];
                     return item_cost(a, L[a.lattice].N) > item_cost(b, L[b.lattice].N);
                   });
  plan->real_items = 0;
  for (int c = 0; c < lfm::kBatchClasses; ++c) plan->class_off[c] = plan->class_n[c] = 0;
  for (int k = 0; k < (int)plan->items.size(); ++k) {
    const lfm::BatchItem& it = plan->items[k];
    plan->real_items += it.level == LFM_REAL;
    const int c = cls[it.lattice];
    if (plan->class_n[c]++ == 0) plan->class_off[c] = k;
  }
  plan->threads = threads;
  plan->smem = t.stages * max_stage * (int)sizeof(float);
  // The sponge tables (one lattice's at a time) after the largest ring, when
  // the largest of them fits; tab[1] lands on a 16-byte boundary (stage
  // floats are multiples of N, N of 4).
  int tab_bytes = 0;
  for (int l = 0; l < count; ++l)
    tab_bytes = std::max(tab_bytes, (4 * (L[l].lut.count + 5) + 15) / 16 * 16);
  plan->tab_off = -1;
  if (plan->smem + tab_bytes <= kBatchSmemLimit) {
    plan->tab_off = t.stages * max_stage + 3;
    plan->smem += tab_bytes;
  }
  if (plan->smem > kBatchSmemLimit)
    return fail(LFM_ERR_UNSUPPORTED, "batch needs %d B of shared memory per CTA (limit %d)",
                plan->smem, kBatchSmemLimit);
  int per_sm = std::min({(228 * 1024) / (plan->smem + 1024), 2048 / threads,
                         65536 / std::max(1, regs * threads)});
  per_sm = std::max(1, per_sm);
  if (t.ctas_per_sm > 0) per_sm = std::min(per_sm, t.ctas_per_sm);
  plan->grid = std::min((int)plan->items.size(), sms * per_sm);
  return LFM_OK;
}

}  // namespace

struct lfm_batch {
  int device = 0;
  int stages = 3;
  int tab_off = -1;
  lfm::BatchLattice* d_lat = nullptr;
  lfm::BatchItem* d_items = nullptr;
  int* d_counters = nullptr;  // next item of each shape class, then retired CTAs
  int nitems = 0, real_items = 0, threads = 0, smem = 0, grid = 0;
  int class_off[lfm::kBatchClasses] = {}, class_n[lfm::kBatchClasses] = {};
};

extern "C" {

int lfm_batch_plan(const lfm_lattice_desc* lattices, int count, const lfm_batch_tuning* tuning,
                   int sms, int32_t* items_out, int max_items, int* nitems_out,
                   int32_t* launch_out) {
  if (!lattices || count <= 0) return fail(LFM_ERR_INVALID_ARG, "empty batch");
  lfm_batch_tuning t;
  int rc = validate_batch_tuning(tuning, &t);
  if (rc) return rc;
  for (int l = 0; l < count; ++l) {
    rc = check_lattice_shape(lattices[l], l);
    if (rc) return rc;
  }
  BatchPlan plan;
  rc = plan_batch(lattices, count, t, 128, sms > 0 ? sms : 148, &plan);
  if (rc) return rc;
  const int total = (int)plan.items.size();
  if (nitems_out) *nitems_out = total;
  if (items_out) {
    if (max_items < total)
      return fail(LFM_ERR_CAPACITY, "%d items > capacity %d", total, max_items);
    for (int k = 0; k < total; ++k) {
      const lfm::BatchItem& it = plan.items[k];
      items_out[6 * k + 0] = it.level;
      items_out[6 * k + 1] = it.lattice;
      items_out[6 * k + 2] = it.j0;
      items_out[6 * k + 3] = it.j1;
      items_out[6 * k + 4] = it.i0;
      items_out[6 * k + 5] = it.i1;
    }
  }
  if (launch_out) {
    launch_out[0] = plan.threads;
    launch_out[1] = plan.smem;
    launch_out[2] = plan.grid;
  }
  return LFM_OK;
}

int lfm_batch_create(const lfm_lattice_desc* lattices, int count,
                     const lfm_batch_tuning* tuning, lfm_batch** out) {
  if (!lattices || count <= 0 || !out) return fail(LFM_ERR_INVALID_ARG, "empty batch");
  lfm_batch_tuning t;
  int rc = validate_batch_tuning(tuning, &t);
  if (rc) return rc;
  int* status = nullptr;
  rc = status_word(&status);
  if (rc) return rc;
  std::vector<lfm::BatchLattice> dev(count);
  for (int l = 0; l < count; ++l) {
    const lfm_lattice_desc& d = lattices[l];
    rc = check_lattice_shape(d, l);
    if (rc) return rc;
    rc = check_lut(d.mask_table, &d.lut, d.N);
    if (rc) return rc;
    const bool cx = d.level == LFM_COMPLEX;
    const float* ptrs[] = {d.psi_r[0], d.psi_r[1], d.chi[0], d.chi[1], cx ? d.psi_i[0] : d.chi[0],
                           cx ? d.psi_i[1] : d.chi[1]};
    for (const float* p : ptrs) {
      if (!p) return fail(LFM_ERR_INVALID_ARG, "lattice %d: null slot", l);
      if (!aligned16(p)) return fail(LFM_ERR_ALIGNMENT, "lattice %d: slot not 16-byte aligned", l);
    }
    lfm::BatchLattice& b = dev[l];
    b.N = d.N;
    b.level = d.level;
    for (int s = 0; s < 2; ++s) {
      b.pr[s] = d.psi_r[s];
      b.pi[s] = cx ? d.psi_i[s] : nullptr;
      b.chi[s] = d.chi[s];
    }
    b.c = lfm::make_step_consts(d.dt2, d.kappa, d.lambda_self, d.chi0, d.e0_sq, d.epsilon_w, 0,
                                0, 0, 0);
    b.lut = device_lut(d.mask_table, &d.lut);
  }
  int regs = 128;
  cudaError_t e = lfm::batch_kernel_regs(&regs);
  if (e != cudaSuccess) return cuda_fail(e, "batch kernel attributes");
  int device = 0, sms = 148;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  BatchPlan plan;
  rc = plan_batch(lattices, count, t, regs, sms, &plan);
  if (rc) return rc;
  for (int l = 0; l < count; ++l) {
    dev[l].TJ = plan.TJ[l];
    dev[l].IC = plan.IC[l];
    dev[l].stage_floats = plan.stage_floats[l];
  }
  lfm_batch* B = new lfm_batch;
  B->device = device;
  B->stages = t.stages;
  B->tab_off = plan.tab_off;
  B->nitems = (int)plan.items.size();
  B->real_items = plan.real_items;
  for (int c = 0; c < lfm::kBatchClasses; ++c) {
    B->class_off[c] = plan.class_off[c];
    B->class_n[c] = plan.class_n[c];
  }
  B->threads = plan.threads;
  B->smem = plan.smem;
  B->grid = plan.grid;
  e = cudaMalloc(&B->d_lat, sizeof(lfm::BatchLattice) * count);
  if (e == cudaSuccess)
    e = cudaMemcpy(B->d_lat, dev.data(), sizeof(lfm::BatchLattice) * count,
                   cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&B->d_items, sizeof(lfm::BatchItem) * plan.items.size());
  if (e == cudaSuccess)
    e = cudaMemcpy(B->d_items, plan.items.data(), sizeof(lfm::BatchItem) * plan.items.size(),
                   cudaMemcpyHostToDevice);
  const size_t counters = (lfm::kBatchClasses + 1) * sizeof(int);
  if (e == cudaSuccess) e = cudaMalloc(&B->d_counters, counters);
  if (e == cudaSuccess) e = cudaMemset(B->d_counters, 0, counters);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    lfm_batch_destroy(B);
    return cuda_fail(e, "batch descriptors");
  }
  *out = B;
  return LFM_OK;
}

int lfm_batch_step(lfm_batch* batch, int parity, int damp_prev, void* stream) {
  if (!batch) return fail(LFM_ERR_INVALID_ARG, "null batch");
  if (parity != 0 && parity != 1) return fail(LFM_ERR_INVALID_ARG, "parity %d", parity);
  int* status = nullptr;
  int rc = status_word(&status);
  if (rc) return rc;
  lfm::BatchParams P{};
  P.lattices = batch->d_lat;
  P.items = batch->d_items;
  P.nitems = batch->nitems;
  P.real_items = batch->real_items;
  for (int c = 0; c < lfm::kBatchClasses; ++c) {
    P.class_off[c] = batch->class_off[c];
    P.class_n[c] = batch->class_n[c];
  }
  P.parity = parity;
  P.damp_prev = damp_prev ? 1 : 0;
  P.stages = batch->stages;
  P.tab_off = batch->tab_off;
  P.status = status;
  P.next_item = batch->d_counters;
  P.retired = batch->d_counters + lfm::kBatchClasses;
  cudaError_t e = lfm::launch_batch_step(P, batch->threads, batch->smem, batch->grid,
                                         static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "batch step launch");
  return LFM_OK;
}

int lfm_batch_info(const lfm_batch* batch, int* items, int* threads, int* grid, int* smem) {
  if (!batch) return fail(LFM_ERR_INVALID_ARG, "null batch");
  if (items) *items = batch->nitems;
  if (threads) *threads = batch->threads;
  if (grid) *grid = batch->grid;
  if (smem) *smem = batch->smem;
  return LFM_OK;
}

int lfm_batch_destroy(lfm_batch* batch) {
  if (!batch) return LFM_OK;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(batch->device);
  if (batch->d_lat) cudaFree(batch->d_lat);
  if (batch->d_items) cudaFree(batch->d_items);
  if (batch->d_counters) cudaFree(batch->d_counters);
  cudaSetDevice(prev);
  delete batch;
  return LFM_OK;
}

int lfm_selftest_device_timeout(unsigned long long limit_ns, void* stream) {
  if (limit_ns < 1000ull || limit_ns > 1000000000ull)
    return fail(LFM_ERR_INVALID_ARG, "limit %llu ns not in [1 us, 1 s]", limit_ns);
  int* status = nullptr;
  int rc = status_word(&status);
  if (rc != LFM_OK) return rc;
  cudaError_t e = lfm::launch_wait_selftest(status, limit_ns, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "wait self-test launch");
  return LFM_OK;
}

int lfm_device_status(int* status_out, int clear) {
  if (!status_out) return fail(LFM_ERR_INVALID_ARG, "null output");
  // Every kernel of this process on the device is finished before the read,
  // whatever stream (blocking or not) it was launched on.
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceSynchronize");
  int v = 0;
  e = cudaMemcpyFromSymbol(&v, g_lfm_status, sizeof v);
  if (e != cudaSuccess) return cuda_fail(e, "read status word");
  if (clear && v) {
    // Clear only the bits just read, atomically on the device: a bit that a
    // kernel launched meanwhile by another host thread sets stays set.
    e = lfm::launch_status_clear(v);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail(e, "clear status word");
  }
  *status_out = v;
  return LFM_OK;
}

}  // extern "C"
