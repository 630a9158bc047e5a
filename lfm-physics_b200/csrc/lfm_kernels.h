// Internal interface between the C ABI (capi.cu) and the kernel files.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "lfm_math.cuh"

namespace lfm {

// Everything one step kernel launch needs.  Protocol mode: all *_out
// pointers set, inputs and outputs distinct, mask = N^3 device array.
// Resident mode: pr_out == pr_prev (and likewise pi, chi), the *_prev_out
// pointers null, mask null and lut set.
struct StepArgs {
  int level;  // lfm_level
  int N;
  StepConsts c;
  const float* pr;
  const float* pi;
  const float* chi;
  const float* pr_prev;
  const float* pi_prev;
  const float* chi_prev;
  float* pr_out;
  float* pi_out;
  float* chi_out;
  float* pr_prev_out;
  float* pi_prev_out;
  float* chi_prev_out;
  const float* mask;   // N^3 mask or null
  MaskLut lut;         // used when mask is null
  const float* sa;     // raw S_a (3*N^3) or null
  float* sa_clip_out;  // clipped S_a copy (protocol colour step) or null
  float* energy_out;   // COLOR: |Psi_a|^2 of the new fields (3*N^3) or null
  int damp_prev;       // multiply the previous-step fields by (1-mask) on read
  int comp;            // compensated Delta form: *_prev hold increments, updated in place
  // Split chi (REAL, COMPLEX; resident layout only): chi = chi0 + hi + lo with
  // hi in chi / chi_prev / chi_out and lo in the three pointers below.
  int split;
  const float* chi_lo;
  const float* chi_lo_prev;
  float* chi_lo_out;
  int* status;         // device status word for bounded waits
  // Slab of a lattice split along i (slab == 0: the whole periodic lattice).
  // The arrays hold ni planes of N x N; the step updates planes [i_lo, i_hi)
  // and reads planes i_lo - 1 and i_hi as they are (ghost planes, no wrap);
  // array plane p is global plane p + i_off (for the sponge).
  int slab;
  int ni, i_lo, i_hi, i_off;
};

cudaError_t launch_direct_step(const StepArgs& a, cudaStream_t stream);

// Fused 2.5D kernel (N % 4 == 0).  Returns cudaErrorNotSupported when the
// size has no tile configuration, so the caller can take the direct path.
cudaError_t launch_tma_step(const StepArgs& a, cudaStream_t stream);

// A bounded wait that must give up (failure-detection test, step_tma.cu).
cudaError_t launch_wait_selftest(int* status, uint64_t limit_ns, cudaStream_t stream);
// Clears `bits` of the device status word (atomically, on the legacy stream).
cudaError_t launch_status_clear(int bits);

// S_a pipeline pieces (helmholtz.cu).
cudaError_t launch_color_energy(const float* pr, const float* pi, float* e, int N,
                                cudaStream_t stream);
cudaError_t launch_helmholtz_multiply_gd(float2* spec, int N, double gamma, double d,
                                         cudaStream_t stream);
cudaError_t launch_clip(const float* in, float* out, int64_t count, cudaStream_t stream);
// The split S_a transform (spectral.cu): which N it serves, the filter table
// ((N/2+1)^3 floats) and the fused pass along i on spec[3][N][N*(N/2+1)].
bool helmholtz_xpass_supported(int N);
cudaError_t launch_helmholtz_table(float* table, int N, double gamma, double d,
                                   cudaStream_t stream);
cudaError_t launch_helmholtz_xpass(float2* spec, const float* table, const float2* twiddles,
                                   int N, cudaStream_t stream);
// Uploads the register DFTs' twiddles to the current device's constant memory
// (once per device, before the first pass along i; synchronous).
cudaError_t upload_dft_twiddles();

// Poisson equilibration pieces (poisson.cu).
cudaError_t launch_poisson_rhs(const float* pr, const float* pi, float* rhs, int N, int colours,
                               float kappa, float e0_sq, cudaStream_t stream);
cudaError_t launch_poisson_divide(const float2* in, double2* out, int N, cudaStream_t stream);
cudaError_t launch_poisson_finish(const double* dchi, float* chi, int N, float chi0,
                                  double radius, int frozen, cudaStream_t stream);

// Adjoint step (adjoint.cu).  g_out / g_in: adjoints of (psi_r, psi_r_prev,
// psi_i, psi_i_prev, chi, chi_prev) after / before the step.
cudaError_t launch_adjoint_step(int level, int N, const float* pr, const float* pi,
                                const float* chi, const float* chi_next, const MaskLut& lut,
                                const float* const g_out[6], float* const g_in[6],
                                const StepConsts& c, cudaStream_t stream);

}  // namespace lfm
