// Device-side description of a batch of lattices (batch.cu, step_tma.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "lfm_math.cuh"

namespace lfm {

// One lattice of the batch: its two slots per field, constants, mask table
// and the tile shape the work list was cut with.
struct BatchLattice {
  int N;
  int level;
  float* pr[2];
  float* pi[2];
  float* chi[2];
  StepConsts c;
  MaskLut lut;
  int TJ;            // rows per tile
  int IC;            // planes per chunk
  int stage_floats;  // floats of one shared-memory stage for this lattice
};

struct BatchItem {
  int lattice;
  int j0, i0, i1;
};

struct BatchParams {
  const BatchLattice* lattices;
  const BatchItem* items;
  int nitems;
  int parity;     // slot holding the current fields
  int damp_prev;  // previous-field slots hold undamped values
  int stages;
  int* status;
};

// Launches one step of every lattice of one level (REAL or COMPLEX).
cudaError_t launch_batch_step(int level, const BatchParams& B, int threads, int smem, int grid,
                              cudaStream_t stream);

// Registers per thread of the batch kernel of a level (for the planner).
cudaError_t batch_kernel_regs(int level, int* regs);

}  // namespace lfm
