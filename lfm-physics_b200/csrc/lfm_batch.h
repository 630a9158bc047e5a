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
  int level;  // LFM_REAL or LFM_COMPLEX, copied from the lattice
  int j0, j1, i0, i1;  // rows [j0, j1), planes [i0, i1)
};

struct BatchParams {
  const BatchLattice* lattices;
  const BatchItem* items;  // REAL items first, then COMPLEX, each sorted by cost
  int nitems;
  int real_items;  // items[0, real_items) are REAL
  int parity;     // slot holding the current fields
  int damp_prev;  // previous-field slots hold undamped values
  int stages;
  int tab_off;     // float offset of the shared-memory sponge table, -1 = read through L1
  int* status;
  int* next_item;  // work-list counters (REAL, COMPLEX), 0 between launches
  int* retired;    // CTAs that took their last item, 0 between launches
};

// Launches one step of every lattice of the batch.
cudaError_t launch_batch_step(const BatchParams& B, int threads, int smem, int grid,
                              cudaStream_t stream);

// Registers per thread of the batch kernel (for the planner).
cudaError_t batch_kernel_regs(int* regs);

}  // namespace lfm
