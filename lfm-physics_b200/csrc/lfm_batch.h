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

// Shape classes of a batch's work list, in the order the CTAs drain them.
// The fixed shapes are the tiles the 256-thread plan cuts the sweep sizes
// into (N, and TJ the lattice's largest tile; step_tma.cu compiles their
// marches with that geometry), REAL then COMPLEX, largest N first; N == 0 is
// a level's class for every other shape (run-time geometry).
struct BatchShape {
  int level, N, TJ;
};
constexpr int kBatchClasses = 12;
constexpr BatchShape kBatchShapes[kBatchClasses] = {
    {LFM_REAL, 96, 10},   {LFM_REAL, 80, 12},   {LFM_REAL, 64, 16},  {LFM_REAL, 48, 16},
    {LFM_REAL, 32, 32},   {LFM_REAL, 0, 0},     {LFM_COMPLEX, 96, 5}, {LFM_COMPLEX, 80, 6},
    {LFM_COMPLEX, 64, 8}, {LFM_COMPLEX, 48, 10}, {LFM_COMPLEX, 32, 16}, {LFM_COMPLEX, 0, 0}};

// The class of a lattice of this level, edge N and largest tile TJ.
constexpr int batch_class_of(int level, int N, int TJ) {
  int any = -1;
  for (int c = 0; c < kBatchClasses; ++c) {
    if (kBatchShapes[c].level != level) continue;
    if (kBatchShapes[c].N == N && kBatchShapes[c].TJ == TJ) return c;
    if (kBatchShapes[c].N == 0) any = c;
  }
  return any;
}

struct BatchParams {
  const BatchLattice* lattices;
  const BatchItem* items;  // grouped by shape class, each group sorted by cost
  int nitems;
  int real_items;  // items[0, real_items) are REAL
  int class_off[kBatchClasses], class_n[kBatchClasses];  // each class's items
  int parity;     // slot holding the current fields
  int damp_prev;  // previous-field slots hold undamped values
  int stages;
  int tab_off;     // float offset of the shared-memory sponge table, -1 = read through L1
  int* status;
  int* next_item;  // work-list counters, one per shape class, 0 between launches
  int* retired;    // CTAs that took their last item, 0 between launches
};

// Launches one step of every lattice of the batch.
cudaError_t launch_batch_step(const BatchParams& B, int threads, int smem, int grid,
                              cudaStream_t stream);

// Registers per thread of the batch kernel (for the planner).
cudaError_t batch_kernel_regs(int* regs);

}  // namespace lfm
