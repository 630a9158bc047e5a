// Tile-configuration table of the fused step kernel: entries forced by the
// autotuner (lfm_tune_set) and the last configuration each (level, N) ran.
#pragma once

namespace lfm {

struct TileConfig {
  int tj;       // rows per tile
  int stages;   // shared-memory ring depth
  int ic;       // planes per chunk (0 = automatic)
  int threads;  // CTA size (recorded)
  int smem;     // dynamic shared memory bytes (recorded)
  int vec;      // cells per thread along k (0 = automatic)
};

bool tune_lookup(int level, int N, TileConfig* out);
void tune_record(int level, int N, const TileConfig& used);

}  // namespace lfm
