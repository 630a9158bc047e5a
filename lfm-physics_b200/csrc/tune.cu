// Tile-configuration table shared by the fused kernels and the C ABI.
#include <map>
#include <mutex>
#include <utility>

#include "lfm_b200.h"
#include "lfm_tune.h"

namespace lfm {
namespace {
std::mutex g_mu;
std::map<std::pair<int, int>, TileConfig> g_forced;
std::map<std::pair<int, int>, TileConfig> g_used;
}  // namespace

bool tune_lookup(int level, int N, TileConfig* out) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_forced.find({level, N});
  if (it == g_forced.end()) return false;
  *out = it->second;
  return true;
}

void tune_record(int level, int N, const TileConfig& used) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_used[{level, N}] = used;
}

}  // namespace lfm

extern "C" {

int lfm_tune_set(int level, int N, int vec, int tj, int stages, int ic) {
  if (level < 0 || level > 2 || N < 2) return LFM_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(lfm::g_mu);
  if (tj <= 0) {
    lfm::g_forced.erase({level, N});
    return LFM_OK;
  }
  if (vec != 0 && vec != 1 && vec != 2 && vec != 4) return LFM_ERR_INVALID_ARG;
  lfm::g_forced[{level, N}] = lfm::TileConfig{tj, stages, ic, 0, 0, vec};
  return LFM_OK;
}

int lfm_tune_get(int level, int N, int* vec, int* tj, int* stages, int* ic, int* threads,
                 int* smem) {
  std::lock_guard<std::mutex> lk(lfm::g_mu);
  auto it = lfm::g_used.find({level, N});
  if (it == lfm::g_used.end()) return LFM_ERR_INVALID_ARG;
  if (vec) *vec = it->second.vec;
  if (tj) *tj = it->second.tj;
  if (stages) *stages = it->second.stages;
  if (ic) *ic = it->second.ic;
  if (threads) *threads = it->second.threads;
  if (smem) *smem = it->second.smem;
  return LFM_OK;
}

}  // extern "C"
