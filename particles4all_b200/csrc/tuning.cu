// tuning.cu — launch shapes of the neighbour kernels per size bucket (p4a_tune_*).
//
// Each tuned kernel is compiled in kVariants launch shapes (threads per block x
// minimum resident blocks per SM, which sets the register budget); the
// per-particle arithmetic is identical in all of them, so a shape changes speed,
// never results. The table maps a launch's particle count (the scene for plain
// launches, the frame's total for batched ones) to a shape; the autotuner
// (particles4all_b200/autotune.py) measures the shapes per size bucket and fills it.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <utility>
#include <vector>

#include "../../include/p4a.h"
#include "p4a_internal.h"

namespace p4a {

const LaunchShape kShapes[TK_COUNT][kVariants] = {
    {{256, 4}, {256, 5}, {256, 6}, {128, 8}, {128, 10}, {128, 12}},   // lambda
    {{256, 5}, {256, 4}, {256, 6}, {128, 10}, {128, 8}, {128, 12}},   // delta
    {{256, 4}, {256, 5}, {256, 3}, {128, 8}, {128, 10}, {128, 6}},    // xsph + normals
    {{128, 10}, {128, 8}, {128, 12}, {256, 5}, {256, 4}, {64, 20}},   // aniso
};

namespace {
std::mutex g_mu;
std::vector<std::pair<int64_t, int>> g_table[kTunedTables];  // (max particles, variant), ascending
// the kernel whose launch shapes table k selects among
int family(int k) { return k < TK_COUNT ? k : k - TK_COUNT; }
int lookup(int table, int64_t particles) {
  for (const auto& b : g_table[table])
    if (particles <= b.first) return b.second;
  return 0;
}
}  // namespace

int tuned_variant(int kernel, int64_t particles) {
  if (kernel < 0 || kernel >= TK_COUNT) return 0;
  std::lock_guard<std::mutex> l(g_mu);
  return lookup(kernel, particles);
}

int tuned_variant_batched(int kernel, int64_t particles) {
  if (kernel < 0 || kernel >= TK_COUNT) return 0;
  std::lock_guard<std::mutex> l(g_mu);
  const int b = TK_COUNT + kernel;
  if (b < kTunedTables && !g_table[b].empty()) return lookup(b, particles);
  return lookup(kernel, particles);
}

}  // namespace p4a

using namespace p4a;

extern "C" {

int p4a_kernel_shapes(int32_t kernel, int32_t* threads, int32_t* min_blocks, int32_t max, int32_t* count) {
  if (kernel < 0 || kernel >= kTunedTables || !count || max < 0) return P4A_ERR_ARG;
  const int32_t c = std::min<int32_t>(max, kVariants);
  const int f = family(kernel);
  for (int32_t v = 0; v < c; v++) {
    if (threads) threads[v] = kShapes[f][v].threads;
    if (min_blocks) min_blocks[v] = kShapes[f][v].minBlocks;
  }
  *count = kVariants;
  return P4A_OK;
}

int p4a_tune_set(int32_t kernel, int64_t max_particles, int32_t variant) {
  if (kernel < 0 || kernel >= kTunedTables || variant < 0 || variant >= kVariants || max_particles < 0)
    return P4A_ERR_ARG;
  std::lock_guard<std::mutex> l(g_mu);
  auto& t = g_table[kernel];
  auto it = std::find_if(t.begin(), t.end(), [&](const std::pair<int64_t, int>& b) { return b.first == max_particles; });
  if (it != t.end()) it->second = variant;
  else t.emplace_back(max_particles, variant);
  std::sort(t.begin(), t.end());
  return P4A_OK;
}

int p4a_tune_clear(int32_t kernel) {
  if (kernel < -1 || kernel >= kTunedTables) return P4A_ERR_ARG;
  std::lock_guard<std::mutex> l(g_mu);
  for (int k = 0; k < kTunedTables; k++)
    if (kernel < 0 || kernel == k) g_table[k].clear();
  return P4A_OK;
}

int p4a_tune_get(int32_t kernel, int64_t particles, int32_t* variant) {
  if (kernel < 0 || kernel >= kTunedTables || !variant) return P4A_ERR_ARG;
  *variant = kernel < TK_COUNT ? tuned_variant(kernel, particles) : tuned_variant_batched(family(kernel), particles);
  return P4A_OK;
}

}  // extern "C"
