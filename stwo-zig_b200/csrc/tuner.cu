// Launch-shape autotuner (declarations in tuner.hpp).
#include "tuner.hpp"

#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <tuple>

namespace sb {

namespace {

using Key = std::tuple<uint32_t, uint32_t, uint32_t>;

struct Table {
  std::mutex mu;
  std::map<Key, TuneEntry> done;
  std::map<Key, bool> tuning;  // keys being tuned by some thread (the others run variant 0 meanwhile)
};

Table& table() {
  static Table t;
  return t;
}

std::atomic<int> g_force{-1};

// One complete run of variant v on `stream`, timed with a pair of events (milliseconds).
cudaError_t time_once(cudaStream_t stream, cudaEvent_t a, cudaEvent_t b, const std::function<cudaError_t(int)>& run,
                      int v, float* ms) {
  cudaError_t e = cudaEventRecord(a, stream);
  if (e == cudaSuccess) e = run(v);
  if (e == cudaSuccess) e = cudaEventRecord(b, stream);
  if (e == cudaSuccess) e = cudaEventSynchronize(b);
  if (e == cudaSuccess) e = cudaEventElapsedTime(ms, a, b);
  return e;
}

}  // namespace

cudaError_t tuned_run(TuneOp op, uint32_t log_size, uint32_t n_cols, int n_variants, bool rerunnable,
                      cudaStream_t stream, const std::function<cudaError_t(int)>& run) {
  const int forced = g_force.load(std::memory_order_relaxed);
  if (forced >= 0) return run(std::min(forced, n_variants - 1));
  if (n_variants <= 1 || !rerunnable) return run(0);
  const Key key{op, log_size, n_cols};
  Table& t = table();
  {
    std::lock_guard<std::mutex> g(t.mu);
    auto it = t.done.find(key);
    if (it != t.done.end()) return run(it->second.variant);
    if (t.tuning.count(key)) return run(0);
    t.tuning[key] = true;
  }
  // Three interleaved rounds over the variants, each keeping its fastest run: work that other
  // streams put on the device at the same time only slows a run down, and interleaving spreads it
  // over the variants.
  TuneEntry entry{op, log_size, n_cols, 0, {0, 0, 0, 0}};
  const int nv = std::min(n_variants, TUNE_MAX_VARIANTS);
  cudaEvent_t a = nullptr, b = nullptr;
  cudaError_t e = cudaEventCreate(&a);
  if (e == cudaSuccess) e = cudaEventCreate(&b);
  for (int round = 0; round < 3 && e == cudaSuccess; ++round)
    for (int v = 0; v < nv && e == cudaSuccess; ++v) {
      float ms = 0;
      e = time_once(stream, a, b, run, v, &ms);
      if (e == cudaSuccess && (round == 0 || ms < entry.ms[v])) entry.ms[v] = ms;
    }
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  for (int v = 1; v < nv; ++v)
    if (entry.ms[v] < entry.ms[entry.variant]) entry.variant = v;
  // The outputs are the last variant's; a run of the chosen one is not needed (same bits).
  std::lock_guard<std::mutex> g(t.mu);
  t.tuning.erase(key);
  if (e == cudaSuccess) t.done[key] = entry;
  return e;
}

void tune_force(int v) { g_force.store(v < 0 ? -1 : v, std::memory_order_relaxed); }

std::vector<TuneEntry> tune_table() {
  Table& t = table();
  std::lock_guard<std::mutex> g(t.mu);
  std::vector<TuneEntry> out;
  for (const auto& kv : t.done) out.push_back(kv.second);
  return out;
}

void tune_clear() {
  Table& t = table();
  std::lock_guard<std::mutex> g(t.mu);
  t.done.clear();
}

}  // namespace sb
