// wg_tune.cu -- the autotuner's cache and timing (see wg_common.cuh).
//
// Tuned operations and their candidates (every candidate gives identical
// results; only the time differs):
//   commute     wg_commutation_bits with algo 0, 1-4 mask words:
//               0 ballot kernel; 1 bit-plane, 2,048-column tiles (256
//               threads); 2 bit-plane, 4,096-column tiles (1,024 threads, 1-2
//               words); 3 and 4 the same two tiles with at most 2,048 lhs rows
//               per CTA instead of up to 16,384;
//   bucket      the bucketed sort's target items per fine bucket:
//               640, 768, 896, 1,024, 1,280;
//   group_qwc   group_commuting chunk length, qwc mode: 256, 512, 1,024;
//   group_full  group_commuting chunk length, full mode: 64, 96, 128, 192.
// Classes: commute (words, log2 n_lhs, log2 n_rhs); bucket (words, log2
// products or terms, 0); group_* (words, log2 terms, 0), logs rounded up.

#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <tuple>

#include "wg_common.cuh"

namespace {

std::atomic<int> g_tune_mode{WG_TUNE_CACHED};
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, int> g_tune_cache;

struct OpInfo {
  int op;
  const char* name;
  int candidates;
};
constexpr OpInfo kOps[] = {
    {wg::kTuneCommute, "commute", 5},
    {wg::kTuneBucket, "bucket", 5},
    {wg::kTuneGroupQwc, "group_qwc", 3},
    {wg::kTuneGroupFull, "group_full", 4},
};

const OpInfo* op_info(int op) {
  for (const auto& o : kOps)
    if (o.op == op) return &o;
  return nullptr;
}

const OpInfo* op_named(const std::string& name) {
  for (const auto& o : kOps)
    if (name == o.name) return &o;
  return nullptr;
}

}  // namespace

namespace wg {

int tune_mode() { return g_tune_mode.load(std::memory_order_relaxed); }

int tune_candidates(int op) {
  const OpInfo* o = op_info(op);
  return o ? o->candidates : 0;
}

int tune_lookup(int op, int words, int a, int b) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune_cache.find({op, words, a, b});
  return it == g_tune_cache.end() ? -1 : it->second;
}

void tune_store(int op, int words, int a, int b, int choice) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_cache[{op, words, a, b}] = choice;
}

int ceil_log2(size_t n) {
  int k = 0;
  while (k < 63 && (size_t{1} << k) < n) ++k;
  return k;
}

float tune_time(cudaStream_t s, bool (*run)(void*), void* ctx) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  check_cuda(cudaEventCreate(&e0), "create tuning event");
  try {
    check_cuda(cudaEventCreate(&e1), "create tuning event");
    check_cuda(cudaStreamSynchronize(s), "start tuning run");
    check_cuda(cudaEventRecord(e0, s), "record tuning event");
    const bool ok = run(ctx);
    check_cuda(cudaEventRecord(e1, s), "record tuning event");
    check_cuda(cudaEventSynchronize(e1), "finish tuning run");
    float ms = -1.0f;
    if (ok) check_cuda(cudaEventElapsedTime(&ms, e0, e1), "read tuning time");
    (void)cudaEventDestroy(e0);
    (void)cudaEventDestroy(e1);
    return ok ? ms : -1.0f;
  } catch (...) {
    (void)cudaEventDestroy(e0);
    if (e1) (void)cudaEventDestroy(e1);
    throw;
  }
}

}  // namespace wg

extern "C" {

int wg_autotune_set_mode(int mode) {
  return wg::guarded([&] {
    if (mode != WG_TUNE_OFF && mode != WG_TUNE_CACHED && mode != WG_TUNE_SEARCH)
      wg::throw_invalid("autotune mode must be WG_TUNE_OFF, WG_TUNE_CACHED or WG_TUNE_SEARCH");
    g_tune_mode.store(mode, std::memory_order_relaxed);
  });
}

int wg_autotune_get_mode(int* mode) {
  return wg::guarded([&] {
    if (!mode) wg::throw_invalid("autotune mode output is null");
    *mode = wg::tune_mode();
  });
}

int wg_autotune_export(char* buf, size_t cap, size_t* needed) {
  return wg::guarded([&] {
    std::string text;
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      for (const auto& [key, choice] : g_tune_cache) {
        const auto& [op, words, a, b] = key;
        const OpInfo* o = op_info(op);
        text += std::string(o ? o->name : "?") + " " + std::to_string(words) + " " + std::to_string(a) + " " +
                std::to_string(b) + " " + std::to_string(choice) + "\n";
      }
    }
    if (needed) *needed = text.size() + 1;
    if (buf && cap) {
      if (cap < text.size() + 1) wg::throw_invalid("autotune export buffer is too small");
      std::memcpy(buf, text.c_str(), text.size() + 1);
    }
  });
}

int wg_autotune_import(const char* text) {
  return wg::guarded([&] {
    if (!text) wg::throw_invalid("autotune import text is null");
    std::istringstream in(text);
    std::string line;
    std::map<std::tuple<int, int, int, int>, int> add;
    int lineno = 0;
    while (std::getline(in, line)) {
      ++lineno;
      if (line.find_first_not_of(" \t\r") == std::string::npos || line[0] == '#') continue;
      std::istringstream ls(line);
      std::string name;
      long long words = -1, a = -1, b = -1, choice = -1;
      std::string rest;
      if (!(ls >> name >> words >> a >> b >> choice) || (ls >> rest))
        wg::throw_invalid("autotune line " + std::to_string(lineno) + ": expected '<op> <words> <a> <b> <choice>'");
      const OpInfo* o = op_named(name);
      if (!o) wg::throw_invalid("autotune line " + std::to_string(lineno) + ": unknown operation '" + name + "'");
      if (words < 0 || a < 0 || a > 63 || b < 0 || b > 63 || choice < 0 || choice >= o->candidates ||
          words > (1 << 20))
        wg::throw_invalid("autotune line " + std::to_string(lineno) + ": value out of range");
      add[{o->op, static_cast<int>(words), static_cast<int>(a), static_cast<int>(b)}] = static_cast<int>(choice);
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (const auto& [k, v] : add) g_tune_cache[k] = v;
  });
}

int wg_autotune_clear(void) {
  return wg::guarded([&] {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache.clear();
  });
}

}  // extern "C"
