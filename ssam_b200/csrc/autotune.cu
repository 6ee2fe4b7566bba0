// Launch-parameter defaults and the measured-choice cache for the 2D kernels.
#include <map>
#include <mutex>
#include <tuple>

#include "autotune.h"
#include "ssam_internal.cuh"

namespace ssam {

namespace {

// Grid sizes are bucketed by log2 so one measurement serves similar grids.
int log2_bucket(int64_t v) {
  int b = 0;
  while (v > 1) {
    v >>= 1;
    ++b;
  }
  return b;
}

using TuneKey = std::tuple<int, int, int, int, int, int, int, int, int>;

struct TuneCache {
  std::mutex mu;
  std::map<TuneKey, TuneChoice> choices;
  std::map<TuneKey, int> depths;  // t field unused (0)
};

TuneCache& cache() {
  static TuneCache c;
  return c;
}

TuneKey make_key(int dtype, int rl, int rr, int rt, int rb, int star, int t, int64_t w,
                 int64_t h) {
  return TuneKey{dtype, rl, rr, rt, rb, star, t, log2_bucket(w), log2_bucket(h)};
}

}  // namespace

bool tune_lookup_2d(int dtype, int rl, int rr, int rt, int rb, int star, int t,
                    int64_t w, int64_t h, TuneChoice* out) {
  TuneCache& c = cache();
  std::lock_guard<std::mutex> g(c.mu);
  auto it = c.choices.find(make_key(dtype, rl, rr, rt, rb, star, t, w, h));
  if (it == c.choices.end()) return false;
  *out = it->second;
  return true;
}

void tune_store_2d(int dtype, int rl, int rr, int rt, int rb, int star, int t, int64_t w,
                   int64_t h, TuneChoice ch) {
  TuneCache& c = cache();
  std::lock_guard<std::mutex> g(c.mu);
  c.choices[make_key(dtype, rl, rr, rt, rb, star, t, w, h)] = ch;
}

TuneChoice tune_default_2d(int dtype, int rl, int rr, int rt, int rb, int star, int t) {
  const int reach = rl > rr ? rl : rr;
  TuneChoice c{8, 4};
  if (dtype == SSAM_F64 && reach > 2) c.p = 4;
  if (reach > 5) c.p = 4;
  (void)rt;
  (void)rb;
  (void)star;
  (void)t;
  return c;
}

int tune_depth_2d(int dtype, int rl, int rr, int rt, int rb, int star, int64_t w,
                  int64_t h, int steps) {
  if (steps <= 1) return 1;
  {
    TuneCache& c = cache();
    std::lock_guard<std::mutex> g(c.mu);
    auto it = c.depths.find(make_key(dtype, rl, rr, rt, rb, star, 0, w, h));
    if (it != c.depths.end()) return it->second;
  }
  const int reach = rl > rr ? rl : rr;
  (void)star;
  (void)rt;
  (void)rb;
  if (reach <= 1) return 4;
  if (reach <= 2) return 2;
  return 1;
}

}  // namespace ssam
