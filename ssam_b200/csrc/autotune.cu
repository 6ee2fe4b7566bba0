// Launch-parameter choice for the 2D kernels: built-in defaults, the cache of
// measured choices, the measuring autotuner (ssam_autotune_stencil2d) and the
// cache file format (ssam_autotune_save / ssam_autotune_load).
#include <stdio.h>

#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

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
  TuneChoice c{8, 4, dtype == SSAM_BF16 || dtype == SSAM_F16 ? 8 : 4};
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

// ------------------------------------------------------------- measuring --

namespace ssam {

// Shared with api.cu.
int check_grid2d(const void* src, const void* dst, int64_t w, int64_t h, int64_t pitch,
                 int dtype, int boundary);
int stencil_matrix(int shape, int radius, const double* coeffs, int steps, int boundary,
                   std::vector<double>* out);

void tune_store_depth_2d(int dtype, int rl, int rr, int rt, int rb, int star, int64_t w,
                         int64_t h, int depth) {
  TuneCache& c = cache();
  std::lock_guard<std::mutex> g(c.mu);
  c.depths[make_key(dtype, rl, rr, rt, rb, star, 0, w, h)] = depth;
}

namespace {

struct Candidate {
  Key2D key;
  Kernel2DInfo info;
};

// Mean time of one launch (ms), after one warm-up launch; enough repetitions
// to cover ~2 ms.
int time_launch(const Kernel2DInfo& info, const Launch2D& a, cudaEvent_t e0, cudaEvent_t e1,
                double* ms_out) {
  cudaError_t e = info.launch(a);
  if (e != cudaSuccess) return fail_cuda(e, "autotune launch");
  SSAM_CUDA_TRY(cudaEventRecord(e0, a.stream));
  e = info.launch(a);
  if (e != cudaSuccess) return fail_cuda(e, "autotune launch");
  SSAM_CUDA_TRY(cudaEventRecord(e1, a.stream));
  SSAM_CUDA_TRY(cudaEventSynchronize(e1));
  float one = 0.f;
  SSAM_CUDA_TRY(cudaEventElapsedTime(&one, e0, e1));
  int reps = one > 0.f ? (int)(2.0f / one) : 20;
  reps = reps < 1 ? 1 : (reps > 20 ? 20 : reps);
  SSAM_CUDA_TRY(cudaEventRecord(e0, a.stream));
  for (int i = 0; i < reps; ++i) {
    e = info.launch(a);
    if (e != cudaSuccess) return fail_cuda(e, "autotune launch");
  }
  SSAM_CUDA_TRY(cudaEventRecord(e1, a.stream));
  SSAM_CUDA_TRY(cudaEventSynchronize(e1));
  float ms = 0.f;
  SSAM_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
  *ms_out = ms / reps;
  return SSAM_OK;
}

// Greedy chain of fused depths (largest first) covering `steps`.
std::vector<int> chain_for(const std::vector<int>& depths_desc, int steps) {
  std::vector<int> chain;
  for (int left = steps; left > 0;) {
    bool placed = false;
    for (int t : depths_desc)
      if (t <= left) {
        chain.push_back(t);
        left -= t;
        placed = true;
        break;
      }
    if (!placed) break;
  }
  return chain;
}

}  // namespace
}  // namespace ssam

using namespace ssam;

extern "C" int ssam_autotune_stencil2d(const void* src, void* dst, int64_t width,
                                       int64_t height, int64_t pitch, int dtype, int shape,
                                       int radius, const double* coeffs, int steps,
                                       int boundary, void* stream,
                                       ssam_tune_report* report) {
  int st = check_grid2d(src, dst, width, height, pitch, dtype, boundary);
  if (st != SSAM_OK) return st;
  std::vector<double> m;
  st = stencil_matrix(shape, radius, coeffs, steps, boundary, &m);
  if (st != SSAM_OK) return st;
  const int r = radius, star = shape == SSAM_STAR ? 1 : 0;
  cudaStream_t s = (cudaStream_t)stream;

  std::vector<Candidate> cands;
  list_2d(dtype, r, r, r, r, star,
          [](const Key2D& k, const Kernel2DInfo& info, void* u) {
            ((std::vector<Candidate>*)u)->push_back(Candidate{k, info});
          },
          &cands);
  if (cands.empty()) return fail(SSAM_ERR_UNSUPPORTED, "no kernel compiled for this stencil");

  cudaEvent_t e0, e1;
  SSAM_CUDA_TRY(cudaEventCreate(&e0));
  SSAM_CUDA_TRY(cudaEventCreate(&e1));
  std::map<int, std::pair<double, TuneChoice>> best;  // fused depth -> (ms, choice)
  int timed = 0;
  for (const Candidate& c : cands) {
    if (c.key.t > steps) continue;
    if (boundary == SSAM_BOUNDARY_CLAMP && c.key.t != 1) continue;
    for (int warps : {2, 4, 8}) {
      Launch2D a{src, dst, width, height, pitch, 0, height, boundary, m.data(), warps, s};
      double ms = 0;
      st = time_launch(c.info, a, e0, e1, &ms);
      if (st != SSAM_OK) break;
      ++timed;
      auto it = best.find(c.key.t);
      if (it == best.end() || ms < it->second.first)
        best[c.key.t] = {ms, TuneChoice{c.key.p, warps, c.key.v}};
    }
    if (st != SSAM_OK) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != SSAM_OK) return st;
  if (best.empty()) return fail(SSAM_ERR_UNSUPPORTED, "no candidate kernel for this run");

  for (auto& kv : best)
    tune_store_2d(dtype, r, r, r, r, star, kv.first, width, height, kv.second.second);

  // temporal depth: the cap whose launch chain is fastest for `steps`
  int best_depth = 1;
  double best_total = -1;
  for (auto& cap : best) {
    std::vector<int> depths;
    for (auto it = best.rbegin(); it != best.rend(); ++it)
      if (it->first <= cap.first) depths.push_back(it->first);
    double total = 0;
    for (int t : chain_for(depths, steps)) total += best[t].first;
    if (best_total < 0 || total < best_total) {
      best_total = total;
      best_depth = cap.first;
    }
  }
  tune_store_depth_2d(dtype, r, r, r, r, star, width, height, best_depth);
  if (report) {
    const TuneChoice& ch = best[best_depth].second;
    report->rows_per_thread = ch.p;
    report->warps_per_block = ch.warps;
    report->columns_per_thread = ch.v;
    report->fused_steps = best_depth;
    report->candidates = timed;
    report->ms_per_step = best_total / steps;
  }
  return SSAM_OK;
}

extern "C" int ssam_autotune_save(const char* path) {
  if (!path) return fail(SSAM_ERR_INVALID, "path must not be NULL");
  FILE* f = fopen(path, "w");
  if (!f) return fail(SSAM_ERR_INVALID, std::string("cannot write ") + path);
  TuneCache& c = cache();
  {
    std::lock_guard<std::mutex> g(c.mu);
    fprintf(f, "# ssam_b200 autotune cache v1\n");
    for (auto& kv : c.choices) {
      const TuneKey& k = kv.first;
      fprintf(f, "choice %d %d %d %d %d %d %d %d %d %d %d %d\n", std::get<0>(k),
              std::get<1>(k), std::get<2>(k), std::get<3>(k), std::get<4>(k),
              std::get<5>(k), std::get<6>(k), std::get<7>(k), std::get<8>(k), kv.second.p,
              kv.second.warps, kv.second.v);
    }
    for (auto& kv : c.depths) {
      const TuneKey& k = kv.first;
      fprintf(f, "depth %d %d %d %d %d %d %d %d %d\n", std::get<0>(k), std::get<1>(k),
              std::get<2>(k), std::get<3>(k), std::get<4>(k), std::get<5>(k), std::get<7>(k),
              std::get<8>(k), kv.second);
    }
  }
  tune3d_for_each(
      [](const int* k, const int* v, void* u) {
        fprintf((FILE*)u, "choice3d %d %d %d %d %d %d %d %d %d %d %d %d %d\n", k[0], k[1],
                k[2], k[3], k[4], k[5], k[6], v[0], v[1], v[2], v[3], v[4], k[7]);
      },
      f);
  depth3d_for_each(
      [](const int* k, int d, void* u) {
        fprintf((FILE*)u, "depth3d %d %d %d %d %d %d %d\n", k[0], k[1], k[2], k[3], k[4], k[5],
                d);
      },
      f);
  fclose(f);
  return SSAM_OK;
}

extern "C" int ssam_autotune_load(const char* path) {
  if (!path) return fail(SSAM_ERR_INVALID, "path must not be NULL");
  FILE* f = fopen(path, "r");
  if (!f) return fail(SSAM_ERR_INVALID, std::string("cannot read ") + path);
  TuneCache& c = cache();
  char line[512];
  int bad = 0;
  std::lock_guard<std::mutex> g(c.mu);
  while (fgets(line, sizeof line, f)) {
    int a[13];
    if (line[0] == '#' || line[0] == '\n') continue;
    if (sscanf(line, "choice %d %d %d %d %d %d %d %d %d %d %d %d", &a[0], &a[1], &a[2],
               &a[3], &a[4], &a[5], &a[6], &a[7], &a[8], &a[9], &a[10], &a[11]) == 12) {
      if (a[9] < 1 || a[10] < 1 || a[10] > 8 || a[11] < 1) { ++bad; continue; }
      c.choices[TuneKey{a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8]}] =
          TuneChoice{a[9], a[10], a[11]};
    } else if (int n3 = sscanf(line, "choice3d %d %d %d %d %d %d %d %d %d %d %d %d %d", &a[0],
                               &a[1], &a[2], &a[3], &a[4], &a[5], &a[6], &a[7], &a[8], &a[9],
                               &a[10], &a[11], &a[12]);
               n3 >= 11 && n3 <= 13) {
      if (n3 < 12) a[11] = 4;  // lines written before the V field: 4 columns a thread
      if (n3 < 13) a[12] = 1;  // lines written before the steps field: one step a launch
      if (a[7] < 1 || a[8] < 1 || a[9] < 1 || a[10] < 0 || a[10] > 1 || a[11] < 1 ||
          a[12] < 1 || a[12] > 2) {
        ++bad;
        continue;
      }
      const int key[8] = {a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[12]};
      tune3d_store(key, a + 7);
    } else if (sscanf(line, "depth3d %d %d %d %d %d %d %d", &a[0], &a[1], &a[2], &a[3], &a[4],
                      &a[5], &a[6]) == 7) {
      if (a[6] < 1 || a[6] > 2) { ++bad; continue; }
      depth3d_store(a, a[6]);
    } else if (sscanf(line, "depth %d %d %d %d %d %d %d %d %d", &a[0], &a[1], &a[2], &a[3],
                      &a[4], &a[5], &a[6], &a[7], &a[8]) == 9) {
      if (a[8] < 1) { ++bad; continue; }
      c.depths[TuneKey{a[0], a[1], a[2], a[3], a[4], a[5], 0, a[6], a[7]}] = a[8];
    } else {
      ++bad;
    }
  }
  fclose(f);
  if (bad) return fail(SSAM_ERR_INVALID, std::to_string(bad) + " malformed line(s) in " + path);
  return SSAM_OK;
}

extern "C" int ssam_autotune_clear(void) {
  {
    TuneCache& c = cache();
    std::lock_guard<std::mutex> g(c.mu);
    c.choices.clear();
    c.depths.clear();
  }
  tune3d_clear();
  return SSAM_OK;
}
