// Project autotuner: picks, for a graph's in-degree distribution, the layout
// bins (lanes-per-row bound of the SELL width classes, chunked-row threshold
// and chunk size), the shared-memory hot prefix and the sweep-kernel variant
// (edges per lane in flight, rows per CTA through CTAs per SM) by timing
// candidates on the graph itself, and remembers the pick per distribution
// signature in a text cache.
//
// No reference counterpart: the reference fixes its launch shape at compile
// time (BLOCK_SIZE, include/common.h:30; warp-per-row or thread-per-row
// chosen by the Makefile, src/pr/Makefile:17-47).
//
// Search (single graph): first the form -- the default exact-order layout
// against the blocked layout (GPR_LAYOUT_BLOCKED, which costs a sort of the
// edges at creation and pays on large graphs); then coordinate descent over
// the chosen form's knobs: for the exact order the kernel variant, hot
// prefix, lanes-per-row bound and chunk threshold / size; for the blocked
// form the rows per block, words per tile and the in-degree above which
// rows are summed in chunks rather than in blocks.  Each candidate is timed as the best of kReps solves of exactly
// `sweeps` sweeps (tol 0), device time of the sweep loop
// (gpr_pr_stats.loop_ms), and taken only when at least kMargin faster than the
// current pick.  The batch tuner first tries the blocked form for the whole
// batch (with its rows per block and words per tile); otherwise it groups
// graphs by signature and tunes the exact-order bins one group at a time on
// the whole batch, the other groups keeping their current picks.
//
// Cache file: one line per entry, later lines override earlier ones:
//   <signature> <sell_max> <chunk> <chunk_min> <hot_entries> <variant> <ms_per_sweep>
//       [<flags> <block_rows> <tile_words> [<blocked_long>]]
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <functional>
#include <map>
#include <string>
#include <vector>

#include "gpr.h"
#include "gpr_guard.h"

namespace {

constexpr int kReps = 3;
constexpr int kDefSell = 64, kDefChunk = 4096, kDefChunkMin = 4096, kDefHot = 32768;

struct Cfg {
  int sell_max = kDefSell, chunk = kDefChunk, chunk_min = kDefChunkMin, hot = kDefHot,
      variant = 0;
  // blocked form (0: library defaults)
  int flags = 0, block_rows = 0, tile_words = 0, blocked_long = 0;
  bool operator==(const Cfg &o) const {
    return sell_max == o.sell_max && chunk == o.chunk && chunk_min == o.chunk_min &&
           hot == o.hot && variant == o.variant && flags == o.flags &&
           block_rows == o.block_rows && tile_words == o.tile_words &&
           blocked_long == o.blocked_long;
  }
};

// Degree-distribution class: rounded log2 of the mean in-degree and a skew
// class from the largest in-degree over the mean (flat < 16, moderate < 256,
// heavy).  Single graphs also carry the rounded log2 of their size.
std::string signature(int m, long long nnz, const int *h_rowptr, int first, bool with_size) {
  long long maxdeg = 0;
  for (int v = 0; v < m; ++v) maxdeg = std::max<long long>(maxdeg, h_rowptr[first + v + 1] - h_rowptr[first + v]);
  const double avg = m > 0 ? (double)nnz / m : 0.0;
  const int db = (int)lround(log2(std::max(avg, 1.0)));
  const double skew = maxdeg / std::max(avg, 1.0);
  const int sc = skew < 16.0 ? 0 : (skew < 256.0 ? 1 : 2);
  char buf[64];
  if (with_size)
    snprintf(buf, sizeof(buf), "pr:m%d:d%d:s%d", (int)lround(log2(std::max(m, 1))), db, sc);
  else
    snprintf(buf, sizeof(buf), "batch:d%d:s%d", db, sc);
  return buf;
}

std::map<std::string, std::pair<Cfg, double>> load_cache(const char *path) {
  std::map<std::string, std::pair<Cfg, double>> c;
  if (!path) return c;
  FILE *f = fopen(path, "r");
  if (!f) return c;
  char line[512];
  while (fgets(line, sizeof(line), f)) {
    char key[128];
    Cfg x;
    double ms = 0;
    const int n = sscanf(line, "%127s %d %d %d %d %d %lf %d %d %d %d", key, &x.sell_max, &x.chunk,
                         &x.chunk_min, &x.hot, &x.variant, &ms, &x.flags, &x.block_rows,
                         &x.tile_words, &x.blocked_long);
    if (n == 7 || n == 10 || n == 11) c[key] = {x, ms};
  }
  fclose(f);
  return c;
}

void save_cache(const char *path, const std::string &key, const Cfg &x, double ms) {
  if (!path) return;
  FILE *f = fopen(path, "a");
  if (!f) return;
  fprintf(f, "%s %d %d %d %d %d %.6f %d %d %d %d\n", key.c_str(), x.sell_max, x.chunk,
          x.chunk_min, x.hot, x.variant, ms, x.flags, x.block_rows, x.tile_words, x.blocked_long);
  fclose(f);
}

gpr_layout_opts to_layout(const Cfg &x) {
  gpr_layout_opts l;
  memset(&l, 0, sizeof(l));
  l.sell_max = x.sell_max;
  l.chunk = x.chunk;
  l.chunk_min = x.chunk_min;
  l.hot_entries = x.hot;
  l.flags = x.flags;
  l.block_rows = x.block_rows;
  l.tile_words = x.tile_words;
  l.blocked_long = x.blocked_long;
  return l;
}

void fill_result(gpr_tune_result *out, const std::string &sig, const Cfg &x, double ms,
                 double ms0, int cands, int cached) {
  if (!out) return;
  memset(out, 0, sizeof(*out));
  out->layout = to_layout(x);
  out->variant = x.variant;
  out->ms_per_sweep = ms;
  out->default_ms_per_sweep = ms0;
  out->candidates = cands;
  out->from_cache = cached;
  snprintf(out->signature, sizeof(out->signature), "%s", sig.c_str());
}

// Host copy of a row-offset array given as host or device memory.
int host_rowptr(const int *any_rowptr, int n, std::vector<int> *h) {
  h->resize((size_t)n);
  return gpr_memcpy(h->data(), any_rowptr, sizeof(int) * (size_t)n);
}

// ---- single graph ---------------------------------------------------------

struct SingleBench {
  int m;
  long long nnz;
  const int *rp, *col, *od;
  int sweeps;
  std::vector<float> init, scores;
  int cands = 0;

  // ms per sweep of configuration x; +inf when it cannot run.
  double time(const Cfg &x) {
    gpr_graph *g = nullptr;
    const gpr_layout_opts l = to_layout(x);
    if (gpr_graph_create_ex(m, nnz, rp, col, od, &l, &g) != GPR_OK) return INFINITY;
    gpr_pr_opts o;
    gpr_pr_opts_default(&o);
    o.tol = 0.0;
    o.max_iter = sweeps;
    o.variant = x.variant;
    o.loop = GPR_LOOP_PERSISTENT;
    double best = INFINITY;
    for (int r = 0; r <= kReps; ++r) {  // first run warms up
      scores = init;
      gpr_pr_stats st;
      if (gpr_pagerank(g, scores.data(), &o, &st) != GPR_OK || st.iterations != sweeps) {
        best = INFINITY;
        break;
      }
      if (r > 0) best = std::min(best, st.loop_ms / sweeps);
    }
    gpr_graph_destroy(g);
    ++cands;
    return best;
  }
};

// A candidate must beat the current pick by this fraction to replace it, so
// run-to-run timing noise does not move the pick.
constexpr double kMargin = 0.03;

// Coordinate descent over one knob: keeps the best of `vals` applied to x.
template <typename F, typename T>
void descend(Cfg *x, double *best, const std::vector<T> &vals, F apply,
             const std::function<double(const Cfg &)> &time) {
  for (const T &v : vals) {
    Cfg y = *x;
    apply(&y, v);
    if (y == *x) continue;
    const double t = time(y);
    if (t < *best * (1.0 - kMargin)) {
      *best = t;
      *x = y;
    }
  }
}

}  // namespace

extern "C" {

int gpr_tune_signature(int m, long long nnz, const int *h_rowptr, int batch, char *buf, int len) {
  GPR_ENTRY_BEGIN
  if (m < 0 || nnz < 0 || (m > 0 && !h_rowptr) || !buf || len < 1) return GPR_EINVAL;
  const std::string s = signature(m, nnz, h_rowptr, 0, batch == 0);
  snprintf(buf, (size_t)len, "%s", s.c_str());
  return GPR_OK;
  GPR_ENTRY_END("gpr_tune_signature")
}

int gpr_tune_cache_lookup(const char *cache_path, const char *sig, gpr_tune_result *out) {
  GPR_ENTRY_BEGIN
  if (!cache_path || !sig || !out) return GPR_EINVAL;
  auto c = load_cache(cache_path);
  auto it = c.find(sig);
  if (it == c.end()) return GPR_EINVAL;
  fill_result(out, sig, it->second.first, it->second.second, 0.0, 0, 1);
  return GPR_OK;
  GPR_ENTRY_END("gpr_tune_cache_lookup")
}

int gpr_tune_graph(int m, long long nnz, const int *any_rowptr, const int *any_col,
                   const int *any_outdeg, const char *cache_path, int sweeps,
                   gpr_tune_result *out) {
  GPR_ENTRY_BEGIN
  if (m < 1 || nnz < 0 || !any_rowptr || !any_outdeg || (nnz > 0 && !any_col) || sweeps < 1 ||
      !out)
    return GPR_EINVAL;
  std::vector<int> hrp;
  int rc = host_rowptr(any_rowptr, m + 1, &hrp);
  if (rc != GPR_OK) return rc;
  const std::string sig = signature(m, nnz, hrp.data(), 0, true);
  auto cache = load_cache(cache_path);
  auto hit = cache.find(sig);
  if (hit != cache.end()) {
    fill_result(out, sig, hit->second.first, hit->second.second, 0.0, 0, 1);
    return GPR_OK;
  }
  SingleBench B{m, nnz, any_rowptr, any_col, any_outdeg, sweeps, {}, {}, 0};
  B.init.assign((size_t)m, 1.0f / (float)m);
  std::function<double(const Cfg &)> time = [&](const Cfg &x) { return B.time(x); };
  Cfg x;
  const double t0 = time(x);
  if (!isfinite(t0)) return GPR_ECUDA;
  double best = t0;
  Cfg xb;
  xb.flags = GPR_LAYOUT_BLOCKED;
  const double tb = time(xb);
  if (tb < best * (1.0 - kMargin)) {
    // the blocked form: its knobs (rows per block also decide one or two
    // CTAs per SM), then which heavy rows are summed in chunks
    x = xb;
    best = tb;
    descend(&x, &best, std::vector<int>{6144, 8192},
            [](Cfg *y, int v) { y->block_rows = v; }, time);
    descend(&x, &best, std::vector<int>{2097152, 4194304},
            [](Cfg *y, int v) { y->tile_words = v; }, time);
    descend(&x, &best, std::vector<int>{16384, 1 << 30},
            [](Cfg *y, int v) { y->blocked_long = v; }, time);
  } else {
    descend(&x, &best, std::vector<int>{1, 2, 3, 4, 5, 6, 7},
            [](Cfg *y, int v) { y->variant = v; }, time);
    descend(&x, &best, std::vector<int>{8192, 16384, 56832},
            [](Cfg *y, int v) { y->hot = v; }, time);
    descend(&x, &best, std::vector<int>{16, 32, 128}, [](Cfg *y, int v) { y->sell_max = v; },
            time);
    descend(&x, &best,
            std::vector<std::pair<int, int>>{{1024, 1024}, {16384, 4096}, {4096, 1024}},
            [](Cfg *y, std::pair<int, int> v) {
              y->chunk_min = v.first;
              y->chunk = v.second;
            },
            time);
  }
  save_cache(cache_path, sig, x, best);
  fill_result(out, sig, x, best, t0, B.cands, 0);
  return GPR_OK;
  GPR_ENTRY_END("gpr_tune_graph")
}

int gpr_tune_multigraph(int n_graphs, const int *h_voff, long long nnz, const int *any_rowptr,
                        const int *any_col, const int *any_outdeg, const char *cache_path,
                        int sweeps, gpr_layout_opts *h_lopts_out, gpr_tune_result *out) {
  GPR_ENTRY_BEGIN
  if (n_graphs < 1 || !h_voff || !any_rowptr || !any_outdeg || sweeps < 1 || !h_lopts_out)
    return GPR_EINVAL;
  const int M = h_voff[n_graphs];
  if (M < 1) return GPR_EINVAL;
  std::vector<int> hrp;
  int rc = host_rowptr(any_rowptr, M + 1, &hrp);
  if (rc != GPR_OK) return rc;
  // Group graphs by signature; groups in descending edge share.
  std::vector<std::string> sig(n_graphs);
  std::map<std::string, long long> share;
  for (int g = 0; g < n_graphs; ++g) {
    const int mg = h_voff[g + 1] - h_voff[g];
    const long long e = (long long)hrp[h_voff[g + 1]] - hrp[h_voff[g]];
    sig[g] = signature(mg, e, hrp.data(), h_voff[g], false);
    share[sig[g]] += e;
  }
  std::vector<std::string> groups;
  for (auto &kv : share) groups.push_back(kv.first);
  std::stable_sort(groups.begin(), groups.end(),
                   [&](const std::string &a, const std::string &b) { return share[a] > share[b]; });
  auto cache = load_cache(cache_path);
  std::map<std::string, Cfg> pick;
  std::map<std::string, bool> cached;
  for (auto &k : groups) {
    auto hit = cache.find(k);
    pick[k] = hit != cache.end() ? hit->second.first : Cfg();
    cached[k] = hit != cache.end();
  }
  std::vector<float> init((size_t)M), scores;
  for (int g = 0; g < n_graphs; ++g)
    for (int v = h_voff[g]; v < h_voff[g + 1]; ++v) init[v] = 1.0f / (float)(h_voff[g + 1] - h_voff[g]);
  int cands = 0;
  auto run = [&](const std::map<std::string, Cfg> &p) -> double {
    std::vector<gpr_layout_opts> l((size_t)n_graphs);
    for (int g = 0; g < n_graphs; ++g) l[g] = to_layout(p.at(sig[g]));
    gpr_multigraph *mg = nullptr;
    if (gpr_multigraph_create(n_graphs, h_voff, nnz, any_rowptr, any_col, any_outdeg, l.data(),
                              &mg) != GPR_OK)
      return INFINITY;
    gpr_pr_opts o;
    gpr_pr_opts_default(&o);
    o.tol = 0.0;
    o.max_iter = sweeps;
    double best = INFINITY;
    for (int r = 0; r <= kReps; ++r) {
      scores = init;
      gpr_pr_stats st;
      if (gpr_multigraph_pagerank(mg, scores.data(), &o, nullptr, nullptr, &st) != GPR_OK) {
        best = INFINITY;
        break;
      }
      if (r > 0) best = std::min(best, st.loop_ms / sweeps);
    }
    gpr_multigraph_destroy(mg);
    ++cands;
    return best;
  };
  const double t0 = run(pick);
  if (!isfinite(t0)) return GPR_ECUDA;
  double best = t0;
  // The blocked form covers the whole batch: it is built when any graph asks
  // for it, with the rows per block and words per tile of the first graph
  // that does.  So it is a batch-wide choice, tried first and carried by the
  // group with the largest edge share; when it wins, only its knobs are
  // searched (the sweep does not read the exact-order bins).
  bool blocked = false;
  for (auto &k : groups) blocked = blocked || (pick[k].flags & GPR_LAYOUT_BLOCKED) != 0;
  const std::string &k0 = groups[0];
  if (!blocked && !cached[k0]) {
    std::function<double(const Cfg &)> time = [&](const Cfg &x) {
      auto p = pick;
      p[k0] = x;
      return run(p);
    };
    Cfg xb = pick[k0];
    xb.flags |= GPR_LAYOUT_BLOCKED;
    const double tb = time(xb);
    if (tb < best * (1.0 - kMargin)) {
      best = tb;
      descend(&xb, &best, std::vector<int>{6144, 8192},
              [](Cfg *y, int v) { y->block_rows = v; }, time);
      descend(&xb, &best, std::vector<int>{2097152, 4194304},
              [](Cfg *y, int v) { y->tile_words = v; }, time);
      pick[k0] = xb;
      blocked = true;
    }
  }
  for (auto &k : groups) {
    if (cached[k]) continue;
    if (blocked) {
      save_cache(cache_path, k, pick[k], best);
      continue;
    }
    std::function<double(const Cfg &)> time = [&](const Cfg &x) {
      auto p = pick;
      p[k] = x;
      return run(p);
    };
    Cfg x = pick[k];
    descend(&x, &best, std::vector<int>{16, 32, 128}, [](Cfg *y, int v) { y->sell_max = v; }, time);
    descend(&x, &best, std::vector<std::pair<int, int>>{{1024, 1024}, {16384, 4096}, {4096, 1024}},
            [](Cfg *y, std::pair<int, int> v) {
              y->chunk_min = v.first;
              y->chunk = v.second;
            },
            time);
    pick[k] = x;
    save_cache(cache_path, k, x, best);
  }
  for (int g = 0; g < n_graphs; ++g) h_lopts_out[g] = to_layout(pick[sig[g]]);
  if (out) {
    fill_result(out, groups.empty() ? "" : groups[0], pick[groups[0]], best, t0, cands,
                cands == 1 ? 1 : 0);
  }
  return GPR_OK;
  GPR_ENTRY_END("gpr_tune_multigraph")
}

}  // extern "C"
