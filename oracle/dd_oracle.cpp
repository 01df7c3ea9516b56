// CPU oracle for the Vamana hot path — TEST INFRASTRUCTURE ONLY (see dd_oracle.h).
//
// Each function restates one step of the reference algorithm and cites the
// reference file:line it follows.  Sorting uses the same library routine the
// reference calls (libstdc++ std::sort / std::set_union / std::set_difference),
// so tie orders come out exactly as in the reference build compiled with the
// same toolchain.  Floating-point sums are written in the reference's order
// (no -march, so the scalar NSGDist path) and this file is compiled with the
// reference's own flags (-O2, no -ffast-math, no FMA on baseline x86-64).
#include "dd_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <thread>
#include <utility>
#include <vector>

namespace {

using id_t_ = uint32_t;
using pid = std::pair<id_t_, float>;

// ---------------------------------------------------------------- distances
// include/utils/NSGDist.h:113-131 (scalar path: groups of 4, then the tail)
float l2_f32(const float* a, const float* b, uint32_t size) {
  float result = 0;
  uint32_t i = 0;
  for (; i + 3 < size; i += 4) {
    float d0 = a[i] - b[i], d1 = a[i + 1] - b[i + 1];
    float d2 = a[i + 2] - b[i + 2], d3 = a[i + 3] - b[i + 3];
    result += d0 * d0 + d1 * d1 + d2 * d2 + d3 * d3;
  }
  for (; i < size; i++) {
    float d0 = a[i] - b[i];
    result += d0 * d0;
  }
  return result;
}
// include/utils/euclidian_point.h:44-60
template <typename T>
float l2_int(const T* p, const T* q, uint32_t d) {
  int result = 0;
  for (uint32_t i = 0; i < d; i++) {
    int32_t t = (int32_t)((int16_t)q[i] - (int16_t)p[i]);
    result += t * t;
  }
  return (float)result;
}
// include/utils/mips_point.h:44-66
float mips_f32(const float* p, const float* q, uint32_t d) {
  float result = 0;
  for (uint32_t i = 0; i < d; i++) result += q[i] * p[i];
  return -result;
}
template <typename T>
float mips_int(const T* p, const T* q, uint32_t d) {
  int result = 0;
  for (uint32_t i = 0; i < d; i++) result += ((int32_t)q[i]) * ((int32_t)p[i]);
  return -((float)result);
}

float dist_any(int dtype, int metric, const void* a, const void* b, uint32_t d) {
  if (metric == 0) {
    if (dtype == 0) return l2_f32((const float*)a, (const float*)b, d);
    if (dtype == 1) return l2_int((const int8_t*)a, (const int8_t*)b, d);
    return l2_int((const uint8_t*)a, (const uint8_t*)b, d);
  }
  if (dtype == 0) return mips_f32((const float*)a, (const float*)b, d);
  if (dtype == 1) return mips_int((const int8_t*)a, (const int8_t*)b, d);
  return mips_int((const uint8_t*)a, (const uint8_t*)b, d);
}

struct Space {
  int dtype, metric;
  const char* base;
  uint64_t n;
  uint32_t d;
  uint64_t stride;
  const void* row(uint64_t i) const { return base + i * stride; }
  float dist(const void* a, const void* b) const { return dist_any(dtype, metric, a, b, d); }
  float dist_ids(uint64_t i, uint64_t j) const { return dist(row(i), row(j)); }
  bool is_metric() const { return metric == 0; }  // mips_point.h:73-74
};

// Graph rows: [deg, nbr_0 .. nbr_{R-1}] (include/utils/graph.h:126-128, 202)
struct GraphView {
  uint32_t* g;
  uint32_t R;
  uint32_t* row(uint64_t i) const { return g + i * (uint64_t)(R + 1); }
  uint32_t size(uint64_t i) const { return row(i)[0]; }
};

// ---------------------------------------------------------------- parallel_for
template <typename F>
void parallel_for(size_t lo, size_t hi, int nthreads, F&& f) {
  if (hi <= lo) return;
  size_t cnt = hi - lo;
  int nt = nthreads > 0 ? nthreads : (int)std::thread::hardware_concurrency();
  if (nt < 1) nt = 1;
  if ((size_t)nt > cnt) nt = (int)cnt;
  if (nt == 1) {
    for (size_t i = lo; i < hi; i++) f(i);
    return;
  }
  std::atomic<size_t> next(lo);
  std::vector<std::thread> ts;
  for (int t = 0; t < nt; t++)
    ts.emplace_back([&]() {
      while (true) {
        size_t s = next.fetch_add(16);
        if (s >= hi) break;
        size_t e = std::min(hi, s + 16);
        for (size_t i = s; i < e; i++) f(i);
      }
    });
  for (auto& t : ts) t.join();
}

// splitmix64 finaliser (include/parlay/utilities.h:145-150)
inline uint64_t hash64_2(uint64_t x) {
  x = (x ^ (x >> 30)) * UINT64_C(0xbf58476d1ce4e5b9);
  x = (x ^ (x >> 27)) * UINT64_C(0x94d049bb133111eb);
  x = x ^ (x >> 31);
  return x;
}

struct BeamResult {
  std::vector<pid> frontier, visited;
  uint64_t dist_cmps = 0;
};

// ---------------------------------------------------------------- beam_search
// include/utils/beamSearch.h:51-184, single start point (:41-48).
BeamResult beam_search(const Space& S, const GraphView& G, const void* p, int64_t self_id,
                       uint32_t start, int64_t k, int64_t L, double cut, int64_t limit,
                       int64_t degree_limit) {
  auto less = [](const pid& a, const pid& b) {
    return a.second < b.second || (a.second == b.second && a.first < b.first);
  };
  // lossy "seen" filter: bits = max(10, ceil(log2(L*L)) - 2)   (:66-73)
  int bits = std::max<int>(10, (int)(std::ceil(std::log2((double)(L * L))) - 2));
  std::vector<id_t_> hash_filter((size_t)1 << bits, (id_t_)-1);
  const uint64_t mask = ((uint64_t)1 << bits) - 1;
  auto has_been_seen = [&](id_t_ a) -> bool {
    size_t loc = (size_t)(hash64_2(a) & mask);
    if (hash_filter[loc] == a) return true;
    hash_filter[loc] = a;
    return false;
  };

  BeamResult res;
  std::vector<pid>& frontier = res.frontier;
  frontier.push_back(pid(start, S.dist(S.row(start), p)));  // :80-82
  std::vector<pid> unvisited(std::max<int64_t>(L, 1));
  unvisited[0] = frontier[0];
  std::vector<pid>& visited = res.visited;
  uint64_t dist_cmps = 1;
  long remain = 1;
  int64_t num_visited = 0;
  std::vector<pid> new_frontier((size_t)(L + G.R));
  std::vector<pid> candidates;
  std::vector<id_t_> keep;
  const float int_max_f = (float)std::numeric_limits<int>::max();

  while (remain > 0 && num_visited < limit) {  // :108
    pid current = unvisited[0];
    visited.insert(std::upper_bound(visited.begin(), visited.end(), current, less), current);
    num_visited++;
    candidates.clear();
    keep.clear();
    int64_t num_elts = std::min<int64_t>(G.size(current.first), degree_limit);
    const uint32_t* nb = G.row(current.first) + 1;
    for (int64_t i = 0; i < num_elts; i++) {  // :126-131
      id_t_ a = nb[i];
      if ((int64_t)a == self_id || has_been_seen(a)) continue;
      keep.push_back(a);
    }
    float cutoff = ((int64_t)frontier.size() < L) ? int_max_f : frontier.back().second;  // :135-137
    for (id_t_ a : keep) {  // :138-145
      float dist = S.dist(S.row(a), p);
      dist_cmps++;
      if (dist >= cutoff) continue;
      candidates.push_back(pid(a, dist));
    }
    std::sort(candidates.begin(), candidates.end(), less);  // :148
    size_t nf = std::set_union(frontier.begin(), frontier.end(), candidates.begin(),
                               candidates.end(), new_frontier.begin(), less) -
                new_frontier.begin();  // :151-154
    nf = std::min<size_t>((size_t)L, nf);  // :157
    if (k > 0 && (int64_t)nf > k && S.is_metric()) {  // :162-167
      pid thr(0, (float)(cut * (double)new_frontier[(size_t)k].second));
      nf = std::upper_bound(new_frontier.begin(), new_frontier.begin() + nf, thr, less) -
           new_frontier.begin();
    }
    frontier.assign(new_frontier.begin(), new_frontier.begin() + nf);
    remain = std::set_difference(frontier.begin(), frontier.end(), visited.begin(),
                                 visited.end(), unvisited.begin(), less) -
             unvisited.begin();  // :175-178
  }
  res.dist_cmps = dist_cmps;
  return res;
}

// ---------------------------------------------------------------- robustPrune
// include/index.h:63-123 (identical copy at src/bsp_index.hpp:483-532)
std::vector<id_t_> robust_prune(const Space& S, const GraphView& G, id_t_ p,
                                const std::vector<pid>& cand, double alpha, uint32_t R) {
  std::vector<pid> candidates(cand.begin(), cand.end());
  uint32_t out_size = G.size(p);
  const uint32_t* nb = G.row(p) + 1;
  for (uint32_t i = 0; i < out_size; i++)
    candidates.push_back(pid(nb[i], S.dist_ids(nb[i], p)));  // :71-74
  std::sort(candidates.begin(), candidates.end(),
            [](pid a, pid b) { return a.second < b.second; });  // :78-79
  std::vector<id_t_> new_nbhs;
  size_t idx = 0;
  while (new_nbhs.size() < R && idx < candidates.size()) {  // :86-106
    int p_star = (int)candidates[idx].first;
    idx++;
    if (p_star == (int)p || p_star == -1) continue;
    new_nbhs.push_back((id_t_)p_star);
    for (size_t i = idx; i < candidates.size(); i++) {
      int p_prime = (int)candidates[i].first;
      if (p_prime != -1) {
        float d_sp = S.dist_ids((id_t_)p_star, (id_t_)p_prime);
        float d_pp = candidates[i].second;
        if (alpha * d_sp <= d_pp) candidates[i].first = (id_t_)-1;
      }
    }
  }
  return new_nbhs;
}

// ---------------------------------------------------------------- schedule
// src/bsp_index.hpp:162-166 (m, max_batch_size) and :238-246 (round bounds);
// knn_index uses n and max_fraction 1.0 (include/index.h:131-132, 233-261).
uint64_t max_batch_of(uint64_t m, double frac) {
  size_t mb = std::min((size_t)(frac * (float)m), (size_t)1000000ul);
  if (mb == 0) mb = m;
  return mb;
}

std::vector<std::pair<uint64_t, uint64_t>> schedule(uint64_t m, uint64_t max_batch) {
  std::vector<std::pair<uint64_t, uint64_t>> rounds;
  size_t inc = 0, count = 0;
  const double base = 2;
  while (count < m) {
    size_t floor_, ceiling;
    if (std::pow(base, (double)inc) <= (double)max_batch) {
      floor_ = (size_t)std::pow(base, (double)inc) - 1;
      ceiling = std::min((size_t)std::pow(base, (double)(inc + 1)), (size_t)m) - 1;
      count = ceiling;
    } else {
      floor_ = count;
      ceiling = std::min(count + (size_t)max_batch, (size_t)m);
      count += (size_t)max_batch;
    }
    rounds.push_back({floor_, ceiling});
    inc++;
  }
  return rounds;
}

// ---------------------------------------------------------------- one round
// New out-lists of the batch points [lo, hi) against the current graph
// (src/bsp_index.hpp:259-277; include/index.h:274-285).
std::vector<std::vector<id_t_>> search_prune_range(const Space& S, const GraphView& G, uint32_t L,
                                                   double alpha, uint32_t start, uint64_t lo,
                                                   uint64_t hi, int nthreads, uint64_t* st) {
  const uint32_t R = G.R;
  const size_t B = hi - lo;
  std::vector<std::vector<id_t_>> new_out(B);
  std::vector<uint64_t> vis_cnt(B), cmp_cnt(B);
  parallel_for(0, B, nthreads, [&](size_t b) {
    id_t_ idx = (id_t_)(lo + b);
    BeamResult r = beam_search(S, G, S.row(idx), idx, start, 0, L, 0.0, (int64_t)S.n,
                               (int64_t)R);
    vis_cnt[b] = r.visited.size();
    cmp_cnt[b] = r.dist_cmps;
    new_out[b] = robust_prune(S, G, idx, r.visited, alpha, R);
  });
  if (st)
    for (size_t b = 0; b < B; b++) st[1] += vis_cnt[b], st[2] += cmp_cnt[b];
  return new_out;
}

// update_neighbors of the batch [floor_, floor_ + B) (:354-357), then the
// reverse edges of the targets t with t % world == rank (:362-407): flatten
// (target, source) in batch order, group by target keeping the input order
// within a target (parlay group_by_key), append or prune.  Returns the
// changed targets in ascending order.
std::vector<id_t_> apply_reverse_owned(const Space& S, GraphView& G, double alpha, uint64_t floor_,
                                       const std::vector<std::vector<id_t_>>& new_out,
                                       uint32_t rank, uint32_t world, int nthreads, uint64_t* st) {
  const uint32_t R = G.R;
  const size_t B = new_out.size();
  for (size_t b = 0; b < B; b++) {
    uint32_t* row = G.row(floor_ + b);
    row[0] = (uint32_t)new_out[b].size();
    for (size_t j = 0; j < new_out[b].size(); j++) row[1 + j] = new_out[b][j];
  }
  std::vector<std::pair<id_t_, id_t_>> pairs;
  for (size_t b = 0; b < B; b++)
    for (id_t_ t : new_out[b])
      if (t % world == rank) pairs.push_back({t, (id_t_)(floor_ + b)});
  std::stable_sort(pairs.begin(), pairs.end(),
                   [](const std::pair<id_t_, id_t_>& a, const std::pair<id_t_, id_t_>& b) {
                     return a.first < b.first;
                   });
  std::vector<size_t> seg;
  for (size_t i = 0; i < pairs.size(); i++)
    if (i == 0 || pairs[i].first != pairs[i - 1].first) seg.push_back(i);
  seg.push_back(pairs.size());
  size_t ngroups = seg.size() - 1;
  std::vector<uint8_t> pruned(ngroups, 0);
  std::vector<uint64_t> pc(ngroups, 0);
  parallel_for(0, ngroups, nthreads, [&](size_t gi) {
    id_t_ t = pairs[seg[gi]].first;
    size_t m = seg[gi + 1] - seg[gi];
    uint32_t* row = G.row(t);
    if (m + row[0] <= R) {
      for (size_t j = 0; j < m; j++) row[1 + row[0] + j] = pairs[seg[gi] + j].second;
      row[0] += (uint32_t)m;
    } else {
      std::vector<pid> cc;
      for (size_t j = 0; j < m; j++) {
        id_t_ c = pairs[seg[gi] + j].second;
        cc.push_back(pid(c, S.dist_ids(c, t)));  // wrapper :536-545
      }
      pc[gi] = m + row[0];
      std::vector<id_t_> nn = robust_prune(S, G, t, cc, alpha, R);
      row[0] = (uint32_t)nn.size();
      for (size_t j = 0; j < nn.size(); j++) row[1 + j] = nn[j];
      pruned[gi] = 1;
    }
  });
  if (st) {
    st[3] += ngroups;
    for (size_t gi = 0; gi < ngroups; gi++) st[4] += pruned[gi], st[5] += pc[gi];
  }
  std::vector<id_t_> changed(ngroups);
  for (size_t gi = 0; gi < ngroups; gi++) changed[gi] = pairs[seg[gi]].first;
  return changed;
}

// ---------------------------------------------------------------- one pass
// include/index.h:250-325 / src/bsp_index.hpp:238-407 with identity order.
void batch_insert(const Space& S, GraphView& G, uint32_t L, double alpha, uint32_t start,
                  const std::vector<std::pair<uint64_t, uint64_t>>& rounds, int nthreads,
                  uint64_t* st) {
  for (auto& rd : rounds) {
    uint64_t floor_ = rd.first, ceiling = rd.second;
    if (st) st[0]++;
    if (ceiling <= floor_) continue;
    auto new_out = search_prune_range(S, G, L, alpha, start, floor_, ceiling, nthreads, st);
    apply_reverse_owned(S, G, alpha, floor_, new_out, 0, 1, nthreads, st);
  }
}

Space make_space(int dtype, int metric, const void* points, uint64_t n, uint32_t d,
                 uint64_t stride) {
  Space S;
  S.dtype = dtype;
  S.metric = metric;
  S.base = (const char*)points;
  S.n = n;
  S.d = d;
  S.stride = stride;
  return S;
}

}  // namespace

extern "C" {

float ddo_distance(int dtype, int metric, const void* a, const void* b, uint32_t d) {
  return dist_any(dtype, metric, a, b, d);
}

uint64_t ddo_schedule(uint64_t n, uint64_t max_build, double xita, int knn_mode,
                      uint64_t* floors, uint64_t* ceilings, uint64_t cap) {
  uint64_t m = n;
  double frac = xita;
  if (knn_mode) {
    frac = 1.0;
  } else if (max_build != 0) {
    m = std::min<uint64_t>(max_build, m);
  }
  auto rounds = schedule(m, max_batch_of(m, frac));
  for (size_t i = 0; i < rounds.size() && i < cap; i++) {
    floors[i] = rounds[i].first;
    ceilings[i] = rounds[i].second;
  }
  return rounds.size();
}

int ddo_build(int dtype, int metric, const void* points, uint64_t n, uint32_t d,
              uint64_t stride, uint32_t R, uint32_t L, double alpha, double xita,
              uint64_t max_build, uint32_t start, int two_pass, int knn_mode, int nthreads,
              uint32_t* graph_out, uint64_t* stats_out) {
  if (!points || !graph_out || n == 0 || R == 0 || L == 0 || start >= n) return -1;
  Space S = make_space(dtype, metric, points, n, d, stride);
  std::memset(graph_out, 0, sizeof(uint32_t) * n * (uint64_t)(R + 1));
  GraphView G{graph_out, R};
  if (stats_out) std::memset(stats_out, 0, sizeof(uint64_t) * 6);
  uint64_t m = n;
  double frac = xita;
  if (knn_mode) {
    frac = 1.0;  // include/index.h:131-132 pass max_fraction 1.00
    start = 0;   // include/index.h:127
  } else if (max_build != 0) {
    m = std::min<uint64_t>(max_build, m);  // src/bsp_index.hpp:162
  }
  auto rounds = schedule(m, max_batch_of(m, frac));
  if (two_pass) batch_insert(S, G, L, 1.0, start, rounds, nthreads, stats_out);
  batch_insert(S, G, L, alpha, start, rounds, nthreads, stats_out);
  if (knn_mode) {
    // include/index.h:133-136: sort each row by distance to its owner
    parallel_for(0, n, nthreads, [&](size_t i) {
      uint32_t* row = G.row(i);
      std::sort(row + 1, row + 1 + row[0], [&](id_t_ j, id_t_ k) {
        return S.dist_ids(i, j) < S.dist_ids(i, k);
      });
    });
  }
  return 0;
}

int ddo_shard_search_prune(int dtype, int metric, const void* points, uint64_t n, uint32_t d,
                           uint64_t stride, const uint32_t* graph, uint32_t R, uint32_t L,
                           double alpha, uint32_t start, uint64_t lo, uint64_t hi, int nthreads,
                           uint32_t* rows_out) {
  if (!points || !graph || !rows_out || hi < lo || hi > n || start >= n) return -1;
  Space S = make_space(dtype, metric, points, n, d, stride);
  GraphView G{const_cast<uint32_t*>(graph), R};
  auto nb = search_prune_range(S, G, L, alpha, start, lo, hi, nthreads, nullptr);
  for (size_t b = 0; b < nb.size(); b++) {
    uint32_t* o = rows_out + b * (uint64_t)(R + 1);
    std::memset(o, 0, 4ull * (R + 1));
    o[0] = (uint32_t)nb[b].size();
    for (size_t j = 0; j < nb[b].size(); j++) o[1 + j] = nb[b][j];
  }
  return 0;
}

int ddo_shard_apply_reverse(int dtype, int metric, const void* points, uint64_t n, uint32_t d,
                            uint64_t stride, uint32_t* graph, uint32_t R, double alpha,
                            uint64_t floor_, uint64_t ceiling, const uint32_t* batch_rows,
                            uint32_t rank, uint32_t world, int nthreads, uint32_t* ids_out,
                            uint32_t* rows_out, uint64_t cap, uint64_t* count) {
  if (!points || !graph || !batch_rows || ceiling < floor_ || ceiling > n || world == 0 ||
      rank >= world)
    return -1;
  Space S = make_space(dtype, metric, points, n, d, stride);
  GraphView G{graph, R};
  std::vector<std::vector<id_t_>> nb(ceiling - floor_);
  for (size_t b = 0; b < nb.size(); b++) {
    const uint32_t* r = batch_rows + b * (uint64_t)(R + 1);
    nb[b].assign(r + 1, r + 1 + r[0]);
  }
  auto changed = apply_reverse_owned(S, G, alpha, floor_, nb, rank, world, nthreads, nullptr);
  *count = changed.size();
  if (changed.size() > cap) return -2;
  for (size_t k = 0; k < changed.size(); k++) {
    ids_out[k] = changed[k];
    std::memcpy(rows_out + k * (uint64_t)(R + 1), G.row(changed[k]), 4ull * (R + 1));
  }
  return 0;
}

int ddo_shard_set_rows(uint32_t* graph, uint64_t n, uint32_t R, const uint32_t* ids,
                       const uint32_t* rows, uint64_t count) {
  for (uint64_t k = 0; k < count; k++) {
    if (ids[k] >= n) return -1;
    std::memcpy(graph + ids[k] * (uint64_t)(R + 1), rows + k * (uint64_t)(R + 1), 4ull * (R + 1));
  }
  return 0;
}

int ddo_beam_search(int dtype, int metric, const void* points, uint64_t n, uint32_t d,
                    uint64_t stride, const uint32_t* graph, uint32_t R, const void* query,
                    int64_t self_id, uint32_t start, int64_t k, int64_t L, double cut,
                    int64_t limit, int64_t degree_limit, uint32_t* fr_ids, float* fr_d,
                    uint32_t* n_fr, uint32_t* vis_ids, float* vis_d, uint32_t* n_vis,
                    uint32_t vis_cap, uint64_t* dist_cmps) {
  Space S = make_space(dtype, metric, points, n, d, stride);
  GraphView G{const_cast<uint32_t*>(graph), R};
  BeamResult r = beam_search(S, G, query, self_id, start, k, L, cut,
                             limit > 0 ? limit : (int64_t)n,
                             degree_limit > 0 ? degree_limit : (int64_t)R);
  *n_fr = (uint32_t)r.frontier.size();
  *n_vis = (uint32_t)r.visited.size();
  if (dist_cmps) *dist_cmps = r.dist_cmps;
  for (size_t i = 0; i < r.frontier.size(); i++) {
    fr_ids[i] = r.frontier[i].first;
    fr_d[i] = r.frontier[i].second;
  }
  if (r.visited.size() > vis_cap) return -1;
  for (size_t i = 0; i < r.visited.size(); i++) {
    vis_ids[i] = r.visited[i].first;
    vis_d[i] = r.visited[i].second;
  }
  return 0;
}

int ddo_search(int dtype, int metric, const void* points, uint64_t n, uint32_t d,
               uint64_t stride, const uint32_t* graph, uint32_t R, const void* queries,
               uint64_t nq, uint64_t qstride, const uint32_t* L_per_query, int64_t k,
               double cut, int64_t limit, int64_t degree_limit, uint32_t start, int nthreads,
               uint32_t* ids_out, uint32_t* visited_out, uint32_t* cmps_out) {
  Space S = make_space(dtype, metric, points, n, d, stride);
  GraphView G{const_cast<uint32_t*>(graph), R};
  parallel_for(0, nq, nthreads, [&](size_t i) {
    const void* q = (const char*)queries + i * qstride;
    BeamResult r = beam_search(S, G, q, (int64_t)i, start, k, L_per_query[i], cut,
                               limit > 0 ? limit : (int64_t)n,
                               degree_limit > 0 ? degree_limit : (int64_t)R);
    for (int64_t j = 0; j < k; j++)
      ids_out[i * k + j] = (size_t)j < r.frontier.size() ? r.frontier[j].first : (uint32_t)-1;
    if (visited_out) visited_out[i] = (uint32_t)r.visited.size();
    if (cmps_out) cmps_out[i] = (uint32_t)r.dist_cmps;
  });
  return 0;
}

int ddo_robust_prune(int dtype, int metric, const void* points, uint64_t n, uint32_t d,
                     uint64_t stride, const uint32_t* graph, uint32_t R, uint32_t p,
                     const uint32_t* cand_ids, const float* cand_d, uint32_t m, double alpha,
                     uint32_t* out, uint32_t* out_len) {
  Space S = make_space(dtype, metric, points, n, d, stride);
  GraphView G{const_cast<uint32_t*>(graph), R};
  std::vector<pid> cand;
  for (uint32_t i = 0; i < m; i++) cand.push_back(pid(cand_ids[i], cand_d[i]));
  auto r = robust_prune(S, G, p, cand, alpha, R);
  *out_len = (uint32_t)r.size();
  for (size_t i = 0; i < r.size(); i++) out[i] = r[i];
  return 0;
}

int ddo_groundtruth(int dtype, int metric, const void* points, uint64_t n, uint32_t d,
                    uint64_t stride, const void* queries, uint64_t nq, uint64_t qstride,
                    uint32_t k, int nthreads, uint32_t* ids_out, float* dists_out) {
  if (k > n) return -1;
  parallel_for(0, nq, nthreads, [&](size_t qi) {
    const char* q = (const char*)queries + qi * qstride;
    std::vector<std::pair<double, uint32_t>> best;  // max-heap by (dist, id)
    best.reserve(k + 1);
    for (uint64_t j = 0; j < n; j++) {
      const char* x = (const char*)points + j * stride;
      double acc = 0;
      if (dtype == 0) {
        const float* a = (const float*)q;
        const float* b = (const float*)x;
        for (uint32_t t = 0; t < d; t++) {
          if (metric == 0) {
            double df = (double)a[t] - (double)b[t];
            acc += df * df;
          } else {
            acc -= (double)a[t] * (double)b[t];
          }
        }
      } else {
        int64_t s = 0;
        for (uint32_t t = 0; t < d; t++) {
          int64_t av = dtype == 1 ? (int64_t)((const int8_t*)q)[t] : (int64_t)((const uint8_t*)q)[t];
          int64_t bv = dtype == 1 ? (int64_t)((const int8_t*)x)[t] : (int64_t)((const uint8_t*)x)[t];
          s += metric == 0 ? (av - bv) * (av - bv) : -(av * bv);
        }
        acc = (double)s;
      }
      std::pair<double, uint32_t> e(acc, (uint32_t)j);
      if (best.size() < k) {
        best.push_back(e);
        std::push_heap(best.begin(), best.end());
      } else if (e < best.front()) {
        std::pop_heap(best.begin(), best.end());
        best.back() = e;
        std::push_heap(best.begin(), best.end());
      }
    }
    std::sort(best.begin(), best.end());
    for (uint32_t t = 0; t < k; t++) {
      ids_out[qi * k + t] = best[t].second;
      dists_out[qi * k + t] = (float)best[t].first;
    }
  });
  return 0;
}

}  // extern "C"
