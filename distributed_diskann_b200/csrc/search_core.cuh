// Warp-cooperative greedy beam search: one warp runs the search of one point.
//
// Semantics follow include/utils/beamSearch.h:51-184 exactly:
//  * frontier = at most L (dist, id) pairs sorted by (dist, id)  (:59-61, :78-82)
//  * each step visits the closest unvisited frontier entry         (:111-117)
//  * its first min(deg, degree_limit) neighbours are filtered by the lossy
//    hash "seen" table (2^bits u32 slots, splitmix64, overwrite on miss) and
//    by p.id()                                                      (:64-73, :125-131)
//  * kept neighbours get exact distances; those below the cutoff (last
//    frontier distance when full, (float)INT_MAX otherwise) are merged into
//    the frontier, which is trimmed to L                            (:135-157)
//  * query mode: the k-cut keeps entries up to cut * dist(k)         (:162-167)
//  * the search ends when no unvisited entry is left or `limit` nodes were
//    visited                                                         (:108, :175-178)
//
// Parallel forms of the sequential steps:
//  * "visited" is a flag bit in the frontier id (ids are unique in the
//    frontier, so set_difference(frontier, visited) is "flag clear").  A node
//    dropped from the frontier after its visit is remembered in an "evicted"
//    list; if it ever re-enters (possible only in query mode, after a k-cut)
//    it re-enters flagged, as set_difference would treat it.
//  * the hash filter is replayed exactly: lanes whose ids fall in the same
//    slot are grouped with __match_any_sync; within a group the table value a
//    lane sees is the id of the previous lane in neighbour order (or the table
//    entry), and the last lane of the group writes the slot.
//  * set_union + trim: candidates are ranked by (dist, id), duplicates of
//    frontier entries dropped (set_union keeps the frontier's copy), and every
//    element moves to its merged position; positions >= L are dropped.
#pragma once
#include "dd_common.cuh"
#include "kernels.cuh"

namespace ddk {

constexpr uint32_t kMaxFrPerLane = kMaxL / 32;
constexpr uint32_t kMaxCandPerLane = kMaxRp / 32;

struct SearchSmem {
  uint8_t* qv;        // query vector (16-byte aligned, zero padded)
  uint32_t* fr_id;    // L entries (id | DD_VBIT when visited)
  float* fr_d;
  uint32_t* c_id;     // Rp per-step candidates
  float* c_d;
  uint32_t* s_id;     // Rp sorted candidates
  float* s_d;
  uint32_t* vis_id;   // visited list in visit order (keep_visited), capacity vcap
  float* vis_d;
  uint32_t* ev_id;    // visited ids pushed out of the frontier (query_mode), capacity vcap
  uint32_t* hash;     // 2^bits slots
};

struct SearchParams {
  const uint8_t* points;
  uint64_t stride;      // bytes between point rows
  const uint32_t* graph;
  uint32_t Rp;          // graph row length (uint32)
  uint64_t n;
  uint32_t d;
  uint32_t start;
  uint32_t L;
  uint32_t k;           // 0 in build mode
  double cut;
  uint64_t limit;
  uint32_t degree_limit;
  uint32_t hbits;
  uint32_t vcap;
  int query_mode;       // track evicted visited entries for re-entry
  int keep_visited;     // record the visited list (build / debug)
  uint32_t* err;
};

struct SearchOut {
  uint32_t fr_n;        // final frontier size
  uint32_t vis_n;       // number of visited nodes (= visited list length when kept)
  uint32_t cmps;        // distance computations (reference dist_cmps)
};

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}
__device__ __forceinline__ uint32_t lanemask_gt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_gt;" : "=r"(m));
  return m;
}

// ceil(log2(L*L)) - 2, at least 10 (beamSearch.h:66), computed exactly in integers
__host__ __device__ inline uint32_t hash_bits_for(uint32_t L) {
  uint64_t sq = (uint64_t)L * L;
  uint32_t c = 0;
  while (((uint64_t)1 << c) < sq) c++;  // ceil(log2(sq)) for sq >= 1
  int b = (int)c - 2;
  return (uint32_t)(b < 10 ? 10 : b);
}

template <int DT, int MT>
__device__ __forceinline__ float point_dist(const SearchParams& P, const uint8_t* qv, uint32_t id) {
  return Dist<DT, MT>::eval(qv, P.points + (uint64_t)id * P.stride, P.d);
}

// Runs one beam search on the warp.  `qv` must already hold the query.
// self_id: the id the reference skips as p.id() (the point itself in the
// build, the query's index in searchAll).
template <int DT, int MT>
__device__ SearchOut warp_beam_search(const SearchParams& P, const SearchSmem& S, uint64_t self_id) {
  const uint32_t lane = lane_id();
  const uint32_t FULL = 0xffffffffu;
  const uint32_t nslots = 1u << P.hbits;
  const uint32_t hmask = nslots - 1;
  for (uint32_t i = lane; i < nslots; i += 32) S.hash[i] = DD_NONE;
  if (lane == 0) {
    S.fr_id[0] = P.start;
    S.fr_d[0] = point_dist<DT, MT>(P, S.qv, P.start);
  }
  __syncwarp();
  uint32_t fr_n = 1;
  uint32_t vis_n = 0;      // visited list length
  uint32_t ev_n = 0;       // evicted list length (query mode)
  uint32_t cmps = 1;       // dist to the start point
  uint64_t num_visited = 0;
  const float int_max_f = 2147483648.0f;  // (float)std::numeric_limits<int>::max()
  const uint32_t dl = P.degree_limit;

  while (num_visited < P.limit) {
    // ---- closest unvisited frontier entry
    int cur_pos = -1;
    for (uint32_t base = 0; base < fr_n; base += 32) {
      uint32_t i = base + lane;
      bool unv = (i < fr_n) && !(S.fr_id[i] & DD_VBIT);
      uint32_t b = __ballot_sync(FULL, unv);
      if (b) { cur_pos = (int)(base + __ffs(b) - 1); break; }
    }
    if (cur_pos < 0) break;
    const uint32_t cur = S.fr_id[cur_pos];
    const float cur_d = S.fr_d[cur_pos];
    __syncwarp();
    if (lane == 0) {
      S.fr_id[cur_pos] = cur | DD_VBIT;
      if (P.keep_visited) {
        if (vis_n < P.vcap) {
          S.vis_id[vis_n] = cur;
          S.vis_d[vis_n] = cur_d;
        } else {
          dd_set_error(P.err, DD_EVIS_CAP);
        }
      }
    }
    if (P.keep_visited && vis_n < P.vcap) vis_n++;
    num_visited++;
    const float cutoff = (fr_n < P.L) ? int_max_f : S.fr_d[fr_n - 1];
    __syncwarp();

    // ---- expand: hash filter (exact replay), distances, compaction
    const uint32_t* row = P.graph + (uint64_t)cur * P.Rp;
    uint32_t nc = 0;
    for (uint32_t base = 0; base < P.Rp && base < dl; base += 32) {
      uint32_t j = base + lane;
      uint32_t a = (j < P.Rp && j < dl) ? __ldg(row + j) : DD_NONE;
      if (a != DD_NONE && a >= P.n) {
        dd_set_error(P.err, DD_EBAD_ID);
        a = DD_NONE;
      }
      bool part = (a != DD_NONE) && ((uint64_t)a != self_id);
      uint32_t loc = part ? (uint32_t)(dd_hash64(a) & hmask) : (0x80000000u | lane);
      uint32_t grp = __match_any_sync(FULL, loc);
      uint32_t before = grp & lanemask_lt();
      uint32_t tval = part ? S.hash[loc] : DD_NONE;
      uint32_t prev_a = __shfl_sync(FULL, a, before ? 31 - __clz(before) : lane);
      uint32_t seen_val = before ? prev_a : tval;
      bool keep = part && (seen_val != a);
      __syncwarp();
      if (part && (grp & lanemask_gt()) == 0) S.hash[loc] = a;
      __syncwarp();
      float dist = 0.f;
      if (keep) dist = point_dist<DT, MT>(P, S.qv, a);
      cmps += __popc(__ballot_sync(FULL, keep));
      bool pass = keep && (dist < cutoff);
      uint32_t pb = __ballot_sync(FULL, pass);
      if (pass) {
        uint32_t pos = nc + __popc(pb & lanemask_lt());
        S.c_id[pos] = a;
        S.c_d[pos] = dist;
      }
      nc += __popc(pb);
    }
    __syncwarp();
    if (nc == 0) continue;

    // ---- rank candidates by (dist, id).  The same id can be kept twice in one
    // step (a row holding it twice, with a colliding id between the copies,
    // defeats the lossy filter); identical copies keep their index order.
    for (uint32_t i = lane; i < nc; i += 32) {
      float di = S.c_d[i];
      uint32_t ii = S.c_id[i];
      uint32_t r = 0;
      for (uint32_t j = 0; j < nc; j++) {
        float dj = S.c_d[j];
        uint32_t ij = S.c_id[j];
        r += (pair_less(dj, ij, di, ii) || (dj == di && ij == ii && j < i)) ? 1u : 0u;
      }
      S.s_id[r] = ii;
      S.s_d[r] = di;
    }
    __syncwarp();
    // set_union as multisets: with m frontier copies of a value and n candidate
    // copies, the candidate copies k >= m are added, after the frontier's copies.
    // A re-entering copy counts as visited while k < (visits of the value):
    // set_difference(frontier, visited) is a multiset difference too.
    bool a_ok[kMaxCandPerLane];
    uint32_t a_id[kMaxCandPerLane], a_ub[kMaxCandPerLane];
    float a_d[kMaxCandPerLane];
#pragma unroll
    for (uint32_t t = 0; t < kMaxCandPerLane; t++) {
      uint32_t i = lane + 32 * t;
      a_ok[t] = false;
      a_id[t] = 0;
      a_ub[t] = 0;
      a_d[t] = 0.f;
      if (i < nc) {
        uint32_t ci = S.s_id[i];
        float cd = S.s_d[i];
        uint32_t k = 0;  // index of this copy among identical candidates
        for (uint32_t u = i; u > 0 && S.s_id[u - 1] == ci && S.s_d[u - 1] == cd; u--) k++;
        uint32_t lo = 0, hi = fr_n;
        while (lo < hi) {
          uint32_t mid = (lo + hi) >> 1;
          if (pair_less(S.fr_d[mid], S.fr_id[mid] & ~DD_VBIT, cd, ci)) lo = mid + 1;
          else hi = mid;
        }
        uint32_t ub = lo, mf = 0;
        while (ub < fr_n && S.fr_d[ub] == cd && (S.fr_id[ub] & ~DD_VBIT) == ci) {
          mf += (S.fr_id[ub] & DD_VBIT) ? 1u : 0u;
          ub++;
        }
        const uint32_t m = ub - lo;
        if (k >= m) {
          a_ok[t] = true;
          if (P.query_mode) {
            uint32_t ev = 0;
            for (uint32_t e = 0; e < ev_n; e++) ev += (S.ev_id[e] == ci) ? 1u : 0u;
            if (k < mf + ev) ci |= DD_VBIT;
          }
          a_id[t] = ci;
          a_d[t] = cd;
          a_ub[t] = ub;
        }
      }
    }
    __syncwarp();
    uint32_t nkeep = 0;
#pragma unroll
    for (uint32_t t = 0; t < kMaxCandPerLane; t++) {
      uint32_t ob = __ballot_sync(FULL, a_ok[t]);
      if (a_ok[t]) {
        uint32_t pos = nkeep + __popc(ob & lanemask_lt());
        // c_* become the kept candidates in sorted order; s_id their frontier upper bound
        S.c_id[pos] = a_id[t];
        S.c_d[pos] = a_d[t];
        S.s_id[pos] = a_ub[t];
      }
      nkeep += __popc(ob);
    }
    __syncwarp();
    if (nkeep == 0) continue;

    // ---- merge: frontier entry i moves to i + #(candidates before it)
    const uint32_t new_n = min(P.L, fr_n + nkeep);
    uint32_t my_id[kMaxFrPerLane];
    float my_d[kMaxFrPerLane];
    uint32_t my_pos[kMaxFrPerLane];
#pragma unroll
    for (uint32_t t = 0; t < kMaxFrPerLane; t++) {
      uint32_t i = lane + 32 * t;
      my_pos[t] = DD_NONE;
      my_id[t] = 0;
      my_d[t] = 0.f;
      if (i < fr_n) {
        uint32_t fi = S.fr_id[i];
        float fd = S.fr_d[i];
        uint32_t lo = 0, hi = nkeep;  // candidates strictly before this entry
        while (lo < hi) {
          uint32_t mid = (lo + hi) >> 1;
          if (pair_less(S.c_d[mid], S.c_id[mid] & ~DD_VBIT, fd, fi & ~DD_VBIT)) lo = mid + 1;
          else hi = mid;
        }
        my_id[t] = fi;
        my_d[t] = fd;
        my_pos[t] = i + lo;
      }
    }
    uint32_t c_ids[kMaxCandPerLane], c_pos[kMaxCandPerLane];
    float c_ds[kMaxCandPerLane];
#pragma unroll
    for (uint32_t t = 0; t < kMaxCandPerLane; t++) {
      uint32_t j = lane + 32 * t;
      c_pos[t] = DD_NONE;
      c_ids[t] = 0;
      c_ds[t] = 0.f;
      if (j < nkeep) {
        c_ids[t] = S.c_id[j];
        c_ds[t] = S.c_d[j];
        c_pos[t] = j + S.s_id[j];
      }
    }
    __syncwarp();
#pragma unroll
    for (uint32_t t = 0; t < kMaxFrPerLane; t++) {
      if (my_pos[t] < new_n) {
        S.fr_id[my_pos[t]] = my_id[t];
        S.fr_d[my_pos[t]] = my_d[t];
      }
    }
#pragma unroll
    for (uint32_t t = 0; t < kMaxCandPerLane; t++) {
      if (c_pos[t] < new_n) {
        S.fr_id[c_pos[t]] = c_ids[t];
        S.fr_d[c_pos[t]] = c_ds[t];
      }
    }
    if (P.query_mode) {
      // visited entries pushed off the end are remembered (in frontier order)
#pragma unroll
      for (uint32_t t = 0; t < kMaxFrPerLane; t++) {
        bool ev = (my_pos[t] != DD_NONE) && (my_pos[t] >= new_n) && (my_id[t] & DD_VBIT);
        uint32_t eb = __ballot_sync(FULL, ev);
        if (ev) {
          uint32_t pos = ev_n + __popc(eb & lanemask_lt());
          if (pos < P.vcap) S.ev_id[pos] = my_id[t] & ~DD_VBIT;
          else dd_set_error(P.err, DD_EVIS_CAP);
        }
        ev_n = min(P.vcap, ev_n + __popc(eb));
      }
    }
    fr_n = new_n;
    __syncwarp();

    // ---- k-cut (query mode, metric spaces only)
    if (P.k > 0 && fr_n > P.k && MT == DD_L2) {
      const float thr = (float)(P.cut * (double)S.fr_d[P.k]);
      uint32_t keep_n = 0;
      for (uint32_t base = 0; base < fr_n; base += 32) {
        uint32_t i = base + lane;
        bool kp = false;
        if (i < fr_n) {
          float fd = S.fr_d[i];
          kp = (fd < thr) || (fd == thr && (S.fr_id[i] & ~DD_VBIT) == 0);
        }
        keep_n += __popc(__ballot_sync(FULL, kp));
      }
      if (P.query_mode) {
        for (uint32_t base = keep_n; base < fr_n; base += 32) {
          uint32_t i = base + lane;
          bool ev = (i < fr_n) && (S.fr_id[i] & DD_VBIT);
          uint32_t eb = __ballot_sync(FULL, ev);
          if (ev) {
            uint32_t pos = ev_n + __popc(eb & lanemask_lt());
            if (pos < P.vcap) S.ev_id[pos] = S.fr_id[i] & ~DD_VBIT;
            else dd_set_error(P.err, DD_EVIS_CAP);
          }
          ev_n = min(P.vcap, ev_n + __popc(eb));
        }
      }
      fr_n = keep_n;
      __syncwarp();
    }
  }
  SearchOut o;
  o.fr_n = fr_n;
  o.vis_n = P.keep_visited ? vis_n : (uint32_t)num_visited;
  o.cmps = cmps;
  return o;
}

}  // namespace ddk
