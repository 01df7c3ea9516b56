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
//  * "visited" is a flag bit in the frontier id.  Within a run of identical
//    frontier entries the flagged copies come first, so the first unflagged
//    entry is the first element of set_difference(frontier, visited) even
//    when the lists are multisets (rows holding an id twice, as two-pass
//    builds produce).  Visited entries dropped from the frontier are kept in
//    an "evicted" list so a re-entering copy is flagged as set_difference
//    would (only possible in query mode, after a k-cut).
//  * the hash filter is replayed exactly: lanes whose ids fall in the same
//    slot are grouped with __match_any_sync; within a group the table value a
//    lane sees is the id of the previous lane in neighbour order (or the table
//    entry), and the last lane of the group writes the slot.  The table lives
//    in the warp's shared memory (24-bit ids when every id is below 0xFFFFFF).
//  * set_union + trim: candidates are ranked by (dist, id), the copies
//    set_union adds are kept, and every element moves to its merged position;
//    positions >= L are dropped.
#pragma once
#include "dd_common.cuh"
#include "kernels.cuh"

namespace ddk {

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
  uint32_t* ev_id;    // visited ids pushed out of the frontier (query_mode), capacity ecap
  uint32_t* ev_bloom; // 1024-bit filter of the ids in ev_id (shared memory, query_mode)
  uint32_t* hash;     // 2^bits slots (shared memory): uint32 ids, or with h24
                      // a uint16 array of the low bits then a uint8 array of the high bits
  int h24;            // ids stored in 24 bits (every id < 0xFFFFFF); 0xFFFFFF = empty
};

// bytes of the lossy "seen" table of 2^hbits slots
__host__ __device__ inline uint32_t hash_table_bytes(uint32_t hbits, bool h24) {
  return (h24 ? 3u : 4u) << hbits;
}

// ---------------------------------------------------------------------------
// The fast form's "seen" filter (build searches of builds whose graph rows
// never hold an id twice, with every id below 2^24 - 1; the host decides,
// rows_without_repeats).  In a build search (k = 0, no k-cut) the filter
// only decides which neighbours get their distance computed: an id it lets
// through twice is re-evaluated, fails the cutoff or is already in the
// frontier, and set_union drops the copy.  So any filter without false
// positives gives the reference's frontier, visited list and graph; only the
// dist_cmps count moves.  This one holds 2^hbits 16-bit tags (2 bytes a slot
// where the reference's table takes 3), set associative: ids are hashed with
// a bijection of [0, 2^24); the low hbits - 2 bits pick a bucket of four tags
// (one 8-byte word) and the remaining 26 - hbits bits are the tag, so a tag
// names exactly one id.  A lookup is one read per lane; a lane that missed
// pushes its tag into the front of the bucket and the oldest tag falls out.
// Lanes that write the same bucket in one step race, and the loser's tag is
// lost: the table only ever holds ids that were evaluated, so a lost tag
// costs a later re-evaluation, never a wrong answer.
// ---------------------------------------------------------------------------
__host__ __device__ inline uint32_t fast_table_bytes(uint32_t hbits) { return 2u << hbits; }

// bijective mix of a 24-bit id (xor-shifts and odd multipliers mod 2^24)
__device__ __forceinline__ uint32_t mix24(uint32_t x) {
  x &= 0xFFFFFFu;
  x ^= x >> 12;
  x = (x * 0x9E3779u) & 0xFFFFFFu;
  x ^= x >> 11;
  x = (x * 0x85EBCBu) & 0xFFFFFFu;
  x ^= x >> 12;
  return x;
}

// the id a slot holds (DD_NONE when empty); h24 is warp-uniform
__device__ __forceinline__ uint32_t hash_get(const SearchSmem& S, uint32_t nslots, uint32_t slot) {
  if (S.h24) {
    const uint16_t* lo = (const uint16_t*)S.hash;
    const uint8_t* hi = (const uint8_t*)(lo + nslots);
    const uint32_t v = (uint32_t)lo[slot] | ((uint32_t)hi[slot] << 16);
    return v == 0xFFFFFFu ? DD_NONE : v;
  }
  return S.hash[slot];
}
__device__ __forceinline__ void hash_set(const SearchSmem& S, uint32_t nslots, uint32_t slot,
                                         uint32_t id) {
  if (S.h24) {
    uint16_t* lo = (uint16_t*)S.hash;
    uint8_t* hi = (uint8_t*)(lo + nslots);
    lo[slot] = (uint16_t)(id & 0xFFFFu);
    hi[slot] = (uint8_t)(id >> 16);
  } else {
    S.hash[slot] = id;
  }
}

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
  uint32_t vcap;        // visited-list capacity (keep_visited)
  uint32_t ecap;        // evicted-list capacity (query_mode)
  int query_mode;       // track evicted visited entries for re-entry
  int keep_visited;     // record the visited list (build / debug)
  uint32_t* err;
  const uint8_t* screen;  // BF16 rows of float data (IndexView::screen), or null
  uint64_t sstride;
  const float* snorm;
  uint32_t fgroup_lg;     // float data: lanes per row of the exact distances (IndexView)
};

struct SearchOut {
  uint32_t fr_n;        // final frontier size
  uint32_t vis_n;       // number of visited nodes (= visited list length when kept)
  uint32_t cmps;        // distance computations (reference dist_cmps)
};

// The evicted list of a query search is scanned only for candidates whose id
// may be in it: a 1024-bit filter of the evicted ids answers "maybe" or "no".
__device__ __forceinline__ uint32_t ev_bloom_bit(uint32_t id) { return (id * 0x9E3779B1u) >> 22; }
__device__ __forceinline__ void ev_bloom_add(uint32_t* bloom, uint32_t id) {
  const uint32_t b = ev_bloom_bit(id);
  atomicOr(&bloom[b >> 5], 1u << (b & 31));
}
__device__ __forceinline__ bool ev_bloom_maybe(const uint32_t* bloom, uint32_t id) {
  const uint32_t b = ev_bloom_bit(id);
  return (bloom[b >> 5] >> (b & 31)) & 1u;
}

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

// slots of the fast filter: half the reference's count (the four-way buckets
// keep tags longer than its one-id slots, and the smaller table lets more
// searches share an SM), at least 2^11 so that a tag (26 - hbits bits) stays
// below the empty marker 0xFFFF
__host__ __device__ inline uint32_t fast_hash_bits(uint32_t L) {
  const uint32_t b = hash_bits_for(L) - 1;
  return b < 11 ? 11u : b;
}

template <int DT, int MT>
__device__ __forceinline__ float point_dist(const SearchParams& P, const uint8_t* qv, uint32_t id) {
  return Dist<DT, MT>::eval(qv, P.points + (uint64_t)id * P.stride, P.d);
}

// ---------------------------------------------------------------------------
// Fast form, float data: BF16 screen + exact FP32 re-rank of one step's kept
// neighbours (ids in S.s_id[0, nk)).  A neighbour enters the frontier only if
// its exact distance (the reference's FP32 order) is below the cutoff
// (include/utils/beamSearch.h:135-145).  Each neighbour's distance is first
// estimated from the BF16 copy of its row (half the bytes; G lanes each, any
// summation order) together with a rigorous bound on how far the exact FP32
// value can lie from the estimate; a neighbour whose lower bound is already at
// or above the cutoff fails for certain and is dropped.  The others (the ones
// that pass, and the few the bound cannot decide) get the exact distance from
// the FP32 row, one lane each, so every frontier entry carries the reference's
// value and the search takes the reference's path.
//
// The bound (u = 2^-24 is FP32's unit roundoff; b~ = bf16(b) is round to
// nearest, so |b~_i - b_i| <= 2^-8 |b~_i| for normal values):
//   L2:   |sum (a_i-b_i)^2 - sum (a_i-b~_i)^2| = |sum e_i (2 t_i + e_i)|
//         <= 2^-7 sum |b~_i| |t_i| + 2^-16 |b~|^2,     t_i = a_i - b~_i
//   MIPS: |sum a_i b_i - sum a_i b~_i| <= 2^-8 sum |a_i b~_i|
// plus the rounding of both FP32 sums: at most (d + 16) 2^-23 (gam) times the
// sum of the absolute terms, taken three times over for the two sums and the
// bound's own arithmetic, an extra 2^-20 for the final subtraction and 1e-20
// for subnormal BF16 values.  A NaN or infinite estimate (data beyond the BF16
// range) never drops a neighbour: the comparison is written to fail on NaN.
// Returns the number of candidates written to S.c_id / S.c_d, which hold the
// same entries in the same (neighbour) order as the exact path would.
// ---------------------------------------------------------------------------
// The exact FP32 distance (Dist<DD_F32, MT>::eval's value, bit for bit) from
// the query q (shared memory) to `row`, computed by a group of G lanes (G =
// 1, 2, 4 or 8, warp-uniform; sub = lane index in the group).  The reference
// sums float L2 as a chain over 4-value groups (each group summed left to
// right) and MIPS as a chain over single products: the terms do not depend on
// the chain, so the G lanes load and compute them in parallel (the row is in
// flight at once instead of in G consecutive batches) and every lane of the
// group then adds them into the chain in the reference's order, taking each
// term from the lane that computed it by shuffle.  Every lane of the warp
// must call it; lanes with act == false return 0.
template <int MT>
__device__ __forceinline__ float exact_dist_group(const float* q, const float* row, uint32_t d,
                                                  uint32_t sub, uint32_t G, bool act) {
  if (G == 1) return act ? Dist<DD_F32, MT>::eval(q, row, d) : 0.f;
  const uint32_t FULL = 0xffffffffu;
  const uint32_t base = lane_id() & ~(G - 1u);
  const uint32_t nv4 = (d + 3) >> 2;  // 4-value words (the query is zero padded to them)
  const float4* r4 = (const float4*)row;
  const float4* q4 = (const float4*)q;
  constexpr int NB = 4;  // words a lane has in flight
  float r = 0.f;
  for (uint32_t w0 = 0; w0 < nv4; w0 += NB * G) {
    float4 y[NB];
#pragma unroll
    for (int i = 0; i < NB; i++) {
      const uint32_t w = w0 + (uint32_t)i * G + sub;
      y[i] = (act && w < nv4) ? __ldg(r4 + w) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int i = 0; i < NB; i++) {
      const uint32_t w = w0 + (uint32_t)i * G + sub;
      const float4 x = w < nv4 ? q4[w] : make_float4(0.f, 0.f, 0.f, 0.f);
      float e[4];
      if (MT == DD_L2) {
        const float t0 = __fsub_rn(x.x, y[i].x), t1 = __fsub_rn(x.y, y[i].y);
        const float t2 = __fsub_rn(x.z, y[i].z), t3 = __fsub_rn(x.w, y[i].w);
        e[0] = __fmul_rn(t0, t0); e[1] = __fmul_rn(t1, t1);
        e[2] = __fmul_rn(t2, t2); e[3] = __fmul_rn(t3, t3);
      } else {
        e[0] = __fmul_rn(x.x, y[i].x); e[1] = __fmul_rn(x.y, y[i].y);
        e[2] = __fmul_rn(x.z, y[i].z); e[3] = __fmul_rn(x.w, y[i].w);
      }
      const float s = __fadd_rn(__fadd_rn(__fadd_rn(e[0], e[1]), e[2]), e[3]);
      // the chain over the words w0 + i G + g, g = 0 .. G-1 (warp-uniform)
      for (uint32_t g = 0; g < G; g++) {
        const uint32_t wg = w0 + (uint32_t)i * G + g;
        if (wg >= nv4) break;
        if (MT == DD_L2 && 4 * wg + 3 < d) {
          r = __fadd_rn(r, __shfl_sync(FULL, s, base + g));
        } else {  // MIPS, and the 0-3 value tail of L2: one value at a time
#pragma unroll
          for (int j = 0; j < 4; j++) {
            const float v = __shfl_sync(FULL, e[j], base + g);
            if (4 * wg + (uint32_t)j < d) r = __fadd_rn(r, v);
          }
        }
      }
    }
  }
  if (!act) return 0.f;
  return MT == DD_L2 ? r : -r;
}

template <int MT>
__device__ __forceinline__ uint32_t screen_and_rerank(const SearchParams& P, const SearchSmem& S,
                                                      uint32_t nk, float cutoff) {
  const uint32_t lane = lane_id();
  const uint32_t FULL = 0xffffffffu;
  const uint32_t nw = (P.d + 7) >> 3;  // 16-byte words of a BF16 row
  const float* qf = (const float*)S.qv;
  const float gam3 = 3.f * (float)(P.d + 16) * 0x1p-23f + 0x1p-20f;
  // G lanes per neighbour: 8 up to 4 neighbours, 4 up to 8, else 2
  const uint32_t lg = nk <= 4 ? 3u : (nk <= 8 ? 2u : 1u);
  const uint32_t G = 1u << lg, per = 32u >> lg, sub = lane & (G - 1);
  constexpr int NB = 4;  // words a lane has in flight
  uint32_t nm = 0;
  for (uint32_t k0 = 0; k0 < nk; k0 += per) {
    const uint32_t k = k0 + (lane >> lg);
    const bool act = k < nk;
    const uint32_t id = act ? S.s_id[k] : 0u;
    const uint4* row = (const uint4*)(P.screen + (uint64_t)id * P.sstride);
    const float nb2 = (MT == DD_L2 && act && sub == 0) ? __ldg(P.snorm + id) : 0.f;
    float acc = 0.f, bnd = 0.f;
    for (uint32_t w0 = sub; w0 < nw; w0 += NB * G) {
      uint4 y[NB];
#pragma unroll
      for (int i = 0; i < NB; i++) {
        const uint32_t w = w0 + (uint32_t)i * G;
        y[i] = (act && w < nw) ? __ldg(row + w) : make_uint4(0, 0, 0, 0);
      }
#pragma unroll
      for (int i = 0; i < NB; i++) {
        const uint32_t w = w0 + (uint32_t)i * G;
        if (w < nw) {
          // the query holds whole 4-value groups; values at or beyond d (the
          // BF16 row's zero padding) are left out, whatever a caller's device
          // query buffer holds there
          const float4 qa = *(const float4*)(qf + 8 * w);
          const float4 qb = (8 * w + 4 < P.d) ? *(const float4*)(qf + 8 * w + 4)
                                              : make_float4(0.f, 0.f, 0.f, 0.f);
          float qs[8] = {qa.x, qa.y, qa.z, qa.w, qb.x, qb.y, qb.z, qb.w};
          if (8 * w + 8 > P.d) {
#pragma unroll
            for (int j = 0; j < 8; j++)
              if (8 * w + (uint32_t)j >= P.d) qs[j] = 0.f;
          }
          const uint32_t ys[4] = {y[i].x, y[i].y, y[i].z, y[i].w};
#pragma unroll
          for (int j = 0; j < 8; j++) {
            const uint32_t hw = ys[j >> 1];
            const float b = __uint_as_float((j & 1) ? (hw & 0xffff0000u) : (hw << 16));
            if (MT == DD_L2) {
              const float t = qs[j] - b;
              acc = fmaf(t, t, acc);
              bnd = fmaf(fabsf(b), fabsf(t), bnd);
            } else {
              acc = fmaf(qs[j], b, acc);
              bnd = fmaf(fabsf(qs[j]), fabsf(b), bnd);
            }
          }
        }
      }
    }
    for (uint32_t o = 1; o < G; o <<= 1) {
      acc += __shfl_xor_sync(FULL, acc, o);
      bnd += __shfl_xor_sync(FULL, bnd, o);
    }
    float lowd;
    if (MT == DD_L2)
      lowd = acc - (1.01f * (0x1p-7f * bnd + 0x1p-16f * nb2) + acc * gam3 + 1e-20f);
    else
      lowd = -acc - (bnd * (1.01f * 0x1p-8f + gam3) + 1e-20f);
    const bool maybe = act && sub == 0 && !(lowd >= cutoff);
    const uint32_t mb = __ballot_sync(FULL, maybe);
    // in place: every id of this pass was read above, and positions before
    // nm + popc(mb) are at or below the ones read
    if (maybe) S.s_id[nm + __popc(mb & lanemask_lt())] = id;
    nm += __popc(mb);
  }
  __syncwarp();
  // exact distances of the survivors: G lanes each (few survivors) or one lane
  // each (many); both give the reference's FP32 value (exact_dist_group)
  const uint32_t lx = nm <= 4 ? 3u : (nm <= 8 ? 2u : (nm <= 16 ? 1u : 0u));
  const uint32_t perx = 32u >> lx, subx = lane & ((1u << lx) - 1u);
  uint32_t nc = 0;
  for (uint32_t k0 = 0; k0 < nm; k0 += perx) {
    const uint32_t k = k0 + (lane >> lx);
    const bool act = k < nm;
    const uint32_t id = act ? S.s_id[k] : 0u;
    const float dist = exact_dist_group<MT>((const float*)S.qv,
                                            (const float*)(P.points + (uint64_t)id * P.stride),
                                            P.d, subx, 1u << lx, act);
    const bool pass = act && subx == 0 && dist < cutoff;
    const uint32_t pb = __ballot_sync(FULL, pass);
    if (pass) {
      const uint32_t pos = nc + __popc(pb & lanemask_lt());
      S.c_id[pos] = id;
      S.c_d[pos] = dist;
    }
    nc += __popc(pb);
  }
  return nc;
}

// Runs one beam search on the warp.  `qv` must already hold the query.
// self_id: the id the reference skips as p.id() (the point itself in the
// build, the query's index in searchAll).
// FPL: frontier entries per lane (L <= 32*FPL); CPL: 32-lane chunks of a row (Rp <= 32*CPL).
// FASTF: the fast form's seen filter (see fast_table_bytes), build searches only.
template <int DT, int MT, int FPL, int CPL, bool FASTF = false>
__device__ SearchOut warp_beam_search(const SearchParams& P, const SearchSmem& S, uint64_t self_id) {
  const uint32_t lane = lane_id();
  const uint32_t FULL = 0xffffffffu;
  const uint32_t nslots = 1u << P.hbits;
  const uint32_t hmask = nslots - 1;
  {
    // all-ones bytes are the empty marker of every layout (a 16-bit tag of
    // the fast filter is below 2^15)
    uint4* h4 = (uint4*)S.hash;
    const uint4 none = make_uint4(DD_NONE, DD_NONE, DD_NONE, DD_NONE);
    const uint32_t n16 =
        (FASTF ? fast_table_bytes(P.hbits) : hash_table_bytes(P.hbits, S.h24 != 0)) / 16u;
    for (uint32_t i = lane; i < n16; i += 32) h4[i] = none;
    if (P.query_mode) S.ev_bloom[lane] = 0u;
  }
  if (lane == 0) {
    S.fr_id[0] = P.start;
    S.fr_d[0] = point_dist<DT, MT>(P, S.qv, P.start);
  }
  __syncwarp();
  uint32_t fr_n = 1;
  uint32_t scan0 = 0;      // lower bound of the first unvisited frontier position
  uint32_t vis_n = 0;      // visited list length
  // Fast form: the visited list is built sorted, from the end of its slice
  // down (see the eviction step), so it leaves the search in the reference's
  // (dist, id) order with no sort: [vtop, vcap) holds it.
  uint32_t vtop = P.vcap;
  uint32_t ev_n = 0;       // evicted list length (query mode)
  uint32_t cmps = 1;       // dist to the start point
  uint64_t num_visited = 0;
  const float int_max_f = 2147483648.0f;  // (float)std::numeric_limits<int>::max()
  const uint32_t dl = min(P.degree_limit, P.Rp);
  // The row of the node expected to be visited next is loaded while the
  // current step is still merging (a speculative load: it is used only if
  // that node is indeed the one visited next).
  uint32_t pred = DD_NONE;
  uint32_t a_pre[CPL];
  auto prefetch_row = [&](uint32_t node) {
    pred = node;
    const uint32_t* prow = P.graph + (uint64_t)node * P.Rp;
#pragma unroll
    for (int t = 0; t < CPL; t++) {
      uint32_t j = 32 * t + lane;
      a_pre[t] = (j < dl) ? __ldg(prow + j) : DD_NONE;
    }
  };

  // Fast form: the register merge knows the next node (the first unvisited
  // entry of the merged frontier), its position and distance, so the next
  // step skips the scan.  known_pos: -1 unknown (scan), -2 none left.
  int known_pos = -1;
  uint32_t known_id = 0;
  float known_d = 0.f;
  while (num_visited < P.limit) {
    // ---- closest unvisited frontier entry (every entry before scan0 is visited)
    int cur_pos = -1;
    uint32_t cur;
    float cur_d;
    if (FASTF && known_pos != -1) {
      if (known_pos < 0) break;
      cur_pos = known_pos;
      cur = known_id;
      cur_d = known_d;
    } else {
      for (uint32_t base = scan0 & ~31u; base < fr_n; base += 32) {
        uint32_t i = base + lane;
        bool unv = (i < fr_n) && !(S.fr_id[i] & DD_VBIT);
        uint32_t b = __ballot_sync(FULL, unv);
        if (b) { cur_pos = (int)(base + __ffs(b) - 1); break; }
      }
      if (cur_pos < 0) break;
      cur = S.fr_id[cur_pos];
      cur_d = S.fr_d[cur_pos];
    }
    known_pos = -1;
    const float cutoff = (fr_n < P.L) ? int_max_f : S.fr_d[fr_n - 1];
    // the row of the node being visited: all chunks loaded up front
    uint32_t a[CPL];
    if (cur == pred) {
#pragma unroll
      for (int t = 0; t < CPL; t++) a[t] = a_pre[t];
    } else {
      const uint32_t* row = P.graph + (uint64_t)cur * P.Rp;
#pragma unroll
      for (int t = 0; t < CPL; t++) {
        uint32_t j = 32 * t + lane;
        a[t] = (j < dl) ? __ldg(row + j) : DD_NONE;
      }
    }
    __syncwarp();
    if (lane == 0) {
      S.fr_id[cur_pos] = cur | DD_VBIT;
      if (P.keep_visited && !FASTF) {
        if (vis_n < P.vcap) {
          S.vis_id[vis_n] = cur;
          S.vis_d[vis_n] = cur_d;
        } else {
          dd_set_error(P.err, DD_EVIS_CAP);
        }
      }
    }
    if (P.keep_visited && (FASTF || vis_n < P.vcap)) vis_n++;
    num_visited++;
    // the next unvisited entry after cur: visited next unless a new candidate beats it
    int nxt_pos = -1;
    for (uint32_t base = (uint32_t)(cur_pos + 1) & ~31u; base < fr_n; base += 32) {
      uint32_t i = base + lane;
      bool unv = (i > (uint32_t)cur_pos) && (i < fr_n) && !(S.fr_id[i] & DD_VBIT);
      uint32_t b = __ballot_sync(FULL, unv);
      if (b) { nxt_pos = (int)(base + __ffs(b) - 1); break; }
    }
    // its row is brought into L2 now (128-byte lines, one per lane); the
    // speculative load of the next row then usually hits L2
    if (nxt_pos >= 0 && lane * 32u < dl) {
      const uint32_t* nrow = P.graph + (uint64_t)S.fr_id[nxt_pos] * P.Rp + lane * 32u;
      asm volatile("prefetch.global.L2 [%0];" ::"l"(nrow));
    }

    // ---- hash filter, replayed chunk by chunk in neighbour order.  The
    // slots, same-slot groups and predecessor ids of all chunks are computed
    // first (they do not depend on the table); the table is then read and
    // written chunk after chunk.
    bool keep[CPL];
    if (FASTF) {
      uint2* tab = (uint2*)S.hash;
      const uint32_t bbits = P.hbits - 2;
      uint32_t slot[CPL];
      uint2 nw[CPL];
#pragma unroll
      for (int t = 0; t < CPL; t++) {
        uint32_t at = a[t];
        if (at != DD_NONE && at >= P.n) {
          dd_set_error(P.err, DD_EBAD_ID);
          at = DD_NONE;
          a[t] = DD_NONE;
        }
        const uint32_t f = mix24(at);
        slot[t] = f & ((1u << bbits) - 1u);
        const uint32_t tag = f >> bbits;
        const uint32_t tt = tag | (tag << 16);
        const uint2 w = tab[slot[t]];
        const bool hit = (__vcmpeq2(w.x, tt) | __vcmpeq2(w.y, tt)) != 0u;
        keep[t] = (at != DD_NONE) && ((uint64_t)at != self_id) && !hit;
        nw[t] = make_uint2((w.x << 16) | tag, (w.y << 16) | (w.x >> 16));
      }
      __syncwarp();
#pragma unroll
      for (int t = 0; t < CPL; t++)
        if (keep[t]) tab[slot[t]] = nw[t];
      __syncwarp();
    } else {
      bool part[CPL];
      uint32_t loc[CPL], grp[CPL], prev_a[CPL];
#pragma unroll
      for (int t = 0; t < CPL; t++) {
        uint32_t at = a[t];
        if (at != DD_NONE && at >= P.n) {
          dd_set_error(P.err, DD_EBAD_ID);
          at = DD_NONE;
          a[t] = DD_NONE;
        }
        part[t] = (at != DD_NONE) && ((uint64_t)at != self_id);
        loc[t] = part[t] ? (uint32_t)(dd_hash64(at) & hmask) : (0x80000000u | lane);
      }
#pragma unroll
      for (int t = 0; t < CPL; t++) {
        grp[t] = __match_any_sync(FULL, loc[t]);
        const uint32_t before = grp[t] & lanemask_lt();
        prev_a[t] = __shfl_sync(FULL, a[t], before ? 31 - __clz(before) : lane);
      }
#pragma unroll
      for (int t = 0; t < CPL; t++) {
        const uint32_t before = grp[t] & lanemask_lt();
        const uint32_t tval = (part[t] && !before) ? hash_get(S, nslots, loc[t]) : DD_NONE;
        const uint32_t seen_val = before ? prev_a[t] : tval;
        keep[t] = part[t] && (seen_val != a[t]);
        __syncwarp();
        if (part[t] && (grp[t] & lanemask_gt()) == 0) hash_set(S, nslots, loc[t], a[t]);
        __syncwarp();
      }
    }

    // ---- the kept neighbours, compacted in neighbour order
    uint32_t nk = 0;
#pragma unroll
    for (int t = 0; t < CPL; t++) {
      const uint32_t kb = __ballot_sync(FULL, keep[t]);
      if (keep[t]) S.s_id[nk + __popc(kb & lanemask_lt())] = a[t];
      nk += __popc(kb);
    }
    cmps += nk;
    __syncwarp();
    // ---- their distances: G lanes per neighbour for integer data (exact in
    // any grouping), one lane for float data (the reference's summation order)
    uint32_t nc = 0;
    if (DT == DD_F32 && P.screen != nullptr && cutoff < int_max_f) {
      // fast form, float data, full frontier: BF16 screen, exact re-rank
      nc = screen_and_rerank<MT>(P, S, nk, cutoff);
    } else {
      // float data: one lane per row in the plain form; in the fast form
      // (fgroup_lg > 0) groups of lanes that load a row together and chain its
      // terms in the reference's order (exact_dist_group): fewer L1 wavefronts
      // per row for more shuffles.  fgroup_lg 1-3: G = 2, 4, 8 lanes; 4: the
      // integer rule (as many lanes as keep one pass, up to 8)
      const uint32_t fg = P.fgroup_lg;
      const uint32_t lg =
          (DT == DD_F32)
              ? (fg < 4 ? fg : (nk <= 4 ? 3u : (nk <= 8 ? 2u : (nk <= 16 ? 1u : 0u))))
              : (nk <= 8 ? 2u : (nk <= 16 ? 1u : 0u));
      const uint32_t G = 1u << lg, per = 32u >> lg, sub = lane & (G - 1);
      for (uint32_t k0 = 0; k0 < nk; k0 += per) {
        const uint32_t k = k0 + (lane >> lg);
        const bool act = k < nk;
        const uint32_t id = act ? S.s_id[k] : 0u;
        float dist;
        if (DT == DD_F32 && fg != 0)
          dist = exact_dist_group<MT>((const float*)S.qv,
                                      (const float*)(P.points + (uint64_t)id * P.stride), P.d,
                                      sub, G, act);
        else
          dist = dist_group<DT, MT, FASTF ? 4 : 8>(
              (const uint4*)S.qv, P.points + (uint64_t)id * P.stride, P.d, sub, G, act);
        const bool pass = act && sub == 0 && dist < cutoff;
        const uint32_t pb = __ballot_sync(FULL, pass);
        if (pass) {
          const uint32_t pos = nc + __popc(pb & lanemask_lt());
          S.c_id[pos] = id;
          S.c_d[pos] = dist;
        }
        nc += __popc(pb);
      }
    }
    __syncwarp();
    if (nc == 0) {
      if (nxt_pos >= 0) {
        prefetch_row(S.fr_id[nxt_pos]);
        if (FASTF) {
          known_pos = nxt_pos;
          known_id = S.fr_id[nxt_pos];
          known_d = S.fr_d[nxt_pos];
        }
      } else if (FASTF) {
        known_pos = -2;
      }
      scan0 = nxt_pos >= 0 ? (uint32_t)nxt_pos : fr_n;
      continue;
    }

    // Every step ends with the same scatter: frontier entry t of this lane
    // moves to my_pos[t] (DD_NONE: no entry), candidate slot t to c_pos[t].
    uint32_t nkeep = 0, ub0 = 0;
    uint32_t my_id[FPL], my_pos[FPL];
    float my_d[FPL];
    uint32_t c_ids[CPL], c_pos[CPL];
    float c_ds[CPL];
    if (FASTF && nc <= 32) {
      // ---- Fast form with at most 32 candidates (nearly every step): one
      // candidate per lane, ordered with shuffles, no shared-memory round
      // trips.  Its rows hold no repeated id and it only runs build searches
      // (no evicted list, no k-cut), so the candidates are distinct, the
      // frontier holds each id at most once, and a candidate is added unless
      // the frontier already holds it.
      const bool cv = lane < nc;
      const float cd = cv ? S.c_d[lane] : 0.f;
      const uint32_t ci = cv ? S.c_id[lane] : 0u;
      uint32_t lo = 0;  // frontier entries below this candidate
      bool keep = false;
      if (cv) {
        uint32_t hi = fr_n;
        while (lo < hi) {
          const uint32_t mid = (lo + hi) >> 1;
          if (pair_less(S.fr_d[mid], S.fr_id[mid] & ~DD_VBIT, cd, ci)) lo = mid + 1;
          else hi = mid;
        }
        keep = !(lo < fr_n && S.fr_d[lo] == cd && (S.fr_id[lo] & ~DD_VBIT) == ci);
      }
      const uint32_t K = __ballot_sync(FULL, keep);
      nkeep = __popc(K);
      // one pass over the kept candidates gives this candidate's rank among
      // them and each frontier entry's shift (#kept candidates placed before it)
      uint32_t krank = 0;
      uint32_t shift[FPL];
#pragma unroll
      for (int t = 0; t < FPL; t++) shift[t] = 0;
      for (uint32_t km = K; km; km &= km - 1) {
        const uint32_t k = __ffs(km) - 1;
        const float dk = __shfl_sync(FULL, cd, k);
        const uint32_t ik = __shfl_sync(FULL, ci, k);
        const uint32_t lk = __shfl_sync(FULL, lo, k);
        krank += pair_less(dk, ik, cd, ci) ? 1u : 0u;
#pragma unroll
        for (int t = 0; t < FPL; t++) shift[t] += (lk <= lane + 32u * t) ? 1u : 0u;
      }
      {
        // the next node: the better of the best new candidate and nxt_pos,
        // which is the first unvisited entry of the merged frontier; in the
        // fast form also its merged position (the best candidate lands at its
        // lower bound, the old entry moves by its shift) unless the trim drops it
        uint32_t nid = DD_NONE, npos = DD_NONE;
        float nd = 0.f;
        if (K) {
          const uint32_t src = __ffs(__ballot_sync(FULL, keep && krank == 0)) - 1;
          nid = __shfl_sync(FULL, ci, src);
          nd = __shfl_sync(FULL, cd, src);
          npos = __shfl_sync(FULL, lo, src);
        }
        if (nxt_pos >= 0) {
          const uint32_t fid = S.fr_id[nxt_pos];
          const float fd = S.fr_d[nxt_pos];
          if (nid == DD_NONE || !pair_less(nd, nid, fd, fid)) {
            nid = fid;
            nd = fd;
            if (FASTF) {
              const uint32_t tn = (uint32_t)nxt_pos >> 5;
              uint32_t sh = 0;
#pragma unroll
              for (int t = 0; t < FPL; t++)
                if ((uint32_t)t == tn) sh = shift[t];
              npos = (uint32_t)nxt_pos + __shfl_sync(FULL, sh, (uint32_t)nxt_pos & 31u);
            }
          }
        }
        if (nid != DD_NONE) prefetch_row(nid);
        if (FASTF) {
          known_pos = (nid != DD_NONE && npos < min(P.L, fr_n + nkeep)) ? (int)npos : -2;
          known_id = nid;
          known_d = nd;
        }
      }
      if (nkeep == 0) {
        scan0 = nxt_pos >= 0 ? (uint32_t)nxt_pos : fr_n;
        continue;
      }
      ub0 = __reduce_min_sync(FULL, keep ? lo : 0xFFFFFFFFu);
#pragma unroll
      for (int t = 0; t < FPL; t++) {
        const uint32_t i = lane + 32 * t;
        my_pos[t] = DD_NONE;
        my_id[t] = 0;
        my_d[t] = 0.f;
        if (i < fr_n) {
          my_pos[t] = i + shift[t];  // entries before ub0 have no shift: not rewritten
          if (i >= ub0) {
            my_id[t] = S.fr_id[i];
            my_d[t] = S.fr_d[i];
          }
        }
      }
      c_ids[0] = ci;
      c_ds[0] = cd;
      c_pos[0] = keep ? lo + krank : DD_NONE;
#pragma unroll
      for (int t = 1; t < CPL; t++) {
        c_ids[t] = 0;
        c_ds[t] = 0.f;
        c_pos[t] = DD_NONE;
      }
    } else {
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
          // (the fast form's rows hold no repeated id, so no identical copies)
          r += (pair_less(dj, ij, di, ii) || (!FASTF && dj == di && ij == ii && j < i)) ? 1u : 0u;
        }
        S.s_id[r] = ii;
        S.s_d[r] = di;
      }
      __syncwarp();
      // set_union as multisets: with m frontier copies of a value and n candidate
      // copies, the candidate copies k >= m are added, after the frontier's copies.
      // A re-entering copy counts as visited while k < (visits of the value):
      // set_difference(frontier, visited) is a multiset difference too.
      bool a_ok[CPL];
      uint32_t a_id[CPL], a_ub[CPL];
      float a_d[CPL];
#pragma unroll
      for (int t = 0; t < CPL; t++) {
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
              if (ev_bloom_maybe(S.ev_bloom, ci))
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
#pragma unroll
      for (int t = 0; t < CPL; t++) {
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
      {
        // expected next node: the better of the best new candidate and nxt_pos
        uint32_t nid = DD_NONE;
        if (nkeep > 0 && !(S.c_id[0] & DD_VBIT)) nid = S.c_id[0];
        if (nxt_pos >= 0 &&
            (nid == DD_NONE || !pair_less(S.c_d[0], nid, S.fr_d[nxt_pos], S.fr_id[nxt_pos])))
          nid = S.fr_id[nxt_pos];
        if (nid != DD_NONE) prefetch_row(nid);
      }
      if (nkeep == 0) {
        scan0 = nxt_pos >= 0 ? (uint32_t)nxt_pos : fr_n;
        continue;
      }

      // ---- merge: frontier entry i moves to i + #(kept candidates placed before
      // it) = i + #{j : ub_j <= i}; candidate j moves to j + ub_j.  Entries
      // before the first insertion point ub_0 stay where they are.
      ub0 = S.s_id[0];
      // Fast form with few kept candidates (the common case once the frontier
      // is full): every entry's shift is counted from the broadcast ub_j, with
      // no per-entry binary search.
      const bool count_shift = FASTF && nkeep <= 8;
      uint32_t shift[FPL];
#pragma unroll
      for (int t = 0; t < FPL; t++) shift[t] = 0;
      if (count_shift) {
        for (uint32_t j = 0; j < nkeep; j++) {
          const uint32_t ubj = S.s_id[j];
#pragma unroll
          for (int t = 0; t < FPL; t++) shift[t] += (ubj <= lane + 32u * t) ? 1u : 0u;
        }
      }
#pragma unroll
      for (int t = 0; t < FPL; t++) {
        uint32_t i = lane + 32 * t;
        my_pos[t] = DD_NONE;
        my_id[t] = 0;
        my_d[t] = 0.f;
        if (i < fr_n) {
          if (i < ub0) {
            my_pos[t] = i;  // unmoved: not rewritten
          } else {
            uint32_t lo = shift[t];
            if (!count_shift) {
              uint32_t hi = nkeep;
              lo = 1;
              while (lo < hi) {
                uint32_t mid = (lo + hi) >> 1;
                if (S.s_id[mid] <= i) lo = mid + 1;
                else hi = mid;
              }
            }
            my_id[t] = S.fr_id[i];
            my_d[t] = S.fr_d[i];
            my_pos[t] = i + lo;
          }
        }
      }
#pragma unroll
      for (int t = 0; t < CPL; t++) {
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
    }
    const uint32_t new_n = min(P.L, fr_n + nkeep);
    // unvisited entries now sit at or after min(ub_0, old nxt_pos)
    scan0 = min(ub0, nxt_pos >= 0 ? (uint32_t)nxt_pos : new_n);
    __syncwarp();
#pragma unroll
    for (int t = 0; t < FPL; t++) {
      if (my_pos[t] < new_n && my_pos[t] != lane + 32u * t) {
        S.fr_id[my_pos[t]] = my_id[t];
        S.fr_d[my_pos[t]] = my_d[t];
      }
    }
#pragma unroll
    for (int t = 0; t < CPL; t++) {
      if (c_pos[t] < new_n) {
        S.fr_id[c_pos[t]] = c_ids[t];
        S.fr_d[c_pos[t]] = c_ds[t];
      }
    }
    if (FASTF && P.keep_visited) {
      // Visited entries pushed off the end of a full frontier never come back
      // in a build search (they fail the cutoff from now on), and every entry
      // pushed off later is smaller in (dist, id) than every one pushed off
      // before (the frontier's last entry only improves, and candidates must
      // beat it).  So each block, in frontier order, goes just below the
      // blocks already written; the final frontier's visited entries go below
      // them at the end.
      uint32_t emask[FPL];
      uint32_t etot = 0;
#pragma unroll
      for (int t = 0; t < FPL; t++) {
        const bool ev = (my_pos[t] != DD_NONE) && (my_pos[t] >= new_n) && (my_id[t] & DD_VBIT);
        emask[t] = __ballot_sync(FULL, ev);
        etot += __popc(emask[t]);
      }
      if (etot > vtop) {
        if (lane == 0) dd_set_error(P.err, DD_EVIS_CAP);
        vtop = 0;
      } else if (etot) {
        const uint32_t base = vtop - etot;
        uint32_t acc = 0;
#pragma unroll
        for (int t = 0; t < FPL; t++) {
          if ((emask[t] >> lane) & 1u) {
            const uint32_t pos = base + acc + __popc(emask[t] & lanemask_lt());
            S.vis_id[pos] = my_id[t] & ~DD_VBIT;
            S.vis_d[pos] = my_d[t];
          }
          acc += __popc(emask[t]);
        }
        vtop = base;
      }
    }
    if (P.query_mode) {
      // visited entries pushed off the end are remembered (in frontier order)
#pragma unroll
      for (int t = 0; t < FPL; t++) {
        bool ev = (my_pos[t] != DD_NONE) && (my_pos[t] >= new_n) && (my_id[t] & DD_VBIT);
        uint32_t eb = __ballot_sync(FULL, ev);
        if (ev) {
          uint32_t pos = ev_n + __popc(eb & lanemask_lt());
          if (pos < P.ecap) {
            S.ev_id[pos] = my_id[t] & ~DD_VBIT;
            ev_bloom_add(S.ev_bloom, my_id[t] & ~DD_VBIT);
          } else {
            dd_set_error(P.err, DD_EVIS_CAP);
          }
        }
        ev_n = min(P.ecap, ev_n + __popc(eb));
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
            if (pos < P.ecap) {
              S.ev_id[pos] = S.fr_id[i] & ~DD_VBIT;
              ev_bloom_add(S.ev_bloom, S.fr_id[i] & ~DD_VBIT);
            } else {
              dd_set_error(P.err, DD_EVIS_CAP);
            }
          }
          ev_n = min(P.ecap, ev_n + __popc(eb));
        }
      }
      fr_n = keep_n;
      __syncwarp();
    }
  }
  if (FASTF && P.keep_visited) {
    // the final frontier's visited entries, in order, below the evicted blocks
    uint32_t nflag = 0;
    for (uint32_t base = 0; base < fr_n; base += 32) {
      const uint32_t i = base + lane;
      nflag += __popc(__ballot_sync(FULL, i < fr_n && (S.fr_id[i] & DD_VBIT)));
    }
    if (nflag > vtop) {
      if (lane == 0) dd_set_error(P.err, DD_EVIS_CAP);
      vtop = 0;
    } else {
      uint32_t pos0 = vtop - nflag;
      for (uint32_t base = 0; base < fr_n; base += 32) {
        const uint32_t i = base + lane;
        const bool f = i < fr_n && (S.fr_id[i] & DD_VBIT);
        const uint32_t fb = __ballot_sync(FULL, f);
        if (f) {
          const uint32_t pos = pos0 + __popc(fb & lanemask_lt());
          S.vis_id[pos] = S.fr_id[i] & ~DD_VBIT;
          S.vis_d[pos] = S.fr_d[i];
        }
        pos0 += __popc(fb);
      }
      vtop -= nflag;
    }
    __syncwarp();
  }
  SearchOut o;
  o.fr_n = fr_n;
  // fast form: the recorded list [vtop, vcap), whose length is the visit count
  o.vis_n = !P.keep_visited ? (uint32_t)num_visited : (FASTF ? P.vcap - vtop : vis_n);
  o.cmps = cmps;
  return o;
}

}  // namespace ddk
