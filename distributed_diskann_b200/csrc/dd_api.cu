// Host side of the C ABI (include/dd_gpu.h): handle management, the batched
// build driver (round schedule of src/bsp_index.hpp:141-246 collapsed onto one
// device-resident index) and the search / ground-truth entry points.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/dd_gpu.h"
#include "dd_common.cuh"
#include "kernels.cuh"
#include "search_core.cuh"
#include "semisort.cuh"
#include "sort_emul.cuh"

using namespace ddk;

struct dd_index {
  int dtype = 0, metric = 0;
  uint64_t n = 0;
  uint32_t d = 0, R = 0, Rp = 0;
  uint64_t stride = 0;  // device row stride in bytes
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = 0;
  uint8_t* points = nullptr;
  uint32_t* graph = nullptr;
  uint32_t* err = nullptr;
  std::string last_error;
  uint64_t launches = 0;
  // build scratch (grown on demand, kept for reuse)
  uint64_t bcap = 0;        // batch capacity of the scratch below
  uint32_t* new_out = nullptr;
  float* new_key = nullptr;  // distances of new_out's entries (fast form)
  float* row_key = nullptr;  // n x Rp: each graph entry's distance to its row's point (fast form)
  bool row_key_ok = false;
  uint32_t* stat_vis = nullptr;
  uint32_t* stat_cmps = nullptr;
  uint32_t* sort_t[2] = {nullptr, nullptr};  // semisort ping-pong buffers
  uint32_t* sort_v[2] = {nullptr, nullptr};
  uint32_t* hist = nullptr;
  uint32_t* heads = nullptr;
  uint32_t* flags = nullptr;
  uint32_t* counters = nullptr;
  uint32_t* big = nullptr;
  uint32_t* block_sums = nullptr;
  unsigned long long* acc = nullptr;  // [0] visited [1] cmps [2] groups [3] prunes [4] cands [5] big
  uint32_t* gcand = nullptr;          // CTA big-target workspace slices
  float* gkey = nullptr;
  int* gpos = nullptr;
  uint32_t* gbits = nullptr;
  int* granges = nullptr;
  uint64_t gcap = 0;
  // per-point visited-list slices of the build searches (grown on demand)
  uint32_t* vis_all = nullptr;
  uint64_t vis_all_words = 0;
  uint32_t* ref_rows = nullptr;  // n x (R+1) reference-layout rows for downloads
  // fast form, float data: BF16 copies of the rows and their squared norms
  // (the search steps' screen), rebuilt after any change of the points
  uint8_t* screen = nullptr;
  float* snorm = nullptr;
  uint64_t sstride = 0;
  bool screen_ok = false;
  bool verbose = false;
  bool hash32 = false;  // DD_HASH32=1: 32-bit hash-table ids even when n < 2^24 - 1
  int search_mode = DD_MODE_FAST;
  // fast form: device work queues (two per round and pass), the CUDA graph of
  // the last build sequence and the stream it is captured on
  uint32_t* queues = nullptr;
  uint64_t queue_words = 0;
  uint64_t scratch_gen = 0;  // bumped whenever build scratch is reallocated
  cudaStream_t own_stream = nullptr;
  cudaGraphExec_t gexec = nullptr;
  uint64_t launches_per_graph = 0;
  uint32_t* qcls = nullptr;  // query class lists, counts and queues (fast search form)
  uint64_t qcls_words = 0;
  uint32_t* qhash = nullptr;  // global seen tables of the wide beam-width classes
  uint64_t qhash_words = 0;
  uint32_t* qev = nullptr;    // evicted lists of the query searches
  uint64_t qev_words = 0;
  // sharded build: the launch shapes and parameters set by dd_shard_begin
  bool shard_ready = false;
  dd_build_params shard_params{};
  uint64_t shard_bmax = 0;
  std::vector<uint64_t> graph_key;  // what the captured graph was built for
};

namespace {

int fail(dd_index* h, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (h) h->last_error = buf;
  return code;
}

#define CK(call)                                                                    \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess)                                                          \
      return fail(h, e_ == cudaErrorMemoryAllocation ? DD_ERR_OOM : DD_ERR_CUDA,    \
                  "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

uint32_t esize(int dtype) { return dtype == DD_F32 ? 4u : 1u; }

IndexView view(dd_index* h) {
  IndexView v;
  v.dtype = h->dtype;
  v.metric = h->metric;
  v.points = h->points;
  v.stride = h->stride;
  v.graph = h->graph;
  v.Rp = h->Rp;
  v.R = h->R;
  v.n = h->n;
  v.d = h->d;
  v.err = h->err;
  return v;
}

// The BF16 screen of float searches (search_core.cuh screen_and_rerank), for
// float data of at most 4096 dimensions, is opt-in: DD_SCREEN=1.  Measured on
// B200 it is slower than computing every candidate's exact FP32 distance (the
// search is bound by instruction issue, not by the bytes the BF16 rows save:
// 1M x 200 MIPS build search 286 against 276 ms, queries at recall 0.95 3.1M
// against 4.2M QPS), so by default the fast form computes them all exactly,
// as the plain form does.
bool screen_enabled(const dd_index* h) {
  if (h->dtype != DD_F32 || h->d > 4096) return false;
  const char* e = getenv("DD_SCREEN");
  return e && e[0] == '1';
}

void attach_screen(const dd_index* h, IndexView* ix) {
  ix->screen = h->screen;
  ix->sstride = h->sstride;
  ix->snorm = h->snorm;
}

// Fast form, float data: how many lanes compute one candidate's exact distance
// in a search step (IndexView::fgroup_lg): one by default; DD_FGROUP=1/2/3
// (2/4/8 lanes) or 4 (per step) asks for lane groups.  Measured on B200 the
// groups are slower (1M x 200 MIPS build search 277 ms with one lane, 307 ms
// per-step groups, 395 ms with pairs): the shuffles of the chain cost more
// than the L1 wavefronts the shared row loads save.
uint32_t fast_fgroup(const dd_index* h) {
  if (h->dtype != DD_F32) return 0;
  uint32_t lg = 0;
  if (const char* e = getenv("DD_FGROUP")) lg = (uint32_t)std::min(4, std::max(0, atoi(e)));
  return lg;
}

template <typename T>
cudaError_t dalloc(T** p, uint64_t count) {
  return cudaMalloc((void**)p, std::max<uint64_t>(count, 1) * sizeof(T));
}

void dfree(void* p) {
  if (p) cudaFree(p);
}

// Makes the BF16 row copies current (stream-ordered after the points' upload).
int ensure_screen(dd_index* h) {
  if (h->screen_ok) return DD_OK;
  if (!h->screen) {
    h->sstride = ((uint64_t)h->d * 2 + 15) / 16 * 16;
    CK(dalloc(&h->screen, h->n * h->sstride));
    CK(dalloc(&h->snorm, h->n));
  }
  launch_screen_rows(view(h), h->screen, h->sstride, h->snorm, h->stream);
  CK(cudaGetLastError());
  h->screen_ok = true;
  return DD_OK;
}

int check_error_word(dd_index* h, uint32_t* bits = nullptr) {
  uint32_t e = 0;
  CK(cudaMemcpyAsync(&e, h->err, 4, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (bits) *bits = e;
  if (e) {
    cudaMemsetAsync(h->err, 0, 4, h->stream);
    std::string m = "device error:";
    if (e & DD_EBAD_ID) m += " neighbour id out of range;";
    if (e & DD_EVIS_CAP) m += " visited list exceeded its capacity (raise vcap);";
    if (e & DD_ECAND_CAP) m += " a per-query beam width was 0, below k or above Lmax;";
    if (e & DD_EDEGREE) m += " row degree exceeds R;";
    if (e & DD_ESEG_CAP) m += " reverse-edge group exceeded the workspace;";
    return fail(h, DD_ERR_DEVICE, "%s", m.c_str());
  }
  return DD_OK;
}

// (floor, ceiling) rounds: src/bsp_index.hpp:162-166, 238-246 (identity order)
std::vector<std::pair<uint64_t, uint64_t>> schedule(uint64_t n, uint64_t max_build, double frac,
                                                    int knn_mode) {
  uint64_t m = n;
  if (knn_mode) frac = 1.0;
  else if (max_build != 0) m = std::min<uint64_t>(max_build, m);
  size_t mb = std::min((size_t)(frac * (float)m), (size_t)1000000ul);
  if (mb == 0) mb = m;
  std::vector<std::pair<uint64_t, uint64_t>> r;
  size_t inc = 0, count = 0;
  while (count < m) {
    size_t fl, ce;
    if (std::pow(2.0, (double)inc) <= (double)mb) {
      fl = (size_t)std::pow(2.0, (double)inc) - 1;
      ce = std::min((size_t)std::pow(2.0, (double)(inc + 1)), (size_t)m) - 1;
      count = ce;
    } else {
      fl = count;
      ce = std::min(count + mb, (size_t)m);
      count += mb;
    }
    r.push_back({fl, ce});
    inc++;
  }
  return r;
}

int ensure_build_scratch(dd_index* h, uint64_t B) {
  if (!h->counters) {
    CK(dalloc(&h->counters, 8));
    CK(dalloc(&h->block_sums, kScanBlocks + 1));
    CK(dalloc(&h->acc, 8));
  }
  if (B <= h->bcap) return DD_OK;
  h->scratch_gen++;
  void* old[] = {h->new_out, h->new_key, h->stat_vis, h->stat_cmps, h->sort_t[0], h->sort_t[1], h->sort_v[0],
                 h->sort_v[1], h->hist, h->heads, h->flags, h->big, h->gcand, h->gkey,
                 h->gpos, h->gbits, h->granges};
  for (void* p : old) dfree(p);
  const uint64_t E = B * h->Rp;
  CK(dalloc(&h->new_out, E));
  CK(dalloc(&h->new_key, E));
  CK(dalloc(&h->stat_vis, B));
  CK(dalloc(&h->stat_cmps, B));
  for (int i = 0; i < 2; i++) {
    CK(dalloc(&h->sort_t[i], E));
    CK(dalloc(&h->sort_v[i], E));
  }
  CK(dalloc(&h->hist, semisort_hist_words(E)));
  CK(dalloc(&h->heads, E));
  CK(dalloc(&h->flags, E));
  CK(dalloc(&h->big, E));
  h->gcap = B + h->Rp;
  CK(dalloc(&h->gcand, kBigSlots * h->gcap));
  CK(dalloc(&h->gkey, kBigSlots * h->gcap));
  CK(dalloc(&h->gpos, kBigSlots * 2 * h->gcap));
  CK(dalloc(&h->gbits, kBigSlots * (h->gcap / 32 + 2)));
  CK(dalloc(&h->granges, kBigSlots * 3 * (h->gcap / 8 + 64)));
  h->bcap = B;
  return DD_OK;
}

SemisortScratch make_ss(dd_index* h) {
  SemisortScratch s;
  for (int i = 0; i < 2; i++) {
    s.t[i] = h->sort_t[i];
    s.v[i] = h->sort_v[i];
  }
  s.hist = h->hist;
  s.heads = h->heads;
  s.flags = h->flags;
  s.block_sums = h->block_sums;
  s.counters = h->counters;
  s.cap = h->bcap * h->Rp;
  return s;
}

// room for `words` uint32 of per-point visited lists
int ensure_vis_all(dd_index* h, uint64_t words) {
  if (words <= h->vis_all_words) return DD_OK;
  h->scratch_gen++;
  dfree(h->vis_all);
  h->vis_all = nullptr;
  h->vis_all_words = 0;
  CK(dalloc(&h->vis_all, words));
  h->vis_all_words = words;
  return DD_OK;
}

// Graph rows never hold an id twice during the build: the fast form's seen
// filter relies on it (search_core.cuh).  Reverse edges are appended without
// a membership check (include/utils/graph.h:84-93), so a row gets a repeat when
// the source is already in it: in the second pass of a two-pass build, and
// when the start point is inserted after points that linked to it (their
// searches start there), because its own reverse edges then reach rows that
// already name it.  A start point inserted first (point 0, the identity
// order's first) or never inserted (beyond max_build) cannot be in a row
// before its own insertion round.
bool rows_without_repeats(const dd_index* h, const dd_build_params* P) {
  if (P->two_pass) return false;
  const uint64_t m = (P->max_build && !P->knn_mode) ? std::min<uint64_t>(P->max_build, h->n) : h->n;
  const uint64_t start = P->knn_mode ? 0 : P->start_point;
  return start == 0 || start >= m;
}

// room for `words` work-queue counters
int ensure_queues(dd_index* h, uint64_t words) {
  if (words <= h->queue_words) return DD_OK;
  h->scratch_gen++;
  dfree(h->queues);
  h->queues = nullptr;
  h->queue_words = 0;
  CK(dalloc(&h->queues, words));
  h->queue_words = words;
  return DD_OK;
}

// ids fit the 24-bit hash table layout (DD_HASH32=1 at dd_create keeps the
// 32-bit layout, which larger indexes use, for testing it on small data)
bool use_h24(const dd_index* h) { return h->n < 0xFFFFFFull && !h->hash32; }

// the reverse-edge scratch of a handle; `res` = semisort result buffer
ReverseScratch make_rs(dd_index* h, int res) {
  ReverseScratch rs;
  rs.st = h->sort_t[res];
  rs.sv = h->sort_v[res];
  rs.heads = h->heads;
  rs.counters = h->counters;
  rs.big = h->big;
  rs.gcand = h->gcand;
  rs.gkey = h->gkey;
  rs.gpos = h->gpos;
  rs.gbits = h->gbits;
  rs.granges = h->granges;
  rs.gcap = h->gcap;
  return rs;
}

__global__ void k_accumulate(const uint32_t* stat_vis, const uint32_t* stat_cmps, uint32_t B,
                             const uint32_t* counters, unsigned long long* acc) {
  unsigned long long sv = 0, sc = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < B; i += gridDim.x * blockDim.x) {
    sv += stat_vis[i];
    sc += stat_cmps[i];
  }
  for (int o = 16; o > 0; o >>= 1) {
    sv += __shfl_down_sync(0xffffffffu, sv, o);
    sc += __shfl_down_sync(0xffffffffu, sc, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&acc[0], sv);
    atomicAdd(&acc[1], sc);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    atomicAdd(&acc[2], (unsigned long long)counters[1]);
    atomicAdd(&acc[3], (unsigned long long)counters[2]);
    atomicAdd(&acc[4], (unsigned long long)counters[3]);
    atomicAdd(&acc[5], (unsigned long long)counters[4]);
  }
}

// Per-round phase events (search+prune kernel, reverse-edge kernels), read once
// at the end of the build so the rounds run back to back without host syncs.
struct PhaseEvents {
  std::vector<cudaEvent_t> ev;
  size_t used = 0;
  cudaEvent_t next() {
    if (used == ev.size()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      ev.push_back(e);
    }
    return ev[used++];
  }
  // events per round: start | search done | prune done | reverse done
  void sum(float* t_search, float* t_prune, float* t_rev) {
    for (size_t i = 0; i + 3 < used; i += 4) {
      float a = 0, b = 0, c = 0;
      cudaEventElapsedTime(&a, ev[i], ev[i + 1]);
      cudaEventElapsedTime(&b, ev[i + 1], ev[i + 2]);
      cudaEventElapsedTime(&c, ev[i + 2], ev[i + 3]);
      *t_search += a;
      *t_prune += b;
      *t_rev += c;
    }
  }
  ~PhaseEvents() {
    for (auto e : ev) cudaEventDestroy(e);
  }
};

// The launch shapes of one build: search and prune layouts and CTA plans.
struct BuildPlan {
  WarpLayout slay;
  LaunchPlan splan;
  PruneLayout play;
  LaunchPlan pplan;
  bool fast;     // DD_MODE_FAST: tensor-core greedy of robustPrune (integer data)
  bool screen;   // fast form, float data: searches screen candidates on BF16 rows
  bool squeue;   // persistent k_search fed by the round's work queue
  bool pqueue;   // persistent k_prune fed by the round's work queue
};

// ---------------------------------------------------------------- autotuner
// The fast form's CTA shapes are picked by timing: at the first round of a
// build with at least kTuneItems points, k_search and k_prune are run on the
// round's first kTuneItems points with every candidate shape (2/4/8/16 warps
// per CTA, with and without the device work queue) and the fastest is kept
// for the rest of the build and for later builds of the same shape.  Both
// kernels only write scratch (visited lists, new out-lists) that the real
// launch of the round then rewrites, so the calibration does not change the
// build.  Results are cached per process, keyed by the shape.
constexpr uint32_t kTuneItems = 32768;

struct TuneResult {
  LaunchPlan splan, pplan;
  bool squeue = true, pqueue = true;
  float search_ms = 0.f, prune_ms = 0.f;  // calibration time of the chosen shapes
};

std::mutex g_tune_mu;
std::vector<std::pair<std::vector<uint64_t>, TuneResult>> g_tune;

std::vector<uint64_t> tune_key(const dd_index* h, const BuildPlan& bp, uint32_t L) {
  return {(uint64_t)h->dtype, (uint64_t)h->metric, h->d, h->Rp, L, bp.slay.vcap, bp.slay.h24,
          bp.slay.fastf, bp.slay.total, bp.play.total, (uint64_t)bp.fast, (uint64_t)bp.screen,
          (uint64_t)fast_fgroup(h), (uint64_t)h->device};
}

bool tune_lookup(const std::vector<uint64_t>& key, TuneResult* out) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  for (auto& e : g_tune)
    if (e.first == key) {
      *out = e.second;
      return true;
    }
  return false;
}

void tune_store(const std::vector<uint64_t>& key, const TuneResult& r) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  for (auto& e : g_tune)
    if (e.first == key) {
      e.second = r;
      return;
    }
  g_tune.push_back({key, r});
}

int grid_for(const LaunchPlan& pl, uint64_t B, int sm_count) {
  const uint64_t wpc = (uint64_t)pl.warps_per_cta;
  return (int)std::min<uint64_t>((B + wpc - 1) / wpc, (uint64_t)pl.blocks_per_sm * sm_count);
}

// Times k_search and then k_prune of round `ra` (its first kTuneItems points)
// for every candidate shape; the work-queue counter used is queues[0].
int tune_round(dd_index* h, RoundArgs ra, BuildPlan* bp, TuneResult* res) {
  IndexView ix = view(h);
  if (bp->screen) attach_screen(h, &ix);
  if (bp->fast) ix.fgroup_lg = fast_fgroup(h);
  ra.B = std::min<uint32_t>(ra.B, kTuneItems);
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  auto timed = [&](auto&& launch, float* ms) -> int {
    CK(cudaMemsetAsync(h->queues, 0, 4, h->stream));
    CK(cudaEventRecord(a, h->stream));
    launch();
    CK(cudaEventRecord(b, h->stream));
    CK(cudaEventSynchronize(b));
    CK(cudaGetLastError());
    CK(cudaEventElapsedTime(ms, a, b));
    return DD_OK;
  };
  float best = 1e30f;
  for (const LaunchPlan& pl : search_plan_candidates(ix, bp->slay, ra.L)) {
    for (int q = 0; q < 2; q++) {
      RoundArgs r2 = ra;
      r2.qsearch = q ? h->queues : nullptr;
      float ms = 0;
      int rc = timed([&] { launch_search(ix, r2, bp->slay, pl, grid_for(pl, r2.B, h->sm_count),
                                         h->stream); }, &ms);
      if (rc) return rc;
      if (ms < best) {
        best = ms;
        res->splan = pl;
        res->squeue = q != 0;
        res->search_ms = ms;
      }
    }
  }
  best = 1e30f;
  for (const LaunchPlan& pl : prune_plan_candidates(ix, bp->play, bp->fast)) {
    for (int q = 0; q < 2; q++) {
      RoundArgs r2 = ra;
      r2.qprune = q ? h->queues : nullptr;
      float ms = 0;
      int rc = timed([&] { launch_prune_round(ix, r2, bp->play, bp->slay.vcap, pl,
                                              grid_for(pl, r2.B, h->sm_count), bp->fast,
                                              h->stream); }, &ms);
      if (rc) return rc;
      if (ms < best) {
        best = ms;
        res->pplan = pl;
        res->pqueue = q != 0;
        res->prune_ms = ms;
      }
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  bp->splan = res->splan;
  bp->squeue = res->squeue;
  bp->pplan = res->pplan;
  bp->pqueue = res->pqueue;
  return DD_OK;
}

// One pass of batch insertions (src/bsp_index.hpp:238-407) as stream-ordered
// work with no host synchronization, so that a build can be captured in a
// CUDA graph.  Round r of this pass uses work-queue counters
// queues[qbase + 2r] (search) and [qbase + 2r + 1] (prune), zeroed by the
// caller.  With `tune` set, the first round large enough is calibrated first
// (tune_round), which synchronizes.
int pass_rounds(dd_index* h, const std::vector<std::pair<uint64_t, uint64_t>>& rounds, double alpha,
                const dd_build_params* P, BuildPlan& bp, uint64_t qbase, PhaseEvents* pe,
                TuneResult* tune) {
  IndexView ix = view(h);
  if (bp.screen) attach_screen(h, &ix);
  if (bp.fast) ix.fgroup_lg = fast_fgroup(h);
  for (size_t r = 0; r < rounds.size(); r++) {
    const auto& rd = rounds[r];
    uint64_t B = rd.second > rd.first ? rd.second - rd.first : 0;
    if (!B) continue;
    RoundArgs ra;
    ra.floor = rd.first;
    ra.B = (uint32_t)B;
    ra.L = P->L;
    ra.alpha = alpha;
    ra.start = P->start_point;
    ra.new_out = h->new_out;
    ra.new_key = bp.fast ? h->new_key : nullptr;
    ra.row_key = bp.fast ? h->row_key : nullptr;
    ra.stat_vis = h->stat_vis;
    ra.stat_cmps = h->stat_cmps;
    ra.vis_all = h->vis_all;
    ra.vis_sorted_tail = bp.slay.fastf ? 1 : 0;
    ra.qsearch = nullptr;
    ra.qprune = nullptr;
    if (tune && B >= kTuneItems) {
      int rc = tune_round(h, ra, &bp, tune);
      if (rc) return rc;
      tune = nullptr;
    }
    if (bp.fast && bp.squeue) ra.qsearch = h->queues + qbase + 2 * r;
    if (bp.fast && bp.pqueue) ra.qprune = h->queues + qbase + 2 * r + 1;
    CK(cudaMemsetAsync(h->counters, 0, 8 * 4, h->stream));
    if (pe) CK(cudaEventRecord(pe->next(), h->stream));
    launch_search(ix, ra, bp.slay, bp.splan, grid_for(bp.splan, B, h->sm_count), h->stream);
    if (pe) CK(cudaEventRecord(pe->next(), h->stream));
    launch_prune_round(ix, ra, bp.play, bp.slay.vcap, bp.pplan,
                       grid_for(bp.pplan, B, h->sm_count), bp.fast, h->stream);
    if (pe) CK(cudaEventRecord(pe->next(), h->stream));
    launch_apply_rows(ix, ra, h->stream);
    SemisortScratch ss = make_ss(h);
    const int res = launch_semisort(h->new_out, B * h->Rp, h->n, ss, h->stream);
    launch_reverse(ix, ra, make_rs(h, res), bp.fast, h->stream, h->sm_count);
    // k_search, k_prune, k_apply_rows, k_reverse, k_reverse_big; per radix
    // pass a histogram, three scans and a scatter; the segment heads' flags,
    // three scans and scatter
    h->launches += 10 + 5 * (uint64_t)((64 - __builtin_clzll(h->n > 1 ? h->n - 1 : 1) + 7) / 8);
    if (P->collect_stats) {
      k_accumulate<<<64, 256, 0, h->stream>>>(h->stat_vis, h->stat_cmps, (uint32_t)B, h->counters,
                                              h->acc);
      h->launches++;
    }
    if (pe) CK(cudaEventRecord(pe->next(), h->stream));
    CK(cudaGetLastError());
    if (h->verbose) {  // per-round diagnostics (DD_VERBOSE=1): synchronizes every round
      uint32_t c[8];
      CK(cudaMemcpyAsync(c, h->counters, sizeof c, cudaMemcpyDeviceToHost, h->stream));
      CK(cudaStreamSynchronize(h->stream));
      fprintf(stderr,
              "[dd] round [%llu, %llu) B=%llu pairs=%u targets=%u pruned=%u cands=%u big=%u "
              "max_big=%u\n",
              (unsigned long long)rd.first, (unsigned long long)rd.second, (unsigned long long)B,
              c[0], c[1], c[2], c[3], c[4], c[5]);
    }
  }
  return DD_OK;
}

// The whole device sequence of one build: reset, both passes, final sort.
int build_sequence(dd_index* h, const std::vector<std::pair<uint64_t, uint64_t>>& rounds,
                   const dd_build_params* Q, BuildPlan& bp, PhaseEvents* pe, TuneResult* tune) {
  // empty graph (the reference starts from Graph(R, n): all degrees 0)
  CK(cudaMemsetAsync(h->graph, 0xff, h->n * h->Rp * 4ull, h->stream));
  CK(cudaMemsetAsync(h->acc, 0, 8 * 8, h->stream));
  CK(cudaMemsetAsync(h->err, 0, 4, h->stream));
  if (bp.fast) CK(cudaMemsetAsync(h->queues, 0, h->queue_words * 4, h->stream));
  const uint64_t per_pass = 2 * rounds.size();
  int rc;
  if (Q->two_pass) {
    rc = pass_rounds(h, rounds, 1.0, Q, bp, 2, pe, tune);
    if (rc) return rc;
    tune = nullptr;
  }
  rc = pass_rounds(h, rounds, Q->alpha, Q, bp, 2 + (Q->two_pass ? per_pass : 0), pe, tune);
  if (rc) return rc;
  if (Q->knn_mode) {
    launch_sort_rows(view(h), h->stream);
    h->launches++;
  }
  return DD_OK;
}

}  // namespace

extern "C" {

int dd_create(int dtype, int metric, uint64_t n, uint32_t d, uint32_t R, int device,
              dd_index** out) {
  dd_index* h = nullptr;
  if (!out) return DD_ERR_ARG;
  *out = nullptr;
  if (dtype < 0 || dtype > 2 || metric < 0 || metric > 1) return DD_ERR_ARG;
  if (n == 0 || n >= 0x7fffffffull || d == 0 || R == 0) return DD_ERR_ARG;
  if (R > kMaxRp) return DD_ERR_UNSUPPORTED;
  if ((uint64_t)d * esize(dtype) > 1024) return DD_ERR_UNSUPPORTED;
  h = new dd_index();
  h->dtype = dtype;
  h->metric = metric;
  h->n = n;
  h->d = d;
  h->R = R;
  h->Rp = (R + 3) & ~3u;
  h->stride = ((uint64_t)d * esize(dtype) + 63) & ~(uint64_t)63;
  h->device = device;
  {
    const char* v = getenv("DD_VERBOSE");
    h->verbose = v && v[0] == '1';
    const char* w = getenv("DD_HASH32");
    h->hash32 = w && w[0] == '1';
  }
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = cudaMalloc((void**)&h->points, n * h->stride);
  if (e == cudaSuccess) e = cudaMalloc((void**)&h->graph, n * h->Rp * 4ull);
  if (e == cudaSuccess) e = cudaMalloc((void**)&h->err, 16);
  if (e == cudaSuccess) e = cudaMemset(h->points, 0, n * h->stride);
  if (e == cudaSuccess) e = cudaMemset(h->graph, 0xff, n * h->Rp * 4ull);
  if (e == cudaSuccess) e = cudaMemset(h->err, 0, 16);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    int code = e == cudaErrorMemoryAllocation ? DD_ERR_OOM : DD_ERR_CUDA;
    dd_destroy(h);
    return code;
  }
  *out = h;
  return DD_OK;
}

int dd_destroy(dd_index* h) {
  if (!h) return DD_OK;
  cudaSetDevice(h->device);
  void* ptrs[] = {h->points, h->graph, h->err, h->new_out, h->new_key, h->stat_vis, h->stat_cmps,
                  h->sort_t[0], h->sort_t[1], h->sort_v[0], h->sort_v[1], h->hist, h->heads,
                  h->flags, h->counters, h->big, h->block_sums, h->acc, h->gcand, h->gkey,
                  h->gpos, h->gbits, h->granges, h->vis_all, h->ref_rows, h->row_key,
                  h->screen, h->snorm};
  for (void* p : ptrs) dfree(p);
  dfree(h->queues);
  dfree(h->qcls);
  dfree(h->qhash);
  dfree(h->qev);
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  delete h;
  return DD_OK;
}

const char* dd_last_error(const dd_index* h) { return h ? h->last_error.c_str() : "null handle"; }

int dd_set_stream(dd_index* h, void* stream) {
  if (!h) return DD_ERR_ARG;
  h->stream = (cudaStream_t)stream;
  return DD_OK;
}

int dd_set_search_mode(dd_index* h, int mode) {
  if (!h) return DD_ERR_ARG;
  if (mode != DD_MODE_FAST && mode != DD_MODE_PLAIN)
    return fail(h, DD_ERR_ARG, "mode must be DD_MODE_FAST or DD_MODE_PLAIN");
  h->search_mode = mode;
  return DD_OK;
}

int dd_check_errors(dd_index* h) {
  if (!h) return DD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  return check_error_word(h);
}

int dd_upload_points(dd_index* h, const void* rows, uint64_t row_stride_bytes) {
  if (!h || !rows) return DD_ERR_ARG;
  h->screen_ok = false;  // the BF16 row copies follow the new points
  uint64_t rb = (uint64_t)h->d * esize(h->dtype);
  if (row_stride_bytes < rb) return fail(h, DD_ERR_ARG, "row stride %llu < row bytes %llu",
                                         (unsigned long long)row_stride_bytes, (unsigned long long)rb);
  CK(cudaSetDevice(h->device));
  CK(cudaMemcpy2DAsync(h->points, h->stride, rows, row_stride_bytes, rb, h->n,
                       cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return DD_OK;
}

int dd_upload_points_device(dd_index* h, const void* rows, uint64_t row_stride_bytes) {
  if (!h || !rows) return DD_ERR_ARG;
  h->screen_ok = false;  // the BF16 row copies follow the new points
  uint64_t rb = (uint64_t)h->d * esize(h->dtype);
  if (row_stride_bytes < rb) return fail(h, DD_ERR_ARG, "row stride too small");
  CK(cudaSetDevice(h->device));
  CK(cudaMemcpy2DAsync(h->points, h->stride, rows, row_stride_bytes, rb, h->n,
                       cudaMemcpyDeviceToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return DD_OK;
}

int dd_upload_points_async(dd_index* h, const void* rows, uint64_t row_stride_bytes) {
  if (!h || !rows) return DD_ERR_ARG;
  h->screen_ok = false;  // the BF16 row copies follow the new points
  uint64_t rb = (uint64_t)h->d * esize(h->dtype);
  if (row_stride_bytes < rb) return fail(h, DD_ERR_ARG, "row stride %llu < row bytes %llu",
                                         (unsigned long long)row_stride_bytes, (unsigned long long)rb);
  CK(cudaSetDevice(h->device));
  CK(cudaMemcpy2DAsync(h->points, h->stride, rows, row_stride_bytes, rb, h->n,
                       cudaMemcpyHostToDevice, h->stream));
  return DD_OK;
}

// PointRange(char*) (include/utils/point_range.h:61-97): the file is read in
// chunks into two pinned staging buffers; the upload of one chunk runs while
// the next one is read from disk.
int dd_load_points_file(dd_index* h, const char* path) {
  if (!h || !path) return DD_ERR_ARG;
  h->screen_ok = false;  // the BF16 row copies follow the new points
  std::ifstream f(path, std::ios::binary);
  if (!f) return fail(h, DD_ERR_IO, "cannot open %s", path);
  uint32_t hdr[2];
  f.read((char*)hdr, 8);
  if (!f || hdr[0] != h->n || hdr[1] != h->d)
    return fail(h, DD_ERR_IO, "%s: header [%u, %u] does not match the index", path, hdr[0], hdr[1]);
  CK(cudaSetDevice(h->device));
  const uint64_t rb = (uint64_t)h->d * esize(h->dtype);
  uint64_t chunk_bytes = 64ull << 20;  // DD_LOAD_CHUNK_BYTES overrides (tests use small chunks)
  if (const char* e = getenv("DD_LOAD_CHUNK_BYTES")) chunk_bytes = std::max<uint64_t>(rb, atoll(e));
  const uint64_t chunk_rows = std::max<uint64_t>(1, std::min<uint64_t>(h->n, chunk_bytes / rb));
  char* stage[2] = {nullptr, nullptr};
  cudaEvent_t done[2] = {nullptr, nullptr};
  int rc = DD_OK;
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < 2 && e == cudaSuccess; i++) {
    e = cudaMallocHost((void**)&stage[i], chunk_rows * rb);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming);
  }
  for (uint64_t r0 = 0, c = 0; e == cudaSuccess && rc == DD_OK && r0 < h->n; r0 += chunk_rows, c++) {
    const int b = (int)(c & 1);
    const uint64_t rows = std::min<uint64_t>(chunk_rows, h->n - r0);
    if (c >= 2) e = cudaEventSynchronize(done[b]);  // the upload that used this buffer ended
    if (e != cudaSuccess) break;
    f.read(stage[b], (std::streamsize)(rows * rb));
    if (!f) {
      rc = fail(h, DD_ERR_IO, "%s: truncated", path);
      break;
    }
    e = cudaMemcpy2DAsync(h->points + r0 * h->stride, h->stride, stage[b], rb, rb, rows,
                          cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaEventRecord(done[b], h->stream);
  }
  cudaError_t e2 = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess) e = e2;
  for (int i = 0; i < 2; i++) {
    if (stage[i]) cudaFreeHost(stage[i]);
    if (done[i]) cudaEventDestroy(done[i]);
  }
  if (rc) return rc;
  CK(e);
  return DD_OK;
}

int dd_upload_graph(dd_index* h, const uint32_t* rows) {
  if (!h || !rows) return DD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  uint32_t* tmp = nullptr;
  CK(dalloc(&tmp, h->n * (h->R + 1)));
  cudaError_t e = cudaMemcpyAsync(tmp, rows, h->n * (h->R + 1) * 4ull, cudaMemcpyHostToDevice,
                                  h->stream);
  if (e == cudaSuccess) {
    launch_from_ref_rows(view(h), tmp, h->stream);
    e = cudaStreamSynchronize(h->stream);
  }
  cudaFree(tmp);
  CK(e);
  return check_error_word(h);
}

int dd_download_graph(dd_index* h, uint32_t* rows) {
  if (!h || !rows) return DD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  // the reference-layout rows are assembled in a buffer kept by the handle
  if (!h->ref_rows) CK(dalloc(&h->ref_rows, h->n * (h->R + 1)));
  launch_to_ref_rows(view(h), h->ref_rows, h->stream);
  CK(cudaMemcpyAsync(rows, h->ref_rows, h->n * (h->R + 1) * 4ull, cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return DD_OK;
}

int dd_save_graph_file(dd_index* h, const char* path) {
  if (!h || !path) return DD_ERR_ARG;
  std::vector<uint32_t> g(h->n * (h->R + 1));
  int rc = dd_download_graph(h, g.data());
  if (rc) return rc;
  // include/utils/graph.h:178-200: [n][R][degrees][edges of each row]
  std::ofstream f(path, std::ios::binary);
  if (!f) return fail(h, DD_ERR_IO, "cannot open %s", path);
  uint32_t pre[2] = {(uint32_t)h->n, h->R};
  f.write((const char*)pre, 8);
  for (uint64_t i = 0; i < h->n; i++) f.write((const char*)&g[i * (h->R + 1)], 4);
  for (uint64_t i = 0; i < h->n; i++)
    f.write((const char*)&g[i * (h->R + 1) + 1], 4ull * g[i * (h->R + 1)]);
  if (!f) return fail(h, DD_ERR_IO, "write failed: %s", path);
  return DD_OK;
}

int dd_load_graph_file(dd_index* h, const char* path) {
  if (!h || !path) return DD_ERR_ARG;
  std::ifstream f(path, std::ios::binary);
  if (!f) return fail(h, DD_ERR_IO, "cannot open %s", path);
  uint32_t pre[2];
  f.read((char*)pre, 8);
  if (!f || pre[0] != h->n || pre[1] != h->R)
    return fail(h, DD_ERR_IO, "%s: [n, R] = [%u, %u] does not match the index", path, pre[0], pre[1]);
  std::vector<uint32_t> deg(h->n);
  f.read((char*)deg.data(), 4ll * h->n);
  std::vector<uint32_t> g(h->n * (h->R + 1), 0);
  for (uint64_t i = 0; i < h->n; i++) {
    if (deg[i] > h->R) return fail(h, DD_ERR_IO, "%s: row %llu degree %u > R", path,
                                   (unsigned long long)i, deg[i]);
    g[i * (h->R + 1)] = deg[i];
    f.read((char*)&g[i * (h->R + 1) + 1], 4ll * deg[i]);
  }
  if (!f) return fail(h, DD_ERR_IO, "%s: truncated", path);
  return dd_upload_graph(h, g.data());
}

int dd_schedule(uint64_t n, uint64_t max_build, double max_fraction, int knn_mode,
                uint64_t* floors, uint64_t* ceilings, uint64_t cap, uint64_t* nrounds) {
  auto r = schedule(n, max_build, max_fraction, knn_mode);
  for (size_t i = 0; i < r.size() && i < cap; i++) {
    floors[i] = r[i].first;
    ceilings[i] = r[i].second;
  }
  if (nrounds) *nrounds = r.size();
  return DD_OK;
}

}  // extern "C"

namespace {

// One build with visited-list capacity vcap; *err_bits = the device error word.
int build_once(dd_index* h, const dd_build_params* P, uint32_t vcap, dd_stats* stats,
               uint32_t* err_bits) {
  *err_bits = 0;
  uint32_t start = P->knn_mode ? 0 : P->start_point;  // include/index.h:127
  h->launches = 0;
  auto rounds = schedule(h->n, P->max_build, P->max_fraction, P->knn_mode);
  uint64_t Bmax = 1;
  for (auto& r : rounds) Bmax = std::max<uint64_t>(Bmax, r.second > r.first ? r.second - r.first : 0);
  int rc = ensure_build_scratch(h, Bmax);
  if (rc) return rc;
  BuildPlan bp;
  bp.fast = P->mode == DD_MODE_FAST;
  const bool fastf = bp.fast && use_h24(h) && rows_without_repeats(h, P);
  bp.slay = make_search_layout(h->d, h->dtype, P->L, h->Rp, vcap, true, use_h24(h), true, fastf);
  if (bp.slay.total > 227 * 1024)
    return fail(h, DD_ERR_UNSUPPORTED, "per-warp shared memory %u B too large (L=%u)",
                bp.slay.total, P->L);
  bp.play = make_prune_layout(h->d, h->dtype, h->Rp, bp.slay.ccap, bp.fast);
  if (bp.play.total > 227 * 1024)
    return fail(h, DD_ERR_UNSUPPORTED, "prune shared memory %u B too large (visited capacity %u)",
                bp.play.total, vcap);
  bp.splan = plan_search(view(h), bp.slay, P->L);
  bp.pplan = plan_prune(view(h), bp.play, bp.fast);
  bp.squeue = bp.pqueue = bp.fast;
  bp.screen = bp.fast && screen_enabled(h);
  if (bp.screen) {
    rc = ensure_screen(h);
    if (rc) return rc;
  }
  if (bp.fast && !h->row_key_ok) {
    // the fast form keeps every graph entry's distance to its row's point
    // beside the graph, so a reverse prune needs no distance of its row
    h->scratch_gen++;
    CK(dalloc(&h->row_key, h->n * (uint64_t)h->Rp));
    h->row_key_ok = true;
  }
  rc = ensure_vis_all(h, Bmax * 2ull * vcap);
  if (rc) return rc;
  rc = ensure_queues(h, 2 + 2 * rounds.size() * (P->two_pass ? 2 : 1));
  if (rc) return rc;

  // fast form: shapes from the autotuner's cache, or calibrated in this build
  TuneResult tuned;
  TuneResult* tune = nullptr;
  const std::vector<uint64_t> tkey = tune_key(h, bp, P->L);
  if (bp.fast) {
    if (tune_lookup(tkey, &tuned)) {
      bp.splan = tuned.splan;
      bp.squeue = tuned.squeue;
      bp.pplan = tuned.pplan;
      bp.pqueue = tuned.pqueue;
    } else if (Bmax >= kTuneItems) {
      tune = &tuned;
    }
  }
  dd_build_params Q = *P;
  Q.start_point = start;
  // A fast build with a settled shape and no statistics runs as one CUDA graph:
  // captured once on the handle's private stream, replayed on later builds.
  const bool use_graph = bp.fast && !tune && !P->collect_stats && !h->verbose;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  PhaseEvents pe;
  PhaseEvents* pep = stats && P->collect_stats ? &pe : nullptr;
  if (use_graph) {
    std::vector<uint64_t> key = tkey;
    uint64_t ab, mf;
    std::memcpy(&ab, &P->alpha, 8);
    std::memcpy(&mf, &P->max_fraction, 8);
    key.insert(key.end(), {ab, mf, P->max_build, start, (uint64_t)P->two_pass,
                           (uint64_t)P->knn_mode, h->scratch_gen,
                           (uint64_t)bp.splan.warps_per_cta, (uint64_t)bp.splan.blocks_per_sm,
                           (uint64_t)bp.pplan.warps_per_cta, (uint64_t)bp.pplan.blocks_per_sm,
                           (uint64_t)bp.squeue, (uint64_t)bp.pqueue});
    if (!h->gexec || h->graph_key != key) {
      if (h->gexec) {
        cudaGraphExecDestroy(h->gexec);
        h->gexec = nullptr;
      }
      if (!h->own_stream) CK(cudaStreamCreate(&h->own_stream));
      cudaStream_t user = h->stream;
      h->stream = h->own_stream;
      cudaGraph_t g = nullptr;
      CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeRelaxed));
      rc = build_sequence(h, rounds, &Q, bp, nullptr, nullptr);
      cudaError_t ce = cudaStreamEndCapture(h->stream, &g);
      h->stream = user;
      if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      CK(ce);
      cudaError_t ie = cudaGraphInstantiate(&h->gexec, g, 0);
      cudaGraphDestroy(g);
      if (ie != cudaSuccess) {
        h->gexec = nullptr;
        CK(ie);
      }
      h->graph_key = key;
      h->launches_per_graph = h->launches;
    }
    h->launches = h->launches_per_graph;
    cudaStream_t ls = h->stream ? h->stream : h->own_stream;
    CK(cudaEventRecord(e0, ls));
    CK(cudaGraphLaunch(h->gexec, ls));
    CK(cudaEventRecord(e1, ls));
  } else {
    CK(cudaEventRecord(e0, h->stream));
    rc = build_sequence(h, rounds, &Q, bp, pep, tune);
    if (rc) return rc;
    CK(cudaEventRecord(e1, h->stream));
    if (tune) tune_store(tkey, tuned);
  }
  CK(cudaEventSynchronize(e1));
  CK(cudaGetLastError());
  rc = check_error_word(h, err_bits);
  if (stats) {
    float ms = 0, ts = 0, tp = 0, tr = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    pe.sum(&ts, &tp, &tr);
    unsigned long long acc[8] = {0};
    cudaMemcpy(acc, h->acc, sizeof acc, cudaMemcpyDeviceToHost);
    std::memset(stats, 0, sizeof *stats);
    stats->rounds = rounds.size() * (P->two_pass ? 2 : 1);
    stats->visited = acc[0];
    stats->dist_cmps = acc[1];
    stats->groups = acc[2];
    stats->reverse_prunes = acc[3];
    stats->prune_cands = acc[4];
    stats->big_groups = acc[5];
    stats->build_ms = ms;
    stats->search_prune_ms = ts + tp;
    stats->reverse_ms = tr;
    stats->search_ms = ts;
    stats->search_warps_per_cta = (uint32_t)bp.splan.warps_per_cta;
    stats->prune_warps_per_cta = (uint32_t)bp.pplan.warps_per_cta;
    stats->search_queue = bp.fast && bp.squeue;
    stats->prune_queue = bp.fast && bp.pqueue;
    stats->graph_replay = use_graph;
    stats->vcap = vcap;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

}  // namespace

extern "C" {

int dd_build(dd_index* h, const dd_build_params* P, dd_stats* stats) {
  if (!h || !P) return DD_ERR_ARG;
  if (P->L == 0 || P->L > kMaxL) return fail(h, DD_ERR_UNSUPPORTED, "L must be in [1, %u]", kMaxL);
  uint32_t start = P->knn_mode ? 0 : P->start_point;  // include/index.h:127
  if (start >= h->n) return fail(h, DD_ERR_ARG, "start point %u >= n", start);
  if (!(P->alpha > 0)) return fail(h, DD_ERR_ARG, "alpha must be positive");
  if (P->mode != DD_MODE_FAST && P->mode != DD_MODE_PLAIN)
    return fail(h, DD_ERR_ARG, "mode must be DD_MODE_FAST or DD_MODE_PLAIN");
  CK(cudaSetDevice(h->device));
  // The reference's build searches have no visited-list limit (limit = n).
  // Here each search keeps its visited list in a slice of vcap entries; when a
  // search overflows it (the kernel flags it and the round goes on), the
  // whole build is run again with twice the capacity, which gives the same
  // graph (the build is deterministic), until the prune's shared memory for
  // vcap + R candidates runs out.
  uint32_t vcap = P->vcap ? P->vcap : 4 * P->L;
  for (;;) {
    uint32_t bits = 0;
    int rc = build_once(h, P, vcap, stats, &bits);
    if (rc == DD_ERR_DEVICE && bits == DD_EVIS_CAP && vcap < (1u << 20)) {
      const uint32_t next = vcap * 2;
      if (make_prune_layout(h->d, h->dtype, h->Rp, next + h->Rp, P->mode == DD_MODE_FAST).total >
          227 * 1024)
        return rc;
      vcap = next;
      continue;
    }
    return rc;
  }
}

// ---------------------------------------------------------------- sharded build
// One rank's share of each round of a build spread over P ranks, one GPU each,
// every rank holding the whole graph (src/bsp_index.hpp:141-434): the batch is
// split into P contiguous slices (:247-252) that the ranks search and prune;
// the new rows are exchanged; each rank runs the reverse edges of the targets
// it owns (t % P == rank, :362-373) and the changed rows are exchanged again.
// Each step gives the same rows as the single-GPU build, so the sharded build
// gives its graph.  The exchanges are the caller's (NCCL all-gathers).

namespace {
BuildPlan shard_plan(dd_index* h) {
  const dd_build_params* P = &h->shard_params;
  const uint32_t vcap = P->vcap ? P->vcap : 8 * P->L;
  BuildPlan bp;
  bp.fast = P->mode == DD_MODE_FAST;
  const bool fastf = bp.fast && use_h24(h) && rows_without_repeats(h, P);
  bp.slay = make_search_layout(h->d, h->dtype, P->L, h->Rp, vcap, true, use_h24(h), true, fastf);
  bp.play = make_prune_layout(h->d, h->dtype, h->Rp, bp.slay.ccap, bp.fast);
  bp.splan = plan_search(view(h), bp.slay, P->L);
  bp.pplan = plan_prune(view(h), bp.play, bp.fast);
  bp.squeue = bp.pqueue = bp.fast;
  bp.screen = bp.fast && screen_enabled(h);
  return bp;
}

RoundArgs shard_round_args(dd_index* h, uint64_t floor, uint64_t B, uint32_t* rows) {
  RoundArgs ra;
  ra.floor = floor;
  ra.B = (uint32_t)B;
  ra.L = h->shard_params.L;
  ra.alpha = h->shard_params.alpha;
  ra.start = h->shard_params.start_point;
  ra.new_out = rows;
  ra.new_key = nullptr;  // the exchanged rows carry no distances: the reverse step recomputes
  ra.row_key = nullptr;
  ra.stat_vis = h->stat_vis;
  ra.stat_cmps = h->stat_cmps;
  ra.vis_all = h->vis_all;
  ra.vis_sorted_tail = shard_plan(h).slay.fastf ? 1 : 0;
  ra.qsearch = nullptr;
  ra.qprune = nullptr;
  return ra;
}
}  // namespace

int dd_shard_begin(dd_index* h, const dd_build_params* P, uint64_t max_batch) {
  if (!h || !P) return DD_ERR_ARG;
  if (P->L == 0 || P->L > kMaxL) return fail(h, DD_ERR_UNSUPPORTED, "L must be in [1, %u]", kMaxL);
  if (P->two_pass || P->knn_mode)
    return fail(h, DD_ERR_UNSUPPORTED, "the sharded build is the single-pass BSP build");
  if (P->start_point >= h->n) return fail(h, DD_ERR_ARG, "start point >= n");
  if (!(P->alpha > 0)) return fail(h, DD_ERR_ARG, "alpha must be positive");
  if (P->mode != DD_MODE_FAST && P->mode != DD_MODE_PLAIN)
    return fail(h, DD_ERR_ARG, "mode must be DD_MODE_FAST or DD_MODE_PLAIN");
  if (max_batch == 0 || max_batch > h->n) return fail(h, DD_ERR_ARG, "bad max_batch");
  CK(cudaSetDevice(h->device));
  h->shard_params = *P;
  h->shard_bmax = max_batch;
  int rc = ensure_build_scratch(h, max_batch);
  if (rc) return rc;
  BuildPlan bp = shard_plan(h);
  if (bp.slay.total > 227 * 1024 || bp.play.total > 227 * 1024)
    return fail(h, DD_ERR_UNSUPPORTED, "shared memory of L=%u too large", P->L);
  rc = ensure_vis_all(h, max_batch * 2ull * bp.slay.vcap);
  if (rc) return rc;
  rc = ensure_queues(h, 2);
  if (rc) return rc;
  if (bp.screen) {
    rc = ensure_screen(h);
    if (rc) return rc;
  }
  CK(cudaMemsetAsync(h->graph, 0xff, h->n * h->Rp * 4ull, h->stream));
  CK(cudaMemsetAsync(h->err, 0, 4, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->shard_ready = true;
  return DD_OK;
}

int dd_shard_search_prune(dd_index* h, uint64_t lo, uint64_t hi, uint32_t* rows) {
  if (!h) return DD_ERR_ARG;
  if (hi == lo) return DD_OK;  // an empty slice (batches smaller than the ranks)
  if (!rows) return fail(h, DD_ERR_ARG, "rows is null");
  if (!h->shard_ready) return fail(h, DD_ERR_ARG, "dd_shard_begin first");
  if (hi < lo || hi > h->n || hi - lo > h->shard_bmax) return fail(h, DD_ERR_ARG, "bad slice");
  if (hi == lo) return DD_OK;
  CK(cudaSetDevice(h->device));
  BuildPlan bp = shard_plan(h);
  RoundArgs ra = shard_round_args(h, lo, hi - lo, rows);
  if (bp.fast) {
    CK(cudaMemsetAsync(h->queues, 0, 8, h->stream));
    ra.qsearch = h->queues;
    ra.qprune = h->queues + 1;
  }
  IndexView ix = view(h);
  if (bp.screen) {
    int rc = ensure_screen(h);
    if (rc) return rc;
    attach_screen(h, &ix);
  }
  if (bp.fast) ix.fgroup_lg = fast_fgroup(h);
  launch_search(ix, ra, bp.slay, bp.splan, grid_for(bp.splan, ra.B, h->sm_count), h->stream);
  launch_prune_round(ix, ra, bp.play, bp.slay.vcap, bp.pplan, grid_for(bp.pplan, ra.B, h->sm_count),
                     bp.fast, h->stream);
  CK(cudaGetLastError());
  return check_error_word(h);
}

int dd_shard_apply_reverse(dd_index* h, uint64_t floor, uint64_t ceiling, const uint32_t* batch_rows,
                           int rank, int world, uint32_t* ids_out, uint32_t* rows_out,
                           uint64_t cap, uint64_t* count) {
  if (!h || !batch_rows || !ids_out || !rows_out || !count) return DD_ERR_ARG;
  if (!h->shard_ready) return fail(h, DD_ERR_ARG, "dd_shard_begin first");
  if (world < 1 || rank < 0 || rank >= world) return fail(h, DD_ERR_ARG, "bad rank / world");
  if (ceiling < floor || ceiling > h->n || ceiling - floor > h->shard_bmax)
    return fail(h, DD_ERR_ARG, "bad round");
  *count = 0;
  if (ceiling == floor) return DD_OK;
  CK(cudaSetDevice(h->device));
  BuildPlan bp = shard_plan(h);
  const uint64_t B = ceiling - floor;
  RoundArgs ra = shard_round_args(h, floor, B, const_cast<uint32_t*>(batch_rows));
  IndexView ix = view(h);
  CK(cudaMemsetAsync(h->counters, 0, 8 * 4, h->stream));
  launch_apply_rows(ix, ra, h->stream);
  SemisortScratch ss = make_ss(h);
  ss.world = (uint32_t)world;
  ss.rank = (uint32_t)rank;
  const int res = launch_semisort(batch_rows, B * h->Rp, h->n, ss, h->stream);
  ReverseScratch rs = make_rs(h, res);
  launch_reverse(ix, ra, rs, bp.fast, h->stream, h->sm_count);
  launch_export_rows(ix, rs.st, rs.heads, h->counters, cap, ids_out, rows_out, h->stream);
  CK(cudaGetLastError());
  uint32_t c[2] = {0, 0};
  CK(cudaMemcpyAsync(c, h->counters, 8, cudaMemcpyDeviceToHost, h->stream));
  int rc = check_error_word(h);  // synchronizes
  if (rc) return rc;
  *count = c[1];
  if (c[1] > cap) return fail(h, DD_ERR_ARG, "%u changed rows exceed the capacity %llu", c[1],
                              (unsigned long long)cap);
  return DD_OK;
}

int dd_shard_set_rows(dd_index* h, const uint32_t* ids, const uint32_t* rows, uint64_t count) {
  if (!h || (count && (!ids || !rows))) return DD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  launch_set_rows(view(h), ids, rows, count, h->stream);
  CK(cudaGetLastError());
  return check_error_word(h);
}

int dd_search_device(dd_index* h, const void* queries, uint64_t nq, uint64_t qstride,
                     const uint32_t* L_per_query, uint32_t Lmax, uint32_t k, double cut,
                     uint64_t limit, uint32_t degree_limit, uint32_t start, int skip_self,
                     uint32_t* ids, float* dists, uint32_t* visited, uint32_t* cmps) {
  if (!h || !queries || !L_per_query || !ids || !dists) return DD_ERR_ARG;
  if (nq == 0) return DD_OK;
  if (Lmax == 0 || Lmax > kMaxL) return fail(h, DD_ERR_UNSUPPORTED, "L must be in [1, %u]", kMaxL);
  if (k == 0 || k > Lmax) return fail(h, DD_ERR_ARG, "k must be in [1, L]");  // beamSearch.h:327-331
  if (start >= h->n) return fail(h, DD_ERR_ARG, "start point >= n");
  if (qstride % 16) return fail(h, DD_ERR_ARG, "device query stride must be a multiple of 16");
  CK(cudaSetDevice(h->device));
  h->launches = 0;
  WarpLayout lay = make_search_layout(h->d, h->dtype, Lmax, h->Rp, 2 * Lmax + 64, false,
                                      use_h24(h), false);
  if ((size_t)lay.total > 227 * 1024)
    return fail(h, DD_ERR_UNSUPPORTED, "query shared memory %u B too large", lay.total);
  QueryArgs qa;
  qa.queries = (const uint8_t*)queries;
  qa.qstride = qstride;
  qa.nq = nq;
  qa.Ls = L_per_query;
  qa.Lmax = Lmax;
  qa.k = k;
  qa.cut = cut;
  qa.limit = limit ? limit : h->n;
  qa.degree_limit = degree_limit ? std::min(degree_limit, h->R) : h->R;
  qa.start = start;
  qa.skip_self = skip_self;
  qa.ids = ids;
  qa.dists = dists;
  qa.visited = visited;
  qa.cmps = cmps;
  qa.cls_items = nullptr;
  qa.cls_count = nullptr;
  qa.cls_queue = nullptr;
  qa.Lvalid = Lmax;
  qa.hash_scratch = nullptr;
  // Evicted lists (visited entries pushed out of the frontier, which a query
  // must still treat as visited if they come back after a k-cut) live in a
  // global slice per resident warp.  Their length is bounded by the visits
  // of the search; ev_cap covers far more than any search here makes, and an
  // overflow is reported through the error word (dd_check_errors).
  qa.ev_cap = 4096 + 8 * Lmax;
  auto ev_slices = [&](uint64_t warps) -> int {
    const uint64_t words = warps * qa.ev_cap;
    if (words > h->qev_words) {
      dfree(h->qev);
      h->qev = nullptr;
      h->qev_words = 0;
      CK(dalloc(&h->qev, words));
      h->qev_words = words;
    }
    qa.ev_scratch = h->qev;
    return DD_OK;
  };
  if (h->search_mode == DD_MODE_PLAIN) {
    // one launch laid out for the largest beam width
    const LaunchPlan plan = plan_query(view(h), lay, Lmax);
    const int wpc = plan.warps_per_cta;
    const int grid = (int)std::min<uint64_t>((nq + wpc - 1) / wpc,
                                             (uint64_t)plan.blocks_per_sm * h->sm_count);
    int rc = ev_slices((uint64_t)grid * wpc);
    if (rc) return rc;
    launch_query(view(h), qa, lay, wpc, grid, h->stream);
    h->launches = 1;
    CK(cudaGetLastError());
    return DD_OK;
  }
  // fast form: the queries are listed by beam-width class on the device, then
  // each class runs as a persistent launch laid out for its own beam width
  // (smaller hash table and frontier: more resident queries per SM), largest
  // class first; classes without queries end at once
  const uint64_t words = (uint64_t)kQueryClasses * nq + 2 * kQueryClasses;
  if (words > h->qcls_words) {
    dfree(h->qcls);
    h->qcls = nullptr;
    h->qcls_words = 0;
    CK(dalloc(&h->qcls, words));
    h->qcls_words = words;
  }
  uint32_t* counts = h->qcls + (uint64_t)kQueryClasses * nq;
  uint32_t* queues = counts + kQueryClasses;
  IndexView ixq = view(h);
  if (screen_enabled(h)) {  // float data: BF16 screen, exact re-rank
    int rc = ensure_screen(h);
    if (rc) return rc;
    attach_screen(h, &ixq);
  }
  ixq.fgroup_lg = fast_fgroup(h);
  CK(cudaMemsetAsync(counts, 0, 2 * kQueryClasses * 4, h->stream));
  launch_bin_queries(L_per_query, nq, k, Lmax, h->qcls, counts, h->stream);
  h->launches = 1;
  for (int c = query_class(Lmax); c >= 0; c--) {
    if ((16u << c) < k && c < query_class(Lmax)) break;  // no valid beam width below k
    const uint32_t Lc = std::min<uint32_t>(16u << c, Lmax);
    // seen tables above 16 KB (beam widths above 128) would cap the resident
    // queries per SM by shared memory: they go to one global slice per warp
    const bool hglob = hash_table_bytes(hash_bits_for(Lc), use_h24(h)) > 16384;
    WarpLayout lc = make_search_layout(h->d, h->dtype, Lc, h->Rp, 2 * Lc + 64, false,
                                       use_h24(h), false, false, hglob);
    const LaunchPlan plan = plan_query(view(h), lc, Lc);
    QueryArgs qc = qa;
    qc.Lmax = Lc;
    qc.cls_items = h->qcls + (uint64_t)c * nq;
    qc.cls_count = counts + c;
    qc.cls_queue = queues + c;
    const int wpc = plan.warps_per_cta;
    const int grid = (int)std::min<uint64_t>((nq + wpc - 1) / wpc,
                                             (uint64_t)plan.blocks_per_sm * h->sm_count);
    int rc = ev_slices((uint64_t)grid * wpc);
    if (rc) return rc;
    qc.ev_scratch = qa.ev_scratch;
    if (hglob) {
      const uint64_t words = (uint64_t)grid * wpc * lc.hash_words;
      if (words > h->qhash_words) {
        dfree(h->qhash);
        h->qhash = nullptr;
        h->qhash_words = 0;
        CK(dalloc(&h->qhash, words));
        h->qhash_words = words;
      }
      qc.hash_scratch = h->qhash;
    }
    launch_query(ixq, qc, lc, wpc, grid, h->stream);
    h->launches++;
  }
  CK(cudaGetLastError());
  return DD_OK;
}

int dd_search(dd_index* h, const void* queries, uint64_t nq, uint64_t qstride,
              const uint32_t* L_per_query, uint32_t k, double cut, uint64_t limit,
              uint32_t degree_limit, uint32_t start, int skip_self, uint32_t* ids, float* dists,
              uint32_t* visited, uint32_t* cmps) {
  if (!h || !queries || !L_per_query || !ids || !dists) return DD_ERR_ARG;
  if (nq == 0) return DD_OK;
  CK(cudaSetDevice(h->device));
  uint64_t rb = (uint64_t)h->d * esize(h->dtype);
  uint64_t ds = h->stride;
  uint32_t Lmax = 0;
  for (uint64_t i = 0; i < nq; i++) Lmax = std::max(Lmax, L_per_query[i]);
  uint8_t* dq = nullptr;
  uint32_t *dL = nullptr, *di = nullptr, *dv = nullptr, *dc = nullptr;
  float* dd = nullptr;
  CK(dalloc(&dq, nq * ds));
  int rc = DD_OK;
  cudaError_t e = dalloc(&dL, nq);
  if (e == cudaSuccess) e = dalloc(&di, nq * k);
  if (e == cudaSuccess) e = dalloc(&dd, nq * k);
  if (e == cudaSuccess) e = dalloc(&dv, nq);
  if (e == cudaSuccess) e = dalloc(&dc, nq);
  if (e == cudaSuccess) e = cudaMemsetAsync(dq, 0, nq * ds, h->stream);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(dq, ds, queries, qstride, rb, nq, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dL, L_per_query, nq * 4, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) {
    rc = dd_search_device(h, dq, nq, ds, dL, Lmax, k, cut, limit, degree_limit, start, skip_self,
                          di, dd, dv, dc);
    if (rc == DD_OK) {
      e = cudaMemcpyAsync(ids, di, nq * k * 4, cudaMemcpyDeviceToHost, h->stream);
      if (e == cudaSuccess) e = cudaMemcpyAsync(dists, dd, nq * k * 4, cudaMemcpyDeviceToHost, h->stream);
      if (e == cudaSuccess && visited) e = cudaMemcpyAsync(visited, dv, nq * 4, cudaMemcpyDeviceToHost, h->stream);
      if (e == cudaSuccess && cmps) e = cudaMemcpyAsync(cmps, dc, nq * 4, cudaMemcpyDeviceToHost, h->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    }
  }
  cudaFree(dq); cudaFree(dL); cudaFree(di); cudaFree(dd); cudaFree(dv); cudaFree(dc);
  if (rc) return rc;
  CK(e);
  return check_error_word(h);
}

int dd_beam_search(dd_index* h, const void* queries, uint64_t nq, uint64_t qstride,
                   const int64_t* self_ids, uint32_t L, uint32_t k, double cut, uint64_t limit,
                   uint32_t degree_limit, uint32_t start, uint32_t vcap, uint32_t* fr_ids,
                   float* fr_dists, uint32_t* fr_sizes, uint32_t* vis_ids, float* vis_dists,
                   uint32_t* vis_sizes, uint32_t* cmps) {
  if (!h || !queries || !self_ids || nq == 0) return DD_ERR_ARG;
  if (L == 0 || L > kMaxL) return fail(h, DD_ERR_UNSUPPORTED, "L must be in [1, %u]", kMaxL);
  if (start >= h->n) return fail(h, DD_ERR_ARG, "start point >= n");
  CK(cudaSetDevice(h->device));
  uint64_t rb = (uint64_t)h->d * esize(h->dtype), ds = h->stride;
  WarpLayout lay = make_search_layout(h->d, h->dtype, L, h->Rp, vcap, false, use_h24(h));
  if (lay.total > 227 * 1024) return fail(h, DD_ERR_UNSUPPORTED, "beam shared memory too large");
  const int bgrid = (int)std::min<uint64_t>(nq, 4096);
  uint8_t* dq = nullptr;
  int64_t* dself = nullptr;
  uint32_t *dfi = nullptr, *dfn = nullptr, *dvi = nullptr, *dvn = nullptr, *dcm = nullptr;
  float *dfd = nullptr, *dvd = nullptr;
  cudaError_t e = dalloc(&dq, nq * ds);
  if (e == cudaSuccess) e = dalloc(&dself, nq);
  if (e == cudaSuccess) e = dalloc(&dfi, nq * L);
  if (e == cudaSuccess) e = dalloc(&dfd, nq * L);
  if (e == cudaSuccess) e = dalloc(&dfn, nq);
  if (e == cudaSuccess) e = dalloc(&dvi, nq * vcap);
  if (e == cudaSuccess) e = dalloc(&dvd, nq * vcap);
  if (e == cudaSuccess) e = dalloc(&dvn, nq);
  if (e == cudaSuccess) e = dalloc(&dcm, nq);
  if (e == cudaSuccess) e = cudaMemsetAsync(dq, 0, nq * ds, h->stream);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(dq, ds, queries, qstride, rb, nq, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dself, self_ids, nq * 8, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) {
    BeamArgs ba;
    ba.queries = dq; ba.qstride = ds; ba.nq = nq; ba.self_ids = dself; ba.L = L; ba.k = k;
    ba.cut = cut; ba.limit = limit ? limit : h->n;
    ba.degree_limit = degree_limit ? std::min(degree_limit, h->R) : h->R;
    ba.start = start; ba.vcap = vcap;
    ba.fr_ids = dfi; ba.fr_d = dfd; ba.fr_n = dfn; ba.vis_ids = dvi; ba.vis_d = dvd;
    ba.vis_n = dvn; ba.cmps = dcm;
    launch_beam(view(h), ba, lay, bgrid, h->stream);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(fr_ids, dfi, nq * L * 4, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(fr_dists, dfd, nq * L * 4, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(fr_sizes, dfn, nq * 4, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(vis_ids, dvi, nq * vcap * 4, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(vis_dists, dvd, nq * vcap * 4, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(vis_sizes, dvn, nq * 4, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(cmps, dcm, nq * 4, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  void* fr[] = {dq, dself, dfi, dfd, dfn, dvi, dvd, dvn, dcm};
  for (void* p : fr) dfree(p);
  CK(e);
  return check_error_word(h);
}

int dd_robust_prune(dd_index* h, uint32_t ntasks, const uint32_t* p, const uint64_t* offsets,
                    const uint32_t* cand_ids, const float* cand_dists, double alpha,
                    uint32_t* out, uint32_t* out_len) {
  if (!h || !p || !offsets || !out || !out_len) return DD_ERR_ARG;
  if (ntasks == 0) return DD_OK;
  for (uint32_t t = 0; t < ntasks; t++)
    if (p[t] >= h->n || offsets[t + 1] < offsets[t]) return fail(h, DD_ERR_ARG, "bad task %u", t);
  for (uint64_t i = 0; i < offsets[ntasks]; i++)
    if (cand_ids[i] >= h->n) return fail(h, DD_ERR_ARG, "candidate id %u >= n", cand_ids[i]);
  CK(cudaSetDevice(h->device));
  uint64_t tot = offsets[ntasks];
  uint64_t ws = tot + (uint64_t)ntasks * h->Rp;
  uint32_t *dp = nullptr, *dci = nullptr, *dout = nullptr, *gc = nullptr;
  uint64_t* doff = nullptr;
  float *dcd = nullptr, *gk = nullptr;
  int* gl = nullptr;
  cudaError_t e = dalloc(&dp, ntasks);
  if (e == cudaSuccess) e = dalloc(&doff, ntasks + 1);
  if (e == cudaSuccess) e = dalloc(&dci, tot);
  if (e == cudaSuccess) e = dalloc(&dcd, tot);
  if (e == cudaSuccess) e = dalloc(&dout, (uint64_t)ntasks * h->Rp);
  if (e == cudaSuccess) e = dalloc(&gc, ws);
  if (e == cudaSuccess) e = dalloc(&gk, ws);
  if (e == cudaSuccess) e = dalloc(&gl, 3 * ws + (uint64_t)ntasks * kGlobalStackInts);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dp, p, ntasks * 4, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(doff, offsets, (ntasks + 1) * 8ull, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess && tot) e = cudaMemcpyAsync(dci, cand_ids, tot * 4, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess && tot) e = cudaMemcpyAsync(dcd, cand_dists, tot * 4, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) {
    PruneArgs pa;
    pa.ntasks = ntasks; pa.p = dp; pa.offsets = doff; pa.cand_ids = dci; pa.cand_d = dcd;
    pa.alpha = alpha; pa.out = dout; pa.gcand = gc; pa.gkey = gk; pa.gws = gl;
    launch_prune_tasks(view(h), pa, h->stream);
    e = cudaGetLastError();
  }
  std::vector<uint32_t> o((uint64_t)ntasks * h->Rp);
  if (e == cudaSuccess) e = cudaMemcpyAsync(o.data(), dout, o.size() * 4, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  void* fr[] = {dp, doff, dci, dcd, dout, gc, gk, gl};
  for (void* q : fr) dfree(q);
  CK(e);
  for (uint32_t t = 0; t < ntasks; t++) {
    uint32_t len = 0;
    while (len < h->R && o[(uint64_t)t * h->Rp + len] != DD_NONE) len++;
    out_len[t] = len;
    for (uint32_t j = 0; j < h->R; j++) out[(uint64_t)t * h->R + j] = j < len ? o[(uint64_t)t * h->Rp + j] : 0u;
  }
  return check_error_word(h);
}

int dd_groundtruth(dd_index* h, const void* queries, uint64_t nq, uint64_t qstride, uint32_t k,
                   uint32_t* ids, float* dists) {
  if (!h || !queries || !ids || !dists) return DD_ERR_ARG;
  if (k == 0 || k > 32 || k > h->n) return fail(h, DD_ERR_UNSUPPORTED, "k must be in [1, 32]");
  if (nq == 0) return DD_OK;
  CK(cudaSetDevice(h->device));
  uint64_t rb = (uint64_t)h->d * esize(h->dtype), ds = h->stride;
  uint32_t nchunks = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(256, h->n / 4096));
  uint8_t* dq = nullptr;
  uint32_t *di = nullptr, *pi = nullptr;
  float* dd = nullptr;
  double* pd = nullptr;
  cudaError_t e = dalloc(&dq, nq * ds);
  if (e == cudaSuccess) e = dalloc(&di, nq * k);
  if (e == cudaSuccess) e = dalloc(&dd, nq * k);
  if (e == cudaSuccess) e = dalloc(&pi, nq * nchunks * k);
  if (e == cudaSuccess) e = dalloc(&pd, nq * nchunks * k);
  if (e == cudaSuccess) e = cudaMemsetAsync(dq, 0, nq * ds, h->stream);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(dq, ds, queries, qstride, rb, nq, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) {
    launch_groundtruth(view(h), dq, ds, nq, k, di, dd, pd, pi, nchunks, h->stream);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(ids, di, nq * k * 4, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dists, dd, nq * k * 4, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  void* fr[] = {dq, di, dd, pi, pd};
  for (void* q : fr) dfree(q);
  CK(e);
  return DD_OK;
}

// the caller may write the points through this pointer: the BF16 row copies
// of the fast float search are rebuilt before their next use
void* dd_device_points(dd_index* h) {
  if (!h) return nullptr;
  h->screen_ok = false;
  return h->points;
}
uint64_t dd_device_row_stride(dd_index* h) { return h ? h->stride : 0; }
void* dd_device_graph(dd_index* h) { return h ? h->graph : nullptr; }
uint32_t dd_device_row_len(dd_index* h) { return h ? h->Rp : 0; }
uint64_t dd_last_launch_count(dd_index* h) { return h ? h->launches : 0; }

}  // extern "C"

// ---- accessors for the other translation units of the library (internal.h)
namespace ddk {
IndexView internal_view(dd_index* h) { return view(h); }
cudaStream_t internal_stream(dd_index* h) { return h->stream; }
int internal_device(dd_index* h) { return h->device; }
int internal_fail(dd_index* h, int code, const char* msg) { return fail(h, code, "%s", msg); }
int internal_check_error_word(dd_index* h) { return check_error_word(h); }
}  // namespace ddk
