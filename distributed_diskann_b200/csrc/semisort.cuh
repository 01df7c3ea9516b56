// Stable grouping of the round's reverse edges by target (the reference's
// flatten + parlay::group_by_key, src/bsp_index.hpp:362-376): a stable LSD
// radix sort of (target, key) pairs, key = b*Rp + j (batch position b, slot j),
// followed by a compaction of the segment heads.  Stability keeps every
// target's sources in batch order, which is the order group_by_key keeps.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace ddk {

constexpr uint32_t kRadixThreads = 256;
constexpr uint32_t kRadixItems = 16;                      // items per thread per tile
constexpr uint32_t kRadixTile = kRadixThreads * kRadixItems;

struct SemisortScratch {
  uint32_t* t[2];      // targets (ping-pong), capacity E
  uint32_t* v[2];      // keys
  uint32_t* hist;      // 256 x tiles
  uint32_t* heads;     // segment starts (capacity E)
  uint32_t* flags;     // capacity E
  uint32_t* block_sums;
  uint32_t* counters;  // [0] valid pairs V, [1] segments T
  uint64_t cap;        // E
  // owner filter of a sharded build: only targets t with t % world == rank
  // are kept (world = 1: every target)
  uint32_t world = 1, rank = 0;
};

// Sorts the valid entries of new_out (E = B*Rp, DD_NONE = empty slot) by
// target; on return the pairs are in t[res], v[res] (res returned), counters[0]
// = V, counters[1] = T and heads[0, T) the segment starts (ascending).
int launch_semisort(const uint32_t* new_out, uint64_t E, uint64_t n, SemisortScratch& s,
                    cudaStream_t st);

uint64_t semisort_hist_words(uint64_t E);

}  // namespace ddk
