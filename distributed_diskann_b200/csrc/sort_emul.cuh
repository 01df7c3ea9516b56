// Exact emulation of the element order produced by libstdc++'s std::sort
// (introsort) with the distance-only comparator robustPrune uses
// (include/index.h:78-79; src/bsp_index.hpp:499-500).  That comparator leaves
// ties unresolved, and introsort is not stable, so the neighbour lists the
// reference builds depend on the exact permutation its std::sort produces
// (g++ 13 libstdc++: introsort with depth limit 2*floor(log2 n), threshold 16,
// median-of-three pivot moved to the front, unguarded Hoare partition,
// heapsort when the depth limit runs out, then a final insertion sort).
//
// The emulation is split in two:
//   1. partition phase: replays the introsort recursion, moving elements
//      exactly as the library does, and records the leaf ranges it stops at
//      (ranges of <= 16 elements, or heap-sorted ranges);
//   2. leaf phase: the library's final insertion sort never moves an element
//      across a leaf boundary (every element of a leaf is <= every element of
//      any later leaf), and insertion sort is stable, so it equals a stable
//      insertion sort inside each leaf.  Leaves are independent and can be
//      finished in parallel.
// Elements are (id, key) pairs held in two parallel arrays; only keys are
// compared.  Works on host and device, on any memory space.
#pragma once
#include <cstdint>

#ifndef DD_HD
#ifdef __CUDACC__
#define DD_HD __host__ __device__ __forceinline__
#else
#define DD_HD inline
#endif
#endif

namespace ddsort {

constexpr int kThreshold = 16;

// count of trailing zero bits of a non-zero word
DD_HD int ctz32(uint32_t w) {
#ifdef __CUDA_ARCH__
  return __ffs(w) - 1;
#else
  return __builtin_ctz(w);
#endif
}

template <typename IdT>
struct Arr {
  IdT* id;
  float* key;
  DD_HD bool less(int a, int b) const { return key[a] < key[b]; }
  DD_HD void swap(int a, int b) const {
    IdT ti = id[a]; id[a] = id[b]; id[b] = ti;
    float tk = key[a]; key[a] = key[b]; key[b] = tk;
  }
};

DD_HD int floor_log2(int n) {
  int k = 0;
  while (n > 1) { n >>= 1; k++; }
  return k;
}

// median of (a, b, c) swapped into `result`
template <typename IdT>
DD_HD void move_median_to_first(const Arr<IdT>& A, int result, int a, int b, int c) {
  if (A.less(a, b)) {
    if (A.less(b, c)) A.swap(result, b);
    else if (A.less(a, c)) A.swap(result, c);
    else A.swap(result, a);
  } else if (A.less(a, c)) {
    A.swap(result, a);
  } else if (A.less(b, c)) {
    A.swap(result, c);
  } else {
    A.swap(result, b);
  }
}

// Hoare partition of [first, last) around the pivot held at `pivot`
template <typename IdT>
DD_HD int unguarded_partition(const Arr<IdT>& A, int first, int last, int pivot) {
  const float pk = A.key[pivot];
  while (true) {
    while (A.key[first] < pk) ++first;
    --last;
    while (pk < A.key[last]) --last;
    if (!(first < last)) return first;
    A.swap(first, last);
    ++first;
  }
}

// The same partition written as rank pairing, the form the parallel device
// code uses.  With the pivot value pk at `pivot` == first - 1:
//   left stops  l_1 < l_2 < ...  : positions in [first, last) with !(key < pk)
//   right stops r_1 > r_2 > ...  : positions in [pivot, last) with !(pk < key)
// the library swaps (l_k, r_k) for every k with l_k < r_k (K such pairs; the
// positions it visits in between are never ones a swap already touched) and
// returns min(l_{K+1}, r_K) (l_1 when K = 0; r_K when l_{K+1} does not exist).
// posL / posR need room for last - pivot entries.
template <typename IdT>
DD_HD int partition_by_rank_pairing(const Arr<IdT>& A, int first, int last, int pivot, int* posL,
                                    int* posR) {
  const float pk = A.key[pivot];
  int nL = 0, nR = 0;
  for (int i = first; i < last; i++)
    if (!(A.key[i] < pk)) posL[nL++] = i;
  for (int i = last - 1; i >= pivot; i--)
    if (!(pk < A.key[i])) posR[nR++] = i;
  int K = 0;
  while (K < nL && K < nR && posL[K] < posR[K]) K++;
  for (int k = 0; k < K; k++) A.swap(posL[k], posR[k]);
  if (K == 0) return posL[0];
  int a = K < nL ? posL[K] : last;
  return a < posR[K - 1] ? a : posR[K - 1];
}

// ---- heap fallback (make_heap + sort_heap over a whole range)
template <typename IdT>
DD_HD void push_heap_(const Arr<IdT>& A, int base, int hole, int top, IdT vid, float vkey) {
  int parent = (hole - 1) / 2;
  while (hole > top && A.key[base + parent] < vkey) {
    A.id[base + hole] = A.id[base + parent];
    A.key[base + hole] = A.key[base + parent];
    hole = parent;
    parent = (hole - 1) / 2;
  }
  A.id[base + hole] = vid;
  A.key[base + hole] = vkey;
}

template <typename IdT>
DD_HD void adjust_heap_(const Arr<IdT>& A, int base, int hole, int len, IdT vid, float vkey) {
  const int top = hole;
  int child = hole;
  while (child < (len - 1) / 2) {
    child = 2 * (child + 1);
    if (A.key[base + child] < A.key[base + child - 1]) child--;
    A.id[base + hole] = A.id[base + child];
    A.key[base + hole] = A.key[base + child];
    hole = child;
  }
  if ((len & 1) == 0 && child == (len - 2) / 2) {
    child = 2 * (child + 1);
    A.id[base + hole] = A.id[base + child - 1];
    A.key[base + hole] = A.key[base + child - 1];
    hole = child - 1;
  }
  push_heap_(A, base, hole, top, vid, vkey);
}

template <typename IdT>
DD_HD void heap_sort_range(const Arr<IdT>& A, int first, int last) {
  int len = last - first;
  if (len < 2) return;
  for (int parent = (len - 2) / 2;; parent--) {
    IdT vid = A.id[first + parent];
    float vk = A.key[first + parent];
    adjust_heap_(A, first, parent, len, vid, vk);
    if (parent == 0) break;
  }
  while (len > 1) {
    --len;
    IdT vid = A.id[first + len];
    float vk = A.key[first + len];
    A.id[first + len] = A.id[first];
    A.key[first + len] = A.key[first];
    adjust_heap_(A, first, 0, len, vid, vk);
  }
}

// stable insertion sort of one leaf
template <typename IdT>
DD_HD void insertion_sort_range(const Arr<IdT>& A, int first, int last) {
  for (int i = first + 1; i < last; i++) {
    IdT vid = A.id[i];
    float vk = A.key[i];
    int j = i;
    while (j > first && vk < A.key[j - 1]) {
      A.id[j] = A.id[j - 1];
      A.key[j] = A.key[j - 1];
      j--;
    }
    A.id[j] = vid;
    A.key[j] = vk;
  }
}

// Leaf sinks of the partition phase.
struct LeafList {  // explicit (lo, hi) pairs, room for n entries each
  int* lo;
  int* hi;
  int n = 0;
  DD_HD void add(int a, int b) { lo[n] = a; hi[n] = b; n++; }
};
struct LeafBits {  // one bit per position, set where a leaf starts ((n + 31) / 32 words)
  uint32_t* bits;
  int n = 0;
  DD_HD void add(int a, int) { bits[a >> 5] |= 1u << (a & 31); n++; }
};

// end of the leaf starting at `lo` in a LeafBits bitmap of n positions
DD_HD int leaf_end(const uint32_t* bits, int lo, int n) {
  int p = lo + 1;
  while (p < n) {
    uint32_t w = bits[p >> 5] & (0xffffffffu << (p & 31));
    if (w) {
      int q = (p & ~31) + (int)ctz32(w);
      return q < n ? q : n;
    }
    p = (p & ~31) + 32;
  }
  return n;
}

// Partition phase with the partition done by rank pairing (posL / posR need
// room for n entries); must give exactly what partition_phase gives.
template <typename IdT, typename Sink>
DD_HD int partition_phase_rank(const Arr<IdT>& A, int n, int* stack, Sink& sink, int* posL,
                               int* posR) {
  if (n <= 0) return 0;
  int sp = 0;
  stack[sp++] = 0;
  stack[sp++] = n;
  stack[sp++] = 2 * floor_log2(n);
  while (sp > 0) {
    int depth = stack[--sp];
    int last = stack[--sp];
    int first = stack[--sp];
    while (last - first > kThreshold) {
      if (depth == 0) {
        heap_sort_range(A, first, last);
        break;
      }
      --depth;
      int mid = first + (last - first) / 2;
      move_median_to_first(A, first, first + 1, mid, last - 1);
      int cut = partition_by_rank_pairing(A, first + 1, last, first, posL, posR);
      stack[sp++] = cut;
      stack[sp++] = last;
      stack[sp++] = depth;
      last = cut;
    }
    sink.add(first, last);
  }
  return sink.n;
}

// Partition phase.  `stack` needs stack_ints(n) ints; every leaf range is
// passed to sink.add(lo, hi); returns the number of leaves.
template <typename IdT, typename Sink>
DD_HD int partition_phase(const Arr<IdT>& A, int n, int* stack, Sink& sink) {
  if (n <= 0) return 0;
  // each stack entry: (first, last, depth) packed as three ints
  int sp = 0;
  stack[sp++] = 0;
  stack[sp++] = n;
  stack[sp++] = 2 * floor_log2(n);
  while (sp > 0) {
    int depth = stack[--sp];
    int last = stack[--sp];
    int first = stack[--sp];
    while (last - first > kThreshold) {
      if (depth == 0) {
        heap_sort_range(A, first, last);
        break;  // the range is fully sorted: record it as a leaf below
      }
      --depth;
      int mid = first + (last - first) / 2;
      move_median_to_first(A, first, first + 1, mid, last - 1);
      int cut = unguarded_partition(A, first + 1, last, first);
      // the library recurses on [cut, last) and loops on [first, cut)
      stack[sp++] = cut;
      stack[sp++] = last;
      stack[sp++] = depth;
      last = cut;
    }
    sink.add(first, last);
  }
  return sink.n;
}

template <typename IdT>
DD_HD int partition_phase(const Arr<IdT>& A, int n, int* stack, int* leaf_lo, int* leaf_hi) {
  LeafList s{leaf_lo, leaf_hi};
  return partition_phase(A, n, stack, s);
}

// Whole std::sort on one thread: the CPU tests check this against std::sort.
template <typename IdT>
DD_HD void introsort_emulated(const Arr<IdT>& A, int n, int* stack, int* leaf_lo, int* leaf_hi) {
  int nl = partition_phase(A, n, stack, leaf_lo, leaf_hi);
  for (int i = 0; i < nl; i++) insertion_sort_range(A, leaf_lo[i], leaf_hi[i]);
}

// Same with the leaves recorded in a bitmap and finished leaf by leaf.
template <typename IdT>
DD_HD void introsort_emulated_bits(const Arr<IdT>& A, int n, int* stack, uint32_t* bits) {
  for (int w = 0; w < (n + 31) / 32; w++) bits[w] = 0;
  LeafBits s{bits};
  partition_phase(A, n, stack, s);
  for (int i = 0; i < n; i++)
    if (bits[i >> 5] & (1u << (i & 31))) insertion_sort_range(A, i, leaf_end(bits, i, n));
}

// stack ints needed by partition_phase for n elements
DD_HD int stack_ints(int n) { return 3 * (2 * floor_log2(n > 1 ? n : 2) + 4); }

}  // namespace ddsort
