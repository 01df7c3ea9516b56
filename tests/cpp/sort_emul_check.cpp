// Checks ddsort::introsort_emulated (the device sort emulation, compiled here
// as host code) against libstdc++ std::sort with the distance-only comparator
// of robustPrune (include/index.h:78-79).  Prints "OK <cases>" on success.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <utility>
#include <vector>

#include "../../distributed_diskann_b200/csrc/sort_emul.cuh"

static int check(const std::vector<std::pair<unsigned, float>>& in, bool* heap_used) {
  std::vector<std::pair<unsigned, float>> ref = in;
  std::sort(ref.begin(), ref.end(),
            [](std::pair<unsigned, float> a, std::pair<unsigned, float> b) { return a.second < b.second; });
  int n = (int)in.size();
  std::vector<unsigned> id(n);
  std::vector<float> key(n);
  for (int i = 0; i < n; i++) id[i] = in[i].first, key[i] = in[i].second;
  std::vector<int> stack(ddsort::stack_ints(n) + 3), lo(n + 1), hi(n + 1);
  ddsort::Arr<unsigned> A{id.data(), key.data()};
  int nl = ddsort::partition_phase(A, n, stack.data(), lo.data(), hi.data());
  for (int i = 0; i < nl; i++) {
    if (hi[i] - lo[i] > ddsort::kThreshold) *heap_used = true;
    ddsort::insertion_sort_range(A, lo[i], hi[i]);
  }
  for (int i = 0; i < n; i++)
    if (id[i] != ref[i].first || key[i] != ref[i].second) return 1;
  // the bitmap-leaf form used by the device prune must agree too
  std::vector<unsigned> id2(n);
  std::vector<float> key2(n);
  for (int i = 0; i < n; i++) id2[i] = in[i].first, key2[i] = in[i].second;
  std::vector<uint32_t> bits((n + 31) / 32 + 1);
  ddsort::Arr<unsigned> B{id2.data(), key2.data()};
  ddsort::introsort_emulated_bits(B, n, stack.data(), bits.data());
  for (int i = 0; i < n; i++)
    if (id2[i] != ref[i].first || key2[i] != ref[i].second) return 2;
  // and the rank-pairing partition (the form the parallel device code uses)
  std::vector<unsigned> id3(n);
  std::vector<float> key3(n);
  for (int i = 0; i < n; i++) id3[i] = in[i].first, key3[i] = in[i].second;
  std::vector<int> posL(n + 1), posR(n + 1), lo3(n + 1), hi3(n + 1);
  ddsort::Arr<unsigned> C{id3.data(), key3.data()};
  ddsort::LeafList sink{lo3.data(), hi3.data()};
  int nl3 = ddsort::partition_phase_rank(C, n, stack.data(), sink, posL.data(), posR.data());
  for (int i = 0; i < nl3; i++) ddsort::insertion_sort_range(C, lo3[i], hi3[i]);
  for (int i = 0; i < n; i++)
    if (id3[i] != ref[i].first || key3[i] != ref[i].second) return 3;
  return 0;
}

int main() {
  std::mt19937_64 rng(12345);
  int cases = 0;
  bool heap_used = false;
  for (int t = 0; t < 40000; t++) {
    int n = (int)(rng() % 700);
    if (t % 7 == 0) n = (int)(rng() % 40);
    int distinct = 1 + (int)(rng() % (t % 3 == 0 ? 4 : (t % 3 == 1 ? 40 : 100000)));
    std::vector<std::pair<unsigned, float>> v(n);
    for (int i = 0; i < n; i++) v[i] = {(unsigned)i, (float)(rng() % distinct)};
    if (t % 5 == 0) std::sort(v.begin(), v.end(), [](auto a, auto b) { return a.second < b.second; });
    if (t % 11 == 0) std::reverse(v.begin(), v.end());
    if (check(v, &heap_used)) { std::printf("MISMATCH case %d n=%d\n", t, n); return 1; }
    cases++;
  }
  // interleaved halves (a[2i] = i, a[2i+1] = n/2 + i) folded mod 97: defeats the
  // median-of-three pivot enough to exhaust the depth limit (heapsort fallback)
  for (int n : {64, 200, 513, 1000, 4096}) {
    std::vector<std::pair<unsigned, float>> v(n);
    for (int i = 0; i < n; i++) {
      int a = (i % 2 == 0) ? i / 2 : n / 2 + i / 2;
      v[i] = {(unsigned)i, (float)(a % 97)};
    }
    if (check(v, &heap_used)) { std::printf("MISMATCH interleaved n=%d\n", n); return 1; }
    cases++;
  }
  // organ-pipe / sawtooth inputs with many ties
  for (int n : {100, 300, 700, 2000}) {
    std::vector<float> key(n);
    std::vector<unsigned> id(n);
    for (int i = 0; i < n; i++) id[i] = i;
    for (int i = 0; i < n; i++) key[i] = (float)((i < n / 2) ? i % 17 : (n - i) % 13);
    std::vector<std::pair<unsigned, float>> v(n);
    for (int i = 0; i < n; i++) v[i] = {id[i], key[i]};
    if (check(v, &heap_used)) { std::printf("MISMATCH pipe n=%d\n", n); return 1; }
    cases++;
  }
  std::printf("OK %d heap=%d\n", cases, heap_used ? 1 : 0);
  return 0;
}
