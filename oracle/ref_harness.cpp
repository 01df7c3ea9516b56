// Test-oracle harness around the reference's own, unmodified sources.
//
// This file is test infrastructure.  It is compiled (oracle/Makefile) against
// the reference tree's headers with the single-rank shims in oracle/ref_shims,
// and its binary lands in oracle/_ref/.  It exposes the reference's build and
// search entry points on files so tests and the CPU baseline can run them:
//
//   build   : BSP_index<Point,PointRange,unsigned>::bsp_build (src/bsp_index.hpp:551-556),
//             the path of `mpirun -np 1 build/distributed_diskann` (src/diskann.cpp:19-39)
//   knnbuild: knn_index<...>::build_index (include/index.h:125-137), the -DORIGINAL_PARLAY path
//   search  : searchAll (include/utils/beamSearch.h:314-346), timed twice like
//             checkRecall (include/utils/check_nn_recall.h:62-66)
//   qps     : the same timing for a list of beam widths on one loaded index
//   beam    : beam_search (include/utils/beamSearch.h:51-184), full frontier + visited
//   prune   : knn_index::robustPrune (include/index.h:63-123)
//
// Nothing here is part of the product library.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "utils/types.h"
#include "utils/point_range.h"
#include "utils/graph.h"
#include "utils/euclidian_point.h"
#include "utils/mips_point.h"
#include "utils/stats.h"
#undef roundup
#include "index.h"
#include "dataset.hpp"
#include "bsp_index.hpp"

namespace {

using idx_t = unsigned int;

void die(const char* m) {
  std::fprintf(stderr, "ref_harness: %s\n", m);
  std::exit(2);
}

std::vector<uint32_t> read_u32_file(const char* fn) {
  std::ifstream f(fn, std::ios::binary);
  if (!f) die("cannot open input file");
  f.seekg(0, std::ios::end);
  size_t bytes = (size_t)f.tellg();
  f.seekg(0);
  std::vector<uint32_t> v(bytes / 4);
  f.read((char*)v.data(), (std::streamsize)(v.size() * 4));
  return v;
}

void write_u32(FILE* f, const std::vector<uint32_t>& v) {
  if (!v.empty()) std::fwrite(v.data(), 4, v.size(), f);
}

double now_s() {
  return std::chrono::duration<double>(
             std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <typename T, typename Point>
int run(int argc, char** argv) {
  using PR = PointRange<T, Point>;
  std::string cmd = argv[1];
  PR Points(argv[4]);

  if (cmd == "build") {
    // build <dtype> <metric> <base> <R> <L> <alpha> <xita> <max> <start> <out_graph>
    if (argc < 12) die("build: bad args");
    dataset_para dp;
    dp.R = (uint32_t)std::atol(argv[5]);
    dp.L = (uint32_t)std::atol(argv[6]);
    dp.alpha = std::atof(argv[7]);
    dp.xita = std::atof(argv[8]);
    dp.max_build = (uint64_t)std::atoll(argv[9]);
    dp.start_point_index = (uint64_t)std::atoll(argv[10]);
    dp.two_pass = false;
    dp.save = true;
    dp.output_path = argv[11];
    BuildParams BP(dp.R, dp.L, dp.alpha, dp.two_pass);
    Graph<unsigned int> G(dp.R, Points.size());
    stats<unsigned int> BuildStats(G.size());
    double t0 = now_s();
    BSP_index<Point, PR, unsigned int> I;
    I.bsp_build(BP, G, Points, BuildStats, dp);
    double t1 = now_s();
    std::printf("HARNESS_BUILD_SECONDS %.9f\n", t1 - t0);
    return 0;
  }
  if (cmd == "knnbuild") {
    // knnbuild <dtype> <metric> <base> <R> <L> <alpha> <two_pass> <out_graph>
    if (argc < 10) die("knnbuild: bad args");
    BuildParams BP(std::atol(argv[5]), std::atol(argv[6]), std::atof(argv[7]),
                   std::atoi(argv[8]) != 0);
    Graph<unsigned int> G(BP.R, Points.size());
    stats<unsigned int> BuildStats(G.size());
    knn_index<Point, PR, unsigned int> I(BP);
    double t0 = now_s();
    I.build_index(G, Points, BuildStats);
    double t1 = now_s();
    std::printf("HARNESS_BUILD_SECONDS %.9f\n", t1 - t0);
    G.save(argv[9]);
    return 0;
  }
  if (cmd == "qps") {
    // qps <dtype> <metric> <base> <graph> <queries> <k> <cut> <start> <L1,L2,...> <out>
    // checkRecall's timing (include/utils/check_nn_recall.h:62-66) for each beam
    // width: searchAll once untimed, then once timed; ids of the timed pass out
    if (argc < 12) die("qps: bad args");
    Graph<unsigned int> G(argv[5]);
    PR Q(argv[6]);
    long k = std::atol(argv[7]);
    double cut = std::atof(argv[8]);
    idx_t start = (idx_t)std::atol(argv[9]);
    FILE* out = std::fopen(argv[11], "wb");
    if (!out) die("cannot open output");
    std::string Ls = argv[10];
    size_t pos = 0;
    while (pos < Ls.size()) {
      size_t e = Ls.find(',', pos);
      if (e == std::string::npos) e = Ls.size();
      long L = std::atol(Ls.substr(pos, e - pos).c_str());
      pos = e + 1;
      QueryParams QP(k, L, cut, (long)G.size(), G.max_degree());
      stats<unsigned int> QS(Q.size());
      auto r1 = searchAll<Point, PR, unsigned int>(Q, G, Points, QS, start, QP);
      QS.clear();
      double t0 = now_s();
      auto r2 = searchAll<Point, PR, unsigned int>(Q, G, Points, QS, start, QP);
      double t1 = now_s();
      std::printf("HARNESS_QPS %ld %.9f\n", L, t1 - t0);
      std::vector<uint32_t> ids;
      for (size_t i = 0; i < Q.size(); i++)
        for (long j = 0; j < k; j++) ids.push_back(r2[i][j]);
      write_u32(out, ids);
    }
    std::fclose(out);
    return 0;
  }
  if (cmd == "search" || cmd == "beam") {
    // search|beam <dtype> <metric> <base> <graph> <queries> <k> <L> <cut> <limit> <degree_limit> <start> <out>
    if (argc < 14) die("search: bad args");
    Graph<unsigned int> G(argv[5]);
    PR Q(argv[6]);
    long k = std::atol(argv[7]);
    long L = std::atol(argv[8]);
    double cut = std::atof(argv[9]);
    long limit = std::atol(argv[10]);
    long dlim = std::atol(argv[11]);
    idx_t start = (idx_t)std::atol(argv[12]);
    if (limit <= 0) limit = (long)G.size();
    if (dlim <= 0) dlim = G.max_degree();
    QueryParams QP(k, L, cut, limit, dlim);
    FILE* out = std::fopen(argv[13], "wb");
    if (!out) die("cannot open output");
    if (cmd == "search") {
      stats<unsigned int> QS(Q.size());
      auto r1 = searchAll<Point, PR, unsigned int>(Q, G, Points, QS, start, QP);
      QS.clear();
      double t0 = now_s();
      auto r2 = searchAll<Point, PR, unsigned int>(Q, G, Points, QS, start, QP);
      double t1 = now_s();
      std::printf("HARNESS_SEARCH_SECONDS %.9f\n", t1 - t0);
      std::vector<uint32_t> ids;
      for (size_t i = 0; i < Q.size(); i++)
        for (long j = 0; j < k; j++) ids.push_back(r2[i][j]);
      write_u32(out, ids);
      write_u32(out, std::vector<uint32_t>(QS.visited.begin(), QS.visited.end()));
      write_u32(out, std::vector<uint32_t>(QS.distances.begin(), QS.distances.end()));
      // searchAll reads frontier[j] for j < k even when the k-cut left fewer than k
      // entries (undefined values); report the frontier sizes so callers can mask them.
      std::vector<uint32_t> fsz(Q.size());
      for (size_t i = 0; i < Q.size(); i++)
        fsz[i] = (uint32_t)beam_search<Point, PR, unsigned int>(Q[i], G, Points, start, QP)
                     .first.first.size();
      write_u32(out, fsz);
    } else {
      // one record per query: [nf][nv][cmps] then nf (id,dist) then nv (id,dist)
      for (size_t i = 0; i < Q.size(); i++) {
        auto res = beam_search<Point, PR, unsigned int>(Q[i], G, Points, start, QP);
        auto& fr = res.first.first;
        auto& vi = res.first.second;
        uint32_t hdr[3] = {(uint32_t)fr.size(), (uint32_t)vi.size(), (uint32_t)res.second};
        std::fwrite(hdr, 4, 3, out);
        for (auto& e : fr) { std::fwrite(&e.first, 4, 1, out); std::fwrite(&e.second, 4, 1, out); }
        for (auto& e : vi) { std::fwrite(&e.first, 4, 1, out); std::fwrite(&e.second, 4, 1, out); }
      }
    }
    std::fclose(out);
    return 0;
  }
  if (cmd == "prune") {
    // prune <dtype> <metric> <base> <graph> <tasks> <R> <alpha> <out>
    // tasks file: repeated [p][m] then m (id, float dist)
    if (argc < 10) die("prune: bad args");
    Graph<unsigned int> G(argv[5]);
    auto tasks = read_u32_file(argv[6]);
    BuildParams BP(std::atol(argv[7]), 1, std::atof(argv[8]), false);
    knn_index<Point, PR, unsigned int> I(BP);
    FILE* out = std::fopen(argv[9], "wb");
    if (!out) die("cannot open output");
    size_t pos = 0;
    while (pos + 2 <= tasks.size()) {
      idx_t p = tasks[pos];
      uint32_t m = tasks[pos + 1];
      pos += 2;
      parlay::sequence<std::pair<idx_t, float>> cand;
      for (uint32_t j = 0; j < m; j++) {
        float d;
        std::memcpy(&d, &tasks[pos + 2 * j + 1], 4);
        cand.push_back(std::make_pair((idx_t)tasks[pos + 2 * j], d));
      }
      pos += 2 * (size_t)m;
      auto r = I.robustPrune(p, cand, G, Points, BP.alpha);
      uint32_t len = (uint32_t)r.size();
      std::fwrite(&len, 4, 1, out);
      if (len) std::fwrite(r.data(), 4, len, out);
    }
    std::fclose(out);
    return 0;
  }
  die("unknown command");
  return 2;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 5) {
    std::fprintf(stderr,
                 "usage: ref_harness <build|knnbuild|search|beam|prune> <f32|i8|u8> <l2|mips> <base.bin> ...\n");
    return 2;
  }
  int mpi_argc = 1;
  MPI_Init(&mpi_argc, &argv);
  std::string dt = argv[2], me = argv[3];
  int rc;
  if (me == "l2") {
    if (dt == "f32") rc = run<float, Euclidian_Point<float>>(argc, argv);
    else if (dt == "i8") rc = run<int8_t, Euclidian_Point<int8_t>>(argc, argv);
    else if (dt == "u8") rc = run<uint8_t, Euclidian_Point<uint8_t>>(argc, argv);
    else die("bad dtype");
  } else if (me == "mips") {
    if (dt == "f32") rc = run<float, Mips_Point<float>>(argc, argv);
    else if (dt == "i8") rc = run<int8_t, Mips_Point<int8_t>>(argc, argv);
    else if (dt == "u8") rc = run<uint8_t, Mips_Point<uint8_t>>(argc, argv);
    else die("bad dtype");
  } else {
    die("bad metric");
  }
  MPI_Finalize();
  return rc;
}
