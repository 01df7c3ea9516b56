// Compiles the drop-in C++ entry points (include/dd_vamana.hpp) against types
// shaped like the reference's PointRange / Graph / BuildParams / QueryParams /
// dataset_para (the members the header reads) and links libdd_gpu.  Without a
// GPU it checks the error path: dd_create fails and the installed handler
// sees the failure (the default prints and aborts, as the reference does).
// With a GPU it runs a small build, saves the graph and searches it.
// Prints "OK <what ran>" on success.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "dd_vamana.hpp"

template <class T>
struct MockPoint {
  static bool is_metric() { return true; }  // Euclidian_Point: L2
};

template <class T, class Point>
struct MockPointRange {
  std::shared_ptr<T[]> values;
  unsigned int dims = 0, aligned_dims = 0;
  size_t n = 0;
  MockPointRange(size_t n_, unsigned d, uint32_t seed) : dims(d), n(n_) {
    aligned_dims = (unsigned)((d * sizeof(T) + 63) / 64 * 64 / sizeof(T));
    values = std::shared_ptr<T[]>(new T[n * aligned_dims]());
    std::mt19937 g(seed);
    for (size_t i = 0; i < n; i++)
      for (unsigned j = 0; j < d; j++) values[i * aligned_dims + j] = (T)(g() % 200);
  }
  size_t size() { return n; }
  unsigned int get_dims() const { return dims; }
  long aligned_dimension() { return aligned_dims; }
};

struct MockEdgeRange {
  uint32_t* row;
  uint32_t* begin() { return row + 1; }
  size_t size() { return row[0]; }
};

struct MockGraph {
  long maxDeg;
  size_t n;
  std::vector<uint32_t> graph;
  MockGraph(long R, size_t n_) : maxDeg(R), n(n_), graph(n_ * (R + 1), 0) {}
  long max_degree() { return maxDeg; }
  size_t size() { return n; }
  MockEdgeRange operator[](uint32_t i) { return MockEdgeRange{graph.data() + i * (maxDeg + 1)}; }
};

struct MockBuildParams {
  long R = 16, L = 32;
  double alpha = 1.2;
  bool two_pass = false;
};
struct MockQueryParams {
  long k = 5, beamSize = 20;
  double cut = 1.35;
  long limit = 0, degree_limit = 0;
};
struct MockDatasetPara {
  double alpha = 1.2, xita = 0.02;
  long max_build = 0, start_point_index = 0;
  bool save = false;
  std::string output_path;
};

struct Failure : std::runtime_error {
  int code;
  Failure(const char* what, int c, const char* msg)
      : std::runtime_error(std::string(what) + ": " + msg), code(c) {}
};

int main(int argc, char** argv) {
  dd::set_error_handler([](const char* what, int code, const char* msg) {
    throw Failure(what, code, msg);
  });
  using Point = MockPoint<uint8_t>;
  MockPointRange<uint8_t, Point> base(2000, 24, 1), queries(50, 24, 2);
  MockGraph G(16, base.size());
  MockBuildParams BP;
  MockDatasetPara dp;
  dp.save = argc > 1;
  if (dp.save) dp.output_path = argv[1];
  try {
    dd::bsp_build<Point>(BP, G, base, dp);
  } catch (const Failure& f) {
    if (std::strstr(f.what(), "dd_create") == nullptr || f.code == DD_OK) {
      std::printf("FAIL unexpected error %s\n", f.what());
      return 1;
    }
    std::printf("OK no device: %s\n", f.what());
    return 0;
  }
  // a device was there: the graph must be filled and searchable
  size_t edges = 0;
  for (size_t i = 0; i < G.size(); i++) edges += G[(uint32_t)i].size();
  MockQueryParams QP;
  QP.limit = (long)base.size();
  QP.degree_limit = G.max_degree();
  std::vector<uint32_t> visited, cmps;
  std::vector<uint32_t> ids = dd::search_all<Point>(queries, G, base, 0, QP, &visited, &cmps);
  if (edges == 0 || ids.size() != queries.size() * QP.k || visited.size() != queries.size()) {
    std::printf("FAIL build/search output\n");
    return 1;
  }
  std::printf("OK built %zu edges, searched %zu queries\n", edges, queries.size());
  return 0;
}
