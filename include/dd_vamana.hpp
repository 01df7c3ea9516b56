/* Drop-in C++ entry points over the C ABI (dd_gpu.h), in the reference's own
 * terms: the reference's PointRange, Graph, BuildParams, QueryParams and
 * dataset_para objects go in as they are, and the calls mirror the ones they
 * replace (paths within Mr1BW/distributed_diskann):
 *
 *   dd::bsp_build        BSP_index<Point,PointRange,indexType>::bsp_build
 *                        (src/bsp_index.hpp:551-556; the batched build with
 *                        dataset_para's xita, max and start_point_index)
 *   dd::knn_build_index  knn_index<Point,PointRange,indexType>::build_index
 *                        (include/index.h:125-137; two_pass, final row sort)
 *   dd::search_all       searchAll (include/utils/beamSearch.h:314-346)
 *
 * Header only; link with -ldd_gpu.  What the templates read from the
 * reference's types (include/utils/point_range.h:53-113, graph.h:120-202,
 * types.h:103-156, src/dataset.hpp:30-89):
 *   PointRange: size(), get_dims(), aligned_dimension(), values (the padded
 *               rows, shared_ptr<T[]>), uploaded in place with their stride;
 *   Point:      is_metric() (Euclidian_Point: L2; Mips_Point: MIPS);
 *   Graph:      size(), max_degree(), operator[](0).begin() - 1 (the n x
 *               (R+1) [deg, nbr...] rows, written by the build);
 *   BuildParams R, L, alpha, two_pass; QueryParams k, beamSize, cut, limit,
 *   degree_limit; dataset_para alpha, xita, max_build, start_point_index,
 *   save, output_path.
 *
 * Errors: the reference prints a message and calls abort() (for example
 * include/utils/graph.h:55-93); dd::check does the same with the library's
 * message unless the caller installed a handler with dd::set_error_handler.
 */
#ifndef DD_VAMANA_HPP
#define DD_VAMANA_HPP

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "dd_gpu.h"

namespace dd {

using ErrorHandler = void (*)(const char* what, int code, const char* message);

inline ErrorHandler& error_handler_slot() {
  static ErrorHandler h = nullptr;
  return h;
}

// A handler replaces the print-and-abort default (it may throw).
inline void set_error_handler(ErrorHandler h) { error_handler_slot() = h; }

// true when rc is DD_OK; otherwise the handler runs (if it returns, the
// calling entry point stops where it is and returns) or the process aborts
inline bool check(dd_index* h, int rc, const char* what) {
  if (rc == DD_OK) return true;
  const char* msg = h ? dd_last_error(h) : "no handle (the call could not create one)";
  if (ErrorHandler eh = error_handler_slot()) {
    eh(what, rc, msg);
    return false;
  }
  std::printf("ERROR in %s (status %d): %s\n", what, rc, msg);
  std::abort();
}

template <class T>
constexpr int dtype_of() {
  static_assert(std::is_same<T, float>::value || std::is_same<T, int8_t>::value ||
                    std::is_same<T, uint8_t>::value,
                "points must be float, int8_t or uint8_t");
  return std::is_same<T, float>::value ? DD_DTYPE_F32
                                       : (std::is_same<T, int8_t>::value ? DD_DTYPE_I8 : DD_DTYPE_U8);
}

template <class Point>
constexpr int metric_of() {
  return Point::is_metric() ? DD_METRIC_L2 : DD_METRIC_MIPS;
}

// element type of a PointRange (its rows are a shared_ptr<T[]>)
template <class PR>
using value_t = typename std::decay<decltype(std::declval<PR&>().values)>::type::element_type;

// One device-resident index (RAII over dd_create / dd_destroy).
class Index {
 public:
  Index(int dtype, int metric, uint64_t n, uint32_t d, uint32_t R, int device = 0) {
    check(nullptr, dd_create(dtype, metric, n, d, R, device, &h_), "dd_create");
  }
  Index() = default;
  Index(Index&& o) noexcept : h_(o.h_) { o.h_ = nullptr; }
  Index& operator=(Index&& o) noexcept {
    std::swap(h_, o.h_);
    return *this;
  }
  Index(const Index&) = delete;
  Index& operator=(const Index&) = delete;
  ~Index() {
    if (h_) dd_destroy(h_);
  }
  dd_index* get() const { return h_; }
  explicit operator bool() const { return h_ != nullptr; }

 private:
  dd_index* h_ = nullptr;
};

// The index of a PointRange with its rows uploaded in place (no host copy).
template <class Point, class PR>
Index upload(PR& Points, uint32_t R, int device = 0) {
  using T = value_t<PR>;
  Index ix(dtype_of<T>(), metric_of<Point>(), (uint64_t)Points.size(), (uint32_t)Points.get_dims(),
           R, device);
  if (ix && !check(ix.get(),
                   dd_upload_points(ix.get(), Points.values.get(),
                                    (uint64_t)Points.aligned_dimension() * sizeof(T)),
                   "dd_upload_points"))
    return Index();
  return ix;
}

template <class Graph>
uint32_t* graph_rows(Graph& G) {
  return (uint32_t*)(G[0].begin() - 1);
}

// BSP_index::bsp_build: the reference leaves its result only in the file
// dp.output_path (G.save); here the graph is also written into G.
template <class Point, class PR, class Graph, class BP, class DP>
void bsp_build(BP& BP_, Graph& G, PR& Points, DP& dp, int device = 0, dd_stats* stats = nullptr,
               int mode = DD_MODE_FAST) {
  Index ix = upload<Point>(Points, (uint32_t)G.max_degree(), device);
  if (!ix) return;
  dd_build_params p{};
  p.L = (uint32_t)BP_.L;
  p.alpha = dp.alpha;
  p.max_fraction = dp.xita;
  p.max_build = (uint64_t)dp.max_build;
  p.start_point = (uint32_t)dp.start_point_index;
  p.collect_stats = stats != nullptr;
  p.mode = mode;
  if (!check(ix.get(), dd_build(ix.get(), &p, stats), "dd_build")) return;
  if (!check(ix.get(), dd_download_graph(ix.get(), graph_rows(G)), "dd_download_graph")) return;
  if (dp.save) check(ix.get(), dd_save_graph_file(ix.get(), dp.output_path.c_str()), "Graph::save");
}

// knn_index::build_index: start point 0, one round per prefix, two_pass, and
// each row sorted by distance at the end.
template <class Point, class PR, class Graph, class BP>
void knn_build_index(BP& BP_, Graph& G, PR& Points, int device = 0, dd_stats* stats = nullptr,
                     int mode = DD_MODE_FAST) {
  Index ix = upload<Point>(Points, (uint32_t)G.max_degree(), device);
  if (!ix) return;
  dd_build_params p{};
  p.L = (uint32_t)BP_.L;
  p.alpha = BP_.alpha;
  p.max_fraction = 1.0;
  p.knn_mode = 1;
  p.two_pass = BP_.two_pass ? 1 : 0;
  p.collect_stats = stats != nullptr;
  p.mode = mode;
  if (!check(ix.get(), dd_build(ix.get(), &p, stats), "dd_build")) return;
  check(ix.get(), dd_download_graph(ix.get(), graph_rows(G)), "dd_download_graph");
}

// searchAll: the first QP.k frontier ids of every query (row-major nq x k);
// base id i is skipped for query i as the reference does.  visited / cmps
// receive each query's visited count and distance computations (the
// reference's QueryStats) when given.
template <class Point, class PR, class Graph, class QP>
std::vector<uint32_t> search_all(PR& Query_Points, Graph& G, PR& Base_Points, uint32_t start,
                                 QP& qp, std::vector<uint32_t>* visited = nullptr,
                                 std::vector<uint32_t>* cmps = nullptr, int device = 0,
                                 int mode = DD_MODE_FAST) {
  using T = value_t<PR>;
  const uint64_t nq = Query_Points.size();
  std::vector<uint32_t> ids((size_t)nq * (size_t)qp.k);
  Index ix = upload<Point>(Base_Points, (uint32_t)G.max_degree(), device);
  if (!ix) return ids;
  if (!check(ix.get(), dd_upload_graph(ix.get(), graph_rows(G)), "dd_upload_graph") ||
      !check(ix.get(), dd_set_search_mode(ix.get(), mode), "dd_set_search_mode"))
    return ids;
  std::vector<uint32_t> Ls((size_t)nq, (uint32_t)qp.beamSize);
  std::vector<float> dists(ids.size());
  if (visited) visited->assign((size_t)nq, 0);
  if (cmps) cmps->assign((size_t)nq, 0);
  check(ix.get(),
        dd_search(ix.get(), Query_Points.values.get(), nq,
                  (uint64_t)Query_Points.aligned_dimension() * sizeof(T), Ls.data(),
                  (uint32_t)qp.k, (double)qp.cut, (uint64_t)qp.limit, (uint32_t)qp.degree_limit,
                  start, /*skip_self=*/1, ids.data(), dists.data(),
                  visited ? visited->data() : nullptr, cmps ? cmps->data() : nullptr),
        "searchAll");
  return ids;
}

}  // namespace dd

#endif  // DD_VAMANA_HPP
