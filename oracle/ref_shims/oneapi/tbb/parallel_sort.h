/* Stand-in for TBB's parallel_sort, referenced only by the unused transport
 * (oracle compile only). */
#pragma once
#include <algorithm>
namespace tbb {
template <typename It, typename C> void parallel_sort(It b, It e, C c) { std::sort(b, e, c); }
template <typename It> void parallel_sort(It b, It e) { std::sort(b, e); }
}
