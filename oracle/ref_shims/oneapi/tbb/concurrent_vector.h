/* Stand-in for TBB's concurrent_vector: the reference only declares message
 * containers of this type on the (unused) point-to-point transport; a plain
 * std::vector gives the same single-threaded behaviour (oracle compile only). */
#pragma once
#include <vector>
namespace tbb {
template <typename T> using concurrent_vector = std::vector<T>;
}
