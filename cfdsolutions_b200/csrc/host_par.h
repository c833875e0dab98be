// Host-side parallel loops of the set-up code (mesh builder, mesh
// installation, ILU ordering): contiguous ranges of an index space, one
// std::thread each.  Every range writes only its own items, so the results do
// not depend on the number of threads.
#pragma once

#include <algorithm>
#include <cstdint>
#include <thread>
#include <vector>

#include "cfd_internal.h"

namespace cfd {

// Ranges [0, n) is split into: up to 16 (or the calling thread's
// g_host_threads), one below 65,536 items.
inline int range_count(int64_t n) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned cap = g_host_threads > 0 ? (unsigned)g_host_threads : 16u;
    return n < 65536 ? 1 : (int)std::min(cap, hw);
}

// fn(t, lo, hi) for the range_count(n) contiguous ranges t of [0, n).
template <typename F>
void parallel_ranges(int64_t n, F fn) {
    const int nt = range_count(n);
    if (nt == 1) {
        fn(0, (int64_t)0, n);
        return;
    }
    std::vector<std::thread> th;
    for (int t = 0; t < nt; t++) th.emplace_back(fn, t, n * t / nt, n * (t + 1) / nt);
    for (auto &x : th) x.join();
}

}  // namespace cfd
