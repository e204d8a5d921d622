// Stand-in for WorkParallelForN (oracle build of the reference sources; test
// infrastructure): splits [0, n) over HDR_REF_THREADS (default: all host cores)
// std::threads in contiguous chunks, like the TBB-backed original.
#pragma once
#include <algorithm>
#include <cstddef>
#include <cstdlib>
#include <thread>
#include <vector>

#include "pxr/pxr.h"

PXR_NAMESPACE_OPEN_SCOPE

inline unsigned WorkShimThreadCount() {
    if (const char *e = std::getenv("HDR_REF_THREADS")) {
        int v = std::atoi(e);
        if (v > 0) return (unsigned)v;
    }
    unsigned n = std::thread::hardware_concurrency();
    return n ? n : 1;
}

template <typename Fn> void WorkParallelForN(std::size_t n, Fn &&fn) {
    if (n == 0) return;
    const std::size_t threads = std::min<std::size_t>(WorkShimThreadCount(), n);
    if (threads <= 1) {
        fn(std::size_t{0}, n);
        return;
    }
    // small chunks handed out round-robin so uneven tiles balance
    const std::size_t chunk = std::max<std::size_t>(1, n / (threads * 8));
    std::vector<std::thread> pool;
    pool.reserve(threads);
    for (std::size_t t = 0; t < threads; ++t) {
        pool.emplace_back([&, t] {
            for (std::size_t b = t * chunk; b < n; b += threads * chunk) fn(b, std::min(n, b + chunk));
        });
    }
    for (auto &th : pool) th.join();
}

PXR_NAMESPACE_CLOSE_SCOPE
