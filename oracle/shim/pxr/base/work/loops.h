// Stand-in for WorkParallelForN (oracle build of the reference sources; test
// infrastructure): hands chunks of [0, n) to HDR_REF_THREADS (default: all host
// cores) std::threads from a shared counter, so uneven tiles balance as under
// the TBB-backed original's work stealing.
//
// Timing a bounded sample of a frame: when WorkShimSelected() holds ranges for
// an iteration space of exactly `total` indices, a loop over that space runs
// only the indices inside the ranges (the passes' 16x16 tile loops then render
// the chosen tile rows of the real frame and nothing else). The harness sets
// and clears the selection around the passes it times.
#pragma once
#include <algorithm>
#include <atomic>
#include <cstddef>
#include <cstdlib>
#include <thread>
#include <utility>
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

struct WorkShimSelection {
    std::size_t total = 0;  // iteration-space size the ranges apply to (0: none)
    std::vector<std::pair<std::size_t, std::size_t>> ranges;  // [begin, end) pieces of [0, total)
};

inline WorkShimSelection &WorkShimSelected() {
    static WorkShimSelection sel;
    return sel;
}

template <typename Fn> void WorkParallelForN(std::size_t n, Fn &&fn) {
    if (n == 0) return;
    std::vector<std::pair<std::size_t, std::size_t>> pieces;
    const WorkShimSelection &sel = WorkShimSelected();
    if (sel.total == n && !sel.ranges.empty())
        pieces = sel.ranges;
    else
        pieces.emplace_back(0, n);
    std::size_t work = 0;
    for (const auto &p : pieces) work += p.second - p.first;
    const std::size_t threads = std::max<std::size_t>(1, std::min<std::size_t>(WorkShimThreadCount(), work));
    // small chunks so uneven tiles balance
    const std::size_t chunk = std::max<std::size_t>(1, work / (threads * 8));
    std::vector<std::pair<std::size_t, std::size_t>> chunks;
    for (const auto &p : pieces)
        for (std::size_t b = p.first; b < p.second; b += chunk) chunks.emplace_back(b, std::min(p.second, b + chunk));
    if (threads <= 1) {
        for (const auto &c : chunks) fn(c.first, c.second);
        return;
    }
    std::atomic<std::size_t> next{0};
    std::vector<std::thread> pool;
    pool.reserve(threads);
    for (std::size_t t = 0; t < threads; ++t) {
        pool.emplace_back([&] {
            for (std::size_t k = next.fetch_add(1); k < chunks.size(); k = next.fetch_add(1))
                fn(chunks[k].first, chunks[k].second);
        });
    }
    for (auto &th : pool) th.join();
}

PXR_NAMESPACE_CLOSE_SCOPE
