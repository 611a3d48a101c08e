// Host-side helpers: a small fork-join loop over all cores, and the error type the C ABI maps to
// status codes.
#pragma once

#include <algorithm>
#include <cstdint>
#include <functional>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "ps_fea.h"

namespace psfea {

struct Error : std::runtime_error {
    ps_status status;
    Error(ps_status s, const std::string& msg) : std::runtime_error(msg), status(s) {}
};

inline unsigned hostThreads() {
    static const unsigned n = [] {
        unsigned t = std::thread::hardware_concurrency();
        return std::max(1u, std::min(t, 64u));
    }();
    return n;
}

// fn(lo, hi) over [0, n) split into contiguous chunks, one thread per chunk; runs inline for
// small n. No reductions: results never depend on the split.
inline void parallelFor(int64_t n, const std::function<void(int64_t, int64_t)>& fn, int64_t grain = 1 << 14) {
    if (n <= 0) return;
    const int64_t chunks = std::min<int64_t>(hostThreads(), std::max<int64_t>(1, n / grain));
    if (chunks <= 1) {
        fn(0, n);
        return;
    }
    std::vector<std::thread> th;
    th.reserve(size_t(chunks));
    for (int64_t c = 0; c < chunks; c++) {
        const int64_t a = n * c / chunks, b = n * (c + 1) / chunks;
        th.emplace_back([&fn, a, b] { fn(a, b); });
    }
    for (auto& t : th) t.join();
}

}  // namespace psfea
