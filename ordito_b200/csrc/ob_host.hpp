// Host-side helpers shared by the library's host setup code (factorisation, hierarchy build).
#pragma once

#include <algorithm>
#include <thread>
#include <vector>

namespace ob {

// Runs fn(begin, end) over [0, n) split across host threads when the work is large; serially
// otherwise. Each part is a contiguous range, so results written per index do not depend on
// the number of threads.
template <typename Fn>
void parallel_range(long long n, bool large, Fn fn) {
    const unsigned hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (!large || hw == 1 || n < 64) {
        fn(0LL, n);
        return;
    }
    const int parts = (int)std::min<long long>(hw, n / 16);
    std::vector<std::thread> pool;
    for (int p = 1; p < parts; ++p)
        pool.emplace_back([=]() { fn(n * p / parts, n * (p + 1) / parts); });
    fn(0LL, n / parts);
    for (auto& th : pool) th.join();
}

// Host threads parallel_range would use for a large job.
inline int host_threads() { return (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency())); }

// Runs fn(p) for p in [0, parts) on `parts` host threads (the caller's thread takes part 0).
template <typename Fn>
void run_parts(int parts, Fn fn) {
    std::vector<std::thread> pool;
    for (int p = 1; p < parts; ++p) pool.emplace_back([=]() { fn(p); });
    if (parts > 0) fn(0);
    for (auto& th : pool) th.join();
}

}  // namespace ob
