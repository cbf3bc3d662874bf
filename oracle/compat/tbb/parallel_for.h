// Test-oracle stand-in for oneTBB's parallel_for over a blocked_range, so the
// reference's TBB-parallel loops compile and run here without TBB.  Work is
// split into chunks handed out dynamically (an atomic cursor) to a pool of
// std::threads; the thread count is MCLCCD_REF_THREADS or all hardware
// threads.  Only scheduling differs from TBB: the loop bodies, and therefore
// every value they compute, are the reference's own.
#pragma once
#include "blocked_range.h"
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <thread>
#include <vector>

namespace tbb {

inline int compat_thread_count()
{
    static int n = [] {
        const char *s = std::getenv("MCLCCD_REF_THREADS");
        int v = s ? std::atoi(s) : 0;
        if (v <= 0) v = int(std::thread::hardware_concurrency());
        return v > 0 ? v : 1;
    }();
    return n;
}

template <typename Value, typename Body>
void parallel_for(const blocked_range<Value> &range, const Body &body)
{
    const Value b = range.begin(), e = range.end();
    if (!(b < e)) return;
    const long long n = (long long)(e - b);
    const int nt = std::min<long long>(compat_thread_count(), n);
    if (nt <= 1) { body(range); return; }
    // Many more chunks than threads so that uneven chunks balance out, but no
    // smaller than the range's grain size.
    long long chunk = std::max<long long>((long long)range.grainsize(), n / ((long long)nt * 64));
    if (chunk < 1) chunk = 1;
    std::atomic<long long> cursor(0);
    auto worker = [&]() {
        for (;;) {
            long long s = cursor.fetch_add(chunk);
            if (s >= n) break;
            long long t = std::min(n, s + chunk);
            body(blocked_range<Value>(Value(b + s), Value(b + t)));
        }
    };
    std::vector<std::thread> pool;
    pool.reserve(nt - 1);
    for (int i = 1; i < nt; ++i) pool.emplace_back(worker);
    worker();
    for (auto &t : pool) t.join();
}

} // namespace tbb
