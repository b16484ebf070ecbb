// Host-side parallel loop for the once-per-mesh work (geometry, layout).
#include <algorithm>
#include <cstdlib>
#include <exception>
#include <thread>

#include "host.hpp"

namespace psst {

int host_threads() {
    static const int n = [] {
        const char *e = std::getenv("PSST_HOST_THREADS");
        int t = e ? std::atoi(e) : (int)std::thread::hardware_concurrency();
        return std::max(1, std::min(t, 64));
    }();
    return n;
}

void parallel_tasks(int ntasks, const std::function<void(int)> &fn) {
    std::vector<std::exception_ptr> err((size_t)std::max(ntasks, 0));
    std::vector<std::thread> pool;
    auto run = [&](int t) {
        try {
            fn(t);
        } catch (...) {
            err[(size_t)t] = std::current_exception();
        }
    };
    for (int t = 1; t < ntasks; ++t) pool.emplace_back(run, t);
    if (ntasks > 0) run(0);
    for (auto &th : pool) th.join();
    for (auto &e : err)
        if (e) std::rethrow_exception(e);
}

void parallel_for(int64_t n, const std::function<void(int64_t, int64_t)> &fn) {
    constexpr int64_t kMinChunk = 16384;
    const int64_t nt = std::min<int64_t>(host_threads(), (n + kMinChunk - 1) / kMinChunk);
    if (nt <= 1) {
        if (n > 0) fn(0, n);
        return;
    }
    std::vector<std::exception_ptr> err((size_t)nt);
    std::vector<std::thread> pool;
    pool.reserve((size_t)nt - 1);
    auto run = [&](int64_t t) {
        try {
            fn(n * t / nt, n * (t + 1) / nt);
        } catch (...) {
            err[(size_t)t] = std::current_exception();
        }
    };
    for (int64_t t = 1; t < nt; ++t) pool.emplace_back(run, t);
    run(0);
    for (auto &th : pool) th.join();
    for (auto &e : err)
        if (e) std::rethrow_exception(e);
}

}  // namespace psst
