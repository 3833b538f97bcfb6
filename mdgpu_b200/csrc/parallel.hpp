// Host-side parallel loop used by the analysis: indices shared out to the
// host's cores from one atomic counter (so uneven items balance), the calling
// thread taking part.
#pragma once

#include <algorithm>
#include <atomic>
#include <exception>
#include <thread>
#include <vector>

namespace mdgpu {

// fn(i) for every i in [0, count); the first exception (lowest index) is
// rethrown after all threads have joined.
template <typename F>
void parallel_for(int count, F&& fn) {
    if (count <= 0) return;
    std::vector<std::exception_ptr> ex(count);
    std::atomic<int> next{0};
    auto work = [&]() {
        for (int i = next.fetch_add(1); i < count; i = next.fetch_add(1)) {
            try {
                fn(i);
            } catch (...) {
                ex[i] = std::current_exception();
            }
        }
    };
    const int nthr = std::max(1, std::min(count, (int)std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (int t = 1; t < nthr; ++t) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    for (auto& e : ex)
        if (e) std::rethrow_exception(e);
}

}  // namespace mdgpu
