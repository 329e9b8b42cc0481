// Host thread helper shared by the graph build and the network loader.
#pragma once

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <exception>
#include <mutex>
#include <system_error>
#include <thread>
#include <vector>

namespace ngx {

// Runs body(task) for every task in [0, tasks) on up to `threads` threads (the calling thread included). A thread that
// cannot be started leaves its share to the others; the first exception a task throws is rethrown here once every
// thread has stopped (the remaining tasks are skipped).
template <typename Body>
inline void parallel_for(int64_t tasks, int threads, const Body& body) {
    const int workers = static_cast<int>(std::min<int64_t>(tasks, threads));
    if (workers <= 1) {
        for (int64_t t = 0; t < tasks; ++t) {
            body(t);
        }
        return;
    }
    std::atomic<int64_t> next{ 0 };
    std::exception_ptr failure;
    std::mutex failure_lock;
    const auto run = [&] {
        for (int64_t t = next.fetch_add(1); t < tasks; t = next.fetch_add(1)) {
            try {
                body(t);
            } catch (...) {
                const std::lock_guard<std::mutex> hold(failure_lock);
                if (!failure) {
                    failure = std::current_exception();
                }
                next.store(tasks);
            }
        }
    };
    std::vector<std::thread> pool;
    pool.reserve(static_cast<size_t>(workers - 1));
    for (int i = 1; i < workers; ++i) {
        try {
            pool.emplace_back(run);
        } catch (const std::system_error&) {
            break;  // fewer threads
        }
    }
    run();
    for (auto& worker : pool) {
        worker.join();
    }
    if (failure) {
        std::rethrow_exception(failure);
    }
}

}  // namespace ngx
