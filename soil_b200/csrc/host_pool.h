// host_pool.h — a small persistent pool of host threads for the batch
// engine's per-box planning (each box's host decisions are independent).
//
// run(n, fn) calls fn(i) for every i in [0, n) across the workers and the
// calling thread, and returns the first non-zero status any call returned
// (every index still runs).  Work is handed out in chunks from an atomic
// cursor, so boxes of uneven cost balance across threads.
#pragma once

#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace soil_host {

class HostPool {
  public:
    explicit HostPool(int threads) {
        for (int t = 1; t < threads; ++t) workers_.emplace_back([this] { loop(); });
    }
    ~HostPool() {
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& w : workers_) w.join();
    }
    HostPool(const HostPool&) = delete;
    HostPool& operator=(const HostPool&) = delete;

    int threads() const { return (int)workers_.size() + 1; }

    int run(size_t n, const std::function<int(size_t)>& fn, size_t min_parallel = 64) {
        if (n == 0) return 0;
        if (workers_.empty() || n < min_parallel) {
            int st = 0;
            for (size_t i = 0; i < n; ++i) {
                const int r = fn(i);
                if (r && !st) st = r;
            }
            return st;
        }
        {
            std::lock_guard<std::mutex> g(mu_);
            fn_ = &fn;
            n_ = n;
            chunk_ = n / ((size_t)threads() * 8) + 1;
            next_.store(0);
            status_.store(0);
            busy_ = (int)workers_.size();
            ++gen_;
        }
        cv_.notify_all();
        work();
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [this] { return busy_ == 0; });
        fn_ = nullptr;
        return status_.load();
    }

  private:
    void work() {
        for (;;) {
            const size_t lo = next_.fetch_add(chunk_);
            if (lo >= n_) return;
            const size_t hi = lo + chunk_ < n_ ? lo + chunk_ : n_;
            for (size_t i = lo; i < hi; ++i) {
                const int r = (*fn_)(i);
                if (r) {
                    int expect = 0;
                    status_.compare_exchange_strong(expect, r);
                }
            }
        }
    }

    void loop() {
        uint64_t seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
            }
            work();
            {
                std::lock_guard<std::mutex> g(mu_);
                if (--busy_ == 0) done_cv_.notify_one();
            }
        }
    }

    std::vector<std::thread> workers_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    const std::function<int(size_t)>* fn_ = nullptr;
    size_t n_ = 0, chunk_ = 1;
    std::atomic<size_t> next_{0};
    std::atomic<int> status_{0};
    int busy_ = 0;
    uint64_t gen_ = 0;
    bool stop_ = false;
};

}  // namespace soil_host
