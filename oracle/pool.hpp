// pool.hpp — TEST INFRASTRUCTURE ONLY (see oracle.hpp).
// A persistent worker pool with dynamic chunked scheduling, standing in for
// rayon's `par_iter_mut().with_min_len(k)` (src/kernel_simd.rs:562,
// src/kernel.rs:187): workers claim chunks of `min_len` items from a shared
// counter until the range is exhausted.
#pragma once
#include <atomic>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace oracle {

class Pool {
  public:
    static Pool& get(int threads) {
        static Pool* p = nullptr;
        static std::mutex m;
        std::lock_guard<std::mutex> g(m);
        if (!p || p->size() != threads) {
            delete p;
            p = new Pool(threads);
        }
        return *p;
    }
    int size() const { return (int)workers_.size() + 1; }

    // Runs fn(i) for i in [0, n), chunks of `chunk` items per claim.
    void parallel_for(long n, long chunk, const std::function<void(long)>& fn) {
        if (n <= 0) return;
        if (workers_.empty()) {
            for (long i = 0; i < n; ++i) fn(i);
            return;
        }
        {
            std::lock_guard<std::mutex> g(mu_);
            fn_ = &fn;
            n_ = n;
            chunk_ = chunk < 1 ? 1 : chunk;
            next_.store(0);
            pending_ = (int)workers_.size();
            ++generation_;
        }
        cv_.notify_all();
        work();
        std::unique_lock<std::mutex> g(mu_);
        done_cv_.wait(g, [&] { return pending_ == 0; });
        fn_ = nullptr;
    }

    ~Pool() {
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
            ++generation_;
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
    }

  private:
    explicit Pool(int threads) {
        for (int i = 1; i < threads; ++i) workers_.emplace_back([this] { loop(); });
    }
    void work() {
        for (;;) {
            long b = next_.fetch_add(chunk_);
            if (b >= n_) break;
            long e = b + chunk_ < n_ ? b + chunk_ : n_;
            for (long i = b; i < e; ++i) (*fn_)(i);
        }
    }
    void loop() {
        unsigned long seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> g(mu_);
                cv_.wait(g, [&] { return generation_ != seen; });
                seen = generation_;
                if (stop_) return;
            }
            work();
            {
                std::lock_guard<std::mutex> g(mu_);
                if (--pending_ == 0) done_cv_.notify_all();
            }
        }
    }
    std::vector<std::thread> workers_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(long)>* fn_ = nullptr;
    long n_ = 0, chunk_ = 1;
    std::atomic<long> next_{0};
    int pending_ = 0;
    unsigned long generation_ = 0;
    bool stop_ = false;
};

inline void parallel_for(int threads, long n, long chunk, const std::function<void(long)>& fn) {
    if (threads <= 1) {
        for (long i = 0; i < n; ++i) fn(i);
        return;
    }
    Pool::get(threads).parallel_for(n, chunk, fn);
}

}  // namespace oracle
