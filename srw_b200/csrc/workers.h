// A fixed set of host worker threads, started once and reused for every call: run(n, fn) calls
// fn(t) for t = 0 .. n-1, t = 0 on the calling thread and the others on workers, and returns when
// all have finished.  Starting and joining threads for every group of electrons cost about as much
// host time as planning a small electron.
#pragma once
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace srwg {

class WorkerPool {
public:
    explicit WorkerPool(int n)
    {
        for (int i = 1; i < n; i++) th_.emplace_back([this, i]() { loop(i); });
    }
    ~WorkerPool()
    {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : th_) t.join();
    }
    WorkerPool(const WorkerPool&) = delete;
    WorkerPool& operator=(const WorkerPool&) = delete;

    int size() const { return (int)th_.size() + 1; }

    // n <= size(); fn must not call run() of the same pool
    void run(int n, const std::function<void(int)>& fn)
    {
        if (n > size()) n = size();
        if (n <= 1) {
            if (n == 1) fn(0);
            return;
        }
        {
            std::lock_guard<std::mutex> lk(mu_);
            job_ = &fn;
            njob_ = n;
            pending_ = n - 1;
            gen_++;
        }
        cv_.notify_all();
        fn(0);
        std::unique_lock<std::mutex> lk(mu_);
        done_.wait(lk, [this]() { return pending_ == 0; });
        job_ = nullptr;
    }

private:
    void loop(int i)
    {
        long long seen = 0;
        for (;;) {
            const std::function<void(int)>* job = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&]() { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
                if (i < njob_) job = job_;
            }
            if (!job) continue;
            (*job)(i);
            std::lock_guard<std::mutex> lk(mu_);
            if (--pending_ == 0) done_.notify_one();
        }
    }

    std::vector<std::thread> th_;
    std::mutex mu_;
    std::condition_variable cv_, done_;
    const std::function<void(int)>* job_ = nullptr;
    int njob_ = 0;
    int pending_ = 0;
    long long gen_ = 0;
    bool stop_ = false;
};

}  // namespace srwg
