// Host work spread over a few worker threads: copies into the page-locked staging
// buffer (a gigabyte of control points for an hour of LFO-modulated voices; one
// thread moves a few GB/s) and the per-job parts of staging a batch.  Work is cut
// into items that the workers and the calling thread take in turn.
#pragma once

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstddef>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace cs {

struct CopyPiece {
    void* dst;
    const void* src;
    size_t bytes;
};

class WorkerPool {
public:
    explicit WorkerPool(unsigned workers)
    {
        for (unsigned i = 0; i < workers; ++i)
            threads_.emplace_back([this] { work(); });
    }

    ~WorkerPool()
    {
        {
            std::lock_guard<std::mutex> lock(mutex_);
            stop_ = true;
        }
        wake_.notify_all();
        for (auto& t : threads_)
            t.join();
    }

    WorkerPool(const WorkerPool&) = delete;
    WorkerPool& operator=(const WorkerPool&) = delete;

    // Copies every piece (cut into pieces of at most `grain` bytes) and returns when
    // all are done.
    void copy(const std::vector<CopyPiece>& pieces, size_t grain = size_t(4) << 20)
    {
        std::vector<CopyPiece> cut;
        for (const auto& p : pieces)
            for (size_t at = 0; at < p.bytes; at += grain)
                cut.push_back({static_cast<char*>(p.dst) + at, static_cast<const char*>(p.src) + at,
                               std::min(grain, p.bytes - at)});
        run(cut.size(), [&](size_t i) { std::memcpy(cut[i].dst, cut[i].src, cut[i].bytes); });
    }

    // Runs task(0) .. task(count - 1) over the workers and the calling thread and
    // returns when all are done.  Tasks must not throw.
    void run(size_t count, const std::function<void(size_t)>& task)
    {
        if (!count)
            return;
        if (threads_.empty() || count == 1) {
            for (size_t i = 0; i < count; ++i)
                task(i);
            return;
        }
        {
            std::lock_guard<std::mutex> lock(mutex_);
            task_ = &task;
            count_ = count;
            next_.store(0);
            pending_ = threads_.size();
            ++generation_;
        }
        wake_.notify_all();
        drain(task, count);
        std::unique_lock<std::mutex> lock(mutex_);
        done_.wait(lock, [this] { return pending_ == 0; });
        task_ = nullptr;
    }

private:
    void drain(const std::function<void(size_t)>& task, size_t count)
    {
        for (size_t i = next_.fetch_add(1); i < count; i = next_.fetch_add(1))
            task(i);
    }

    void work()
    {
        size_t seen = 0;
        for (;;) {
            const std::function<void(size_t)>* task;
            size_t count;
            {
                std::unique_lock<std::mutex> lock(mutex_);
                wake_.wait(lock, [&] { return stop_ || generation_ != seen; });
                if (stop_)
                    return;
                seen = generation_;
                task = task_;
                count = count_;
            }
            drain(*task, count);
            {
                std::lock_guard<std::mutex> lock(mutex_);
                if (--pending_ == 0)
                    done_.notify_one();
            }
        }
    }

    std::vector<std::thread> threads_;
    std::mutex mutex_;
    std::condition_variable wake_, done_;
    const std::function<void(size_t)>* task_ = nullptr;
    size_t count_ = 0;
    std::atomic<size_t> next_{0};
    size_t pending_ = 0, generation_ = 0;
    bool stop_ = false;
};

} // namespace cs
