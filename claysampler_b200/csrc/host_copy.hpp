// Host-memory copies spread over a few worker threads.  Staging a batch copies its
// plans' control points (a gigabyte for an hour of LFO-modulated voices) into
// page-locked memory; one thread moves a few GB/s, so the copy is cut into pieces
// that the workers and the calling thread take in turn.
#pragma once

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstddef>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

namespace cs {

struct CopyPiece {
    void* dst;
    const void* src;
    size_t bytes;
};

class CopyPool {
public:
    explicit CopyPool(unsigned workers)
    {
        for (unsigned i = 0; i < workers; ++i)
            threads_.emplace_back([this] { work(); });
    }

    ~CopyPool()
    {
        {
            std::lock_guard<std::mutex> lock(mutex_);
            stop_ = true;
        }
        wake_.notify_all();
        for (auto& t : threads_)
            t.join();
    }

    CopyPool(const CopyPool&) = delete;
    CopyPool& operator=(const CopyPool&) = delete;

    // Copies every piece (cut into pieces of at most `grain` bytes) and returns when
    // all are done.
    void copy(const std::vector<CopyPiece>& pieces, size_t grain = size_t(4) << 20)
    {
        std::vector<CopyPiece> cut;
        for (const auto& p : pieces)
            for (size_t at = 0; at < p.bytes; at += grain)
                cut.push_back({static_cast<char*>(p.dst) + at, static_cast<const char*>(p.src) + at,
                               std::min(grain, p.bytes - at)});
        if (cut.empty())
            return;
        if (threads_.empty() || cut.size() == 1) {
            for (const auto& p : cut)
                std::memcpy(p.dst, p.src, p.bytes);
            return;
        }
        {
            std::lock_guard<std::mutex> lock(mutex_);
            work_ = &cut;
            next_.store(0);
            pending_ = threads_.size();
            ++generation_;
        }
        wake_.notify_all();
        drain(cut);
        std::unique_lock<std::mutex> lock(mutex_);
        done_.wait(lock, [this] { return pending_ == 0; });
        work_ = nullptr;
    }

private:
    void drain(const std::vector<CopyPiece>& cut)
    {
        for (size_t i = next_.fetch_add(1); i < cut.size(); i = next_.fetch_add(1))
            std::memcpy(cut[i].dst, cut[i].src, cut[i].bytes);
    }

    void work()
    {
        size_t seen = 0;
        for (;;) {
            const std::vector<CopyPiece>* cut;
            {
                std::unique_lock<std::mutex> lock(mutex_);
                wake_.wait(lock, [&] { return stop_ || generation_ != seen; });
                if (stop_)
                    return;
                seen = generation_;
                cut = work_;
            }
            drain(*cut);
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
    const std::vector<CopyPiece>* work_ = nullptr;
    std::atomic<size_t> next_{0};
    size_t pending_ = 0, generation_ = 0;
    bool stop_ = false;
};

} // namespace cs
