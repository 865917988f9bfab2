// pl_budget.h -- a soft device-memory budget shared by the states of a batch
// or a serving loop.
#pragma once

#include <chrono>
#include <condition_variable>
#include <cstddef>
#include <mutex>

namespace pl {

// The states of a batch count their buffers against `limit`.  A state that
// must grow past the limit waits until other states release memory, unless
// every other holder is waiting as well; then it proceeds, so the batch
// cannot deadlock (the limit is set below the device's memory, so a short
// overshoot still fits).
struct MemBudget {
    std::mutex mu;
    std::condition_variable cv;
    size_t limit = 0;
    size_t used = 0;
    size_t peak = 0;
    int holders = 0;
    int waiting = 0;
    unsigned long long waits = 0;
    size_t reserved = 0;  // admission reserves of the running jobs

    // Replace `old_bytes` held by the caller with `new_bytes`.
    void resize(size_t old_bytes, size_t new_bytes) {
        std::unique_lock<std::mutex> lock(mu);
        if (new_bytes > old_bytes) {
            bool counted = false;
            while (used - old_bytes + new_bytes > limit && waiting + 1 < holders) {
                if (!counted) {
                    ++waits;
                    counted = true;
                }
                ++waiting;
                cv.wait_for(lock, std::chrono::milliseconds(50));
                --waiting;
            }
        }
        used = used - old_bytes + new_bytes;
        if (used > peak) peak = used;
        if (new_bytes < old_bytes) cv.notify_all();
    }
    // A job starts holding memory: it needs `need` more bytes than its lane
    // already holds (its admission reserve).  Wait while that does not fit
    // beside the running jobs -- the larger of what they hold and what they
    // reserved at admission; a job is always admitted when no other job
    // runs.  Returns whether the job was deferred.
    bool admit(size_t need = 0) {
        std::unique_lock<std::mutex> lock(mu);
        bool deferred = false;
        for (;;) {
            const size_t busy = used > reserved ? used : reserved;
            if (holders == 0 || (busy < limit && need <= limit - busy)) break;
            if (!deferred) {
                ++waits;
                deferred = true;
            }
            cv.wait_for(lock, std::chrono::milliseconds(50));
        }
        reserved += need;
        ++holders;
        return deferred;
    }
    void leave(size_t need = 0) {
        std::lock_guard<std::mutex> lock(mu);
        reserved -= need;
        --holders;
        cv.notify_all();
    }
};

}  // namespace pl
