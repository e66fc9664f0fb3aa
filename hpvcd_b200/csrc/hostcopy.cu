// hostcopy.cu -- the host copy pool (host code only; see hostcopy.h).
//
// A job is a list of pieces of at most kPiece bytes with an atomic cursor.
// The caller queues its job, then takes pieces itself; idle workers take the
// front job's pieces until its cursor runs past the end.  The caller returns
// once the done count reaches the piece count, so every byte has landed even
// when a worker still holds the job.
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "hostcopy.h"

namespace hpvcd_host {
namespace {

constexpr size_t kPiece = 1u << 20;
// below this a job is copied inline: waking workers costs more than it saves
constexpr size_t kInline = 2u << 20;

struct Job {
    std::vector<CopyTask> pieces;
    std::atomic<size_t> next{0};
    std::atomic<size_t> done{0};
    std::mutex mu;
    std::condition_variable cv;

    // Copy pieces until none are left; true when this call copied the last.
    void work() {
        const size_t n = pieces.size();
        for (size_t i = next.fetch_add(1); i < n; i = next.fetch_add(1)) {
            memcpy(pieces[i].dst, pieces[i].src, pieces[i].bytes);
            if (done.fetch_add(1) + 1 == n) {
                std::lock_guard<std::mutex> l(mu);
                cv.notify_all();
            }
        }
    }
};

class Pool {
  public:
    explicit Pool(int threads) : n_(threads) {
        for (int i = 0; i < n_; ++i) std::thread([this]() { loop(); }).detach();
    }
    int threads() const { return n_; }

    void run(const std::shared_ptr<Job>& j) {
        if (n_ > 0) {
            {
                std::lock_guard<std::mutex> l(mu_);
                q_.push_back(j);
            }
            cv_.notify_all();
        }
        j->work();
        std::unique_lock<std::mutex> l(j->mu);
        j->cv.wait(l, [&]() { return j->done.load() == j->pieces.size(); });
    }

  private:
    void loop() {
        for (;;) {
            std::shared_ptr<Job> j;
            {
                std::unique_lock<std::mutex> l(mu_);
                cv_.wait(l, [&]() { return !q_.empty(); });
                j = q_.front();
                if (j->next.load() >= j->pieces.size()) {  // exhausted: drop it from the queue
                    q_.pop_front();
                    continue;
                }
            }
            j->work();
            std::lock_guard<std::mutex> l(mu_);
            auto it = std::find(q_.begin(), q_.end(), j);
            if (it != q_.end()) q_.erase(it);
        }
    }

    int n_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<std::shared_ptr<Job>> q_;
};

Pool& pool() {
    // leaked on purpose: detached workers may still be parked in it at exit
    static Pool* p = []() {
        int n;
        if (const char* e = getenv("HPVCD_COPY_THREADS")) {
            n = std::max(0, std::min(64, atoi(e)));
        } else {
            const unsigned hw = std::thread::hardware_concurrency();
            n = std::max(1, std::min(8, (int)(hw ? hw : 2) / 2));
        }
        return new Pool(n);
    }();
    return *p;
}

}  // namespace

void parallel_copy(const CopyTask* tasks, size_t n) {
    size_t total = 0;
    for (size_t i = 0; i < n; ++i) total += tasks[i].bytes;
    if (total < kInline || pool().threads() == 0) {
        for (size_t i = 0; i < n; ++i)
            if (tasks[i].bytes) memcpy(tasks[i].dst, tasks[i].src, tasks[i].bytes);
        return;
    }
    auto j = std::make_shared<Job>();
    j->pieces.reserve(total / kPiece + n);
    for (size_t i = 0; i < n; ++i) {
        unsigned char* d = (unsigned char*)tasks[i].dst;
        const unsigned char* s = (const unsigned char*)tasks[i].src;
        for (size_t o = 0; o < tasks[i].bytes; o += kPiece)
            j->pieces.push_back(CopyTask{d + o, s + o, std::min(kPiece, tasks[i].bytes - o)});
    }
    pool().run(j);
}

int copy_threads() { return pool().threads(); }

}  // namespace hpvcd_host
