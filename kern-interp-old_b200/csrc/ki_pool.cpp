#include "ki_pool.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <mutex>
#include <thread>
#include <vector>

namespace kib {

namespace {

// set while a thread runs pool work: a parallel_for issued from inside a job
// runs inline instead of waiting for the (busy) pool
thread_local bool t_in_job = false;

// Workers spin on the job counter for a while after each job before they
// sleep on the condition variable: the factorization issues many short
// jobs back to back (one or two per level and phase), and a sleeping
// worker takes tens of microseconds to wake.  The window (1 ms) outlasts
// most of a level's GPU work, during which the host only waits, so the next
// level's bookkeeping finds the workers awake (measured on a B200 host: the
// 256-problem batch factorization 65 -> 61 ms against a 200 us window).
class Pool {
 public:
  Pool() {
    // KI_THREADS (if set) is the total thread count, the caller's included
    const unsigned hw = std::thread::hardware_concurrency();
    int n = static_cast<int>(std::min(16u, hw > 1 ? hw - 1 : 0u));
    if (const char* e = std::getenv("KI_THREADS")) {
      const int want = std::atoi(e);
      if (want >= 1) n = std::min(want - 1, 63);
    }
    for (int i = 0; i < n; i++) workers_.emplace_back([this] { loop(); });
  }
  ~Pool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_.store(true);
      gen_.fetch_add(1);
    }
    cv_.notify_all();
    for (std::thread& t : workers_) t.join();
  }
  int size() const { return static_cast<int>(workers_.size()) + 1; }

  void run(int n, int grain, const std::function<void(int, int)>& fn) {
    std::lock_guard<std::mutex> job_lock(job_mu_);  // one job at a time
    fn_ = &fn;
    n_ = n;
    grain_ = grain;
    next_.store(0, std::memory_order_relaxed);
    active_.store(static_cast<int>(workers_.size()), std::memory_order_relaxed);
    {
      std::lock_guard<std::mutex> lk(mu_);
      gen_.fetch_add(1, std::memory_order_release);
    }
    if (sleepers_.load() > 0) cv_.notify_all();
    work();
    // the workers finish within microseconds of the last chunk
    for (int spin = 0; active_.load(std::memory_order_acquire) != 0; spin++)
      if (spin > 2000) std::this_thread::yield();
    fn_ = nullptr;
  }

 private:
  void work() {
    t_in_job = true;
    for (;;) {
      const int b = next_.fetch_add(grain_);
      if (b >= n_) break;
      (*fn_)(b, std::min(n_, b + grain_));
    }
    t_in_job = false;
  }
  void loop() {
    long long seen = 0;
    for (;;) {
      bool got = false;
      const auto t0 = std::chrono::steady_clock::now();
      for (int spin = 0;; spin++) {
        if (gen_.load(std::memory_order_acquire) != seen) {
          got = true;
          break;
        }
        if ((spin & 255) == 255 &&
            std::chrono::steady_clock::now() - t0 > std::chrono::microseconds(1000))
          break;
      }
      if (!got) {
        std::unique_lock<std::mutex> lk(mu_);
        sleepers_.fetch_add(1);
        cv_.wait(lk, [&] { return gen_.load() != seen; });
        sleepers_.fetch_sub(1);
      }
      seen = gen_.load(std::memory_order_acquire);
      if (stop_.load()) return;
      work();
      active_.fetch_sub(1, std::memory_order_release);
    }
  }

  std::vector<std::thread> workers_;
  std::mutex mu_, job_mu_;
  std::condition_variable cv_;
  const std::function<void(int, int)>* fn_ = nullptr;
  std::atomic<int> next_{0}, active_{0}, sleepers_{0};
  int n_ = 0, grain_ = 1;
  std::atomic<long long> gen_{0};
  std::atomic<bool> stop_{false};
};

Pool& pool() {
  static Pool p;
  return p;
}

}  // namespace

int pool_threads() { return pool().size(); }

void parallel_for(int n, int grain, const std::function<void(int, int)>& fn, int serial_below) {
  if (n <= 0) return;
  grain = std::max(1, grain);
  if (n < serial_below || n <= grain || t_in_job || pool().size() == 1) {
    fn(0, n);
    return;
  }
  pool().run(n, grain, fn);
}

}  // namespace kib
