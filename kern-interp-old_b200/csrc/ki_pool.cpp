#include "ki_pool.h"

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <vector>

namespace kib {

namespace {

// set while a thread runs pool work: a parallel_for issued from inside a job
// runs inline instead of waiting for the (busy) pool
thread_local bool t_in_job = false;

class Pool {
 public:
  Pool() {
    const unsigned hw = std::thread::hardware_concurrency();
    const int n = static_cast<int>(std::min(16u, hw > 1 ? hw - 1 : 0u));
    for (int i = 0; i < n; i++) workers_.emplace_back([this] { loop(); });
  }
  ~Pool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
      gen_++;
    }
    cv_.notify_all();
    for (std::thread& t : workers_) t.join();
  }
  int size() const { return static_cast<int>(workers_.size()) + 1; }

  void run(int n, int grain, const std::function<void(int, int)>& fn) {
    std::lock_guard<std::mutex> job_lock(job_mu_);  // one job at a time
    {
      std::lock_guard<std::mutex> lk(mu_);
      fn_ = &fn;
      n_ = n;
      grain_ = grain;
      next_.store(0);
      active_ = static_cast<int>(workers_.size());
      gen_++;
    }
    cv_.notify_all();
    work();
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [this] { return active_ == 0; });
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
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return gen_ != seen; });
        seen = gen_;
        if (stop_) return;
      }
      work();
      {
        std::lock_guard<std::mutex> lk(mu_);
        if (--active_ == 0) done_cv_.notify_one();
      }
    }
  }

  std::vector<std::thread> workers_;
  std::mutex mu_, job_mu_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(int, int)>* fn_ = nullptr;
  std::atomic<int> next_{0};
  int n_ = 0, grain_ = 1, active_ = 0;
  long long gen_ = 0;
  bool stop_ = false;
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
