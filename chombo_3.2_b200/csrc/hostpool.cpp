#include "hostpool.H"

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <deque>
#include <exception>
#include <mutex>
#include <thread>
#include <vector>

namespace cmg {

namespace {

struct Job {
  const std::function<void(size_t)>* fn = nullptr;
  size_t n = 0;
  std::atomic<size_t> next{0};
  std::atomic<size_t> done{0};
  int active = 0;  // workers inside this job (guarded by the pool mutex)
  std::mutex em;
  std::exception_ptr err;
};

class Pool {
 public:
  Pool() {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    // the caller works too: hw - 1 workers keep one thread per core (at most
    // 32 threads on one loop, beyond which these loops stop gaining)
    for (unsigned t = 0; t + 1 < std::min(hw, 32u); ++t) workers_.emplace_back([this]() { loop(); });
    for (auto& w : workers_) w.detach();  // they wait on the queue until the process ends
  }

  void run(size_t n, const std::function<void(size_t)>& fn) {
    if (n == 0) return;
    Job job;
    job.fn = &fn;
    job.n = n;
    const bool share = n > 1 && !workers_.empty();
    if (share) {
      {
        std::lock_guard<std::mutex> lk(m_);
        q_.push_back(&job);
      }
      cv_.notify_all();
    }
    work(job);
    if (share) {
      // no worker takes the job from here on; wait for the ones inside it
      std::unique_lock<std::mutex> lk(m_);
      auto it = std::find(q_.begin(), q_.end(), &job);
      if (it != q_.end()) q_.erase(it);
      doneCv_.wait(lk, [&]() { return job.active == 0 && job.done.load() == job.n; });
    }
    if (job.err) std::rethrow_exception(job.err);
  }

 private:
  std::mutex m_;
  std::condition_variable cv_, doneCv_;
  std::deque<Job*> q_;
  std::vector<std::thread> workers_;

  void work(Job& j) {
    for (size_t i = j.next++; i < j.n; i = j.next++) {
      try {
        (*j.fn)(i);
      } catch (...) {
        std::lock_guard<std::mutex> lk(j.em);
        if (!j.err) j.err = std::current_exception();
      }
      if (++j.done == j.n) {
        std::lock_guard<std::mutex> lk(m_);
        doneCv_.notify_all();
      }
    }
  }

  void loop() {
    std::unique_lock<std::mutex> lk(m_);
    for (;;) {
      cv_.wait(lk, [&]() { return !q_.empty(); });
      Job* j = q_.front();
      if (j->next.load() >= j->n) {  // every item claimed: the job leaves the queue
        q_.pop_front();
        continue;
      }
      ++j->active;
      lk.unlock();
      work(*j);
      lk.lock();
      if (--j->active == 0) doneCv_.notify_all();
    }
  }
};

Pool& pool() {
  static Pool* p = new Pool();  // never destroyed: its detached workers outlive static destructors
  return *p;
}

}  // namespace

void hostParallel(size_t n, const std::function<void(size_t)>& fn) { pool().run(n, fn); }

}  // namespace cmg
