// host_threads.h -- TEST INFRASTRUCTURE (CPU timing baseline only).  A
// persistent pool of host threads for the ORC_THREADS build of the oracle
// (oracle/Makefile: libab2_oracle_threads.so): parallel loops split [0, n)
// into one contiguous block per thread; the calling thread runs block 0.
// Thread count: AB2_CPU_THREADS if set, else std::thread::hardware_concurrency().
#pragma once

#include <condition_variable>
#include <cstdlib>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace ab2_oracle {

class HostPool {
 public:
  static HostPool& get() {
    static HostPool pool;
    return pool;
  }
  int size() const { return m_n; }

  // f(t, lo, hi) for every thread t and its block [lo, hi) of [0, n).
  void run(long long n, const std::function<void(int, long long, long long)>& f) {
    if (m_n == 1 || n < 4096) {
      f(0, 0, n);
      return;
    }
    {
      std::unique_lock<std::mutex> lk(m_mu);
      m_job = &f;
      m_len = n;
      m_pending = m_n - 1;
      ++m_gen;
    }
    m_cv.notify_all();
    f(0, 0, n / m_n);
    std::unique_lock<std::mutex> lk(m_mu);
    m_done.wait(lk, [this] { return m_pending == 0; });
    m_job = nullptr;
  }

  ~HostPool() {
    {
      std::unique_lock<std::mutex> lk(m_mu);
      m_stop = true;
      ++m_gen;
    }
    m_cv.notify_all();
    for (auto& t : m_threads) t.join();
  }

 private:
  HostPool() {
    const char* env = std::getenv("AB2_CPU_THREADS");
    int n = env ? std::atoi(env) : (int)std::thread::hardware_concurrency();
    m_n = n > 0 ? n : 1;
    for (int t = 1; t < m_n; ++t) m_threads.emplace_back([this, t] { worker(t); });
  }
  void worker(int t) {
    unsigned long long seen = 0;
    for (;;) {
      const std::function<void(int, long long, long long)>* job;
      long long n;
      {
        std::unique_lock<std::mutex> lk(m_mu);
        m_cv.wait(lk, [&] { return m_gen != seen; });
        seen = m_gen;
        if (m_stop) return;
        job = m_job;
        n = m_len;
      }
      (*job)(t, n * t / m_n, n * (t + 1) / m_n);
      std::unique_lock<std::mutex> lk(m_mu);
      if (--m_pending == 0) m_done.notify_one();
    }
  }

  int m_n = 1;
  std::vector<std::thread> m_threads;
  std::mutex m_mu;
  std::condition_variable m_cv, m_done;
  const std::function<void(int, long long, long long)>* m_job = nullptr;
  long long m_len = 0;
  int m_pending = 0;
  unsigned long long m_gen = 0;
  bool m_stop = false;
};

}  // namespace ab2_oracle
