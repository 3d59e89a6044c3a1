// Minimal std-based stand-in for the parts of boost.thread the reference uses
// (thread objects, a scoped-lock mutex, sleep). Only for the headless oracle build.
#pragma once
#include <thread>
#include <mutex>
#include <chrono>
#include <functional>
namespace boost {
class mutex : public std::mutex {
public:
  typedef std::unique_lock<std::mutex> scoped_lock;
};
class thread {
  std::thread t_;
public:
  thread() {}
  template <class F, class... A> explicit thread(F&& f, A&&... a) : t_(std::forward<F>(f), std::forward<A>(a)...) {}
  void join() { if (t_.joinable()) t_.join(); }
  bool joinable() const { return t_.joinable(); }
  ~thread() { if (t_.joinable()) t_.join(); }
};
namespace posix_time {
inline std::chrono::microseconds microseconds(long v) { return std::chrono::microseconds(v); }
}
namespace this_thread {
inline void sleep(std::chrono::microseconds d) { std::this_thread::sleep_for(d); }
}
}  // namespace boost
