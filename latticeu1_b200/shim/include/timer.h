// Wall-clock timer with the interface of the reference's Timer
// (reference include/timer.h, src/timer.cpp): start/stop/getElapsedTime*.
#ifndef U1_SHIM_TIMER_H
#define U1_SHIM_TIMER_H
#include <chrono>

class Timer {
  std::chrono::steady_clock::time_point t0_, t1_;
  bool running_ = false;

 public:
  Timer() : t0_(std::chrono::steady_clock::now()), t1_(t0_) {}
  void start() { t0_ = std::chrono::steady_clock::now(); running_ = true; }
  void stop() { t1_ = std::chrono::steady_clock::now(); running_ = false; }
  double getElapsedTimeInMicroSec() {
    const auto end = running_ ? std::chrono::steady_clock::now() : t1_;
    return std::chrono::duration<double, std::micro>(end - t0_).count();
  }
  double getElapsedTimeInMilliSec() { return getElapsedTimeInMicroSec() * 1e-3; }
  double getElapsedTimeInSec() { return getElapsedTimeInMicroSec() * 1e-6; }
  double getElapsedTime() { return getElapsedTimeInSec(); }
};

#endif
