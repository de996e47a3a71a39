/*
 * gardenia_timer.h -- wall-clock Timer with the reference's interface
 * (include/timer.h:19-48): Start / Stop / Seconds / Millisecs / Microsecs,
 * measured with gettimeofday like the reference.
 */
#ifndef GARDENIA_TIMER_H_
#define GARDENIA_TIMER_H_

#include <sys/time.h>

class Timer {
 public:
  void Start() { gettimeofday(&t0_, nullptr); }
  void Stop() { gettimeofday(&t1_, nullptr); }
  double Microsecs() const {
    return (double)(t1_.tv_sec - t0_.tv_sec) * 1e6 + (double)(t1_.tv_usec - t0_.tv_usec);
  }
  double Millisecs() const { return Microsecs() / 1e3; }
  double Seconds() const { return Microsecs() / 1e6; }

 private:
  struct timeval t0_ = {0, 0}, t1_ = {0, 0};
};

#define TIME_OP(t, op) \
  {                    \
    (t).Start();       \
    (op);              \
    (t).Stop();        \
  }

#endif
