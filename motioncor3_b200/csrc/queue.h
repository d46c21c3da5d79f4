// Movie queue of a context (mc3_submit / mc3_wait): the role of the
// reference's processing thread and its package queue
// (CProcessThread::ThreadMain, CProcessThread.cpp:39-80), which takes the
// loaded movies in order and processes them, with the loader thread copying
// the next movie meanwhile (MrcUtil/CLoadCryoEMStack.cpp:104-152).
#pragma once
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>

#include "engine.h"

namespace mc3 {

class MovieQueue {
 public:
  explicit MovieQueue(Engine* e);
  ~MovieQueue();  // finishes the queued movies, then joins the worker
  // Hands a movie to the worker; returns its ticket in *ticket.
  int submit(const mc3_movie& mv, mc3_result* out, int* ticket);
  // Blocks until the ticket's movie is done; its status, and the time from
  // submission to the end of processing in *latency_ms.
  int wait(int ticket, double* latency_ms);
  // Tickets submitted and not yet waited for.
  int outstanding();

 private:
  using Clock = std::chrono::steady_clock;
  struct Job {
    int ticket;
    mc3_movie mv;
    mc3_result* out;
    Clock::time_point t_submit, t_done;
    int status = kOk;
    bool done = false;
    bool prefetched = false;
  };
  void run();

  Engine* eng_;
  std::mutex mu_;
  std::condition_variable cv_work_, cv_done_;
  std::deque<Job*> pending_;     // submitted, not started (in order)
  std::map<int, Job*> jobs_;     // every job not yet waited for
  bool stop_ = false;
  int next_ticket_ = 1;
  std::thread worker_;           // started last
};

}  // namespace mc3
