// Movie queue: one worker thread per context processes submitted movies in
// submission order.  Before each movie is processed, the raw frames of the
// movie queued after it start their host->device copy on the engine's copy
// stream (Engine::prefetch), so that copy overlaps this movie's kernels;
// movies of any size follow one another (the engine's buffers grow to the
// largest geometry seen and are reused).
#include "queue.h"

namespace mc3 {

MovieQueue::MovieQueue(Engine* e) : eng_(e) { worker_ = std::thread([this] { run(); }); }

MovieQueue::~MovieQueue() {
  {
    std::lock_guard<std::mutex> lk(mu_);
    stop_ = true;
  }
  cv_work_.notify_all();
  if (worker_.joinable()) worker_.join();
  for (auto& kv : jobs_) delete kv.second;
}

int MovieQueue::submit(const mc3_movie& mv, mc3_result* out, int* ticket) {
  Job* j = new (std::nothrow) Job;
  if (!j) return kENoMem;
  {
    std::lock_guard<std::mutex> lk(mu_);
    j->ticket = next_ticket_++;
    j->mv = mv;
    j->out = out;
    j->t_submit = Clock::now();
    jobs_[j->ticket] = j;
    pending_.push_back(j);
    *ticket = j->ticket;
  }
  cv_work_.notify_one();
  return kOk;
}

int MovieQueue::wait(int ticket, double* latency_ms) {
  std::unique_lock<std::mutex> lk(mu_);
  auto it = jobs_.find(ticket);
  if (it == jobs_.end()) return kEInval;
  Job* j = it->second;
  cv_done_.wait(lk, [&] { return j->done; });
  const int s = j->status;
  if (latency_ms)
    *latency_ms = std::chrono::duration<double, std::milli>(j->t_done - j->t_submit).count();
  jobs_.erase(it);
  delete j;
  return s;
}

int MovieQueue::outstanding() {
  std::lock_guard<std::mutex> lk(mu_);
  return (int)jobs_.size();
}

void MovieQueue::run() {
  for (;;) {
    Job* j = nullptr;
    Job* next = nullptr;
    {
      std::unique_lock<std::mutex> lk(mu_);
      cv_work_.wait(lk, [&] { return stop_ || !pending_.empty(); });
      if (pending_.empty()) return;  // stop requested and nothing left
      j = pending_.front();
      pending_.pop_front();
      if (!pending_.empty()) next = pending_.front();
    }
    int s = kOk;
    // this movie's copy (if it was not started while the previous one ran),
    // then the next movie's, both on the copy stream
    if (!j->prefetched && !j->mv.on_device) {
      s = eng_->prefetch(j->mv);
      j->prefetched = s == kOk;
    }
    if (s == kOk && next && !next->mv.on_device && eng_->prefetch(next->mv) == kOk) {
      std::lock_guard<std::mutex> lk(mu_);
      next->prefetched = true;
    }
    if (s == kOk) s = eng_->process(j->mv, j->out);
    if (s != kOk) {
      // a movie that failed before reading its prefetched frames would leave
      // the copies out of order: drop them, the next movie copies again
      eng_->drop_prefetched();
      std::lock_guard<std::mutex> lk(mu_);
      if (next) next->prefetched = false;
    }
    {
      std::lock_guard<std::mutex> lk(mu_);
      j->status = s;
      j->t_done = Clock::now();
      j->done = true;
    }
    cv_done_.notify_all();
  }
}

}  // namespace mc3
