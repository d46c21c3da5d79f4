// Per-kernel launch accounting (see profile.h).
#include "profile.h"

#include <atomic>
#include <cstdio>
#include <map>
#include <mutex>
#include <vector>

namespace mc3 {
namespace prof {

namespace {
struct Pending {
  std::string k;
  cudaEvent_t a, b;
  double bytes;
};
struct Total {
  unsigned long long n = 0;
  double ms = 0.0;
  double bytes = 0.0;
};
std::mutex mu;
bool on = false;
std::atomic<unsigned long long> count{0};
std::vector<Pending> pending;
std::vector<cudaEvent_t> pool;
std::map<std::string, Total> totals;
thread_local cudaEvent_t cur_a = nullptr;

cudaEvent_t get_event() {
  if (!pool.empty()) {
    cudaEvent_t e = pool.back();
    pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}
}  // namespace

void enable(bool o) {
  std::lock_guard<std::mutex> lk(mu);
  on = o;
}

bool enabled() { return on; }

void begin(const char* kernel, cudaStream_t st) {
  (void)kernel;
  if (!on) return;
  std::lock_guard<std::mutex> lk(mu);
  cur_a = get_event();
  cudaEventRecord(cur_a, st);
}

void end(const char* kernel, double bytes, cudaStream_t st) {
  count.fetch_add(1, std::memory_order_relaxed);
  if (!on || !cur_a) return;
  std::lock_guard<std::mutex> lk(mu);
  cudaEvent_t b = get_event();
  cudaEventRecord(b, st);
  pending.push_back(Pending{kernel, cur_a, b, bytes});
  cur_a = nullptr;
}

void collect() {
  std::lock_guard<std::mutex> lk(mu);
  for (auto& p : pending) {
    float ms = 0.f;
    if (cudaEventSynchronize(p.b) == cudaSuccess && cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
      Total& t = totals[p.k];
      t.n += 1;
      t.ms += ms;
      t.bytes += p.bytes;
    }
    pool.push_back(p.a);
    pool.push_back(p.b);
  }
  pending.clear();
  cudaGetLastError();
}

void reset() {
  collect();
  std::lock_guard<std::mutex> lk(mu);
  totals.clear();
}

std::string json() {
  collect();
  std::lock_guard<std::mutex> lk(mu);
  std::string s = "{";
  bool first = true;
  for (auto& kv : totals) {
    char buf[256];
    std::snprintf(buf, sizeof(buf), "%s\"%s\": [%llu, %.6f, %.1f]", first ? "" : ", ", kv.first.c_str(),
                  kv.second.n, kv.second.ms, kv.second.bytes);
    s += buf;
    first = false;
  }
  s += "}";
  return s;
}

unsigned long long launches() { return count.load(); }

}  // namespace prof
}  // namespace mc3
