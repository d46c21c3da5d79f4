// Per-kernel launch accounting: every launch wrapper reports its kernel
// name and algorithmic bytes; when profiling is enabled a pair of CUDA
// events brackets each launch on its stream, and the elapsed times are
// collected after the stream has been synchronised.
#pragma once
#include <cuda_runtime.h>

#include <string>

namespace mc3 {
namespace prof {

void enable(bool on);
bool enabled();
// Called around a kernel launch on `st`.  `bytes` = algorithmic HBM bytes
// the launch must move (each input read once, each output written once).
void begin(const char* kernel, cudaStream_t st);
void end(const char* kernel, double bytes, cudaStream_t st);
// Folds completed launches into the totals (call after a stream sync).
void collect();
void reset();
// {"kernel": [launches, total_ms, total_bytes], ...}
std::string json();
unsigned long long launches();

struct Scope {
  const char* k;
  double bytes;
  cudaStream_t st;
  Scope(const char* kernel, double b, cudaStream_t s) : k(kernel), bytes(b), st(s) { begin(k, st); }
  ~Scope() { end(k, bytes, st); }
};

}  // namespace prof
}  // namespace mc3
