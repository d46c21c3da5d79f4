// mc3_phase_shift_noalloc: the phase shift of mc3_phase_shift with its
// scratch (the shift and the two phase tables) in a fixed device array
// instead of cudaMalloc'd buffers.
//
// Who needs it: callers that must not allocate device memory while they
// run -- code that executes with a memory pool or budget fixed up front
// (an embedding application that owns all of the GPU's memory, a process
// whose allocations are reserved at start-up), and callers on paths where
// cudaMalloc/cudaFree would add a device-wide synchronisation and
// unpredictable latency.  mc3_phase_shift allocates and frees three small
// buffers per call; this entry point allocates nothing.
//
// The scratch is one file-scope __device__ array shared by every call on a
// device.  Its address is looked up once per device (cudaGetSymbolAddress,
// with that device current) on the first call made on that device and kept
// for the life of the process; a cudaDeviceReset (which ends the context the
// address belongs to) makes the kept address stale, so a process that resets
// a device must not call this entry point on it afterwards.  The shift is
// passed to the device as a kernel argument: no host memory is read.
#include <mutex>

#include "kernels.cuh"
#include "../../include/mc3.h"

namespace {

// Slots, in float2 (8-byte) units; each region starts on a 256-byte boundary.
constexpr int kShiftSlots = 32;                                       // (sx, sy) + padding
constexpr int kExSlots = (MC3_NOALLOC_MAX_CMP_X + 31) / 32 * 32;      // x phase table
constexpr int kEySlots = (MC3_NOALLOC_MAX_CMP_Y + 31) / 32 * 32;      // y phase table
constexpr int kScratchSlots = kShiftSlots + kExSlots + kEySlots;     // 24,640 -> 197,120 bytes

static __device__ __align__(256) float2 g_noalloc_scratch[kScratchSlots];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
float2* g_scratch_ptr[kMaxDevices] = {};

// Set-up for the current device: resolve the symbol's device address once.
int scratch_for_current_device(float2** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return MC3_ECUDA;
  if (dev < 0 || dev >= kMaxDevices) return MC3_EUNSUPPORTED;
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return MC3_ECUDA;
    g_scratch_ptr[dev] = static_cast<float2*>(p);
  }
  *out = g_scratch_ptr[dev];
  return MC3_OK;
}

// Writes the shift into its scratch slot from the kernel's own argument, so
// that no host memory is read by the device.
__global__ void k_noalloc_store_shift(float2* slot, float2 v) { *slot = v; }

}  // namespace

extern "C" int mc3_phase_shift_noalloc(const float* in, float* out, int cmp_x, int cmp_y,
                                       float sx, float sy, int accumulate, void* stream) {
  if (!in || !out || cmp_x < 2 || cmp_y < 1) return MC3_EINVAL;
  if (cmp_x > MC3_NOALLOC_MAX_CMP_X || cmp_y > MC3_NOALLOC_MAX_CMP_Y) return MC3_ETOOBIG;
  float2* base = nullptr;
  int s = scratch_for_current_device(&base);
  if (s != MC3_OK) return s;
  // Nothing in the scratch has to start at zero: the shift is written here
  // and both tables are fully written by k_phase_tables before they are read.
  float2* sh = base;
  float2* ex = base + kShiftSlots;
  float2* ey = ex + kExSlots;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  {
    mc3::prof::Scope ps("k_noalloc_store_shift", 8.0, st);
    k_noalloc_store_shift<<<1, 1, 0, st>>>(sh, make_float2(sx, sy));
    if (cudaGetLastError() != cudaSuccess) return MC3_ECUDA;
  }
  s = mc3::phase_tables(sh, 1, cmp_x, cmp_y, ex, ey, false, st);
  if (s != MC3_OK) return s;
  return mc3::phase_apply(reinterpret_cast<const float2*>(in), reinterpret_cast<float2*>(out),
                          cmp_x, cmp_y, ex, ey, accumulate != 0, st);
}
