// Row and column passes built on the radix-16 register FFT (fft_r16.cuh):
// the first stage reads global memory directly, the last stage writes it
// directly, and shared memory only carries the exchanges between stages.
// 512 threads per CTA, up to 72 KB of shared memory, two CTAs per SM.
#include <algorithm>
#include <cstdlib>

#include "fft.cuh"
#include "fft_r16.cuh"
#include "tuning.h"

namespace mc3 {

namespace {
constexpr int kR16Threads = 512;
constexpr int kR16Budget = 72 * 1024;
// Sequences per CTA: one per N/16 threads.
__host__ __device__ constexpr int r16_batch(int n) { return kR16Threads / (n / 16); }
}  // namespace

bool r16_enabled() { return active_tuning().fft_r16 != 0; }

// ---------------------------------------------------------------------
// Column pass: NB adjacent columns per CTA; thread t -> column t % NB,
// slot t / NB, so a warp's loads cover NB adjacent columns of 32/NB rows.
// ---------------------------------------------------------------------
// PHASE / CROP: the phase-shift prologue and the crop epilogue are compiled
// in only where used.  T threads: 512 (two CTAs per SM) or 1024 (the wide
// form: twice the columns per CTA, so that each warp's loads and stores
// cover whole 32-byte sectors at 4096 points; one CTA per SM).
template <int H, bool PHASE, bool CROP, int T = kR16Threads>
__global__ void __launch_bounds__(T, kR16Threads * 2 / T) k_col_fft_r16(const float2* in, float2* out,
                                                                long pitch, int cmpX, Batch bt,
                                                                const float2* __restrict__ tw,
                                                                ColOps ops) {
  constexpr int NB = T / (H / 16);
  constexpr int LD = spad16_col_stride(H, NB);
  static_assert(NB * LD * (int)sizeof(float2) <= (T == kR16Threads ? kR16Budget : 2 * kR16Budget),
                "shared memory budget");
  extern __shared__ float2 sm[];
  const int item = blockIdx.y;
  const int c = threadIdx.x % NB;
  const int j = threadIdx.x / NB;
  const int x = blockIdx.x * NB + c;
  const bool live = x < cmpX;
  const float2* src = in + batch_in_off(bt, item) + x;
  const float2* ey = PHASE ? ops.ey + (long)item * H : nullptr;
  const float2 exx = (PHASE && live) ? ops.ex[(long)item * cmpX + x] : c2(1.f, 0.f);
  float2* dst = out + (long)item * bt.out_stride + x;
  float2* crop = CROP ? ops.crop + (long)item * ops.crop_x * ops.crop_y + x : nullptr;
  const bool in_crop = CROP && x < ops.crop_x;
  auto load = [&](int y) {
    if (!live) return c2(0.f, 0.f);
    float2 v = src[(long)y * pitch];
    if constexpr (PHASE) v = cmul(v, cmul(exx, ey[y]));
    return v;
  };
  auto store = [&](int y, float2 v) {
    if (!live) return;
    v = cscale(v, ops.scale);
    dst[(long)y * pitch] = v;
    if (CROP && in_crop) {
      int yo = -1;
      if (y <= ops.crop_y / 2) yo = y;
      else if (y > H - ops.crop_y / 2) yo = y - H + ops.crop_y;
      if (yo >= 0) crop[(long)yo * ops.crop_x] = v;
    }
  };
  float2* buf = sm + c * LD;
  if (ops.dir < 0) fft_r16<-1, H, false, false>(buf, j, tw, 1, load, store);
  else fft_r16<1, H, false, false>(buf, j, tw, 1, load, store);
}

// ---------------------------------------------------------------------
// Pipelined 4096-point column pass (persistent, one 1024-thread CTA per
// SM).  Work unit = 4 adjacent columns of one item.  While a unit is
// transformed in registers, the next unit's 4 x 4096 values are copied
// into a 128 KB staging buffer by 8-byte cp.async (each warp copies 8 rows
// x 32 bytes: whole sectors), so DRAM reads run under the arithmetic of the
// previous unit instead of in a separate load phase.  The two exchanges
// between the three radix-16 stages go through a second buffer that holds
// two columns at a time (columns 0-1, then 2-3), which keeps the whole CTA
// within 196 KB of shared memory.  The row pitch of the spectra (W/2+1
// complex) is odd for every even W, so the rows are not 16-byte aligned
// and the copies are 8-byte cp.async rather than tensor-map bulk copies.
// ---------------------------------------------------------------------
namespace {
constexpr int kPipeH = 4096;
constexpr int kPipeNB = 4;
constexpr int kPipeT = kPipeH / 16 * kPipeNB;  // 1024
constexpr int kPipeLDX = spad16_col_stride(kPipeH, 2);
constexpr size_t kPipeSmem =
    (size_t)kPipeH * kPipeNB * sizeof(float2) + 2 * (size_t)kPipeLDX * sizeof(float2);

__device__ __forceinline__ void cp_async8(float2* dst, const float2* src, int bytes) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Exchange after stage S: the 16 outputs in v (indices base + r*NS) are
// written to the exchange buffer and the next stage's 16 inputs read back,
// for columns 0-1 (c < 2) and then columns 2-3.
template <int S>
__device__ __forceinline__ void pipe_exchange(float2 (&v)[16], int j, int c, float2* xb) {
  using St = R16Stage<kPipeH, S>;
  constexpr int NS = St::NS;
  const int base = (j / NS) * NS * 16 + j % NS;
  float2* buf = xb + (c & 1) * kPipeLDX;
#pragma unroll
  for (int half = 0; half < 2; ++half) {
    if ((c >> 1) == half) {
#pragma unroll
      for (int r = 0; r < 16; ++r) buf[spad16(base + r * NS)] = v[r];
    }
    __syncthreads();
    if ((c >> 1) == half) {
#pragma unroll
      for (int r = 0; r < 16; ++r) v[r] = buf[spad16(r16_in_index<kPipeH, S + 1>(j, 0, r))];
    }
    __syncthreads();
  }
}
}  // namespace

template <int DIR, bool PHASE, bool CROP>
__global__ void __launch_bounds__(kPipeT, 1) k_col_fft_r16p(const float2* in, float2* out,
                                                            long pitch, int cmpX, Batch bt,
                                                            const float2* __restrict__ tw,
                                                            ColOps ops, int ngroups, int nunits) {
  static_assert(r16_nstages(kPipeH) == 3 && R16Stage<kPipeH, 0>::NB == 1, "three radix-16 stages");
  extern __shared__ float2 sm[];
  float2* pre = sm;                         // [kPipeH][kPipeNB]
  float2* xb = sm + kPipeH * kPipeNB;       // two columns, kPipeLDX apart
  const int c = threadIdx.x % kPipeNB;
  const int j = threadIdx.x / kPipeNB;
  auto prefetch = [&](int u) {
    const int item = u / ngroups, x = (u % ngroups) * kPipeNB + c;
    const int bytes = x < cmpX ? 8 : 0;     // columns past cmpX are zero-filled
    const float2* src = in + batch_in_off(bt, item) + min(x, cmpX - 1) + (long)j * pitch;
#pragma unroll
    for (int r = 0; r < 16; ++r)
      cp_async8(pre + (j + 256 * r) * kPipeNB + c, src + (long)(256 * r) * pitch, bytes);
    cp_async_commit();
  };
  int u = blockIdx.x;
  if (u < nunits) prefetch(u);
  for (; u < nunits; u += gridDim.x) {
    const int item = u / ngroups, x = (u % ngroups) * kPipeNB + c;
    const bool live = x < cmpX;
    cp_async_wait_all();
    __syncthreads();
    float2 v[16];
    {
      const float2* ey = PHASE ? ops.ey + (long)item * kPipeH : nullptr;
      const float2 exx = (PHASE && live) ? ops.ex[(long)item * cmpX + x] : c2(1.f, 0.f);
#pragma unroll
      for (int r = 0; r < 16; ++r) {
        const int y = r16_in_index<kPipeH, 0>(j, 0, r);
        v[r] = pre[y * kPipeNB + c];
        if constexpr (PHASE) v[r] = cmul(v[r], cmul(exx, ey[y]));
      }
    }
    __syncthreads();                        // the staging buffer is free again
    if (u + (int)gridDim.x < nunits) prefetch(u + gridDim.x);
    auto none = [](int, float2) {};
    r16_compute<DIR, kPipeH, 0>(v, j, tw, 1, none);
    pipe_exchange<0>(v, j, c, xb);
    r16_compute<DIR, kPipeH, 1>(v, j, tw, 1, none);
    pipe_exchange<1>(v, j, c, xb);
    float2* dst = out + (long)item * bt.out_stride + x;
    float2* crop = CROP ? ops.crop + (long)item * ops.crop_x * ops.crop_y + x : nullptr;
    const bool in_crop = CROP && x < ops.crop_x;
    r16_compute<DIR, kPipeH, 2>(v, j, tw, 1, [&](int y, float2 w) {
      if (!live) return;
      w = cscale(w, ops.scale);
      dst[(long)y * pitch] = w;
      if (CROP && in_crop) {
        int yo = -1;
        if (y <= ops.crop_y / 2) yo = y;
        else if (y > kPipeH - ops.crop_y / 2) yo = y - kPipeH + ops.crop_y;
        if (yo >= 0) crop[(long)yo * ops.crop_x] = w;
      }
    });
  }
  cp_async_wait_all();
}

// ---------------------------------------------------------------------
// Row R2C: ROWS rows per CTA, M = W/2 complex points per row (the real row
// read as complex pairs), thread t -> row t / (M/16), slot t % (M/16).  The
// transform ends in shared memory for the paired post-processing, then the
// W/2+1 outputs of each row are stored.
// ---------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(kR16Threads, 2) k_row_r2c_r16(const float* __restrict__ in,
                                                                long in_pitch, float2* out,
                                                                long out_pitch, int H, Batch bt,
                                                                const float2* __restrict__ tw,
                                                                float scale) {
  constexpr int ROWS = r16_batch(M);
  constexpr int LD = spad16_len(M + 1);
  static_assert(ROWS * LD * (int)sizeof(float2) <= kR16Budget, "shared memory budget");
  extern __shared__ float2 sm[];
  const int item = blockIdx.y;
  const int rr = threadIdx.x / (M / 16);
  const int j = threadIdx.x % (M / 16);
  const int r0 = blockIdx.x * ROWS;
  const int nr = min(ROWS, H - r0);
  const bool live = rr < nr;
  const float* src = in + batch_in_off(bt, item) + (long)(r0 + rr) * in_pitch;
  const bool pair = ((reinterpret_cast<uintptr_t>(in + batch_in_off(bt, item)) & 7) == 0) &&
                    !(in_pitch & 1);
  auto load = [&](int m) {
    if (!live) return c2(0.f, 0.f);
    const float* p = src + 2 * m;
    return pair ? *reinterpret_cast<const float2*>(p) : c2(p[0], p[1]);
  };
  auto none = [](int, float2) {};
  // tw: the W-point table; the M-point stages read every second entry
  fft_r16<-1, M, false, true>(sm + rr * LD, j, tw, 2, load, none);
  constexpr int NP = M / 2 + 1;
  for (int t = threadIdx.x; t < nr * NP; t += kR16Threads) {
    const int r = t / NP, p = t % NP;
    r2c_post_pair<4>(sm + r * LD, M, p, tw, scale);
  }
  __syncthreads();
  float2* dst = out + (long)item * bt.out_stride + (long)r0 * out_pitch;
  for (int t = threadIdx.x; t < nr * (M + 1); t += kR16Threads) {
    const int r = t / (M + 1), k = t % (M + 1);
    dst[(long)r * out_pitch + k] = sm[r * LD + spad16(k)];
  }
}

// ---------------------------------------------------------------------
// Pipelined row R2C for rows of 4096 reals (M = 2048 complex points):
// persistent CTAs of 256 threads, two rows per unit, three CTAs per SM.
// Each row of the next unit arrives by one bulk copy (cp.async.bulk on the
// TMA unit, completing on an mbarrier), issued as soon as the current
// unit's first radix-16 stage has read the staging slots, so the copy runs
// under the rest of the transform, the post-processing and the stores.
// The padded rows (W+2 floats) start on 8-byte boundaries, so each copy
// starts at the 16-byte boundary at or below its row and ends at most 8
// bytes past the row's data, inside the row's own padding; the leading
// bytes belong to the previous row and are not used.  Every wait on the
// mbarrier is bounded; a CTA that gives up records it in g_fft_pipe_error
// (fft_pipe_error) and leaves.
// ---------------------------------------------------------------------
namespace {
constexpr int kRowPM = 2048;
constexpr int kRowPRows = 2;
constexpr int kRowPT = kRowPM / 16 * kRowPRows;  // 256
constexpr int kRowPSlot = 2 * kRowPM + 8;        // floats per staged row (16-byte multiple)
constexpr int kRowPLD = spad16_len(kRowPM + 1);
constexpr size_t kRowPStage = (size_t)kRowPRows * kRowPSlot * sizeof(float);
constexpr size_t kRowPSmem = 16 + kRowPStage + (size_t)kRowPRows * kRowPLD * sizeof(float2);
static_assert(kRowPStage % 16 == 0, "bulk copy destinations on 16-byte boundaries");
// Longest wait on one mbarrier (about 1 s at the B200's clock).
constexpr long long kPipeWaitCycles = 2000000000ll;

__device__ int g_fft_pipe_error;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Polls the mbarrier phase of the given parity; false after
// kPipeWaitCycles or once another CTA has recorded an error.
__device__ __forceinline__ bool pipe_wait(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  for (unsigned i = 0;; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if ((i & 255u) == 255u) {
      if (*reinterpret_cast<volatile int*>(&g_fft_pipe_error)) return false;
      if (clock64() - t0 > kPipeWaitCycles) return false;
    }
  }
}
}  // namespace

__global__ void __launch_bounds__(kRowPT, 3) k_row_r2c_r16p(const float* in, long in_pitch,
                                                            float2* out, long out_pitch, int H,
                                                            Batch bt, const float2* __restrict__ tw,
                                                            float scale, int rgroups, int nunits) {
  constexpr int M = kRowPM;
  extern __shared__ __align__(16) unsigned char smraw[];
  float* stage = reinterpret_cast<float*>(smraw + 16);
  float2* A = reinterpret_cast<float2*>(smraw + 16 + kRowPStage);
  const uint32_t bar = smem_addr(smraw);
  const int rr = threadIdx.x / (M / 16);
  const int j = threadIdx.x % (M / 16);
  // One arrive with the unit's byte count, then one copy per row.
  auto issue = [&](int u) {
    const int item = u / rgroups, r0 = (u % rgroups) * kRowPRows;
    const int nr = min(kRowPRows, H - r0);
    const float* base = in + batch_in_off(bt, item) + (long)r0 * in_pitch;
    uint32_t total = 0;
    for (int r = 0; r < nr; ++r) {
      const uintptr_t a = reinterpret_cast<uintptr_t>(base + (long)r * in_pitch);
      total += ((uint32_t)(a & 15) + 2 * M * 4 + 15) & ~15u;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(total)
                 : "memory");
    for (int r = 0; r < nr; ++r) {
      const uintptr_t a = reinterpret_cast<uintptr_t>(base + (long)r * in_pitch);
      const uint32_t lead = (uint32_t)(a & 15);
      const uint32_t bytes = (lead + 2 * M * 4 + 15) & ~15u;
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              smem_addr(stage + r * kRowPSlot)),
          "l"(a - lead), "r"(bytes), "r"(bar)
          : "memory");
    }
  };
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  int u = blockIdx.x;
  if (threadIdx.x == 0 && u < nunits) issue(u);
  for (int k = 0; u < nunits; u += gridDim.x, ++k) {
    const bool ok = pipe_wait(bar, (uint32_t)(k & 1));
    // also the barrier after the previous unit's stores from A
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) atomicOr(&g_fft_pipe_error, 1);
      return;
    }
    const int item = u / rgroups, r0 = (u % rgroups) * kRowPRows;
    const int nr = min(kRowPRows, H - r0);
    const bool live = rr < nr;
    const uintptr_t a = reinterpret_cast<uintptr_t>(in + batch_in_off(bt, item) +
                                                    (long)(r0 + rr) * in_pitch);
    const float* srow = stage + rr * kRowPSlot + ((a & 15) >> 2);
    auto load = [&](int m) {
      return live ? *reinterpret_cast<const float2*>(srow + 2 * m) : c2(0.f, 0.f);
    };
    auto none = [](int, float2) {};
    const int next = u + (int)gridDim.x;
    auto after_first = [&]() {
      if (threadIdx.x == 0 && next < nunits) issue(next);
    };
    fft_r16<-1, M, false, true>(A + rr * kRowPLD, j, tw, 2, load, none, after_first);
    constexpr int NP = M / 2 + 1;
    for (int t = threadIdx.x; t < nr * NP; t += kRowPT) {
      const int r = t / NP, p = t % NP;
      r2c_post_pair<4>(A + r * kRowPLD, M, p, tw, scale);
    }
    __syncthreads();
    float2* dst = out + (long)item * bt.out_stride + (long)r0 * out_pitch;
    for (int t = threadIdx.x; t < nr * (M + 1); t += kRowPT) {
      const int r = t / (M + 1), kk = t % (M + 1);
      dst[(long)r * out_pitch + kk] = A[r * kRowPLD + spad16(kk)];
    }
  }
}

// Pipelined row C2R for rows of 4096 reals, the counterpart of
// k_row_r2c_r16p: the next unit's half-spectrum rows (2049 complex) arrive
// by bulk copies issued once the current unit's rows have been moved into
// the padded work buffer.  A row that starts on a 16-byte boundary is copied
// without its Nyquist term (2048 values: the whole row would end 8 bytes
// into the next one), and that term is read directly; a row that starts 8
// bytes past a boundary is copied with the previous row's last value in
// front, which is not used.
__global__ void __launch_bounds__(kRowPT, 3) k_row_c2r_r16p(const float2* in, long in_pitch,
                                                            float* out, long out_pitch, int H,
                                                            Batch bt, const float2* __restrict__ tw,
                                                            int keep_im, int rgroups, int nunits) {
  constexpr int M = kRowPM;
  constexpr int SLOT = kRowPSlot / 2;  // float2 per staged row
  extern __shared__ __align__(16) unsigned char smraw[];
  float2* stage = reinterpret_cast<float2*>(smraw + 16);
  float2* A = reinterpret_cast<float2*>(smraw + 16 + kRowPStage);
  const uint32_t bar = smem_addr(smraw);
  const int rr = threadIdx.x / (M / 16);
  const int j = threadIdx.x % (M / 16);
  auto row_bytes = [](uintptr_t a) -> uint32_t { return (a & 15) ? 8u + 8u * (M + 1) : 8u * M; };
  auto issue = [&](int u) {
    const int item = u / rgroups, r0 = (u % rgroups) * kRowPRows;
    const int nr = min(kRowPRows, H - r0);
    const float2* base = in + batch_in_off(bt, item) + (long)r0 * in_pitch;
    uint32_t total = 0;
    for (int r = 0; r < nr; ++r) total += row_bytes(reinterpret_cast<uintptr_t>(base + (long)r * in_pitch));
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(total)
                 : "memory");
    for (int r = 0; r < nr; ++r) {
      const uintptr_t a = reinterpret_cast<uintptr_t>(base + (long)r * in_pitch);
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              smem_addr(stage + r * SLOT)),
          "l"(a & ~(uintptr_t)15), "r"(row_bytes(a)), "r"(bar)
          : "memory");
    }
  };
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  int u = blockIdx.x;
  if (threadIdx.x == 0 && u < nunits) issue(u);
  for (int k = 0; u < nunits; u += gridDim.x, ++k) {
    const bool ok = pipe_wait(bar, (uint32_t)(k & 1));
    // also the barrier after the previous unit's last stage read A
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) atomicOr(&g_fft_pipe_error, 1);
      return;
    }
    const int item = u / rgroups, r0 = (u % rgroups) * kRowPRows;
    const int nr = min(kRowPRows, H - r0);
    const float2* src = in + batch_in_off(bt, item) + (long)r0 * in_pitch;
    for (int t = threadIdx.x; t < nr * (M + 1); t += kRowPT) {
      const int r = t / (M + 1), kk = t % (M + 1);
      const float2* row = src + (long)r * in_pitch;
      const bool lead = (reinterpret_cast<uintptr_t>(row) & 15) != 0;
      A[r * kRowPLD + spad16(kk)] =
          (kk == M && !lead) ? row[M] : stage[r * SLOT + (lead ? 1 : 0) + kk];
    }
    __syncthreads();  // the staging slots are free again
    const int next = u + (int)gridDim.x;
    if (threadIdx.x == 0 && next < nunits) issue(next);
    constexpr int NP = M / 2 + 1;
    for (int t = threadIdx.x; t < nr * NP; t += kRowPT) {
      const int r = t / NP, p = t % NP;
      c2r_pre_pair<4>(A + r * kRowPLD, M, p, tw, keep_im);
    }
    __syncthreads();
    const bool live = rr < nr;
    float* dst = out + (long)item * bt.out_stride + (long)(r0 + rr) * out_pitch;
    const bool pair = ((reinterpret_cast<uintptr_t>(out + (long)item * bt.out_stride) & 7) == 0) &&
                      !(out_pitch & 1);
    auto none = [](int) { return c2(0.f, 0.f); };
    auto store = [&](int m, float2 v) {
      if (!live) return;
      float* p = dst + 2 * m;
      if (pair) {
        *reinterpret_cast<float2*>(p) = v;
      } else {
        p[0] = v.x;
        p[1] = v.y;
      }
    };
    fft_r16<1, M, true, false>(A + rr * kRowPLD, j, tw, 2, none, store);
  }
}

int fft_pipe_error(bool reset, int* flag) {
  int v = 0;
  MC3_CUDA(cudaMemcpyFromSymbol(&v, g_fft_pipe_error, sizeof(int)));
  if (reset && v) {
    const int z = 0;
    MC3_CUDA(cudaMemcpyToSymbol(g_fft_pipe_error, &z, sizeof(int)));
  }
  *flag = v;
  return kOk;
}

// ---------------------------------------------------------------------
// Row C2R (unnormalised): rows loaded to shared memory, paired
// pre-processing in place, then the transform from shared memory with the
// last stage storing real pairs straight to global memory.
// ---------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(kR16Threads, 2) k_row_c2r_r16(const float2* in, long in_pitch,
                                                                float* out, long out_pitch, int H,
                                                                Batch bt,
                                                                const float2* __restrict__ tw,
                                                                int keep_im) {
  constexpr int ROWS = r16_batch(M);
  constexpr int LD = spad16_len(M + 1);
  static_assert(ROWS * LD * (int)sizeof(float2) <= kR16Budget, "shared memory budget");
  extern __shared__ float2 sm[];
  const int item = blockIdx.y;
  const int r0 = blockIdx.x * ROWS;
  const int nr = min(ROWS, H - r0);
  const float2* src = in + batch_in_off(bt, item) + (long)r0 * in_pitch;
  for (int t = threadIdx.x; t < nr * (M + 1); t += kR16Threads) {
    const int r = t / (M + 1), k = t % (M + 1);
    sm[r * LD + spad16(k)] = src[(long)r * in_pitch + k];
  }
  __syncthreads();
  constexpr int NP = M / 2 + 1;
  for (int t = threadIdx.x; t < nr * NP; t += kR16Threads) {
    const int r = t / NP, p = t % NP;
    c2r_pre_pair<4>(sm + r * LD, M, p, tw, keep_im);
  }
  __syncthreads();
  const int rr = threadIdx.x / (M / 16);
  const int j = threadIdx.x % (M / 16);
  const bool live = rr < nr;
  float* dst = out + (long)item * bt.out_stride + (long)(r0 + rr) * out_pitch;
  const bool pair = ((reinterpret_cast<uintptr_t>(out + (long)item * bt.out_stride) & 7) == 0) &&
                    !(out_pitch & 1);
  auto none = [](int) { return c2(0.f, 0.f); };
  auto store = [&](int m, float2 v) {
    if (!live) return;
    float* p = dst + 2 * m;
    if (pair) {
      *reinterpret_cast<float2*>(p) = v;
    } else {
      p[0] = v.x;
      p[1] = v.y;
    }
  };
  fft_r16<1, M, true, false>(sm + rr * LD, j, tw, 2, none, store);
}

// ---------------------------------------------------------------------
// Launchers (compile-time lengths 256..4096 columns, 128..2048 row pairs).
// ---------------------------------------------------------------------
namespace {
template <int H, int T = kR16Threads>
int launch_col(const float2* in, float2* out, long pitch, int cmpX, const Batch& b,
               const float2* tw, const ColOps& ops, const char* name, cudaStream_t st) {
  constexpr int NB = T / (H / 16);
  const size_t smem = (size_t)NB * spad16_col_stride(H, NB) * sizeof(float2);
  dim3 grid(ceil_div(cmpX, NB), b.items);
  prof::Scope ps(name, (double)b.items * ((double)cmpX * H * 16.0 + (ops.crop ? (double)ops.crop_x * ops.crop_y * 8.0 : 0.0)), st);
  const bool phase = ops.ex && ops.ey, crop = ops.crop != nullptr;
#define MC3_COLK(P, C)                                                                   \
  {                                                                                      \
    MC3_TRY(set_smem_attr(k_col_fft_r16<H, P, C, T>, smem));                             \
    k_col_fft_r16<H, P, C, T><<<grid, T, smem, st>>>(in, out, pitch, cmpX, b, tw, ops);  \
  }
  if (phase && crop) MC3_COLK(true, true)
  else if (phase) MC3_COLK(true, false)
  else if (crop) MC3_COLK(false, true)
  else MC3_COLK(false, false)
#undef MC3_COLK
  MC3_CHECK_LAUNCH(name);
  return kOk;
}
int sm_count() {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
    n = 148;
  return n;
}
int launch_col_pipe(const float2* in, float2* out, long pitch, int cmpX, const Batch& b,
                    const float2* tw, const ColOps& ops, const char* name, cudaStream_t st) {
  const int ngroups = ceil_div(cmpX, kPipeNB);
  const long nunits_l = (long)ngroups * b.items;
  if (nunits_l > 0x7fffffffL) return kEUnsupported;
  const int nunits = (int)nunits_l;
  const int grid = std::min(nunits, sm_count());
  prof::Scope ps(name, (double)b.items * ((double)cmpX * kPipeH * 16.0 + (ops.crop ? (double)ops.crop_x * ops.crop_y * 8.0 : 0.0)), st);
  const bool phase = ops.ex && ops.ey, crop = ops.crop != nullptr;
#define MC3_PIPEK(D, P, C)                                                                  \
  {                                                                                         \
    MC3_TRY(set_smem_attr(k_col_fft_r16p<D, P, C>, kPipeSmem));                             \
    k_col_fft_r16p<D, P, C><<<grid, kPipeT, kPipeSmem, st>>>(in, out, pitch, cmpX, b, tw,   \
                                                             ops, ngroups, nunits);         \
  }
#define MC3_PIPED(D)                          \
  if (phase && crop) MC3_PIPEK(D, true, true) \
  else if (phase) MC3_PIPEK(D, true, false)   \
  else if (crop) MC3_PIPEK(D, false, true)    \
  else MC3_PIPEK(D, false, false)
  if (ops.dir < 0) {
    MC3_PIPED(-1)
  } else {
    MC3_PIPED(1)
  }
#undef MC3_PIPED
#undef MC3_PIPEK
  MC3_CHECK_LAUNCH(name);
  return kOk;
}
template <int M>
int launch_r2c(const float* in, long in_pitch, float2* out, long out_pitch, int H, const Batch& b,
               const float2* tw, float scale, const char* name, cudaStream_t st) {
  constexpr int ROWS = r16_batch(M);
  const size_t smem = (size_t)ROWS * spad16_len(M + 1) * sizeof(float2);
  MC3_TRY(set_smem_attr(k_row_r2c_r16<M>, smem));
  dim3 grid(ceil_div(H, ROWS), b.items);
  prof::Scope ps(name, (double)b.items * H * (2 * M * 4.0 + (M + 1) * 8.0), st);
  k_row_r2c_r16<M><<<grid, kR16Threads, smem, st>>>(in, in_pitch, out, out_pitch, H, b, tw, scale);
  MC3_CHECK_LAUNCH(name);
  return kOk;
}
// The pipelined R2C's copies need every row to start on an 8-byte boundary
// of a 16-byte-aligned buffer, with the row's 8 bytes of padding after it.
bool row_pipe_fits(const float* in, long in_pitch, int W, const Batch& b) {
  return W == 2 * kRowPM && (reinterpret_cast<uintptr_t>(in) & 15) == 0 && in_pitch % 2 == 0 &&
         in_pitch >= W + 2 && (b.nf <= 1 || b.in_stride % 2 == 0) && b.patch_off == nullptr;
}
int launch_r2c_pipe(const float* in, long in_pitch, float2* out, long out_pitch, int H,
                    const Batch& b, const float2* tw, float scale, cudaStream_t st) {
  const int rgroups = ceil_div(H, kRowPRows);
  const long nunits_l = (long)rgroups * b.items;
  if (nunits_l > 0x7fffffffL) return kEUnsupported;
  const int nunits = (int)nunits_l;
  const int grid = std::min(nunits, 3 * sm_count());
  MC3_TRY(set_smem_attr(k_row_r2c_r16p, kRowPSmem));
  prof::Scope ps("k_row_r2c_r16p<2048>", (double)b.items * H * (2 * kRowPM * 4.0 + (kRowPM + 1) * 8.0), st);
  k_row_r2c_r16p<<<grid, kRowPT, kRowPSmem, st>>>(in, in_pitch, out, out_pitch, H, b, tw, scale,
                                                  rgroups, nunits);
  MC3_CHECK_LAUNCH("k_row_r2c_r16p<2048>");
  return kOk;
}
int launch_c2r_pipe(const float2* in, long in_pitch, float* out, long out_pitch, int H,
                    const Batch& b, const float2* tw, int keep_im, cudaStream_t st) {
  const int rgroups = ceil_div(H, kRowPRows);
  const long nunits_l = (long)rgroups * b.items;
  if (nunits_l > 0x7fffffffL) return kEUnsupported;
  const int nunits = (int)nunits_l;
  const int grid = std::min(nunits, 3 * sm_count());
  MC3_TRY(set_smem_attr(k_row_c2r_r16p, kRowPSmem));
  prof::Scope ps("k_row_c2r_r16p<2048>", (double)b.items * H * (2 * kRowPM * 4.0 + (kRowPM + 1) * 8.0), st);
  k_row_c2r_r16p<<<grid, kRowPT, kRowPSmem, st>>>(in, in_pitch, out, out_pitch, H, b, tw, keep_im,
                                                  rgroups, nunits);
  MC3_CHECK_LAUNCH("k_row_c2r_r16p<2048>");
  return kOk;
}
template <int M>
int launch_c2r(const float2* in, long in_pitch, float* out, long out_pitch, int H, const Batch& b,
               const float2* tw, const char* name, int keep_im, cudaStream_t st) {
  constexpr int ROWS = r16_batch(M);
  const size_t smem = (size_t)ROWS * spad16_len(M + 1) * sizeof(float2);
  MC3_TRY(set_smem_attr(k_row_c2r_r16<M>, smem));
  dim3 grid(ceil_div(H, ROWS), b.items);
  prof::Scope ps(name, (double)b.items * H * (2 * M * 4.0 + (M + 1) * 8.0), st);
  k_row_c2r_r16<M><<<grid, kR16Threads, smem, st>>>(in, in_pitch, out, out_pitch, H, b, tw, keep_im);
  MC3_CHECK_LAUNCH(name);
  return kOk;
}
}  // namespace

int col_fft_r16(const float2* in, float2* out, long pitch, int cmpX, int H, const Batch& b,
                const ColOps& ops, cudaStream_t st) {
  if (!r16_enabled()) return kEUnsupported;
  FftDesc d;
  switch (H) {
    case 256: case 512: case 1024: case 2048: case 4096: break;
    default: return kEUnsupported;
  }
  MC3_TRY(make_desc(H, H, &d));
  switch (H) {
    case 256: return launch_col<256>(in, out, pitch, cmpX, b, d.tw, ops, "k_col_fft_r16<256>", st);
    case 512: return launch_col<512>(in, out, pitch, cmpX, b, d.tw, ops, "k_col_fft_r16<512>", st);
    case 1024: return launch_col<1024>(in, out, pitch, cmpX, b, d.tw, ops, "k_col_fft_r16<1024>", st);
    case 2048: return launch_col<2048>(in, out, pitch, cmpX, b, d.tw, ops, "k_col_fft_r16<2048>", st);
    default:
      if (active_tuning().col_wide == 2)
        return launch_col_pipe(in, out, pitch, cmpX, b, d.tw, ops, "k_col_fft_r16p<4096>", st);
      if (active_tuning().col_wide)
        return launch_col<4096, 2 * kR16Threads>(in, out, pitch, cmpX, b, d.tw, ops,
                                                 "k_col_fft_r16w<4096>", st);
      return launch_col<4096>(in, out, pitch, cmpX, b, d.tw, ops, "k_col_fft_r16<4096>", st);
  }
}

int row_r2c_r16(const float* in, long in_pitch, float2* out, long out_pitch, int W, int H,
                const Batch& b, float scale, cudaStream_t st) {
  if (!r16_enabled()) return kEUnsupported;
  const int M = W / 2;
  switch (M) {
    case 256: case 512: case 1024: case 2048: break;
    default: return kEUnsupported;
  }
  FftDesc d;
  MC3_TRY(make_desc(M, W, &d));
  switch (M) {
    case 256: return launch_r2c<256>(in, in_pitch, out, out_pitch, H, b, d.tw, scale, "k_row_r2c_r16<256>", st);
    case 512: return launch_r2c<512>(in, in_pitch, out, out_pitch, H, b, d.tw, scale, "k_row_r2c_r16<512>", st);
    case 1024: return launch_r2c<1024>(in, in_pitch, out, out_pitch, H, b, d.tw, scale, "k_row_r2c_r16<1024>", st);
    default:
      if (active_tuning().row_pipe && row_pipe_fits(in, in_pitch, W, b))
        return launch_r2c_pipe(in, in_pitch, out, out_pitch, H, b, d.tw, scale, st);
      return launch_r2c<2048>(in, in_pitch, out, out_pitch, H, b, d.tw, scale, "k_row_r2c_r16<2048>", st);
  }
}

int row_c2r_r16(const float2* in, long in_pitch, float* out, long out_pitch, int W, int H,
                const Batch& b, cudaStream_t st, int keep_im) {
  if (!r16_enabled()) return kEUnsupported;
  const int M = W / 2;
  switch (M) {
    case 256: case 512: case 1024: case 2048: break;
    default: return kEUnsupported;
  }
  FftDesc d;
  MC3_TRY(make_desc(M, W, &d));
  switch (M) {
    case 256: return launch_c2r<256>(in, in_pitch, out, out_pitch, H, b, d.tw, "k_row_c2r_r16<256>", keep_im, st);
    case 512: return launch_c2r<512>(in, in_pitch, out, out_pitch, H, b, d.tw, "k_row_c2r_r16<512>", keep_im, st);
    case 1024: return launch_c2r<1024>(in, in_pitch, out, out_pitch, H, b, d.tw, "k_row_c2r_r16<1024>", keep_im, st);
    default:
      // the copies need a 16-byte-aligned buffer; rows then start on 8-byte boundaries
      if (active_tuning().row_pipe && (reinterpret_cast<uintptr_t>(in) & 15) == 0 &&
          b.patch_off == nullptr)
        return launch_c2r_pipe(in, in_pitch, out, out_pitch, H, b, d.tw, keep_im, st);
      return launch_c2r<2048>(in, in_pitch, out, out_pitch, H, b, d.tw, "k_row_c2r_r16<2048>", keep_im, st);
  }
}

}  // namespace mc3
