// Shared-memory 2D FFT passes (see fft.cuh).
#include <cmath>
#include <map>
#include <mutex>
#include <vector>

#include "fft.cuh"
#include "tuning.h"

namespace mc3 {

namespace {
std::mutex g_tw_mu;
std::map<std::pair<int, int>, float2*> g_tw;  // (device, n) -> table
constexpr int kSmemBudget = 100 * 1024;
}  // namespace

const float2* twiddles(int n) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_tw_mu);
  auto key = std::make_pair(dev, n);
  auto it = g_tw.find(key);
  if (it != g_tw.end()) return it->second;
  std::vector<float2> h(n);
  for (int k = 0; k < n; ++k) {
    const double a = -2.0 * M_PI * (double)k / (double)n;
    h[k].x = (float)std::cos(a);
    h[k].y = (float)std::sin(a);
  }
  float2* d = nullptr;
  if (cudaMalloc(&d, sizeof(float2) * n) != cudaSuccess) return nullptr;
  if (cudaMemcpy(d, h.data(), sizeof(float2) * n, cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(d);
    return nullptr;
  }
  g_tw[key] = d;
  return d;
}

int make_desc(int n, int table_n, FftDesc* d) {
  d->n = n;
  d->nstages = fft_factorize(n, d->radix);
  if (d->nstages < 0 || table_n % n) return kEInval;
  d->tw = twiddles(table_n);
  if (!d->tw) return kENoMem;
  d->tws = table_n / n;
  return kOk;
}

// Global -> shared staging with kStage independent global loads in flight
// per thread before their shared-memory stores: element t of `total` is
// produced by load(t) and consumed by store(t, v).
template <int kStage, class LoadF, class StoreF>
__device__ __forceinline__ void staged_copy(int total, LoadF load, StoreF store) {
  const int step = blockDim.x;
  for (int t0 = threadIdx.x; t0 < total; t0 += step * kStage) {
    float2 v[kStage];
#pragma unroll
    for (int j = 0; j < kStage; ++j) {
      const int t = t0 + j * step;
      if (t < total) v[j] = load(t);
    }
#pragma unroll
    for (int j = 0; j < kStage; ++j) {
      const int t = t0 + j * step;
      if (t < total) store(t, v[j]);
    }
  }
}
constexpr int kStageLoads = 8;


// ---------------------------------------------------------------------
// Row real FFT (R2C): each CTA transforms `rows` rows of one batch item.
// ---------------------------------------------------------------------
__global__ void __launch_bounds__(256, 2) k_row_r2c(const float* __restrict__ in, long in_pitch, float2* out, long out_pitch,
                          int W, int H, int rows, Batch bt, FftDesc dM, float scale) {
  extern __shared__ float2 sm[];
  const int M = W / 2;
  const int ld = M + 1;
  float2* A = sm;
  float2* B = sm + rows * ld;
  const int item = blockIdx.y;
  const int r0 = blockIdx.x * rows;
  const int nr = min(rows, H - r0);
  const float* src = in + batch_in_off(bt, item) + (long)r0 * in_pitch;
  const bool pair = ((reinterpret_cast<uintptr_t>(src) & 7) == 0) && !(in_pitch & 1);
  staged_copy<kStageLoads>(
      nr * M,
      [&](int t) {
        const int r = t / M, m = t - r * M;
        const float* p = src + (long)r * in_pitch + 2 * m;
        return pair ? *reinterpret_cast<const float2*>(p) : c2(p[0], p[1]);
      },
      [&](int t, float2 v) {
        const int r = t / M, m = t - r * M;
        A[r * ld + m] = v;
      });
  __syncthreads();
  float2* R = cta_fft<-1>(A, B, dM, nr, 1, ld);
  float2* dst = out + (long)item * bt.out_stride + (long)r0 * out_pitch;
  for (int t = threadIdx.x; t < nr * (M + 1); t += blockDim.x) {
    const int r = t / (M + 1), k = t - r * (M + 1);
    float2 v = r2c_post(R + r * ld, M, k, dM.tw, 1);
    dst[(long)r * out_pitch + k] = cscale(v, scale);
  }
}

// ---------------------------------------------------------------------
// Row real inverse (C2R), unnormalised.
// ---------------------------------------------------------------------
__global__ void __launch_bounds__(256, 2) k_row_c2r(const float2* in, long in_pitch, float* out, long out_pitch, int W,
                          int H, int rows, Batch bt, FftDesc dM, int keep_im) {
  extern __shared__ float2 sm[];
  const int M = W / 2;
  const int ld = M + 1;
  float2* A = sm;
  float2* B = sm + rows * ld;
  const int item = blockIdx.y;
  const int r0 = blockIdx.x * rows;
  const int nr = min(rows, H - r0);
  const float2* src = in + batch_in_off(bt, item) + (long)r0 * in_pitch;
  staged_copy<kStageLoads>(
      nr * (M + 1),
      [&](int t) {
        const int r = t / (M + 1), k = t - r * (M + 1);
        return src[(long)r * in_pitch + k];
      },
      [&](int t, float2 v) {
        const int r = t / (M + 1), k = t - r * (M + 1);
        B[r * ld + k] = v;
      });
  __syncthreads();
  for (int t = threadIdx.x; t < nr * M; t += blockDim.x) {
    const int r = t / M, k = t - r * M;
    A[r * ld + k] = c2r_pre(B + r * ld, M, k, dM.tw, 1, keep_im);
  }
  __syncthreads();
  float2* R = cta_fft<1>(A, B, dM, nr, 1, ld);
  float* dst = out + (long)item * bt.out_stride + (long)r0 * out_pitch;
  for (int t = threadIdx.x; t < nr * M; t += blockDim.x) {
    const int r = t / M, m = t - r * M;
    const float2 v = R[r * ld + m];
    float* p = dst + (long)r * out_pitch + 2 * m;
    p[0] = v.x;
    p[1] = v.y;
  }
}

// ---------------------------------------------------------------------
// Column complex FFT with optional phase-shift prologue and crop epilogue.
// ---------------------------------------------------------------------
__global__ void __launch_bounds__(256, 2) k_col_fft(const float2* in, float2* out, long pitch, int cmpX, int H, int TX,
                          Batch bt, FftDesc dH, ColOps ops) {
  extern __shared__ float2 sm[];
  const int ld = H + 1;
  float2* A = sm;
  float2* B = sm + TX * ld;
  const int item = blockIdx.y;
  const int x0 = blockIdx.x * TX;
  const float2* src = in + batch_in_off(bt, item);
  const float2* ex = ops.ex ? ops.ex + (long)item * cmpX : nullptr;
  const float2* ey = ops.ey ? ops.ey + (long)item * H : nullptr;
  staged_copy<kStageLoads>(
      TX * H,
      [&](int t) {
        const int y = t / TX, c = t - y * TX;
        const int x = x0 + c;
        float2 v = c2(0.f, 0.f);
        if (x < cmpX) {
          v = src[(long)y * pitch + x];
          if (ex) v = cmul(v, cmul(ex[x], ey[y]));
        }
        return v;
      },
      [&](int t, float2 v) {
        const int y = t / TX, c = t - y * TX;
        A[c * ld + y] = v;
      });
  __syncthreads();
  float2* R = ops.dir < 0 ? cta_fft<-1>(A, B, dH, TX, 1, ld) : cta_fft<1>(A, B, dH, TX, 1, ld);
  float2* dst = out + (long)item * bt.out_stride;
  float2* crop = ops.crop ? ops.crop + (long)item * ops.crop_x * ops.crop_y : nullptr;
  for (int t = threadIdx.x; t < TX * H; t += blockDim.x) {
    const int y = t / TX, c = t - y * TX;
    const int x = x0 + c;
    if (x >= cmpX) continue;
    const float2 v = cscale(R[c * ld + y], ops.scale);
    dst[(long)y * pitch + x] = v;
    if (crop && x < ops.crop_x) {
      // GFourierResize2D::mGResize row mapping (Util/GFourierResize2D.cu:7-37)
      int yo = -1;
      if (y <= ops.crop_y / 2) yo = y;
      else if (y > H - ops.crop_y / 2) yo = y - H + ops.crop_y;
      if (yo >= 0) crop[(long)yo * ops.crop_x + x] = v;
    }
  }
}

// ---------------------------------------------------------------------
// In-place variants (plans made only of radices 2, 3, 4, 8): one padded
// buffer per sequence, register-staged stages.  Used whenever the plan
// allows; the ping-pong kernels above cover every other length.
// ---------------------------------------------------------------------
template <int MAXB>
__global__ void __launch_bounds__(512, 2) k_row_r2c_ip(const float* __restrict__ in, long in_pitch,
                                                    float2* out, long out_pitch, int W, int H,
                                                    int rows, Batch bt, FftDesc dM, float scale) {
  extern __shared__ float2 sm[];
  const int M = W / 2;
  const int ld = spad_len(M + 1);
  const int item = blockIdx.y;
  const int r0 = blockIdx.x * rows;
  const int nr = min(rows, H - r0);
  const float* src = in + batch_in_off(bt, item) + (long)r0 * in_pitch;
  // 8-byte loads when every row start is 8-byte aligned (patch extraction
  // offsets can be odd).
  const bool pair = ((reinterpret_cast<uintptr_t>(src) & 7) == 0) && !(in_pitch & 1);
  staged_copy<kStageLoads>(
      nr * M,
      [&](int t) {
        const int r = t / M, m = t - r * M;
        const float* p = src + (long)r * in_pitch + 2 * m;
        return pair ? *reinterpret_cast<const float2*>(p) : c2(p[0], p[1]);
      },
      [&](int t, float2 v) {
        const int r = t / M, m = t - r * M;
        sm[r * ld + spad(m)] = v;
      });
  __syncthreads();
  cta_fft_inplace<-1, MAXB>(sm, dM, nr, ld);
  const int np = M / 2 + 1;
  for (int t = threadIdx.x; t < nr * np; t += blockDim.x) {
    const int r = t / np, p = t - r * np;
    r2c_post_pair(sm + r * ld, M, p, dM.tw, scale);
  }
  __syncthreads();
  float2* dst = out + (long)item * bt.out_stride + (long)r0 * out_pitch;
  for (int t = threadIdx.x; t < nr * (M + 1); t += blockDim.x) {
    const int r = t / (M + 1), k = t - r * (M + 1);
    dst[(long)r * out_pitch + k] = sm[r * ld + spad(k)];
  }
}

template <int MAXB>
__global__ void __launch_bounds__(512, 2) k_row_c2r_ip(const float2* in, long in_pitch, float* out,
                                                    long out_pitch, int W, int H, int rows,
                                                    Batch bt, FftDesc dM, int keep_im) {
  extern __shared__ float2 sm[];
  const int M = W / 2;
  const int ld = spad_len(M + 1);
  const int item = blockIdx.y;
  const int r0 = blockIdx.x * rows;
  const int nr = min(rows, H - r0);
  const float2* src = in + batch_in_off(bt, item) + (long)r0 * in_pitch;
  staged_copy<kStageLoads>(
      nr * (M + 1),
      [&](int t) {
        const int r = t / (M + 1), k = t - r * (M + 1);
        return src[(long)r * in_pitch + k];
      },
      [&](int t, float2 v) {
        const int r = t / (M + 1), k = t - r * (M + 1);
        sm[r * ld + spad(k)] = v;
      });
  __syncthreads();
  const int np = M / 2 + 1;
  for (int t = threadIdx.x; t < nr * np; t += blockDim.x) {
    const int r = t / np, p = t - r * np;
    c2r_pre_pair(sm + r * ld, M, p, dM.tw, keep_im);
  }
  __syncthreads();
  cta_fft_inplace<1, MAXB>(sm, dM, nr, ld);
  float* dst = out + (long)item * bt.out_stride + (long)r0 * out_pitch;
  const bool pair = ((reinterpret_cast<uintptr_t>(dst) & 7) == 0) && !(out_pitch & 1);
  for (int t = threadIdx.x; t < nr * M; t += blockDim.x) {
    const int r = t / M, m = t - r * M;
    const float2 v = sm[r * ld + spad(m)];
    float* p = dst + (long)r * out_pitch + 2 * m;
    if (pair) {
      *reinterpret_cast<float2*>(p) = v;
    } else {
      p[0] = v.x;
      p[1] = v.y;
    }
  }
}

template <int MAXB>
__global__ void __launch_bounds__(512, 2) k_col_fft_ip(const float2* in, float2* out, long pitch,
                                                    int cmpX, int H, int TX, Batch bt, FftDesc dH,
                                                    ColOps ops) {
  extern __shared__ float2 sm[];
  const int ld = spad_len(H);
  const int item = blockIdx.y;
  const int x0 = blockIdx.x * TX;
  const float2* src = in + batch_in_off(bt, item);
  const float2* ex = ops.ex ? ops.ex + (long)item * cmpX : nullptr;
  const float2* ey = ops.ey ? ops.ey + (long)item * H : nullptr;
  staged_copy<kStageLoads>(
      TX * H,
      [&](int t) {
        const int y = t / TX, c = t - y * TX;
        const int x = x0 + c;
        float2 v = c2(0.f, 0.f);
        if (x < cmpX) {
          v = src[(long)y * pitch + x];
          if (ex) v = cmul(v, cmul(ex[x], ey[y]));
        }
        return v;
      },
      [&](int t, float2 v) {
        const int y = t / TX, c = t - y * TX;
        sm[c * ld + spad(y)] = v;
      });
  __syncthreads();
  if (ops.dir < 0) cta_fft_inplace<-1, MAXB>(sm, dH, TX, ld);
  else cta_fft_inplace<1, MAXB>(sm, dH, TX, ld);
  float2* dst = out + (long)item * bt.out_stride;
  float2* crop = ops.crop ? ops.crop + (long)item * ops.crop_x * ops.crop_y : nullptr;
  for (int t = threadIdx.x; t < TX * H; t += blockDim.x) {
    const int y = t / TX, c = t - y * TX;
    const int x = x0 + c;
    if (x >= cmpX) continue;
    const float2 v = cscale(sm[c * ld + spad(y)], ops.scale);
    dst[(long)y * pitch + x] = v;
    if (crop && x < ops.crop_x) {
      int yo = -1;
      if (y <= ops.crop_y / 2) yo = y;
      else if (y > H - ops.crop_y / 2) yo = y - H + ops.crop_y;
      if (yo >= 0) crop[(long)yo * ops.crop_x + x] = v;
    }
  }
}

// ---------------------------------------------------------------------
// Compile-time variants of the in-place kernels for power-of-two lengths
// (M complex per row, H per column): the sequence length, the sequences
// per CTA and the padded stride are template constants.
// ---------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(kCtThreads, 2) k_row_r2c_ct(const float* __restrict__ in,
                                                              long in_pitch, float2* out,
                                                              long out_pitch, int H, Batch bt,
                                                              const float2* __restrict__ tw,
                                                              float scale) {
  constexpr int LD = ct_spad_len(M + 1);
  constexpr int ROWS = ct_batch(LD);
  extern __shared__ float2 sm[];
  const int item = blockIdx.y;
  const int r0 = blockIdx.x * ROWS;
  const int nr = min(ROWS, H - r0);
  const float* src = in + batch_in_off(bt, item) + (long)r0 * in_pitch;
  const bool pair = ((reinterpret_cast<uintptr_t>(src) & 7) == 0) && !(in_pitch & 1);
  staged_copy<kStageLoads>(
      nr * M,
      [&](int t) {
        const int r = t / M, m = t % M;
        const float* p = src + (long)r * in_pitch + 2 * m;
        return pair ? *reinterpret_cast<const float2*>(p) : c2(p[0], p[1]);
      },
      [&](int t, float2 v) {
        const int r = t / M, m = t % M;
        sm[r * LD + spad(m)] = v;
      });
  __syncthreads();
  // tw: the 2M-point table, read every second entry by the M-point stages
  cta_fft_ct<-1, M, ROWS, kCtThreads, LD>(sm, tw, 2);
  constexpr int NP = M / 2 + 1;
  for (int t = threadIdx.x; t < nr * NP; t += kCtThreads) {
    const int r = t / NP, p = t % NP;
    r2c_post_pair(sm + r * LD, M, p, tw, scale);
  }
  __syncthreads();
  float2* dst = out + (long)item * bt.out_stride + (long)r0 * out_pitch;
  for (int t = threadIdx.x; t < nr * (M + 1); t += kCtThreads) {
    const int r = t / (M + 1), k = t % (M + 1);
    dst[(long)r * out_pitch + k] = sm[r * LD + spad(k)];
  }
}

template <int M>
__global__ void __launch_bounds__(kCtThreads, 2) k_row_c2r_ct(const float2* in, long in_pitch,
                                                              float* out, long out_pitch, int H,
                                                              Batch bt,
                                                              const float2* __restrict__ tw,
                                                              int keep_im) {
  constexpr int LD = ct_spad_len(M + 1);
  constexpr int ROWS = ct_batch(LD);
  extern __shared__ float2 sm[];
  const int item = blockIdx.y;
  const int r0 = blockIdx.x * ROWS;
  const int nr = min(ROWS, H - r0);
  const float2* src = in + batch_in_off(bt, item) + (long)r0 * in_pitch;
  staged_copy<kStageLoads>(
      nr * (M + 1),
      [&](int t) {
        const int r = t / (M + 1), k = t % (M + 1);
        return src[(long)r * in_pitch + k];
      },
      [&](int t, float2 v) {
        const int r = t / (M + 1), k = t % (M + 1);
        sm[r * LD + spad(k)] = v;
      });
  __syncthreads();
  constexpr int NP = M / 2 + 1;
  for (int t = threadIdx.x; t < nr * NP; t += kCtThreads) {
    const int r = t / NP, p = t % NP;
    c2r_pre_pair(sm + r * LD, M, p, tw, keep_im);
  }
  __syncthreads();
  cta_fft_ct<1, M, ROWS, kCtThreads, LD>(sm, tw, 2);
  float* dst = out + (long)item * bt.out_stride + (long)r0 * out_pitch;
  const bool pair = ((reinterpret_cast<uintptr_t>(dst) & 7) == 0) && !(out_pitch & 1);
  for (int t = threadIdx.x; t < nr * M; t += kCtThreads) {
    const int r = t / M, m = t % M;
    const float2 v = sm[r * LD + spad(m)];
    float* p = dst + (long)r * out_pitch + 2 * m;
    if (pair) {
      *reinterpret_cast<float2*>(p) = v;
    } else {
      p[0] = v.x;
      p[1] = v.y;
    }
  }
}

// TX columns per CTA (default: two CTAs of kCtThreads per SM); the wide
// form (TX doubled, 2*kCtThreads threads, one CTA per SM) reads full 32-byte
// sectors at H = 4096.
template <int H, int TX, int T>
__global__ void __launch_bounds__(T, 1024 / T) k_col_fft_ct(const float2* in, float2* out,
                                                           long pitch, int cmpX, Batch bt,
                                                           const float2* __restrict__ tw,
                                                           ColOps ops) {
  constexpr int LD = ct_spad_len(H);
  extern __shared__ float2 sm[];
  const int item = blockIdx.y;
  const int x0 = blockIdx.x * TX;
  const float2* src = in + batch_in_off(bt, item);
  const float2* ex = ops.ex ? ops.ex + (long)item * cmpX : nullptr;
  const float2* ey = ops.ey ? ops.ey + (long)item * H : nullptr;
  staged_copy<kStageLoads>(
      TX * H,
      [&](int t) {
        const int y = t / TX, c = t % TX;
        const int x = x0 + c;
        float2 v = c2(0.f, 0.f);
        if (x < cmpX) {
          v = src[(long)y * pitch + x];
          if (ex) v = cmul(v, cmul(ex[x], ey[y]));
        }
        return v;
      },
      [&](int t, float2 v) {
        const int y = t / TX, c = t % TX;
        sm[c * LD + spad(y)] = v;
      });
  __syncthreads();
  if (ops.dir < 0) cta_fft_ct<-1, H, TX, T, LD>(sm, tw, 1);
  else cta_fft_ct<1, H, TX, T, LD>(sm, tw, 1);
  float2* dst = out + (long)item * bt.out_stride;
  float2* crop = ops.crop ? ops.crop + (long)item * ops.crop_x * ops.crop_y : nullptr;
  for (int t = threadIdx.x; t < TX * H; t += T) {
    const int y = t / TX, c = t % TX;
    const int x = x0 + c;
    if (x >= cmpX) continue;
    const float2 v = cscale(sm[c * LD + spad(y)], ops.scale);
    dst[(long)y * pitch + x] = v;
    if (crop && x < ops.crop_x) {
      int yo = -1;
      if (y <= ops.crop_y / 2) yo = y;
      else if (y > H - ops.crop_y / 2) yo = y - H + ops.crop_y;
      if (yo >= 0) crop[(long)yo * ops.crop_x + x] = v;
    }
  }
}

namespace {
template <int M>
int launch_row_r2c_ct(const float* in, long in_pitch, float2* out, long out_pitch, int H,
                      const Batch& b, const float2* tw, float scale, cudaStream_t st) {
  constexpr int LD = ct_spad_len(M + 1);
  constexpr int ROWS = ct_batch(LD);
  const size_t smem = (size_t)ROWS * LD * sizeof(float2);
  MC3_TRY(set_smem_attr(k_row_r2c_ct<M>, smem));
  dim3 grid(ceil_div(H, ROWS), b.items);
  k_row_r2c_ct<M><<<grid, kCtThreads, smem, st>>>(in, in_pitch, out, out_pitch, H, b, tw, scale);
  MC3_CHECK_LAUNCH("k_row_r2c_ct");
  return kOk;
}
template <int M>
int launch_row_c2r_ct(const float2* in, long in_pitch, float* out, long out_pitch, int H,
                      const Batch& b, const float2* tw, int keep_im, cudaStream_t st) {
  constexpr int LD = ct_spad_len(M + 1);
  constexpr int ROWS = ct_batch(LD);
  const size_t smem = (size_t)ROWS * LD * sizeof(float2);
  MC3_TRY(set_smem_attr(k_row_c2r_ct<M>, smem));
  dim3 grid(ceil_div(H, ROWS), b.items);
  k_row_c2r_ct<M><<<grid, kCtThreads, smem, st>>>(in, in_pitch, out, out_pitch, H, b, tw, keep_im);
  MC3_CHECK_LAUNCH("k_row_c2r_ct");
  return kOk;
}
template <int H, bool WIDE = false>
int launch_col_fft_ct(const float2* in, float2* out, long pitch, int cmpX, const Batch& b,
                      const float2* tw, const ColOps& ops, cudaStream_t st) {
  constexpr int LD = ct_spad_len(H);
  constexpr int TX = ct_batch(LD) * (WIDE ? 2 : 1);
  constexpr int T = kCtThreads * (WIDE ? 2 : 1);
  const size_t smem = (size_t)TX * LD * sizeof(float2);
  MC3_TRY(set_smem_attr(k_col_fft_ct<H, TX, T>, smem));
  dim3 grid(ceil_div(cmpX, TX), b.items);
  k_col_fft_ct<H, TX, T><<<grid, T, smem, st>>>(in, out, pitch, cmpX, b, tw, ops);
  MC3_CHECK_LAUNCH("k_col_fft_ct");
  return kOk;
}
// MC3_FFT_COL_WIDE=1 selects the wide 4096-point column form (A/B runs).
bool col_wide() { return active_tuning().col_wide != 0; }
// MC3_FFT_RUNTIME_PLAN=1 keeps the runtime-plan in-place kernels (A/B runs).
bool ct_off() {
  static const bool off = [] {
    const char* e = getenv("MC3_FFT_RUNTIME_PLAN");
    return e && e[0] == '1';
  }();
  return off;
}
}  // namespace

namespace {
constexpr int kIpThreads = 512;
constexpr int kIpBudget = 72 * 1024;   // shared memory per CTA, in-place kernels
int min_radix(const FftDesc& d) {
  int r = 64;
  for (int s = 0; s < d.nstages; ++s) r = d.radix[s] < r ? d.radix[s] : r;
  return r;
}
// Sequences per CTA for an in-place pass: bounded by the register staging
// capacity (MAXB butterflies per thread) and the shared-memory budget.
// MC3_FFT_PINGPONG=1 forces the generic kernels (A/B comparisons).
bool use_inplace(const FftDesc& d) {
  static const bool off = [] {
    const char* e = getenv("MC3_FFT_PINGPONG");
    return e && e[0] == '1';
  }();
  return !off && all_dedicated(d);
}
int ip_batch(const FftDesc& d, int ld, int maxb) {
  const int per = d.n / min_radix(d);
  int nb = (maxb * kIpThreads) / per;
  const int by_smem = kIpBudget / (ld * (int)sizeof(float2));
  if (by_smem < nb) nb = by_smem;
  if (nb > 16) nb = 16;
  return nb;
}
}  // namespace

int row_tile(int M) {
  int rows = kSmemBudget / (2 * (M + 1) * (int)sizeof(float2));
  if (rows < 1) rows = 1;
  if (rows > 16) rows = 16;
  return rows;
}
int col_tile(int H) {
  int tx = kSmemBudget / (2 * (H + 1) * (int)sizeof(float2));
  int p = 1;
  while (p * 2 <= tx && p < 16) p *= 2;
  return p;
}

int row_r2c(const float* in, long in_pitch, float2* out, long out_pitch, int W, int H,
            const Batch& b, float scale, cudaStream_t st) {
  if (W < 2 || (W & 1) || H < 1 || b.items < 1) return kEInval;
  {
    const int s = row_r2c_r16(in, in_pitch, out, out_pitch, W, H, b, scale, st);
    if (s != kEUnsupported) return s;
  }
  const int M = W / 2;
  FftDesc d;
  MC3_TRY(make_desc(M, W, &d));
  if (use_inplace(d) && !ct_off()) {
    const double bytes = (double)b.items * H * (W * 4.0 + (W / 2 + 1) * 8.0);
#define MC3_CT(NAME, MM)                                                                   \
  case MM: {                                                                               \
    prof::Scope ps(NAME, bytes, st);                                                       \
    return launch_row_r2c_ct<MM>(in, in_pitch, out, out_pitch, H, b, d.tw, scale, st);    \
  }
    switch (M) {
      MC3_CT("k_row_r2c_ct<128>", 128)
      MC3_CT("k_row_r2c_ct<256>", 256)
      MC3_CT("k_row_r2c_ct<512>", 512)
      MC3_CT("k_row_r2c_ct<1024>", 1024)
      MC3_CT("k_row_r2c_ct<2048>", 2048)
      default: break;
    }
#undef MC3_CT
  }
  if (use_inplace(d)) {
    const int ld = spad_len(M + 1);
    const int rows = ip_batch(d, ld, 2);
    if (rows >= 1) {
      const size_t smem = (size_t)rows * ld * sizeof(float2);
      MC3_TRY(set_smem_attr(k_row_r2c_ip<2>, smem));
      dim3 grid(ceil_div(H, rows), b.items);
      prof::Scope ps("k_row_r2c", (double)b.items * H * (W * 4.0 + (W / 2 + 1) * 8.0), st);
      k_row_r2c_ip<2><<<grid, kIpThreads, smem, st>>>(in, in_pitch, out, out_pitch, W, H, rows, b, d, scale);
      MC3_CHECK_LAUNCH("k_row_r2c_ip");
      return kOk;
    }
  }
  const int rows = row_tile(M);
  const size_t smem = 2 * (size_t)rows * (M + 1) * sizeof(float2);
  if (smem > 200 * 1024) return kEUnsupported;
  MC3_TRY(set_smem_attr(k_row_r2c, smem));
  dim3 grid(ceil_div(H, rows), b.items);
  prof::Scope ps("k_row_r2c", (double)b.items * H * (W * 4.0 + (W / 2 + 1) * 8.0), st);
  k_row_r2c<<<grid, 256, smem, st>>>(in, in_pitch, out, out_pitch, W, H, rows, b, d, scale);
  MC3_CHECK_LAUNCH("k_row_r2c");
  return kOk;
}

// cufftPlan2d C2R, probed on the B200 with a single imaginary DC or Nyquist
// term per row: the imaginary parts of X[0] and X[W/2] reach the output
// (-(b0 + bM) on even samples, b0 - bM on odd ones) for 2048^2, 4096^2,
// 4096 x 2048, 2048 x 4096 and 1024 x 2048 (W x H), and are dropped for
// 64^2 .. 1536^2, 384 x 320, 192 x 160, 408^2, 410 x 408, 2882 x 2048,
// 5760 x 4092 and 2048 x 1024: both sides powers of two and H >= 2048.
bool c2r_keep_edge_imag(int W, int H) {
  auto pow2 = [](int n) { return n > 0 && (n & (n - 1)) == 0; };
  return pow2(W) && pow2(H) && H >= 2048;
}

int row_c2r(const float2* in, long in_pitch, float* out, long out_pitch, int W, int H,
            const Batch& b, cudaStream_t st) {
  const int keep_im = c2r_keep_edge_imag(W, H) ? 1 : 0;
  if (W < 2 || (W & 1) || H < 1 || b.items < 1) return kEInval;
  {
    const int s = row_c2r_r16(in, in_pitch, out, out_pitch, W, H, b, st, keep_im);
    if (s != kEUnsupported) return s;
  }
  const int M = W / 2;
  FftDesc d;
  MC3_TRY(make_desc(M, W, &d));
  if (use_inplace(d) && !ct_off()) {
    const double bytes = (double)b.items * H * (W * 4.0 + (W / 2 + 1) * 8.0);
#define MC3_CT(NAME, MM)                                                              \
  case MM: {                                                                          \
    prof::Scope ps(NAME, bytes, st);                                                  \
    return launch_row_c2r_ct<MM>(in, in_pitch, out, out_pitch, H, b, d.tw, keep_im, st); \
  }
    switch (M) {
      MC3_CT("k_row_c2r_ct<128>", 128)
      MC3_CT("k_row_c2r_ct<256>", 256)
      MC3_CT("k_row_c2r_ct<512>", 512)
      MC3_CT("k_row_c2r_ct<1024>", 1024)
      MC3_CT("k_row_c2r_ct<2048>", 2048)
      default: break;
    }
#undef MC3_CT
  }
  if (use_inplace(d)) {
    const int ld = spad_len(M + 1);
    const int rows = ip_batch(d, ld, 2);
    if (rows >= 1) {
      const size_t smem = (size_t)rows * ld * sizeof(float2);
      MC3_TRY(set_smem_attr(k_row_c2r_ip<2>, smem));
      dim3 grid(ceil_div(H, rows), b.items);
      prof::Scope ps("k_row_c2r", (double)b.items * H * (W * 4.0 + (W / 2 + 1) * 8.0), st);
      k_row_c2r_ip<2><<<grid, kIpThreads, smem, st>>>(in, in_pitch, out, out_pitch, W, H, rows, b, d,
                                                       keep_im);
      MC3_CHECK_LAUNCH("k_row_c2r_ip");
      return kOk;
    }
  }
  const int rows = row_tile(M);
  const size_t smem = 2 * (size_t)rows * (M + 1) * sizeof(float2);
  if (smem > 200 * 1024) return kEUnsupported;
  MC3_TRY(set_smem_attr(k_row_c2r, smem));
  dim3 grid(ceil_div(H, rows), b.items);
  prof::Scope ps("k_row_c2r", (double)b.items * H * (W * 4.0 + (W / 2 + 1) * 8.0), st);
  k_row_c2r<<<grid, 256, smem, st>>>(in, in_pitch, out, out_pitch, W, H, rows, b, d, keep_im);
  MC3_CHECK_LAUNCH("k_row_c2r");
  return kOk;
}

int col_fft(const float2* in, float2* out, long pitch, int cmpX, int H, const Batch& b,
            const ColOps& ops, cudaStream_t st) {
  if (cmpX < 1 || H < 1 || b.items < 1) return kEInval;
  if (ops.crop && (ops.crop_x > cmpX || ops.crop_y > H)) return kEInval;
  {
    const int s = col_fft_r16(in, out, pitch, cmpX, H, b, ops, st);
    if (s != kEUnsupported) return s;
  }
  FftDesc d;
  MC3_TRY(make_desc(H, H, &d));
  if (use_inplace(d) && !ct_off()) {
    const double bytes = (double)b.items * ((double)cmpX * H * 16.0 + (ops.crop ? (double)ops.crop_x * ops.crop_y * 8.0 : 0.0));
#define MC3_CT(NAME, HH)                                                              \
  case HH: {                                                                          \
    prof::Scope ps(NAME, bytes, st);                                                  \
    if constexpr (HH == 4096) {                                                       \
      if (col_wide())                                                                 \
        return launch_col_fft_ct<HH, true>(in, out, pitch, cmpX, b, d.tw, ops, st);   \
    }                                                                                 \
    return launch_col_fft_ct<HH>(in, out, pitch, cmpX, b, d.tw, ops, st);             \
  }
    switch (H) {
      MC3_CT("k_col_fft_ct<256>", 256)
      MC3_CT("k_col_fft_ct<512>", 512)
      MC3_CT("k_col_fft_ct<1024>", 1024)
      MC3_CT("k_col_fft_ct<2048>", 2048)
      MC3_CT("k_col_fft_ct<4096>", 4096)
      default: break;
    }
#undef MC3_CT
  }
  if (use_inplace(d)) {
    const int ld = spad_len(H);
    const int tx = ip_batch(d, ld, 2);
    if (tx >= 1) {
      const size_t smem = (size_t)tx * ld * sizeof(float2);
      MC3_TRY(set_smem_attr(k_col_fft_ip<2>, smem));
      dim3 grid(ceil_div(cmpX, tx), b.items);
      prof::Scope ps("k_col_fft", (double)b.items * ((double)cmpX * H * 16.0 + (ops.crop ? (double)ops.crop_x * ops.crop_y * 8.0 : 0.0)), st);
      k_col_fft_ip<2><<<grid, kIpThreads, smem, st>>>(in, out, pitch, cmpX, H, tx, b, d, ops);
      MC3_CHECK_LAUNCH("k_col_fft_ip");
      return kOk;
    }
  }
  const int tx = col_tile(H);
  const size_t smem = 2 * (size_t)tx * (H + 1) * sizeof(float2);
  if (smem > 200 * 1024) return kEUnsupported;
  MC3_TRY(set_smem_attr(k_col_fft, smem));
  dim3 grid(ceil_div(cmpX, tx), b.items);
  prof::Scope ps("k_col_fft", (double)b.items * ((double)cmpX * H * 16.0 + (ops.crop ? (double)ops.crop_x * ops.crop_y * 8.0 : 0.0)), st);
  k_col_fft<<<grid, 256, smem, st>>>(in, out, pitch, cmpX, H, tx, b, d, ops);
  MC3_CHECK_LAUNCH("k_col_fft");
  return kOk;
}

}  // namespace mc3
