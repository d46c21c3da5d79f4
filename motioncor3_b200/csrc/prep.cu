// Frame preparation: gain application, frame sum, hot-pixel and defect
// detection, defect fill, image moments.  Restates MrcUtil/GApplyRefsToFrame.cu,
// MrcUtil/CSumFFTStack.cpp, BadPixel/GDetectHot.cu, BadPixel/GLocalCC.cu,
// BadPixel/GDetectPatch.cu, BadPixel/GCorrectBad.cu and Util/GCalcMoment2D.cu.
#include "kernels.cuh"

namespace mc3 {

// ---- gain + running frame sum --------------------------------------------
// One thread per pixel walks all frames: frame_f = raw_f * gain is written
// to the padded frame stack and accumulated (in frame order, as the
// reference's CSumFFTStack does) into the padded sum image.
template <typename T>
__global__ void k_gain_sum(const T* __restrict__ raw, long raw_stride, const float* __restrict__ dark,
                           const float* __restrict__ gain, float* frames, long fr_stride, float* sum,
                           int W, int H, int N, int padX) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= W) return;
  const float g = gain ? gain[(long)y * W + x] : 1.0f;
  const float d = dark ? dark[(long)y * W + x] : 0.0f;
  float s = 0.0f;
  for (int f = 0; f < N; ++f) {
    float v = (float)raw[(long)f * raw_stride + (long)y * W + x];
    if (dark) v -= d;  // (raw - dark) * gain, GApplyRefsToFrame.cu:66-70
    if (gain) v *= g;
    frames[(long)f * fr_stride + (long)y * padX + x] = v;
    s += v;
  }
  if (sum) sum[(long)y * padX + x] = s;
}

// Mode 101 (4-bit, two pixels per byte, rows of (W+1)/2 bytes): pixel x is
// the low nibble of byte x/2 for even x, the high nibble for odd x
// (GApplyRefsToFrame mGDoPkd, MrcUtil/GApplyRefsToFrame.cu:30-53).
__global__ void k_gain_sum_pkd(const uint8_t* __restrict__ raw, long raw_stride,
                               const float* __restrict__ dark, const float* __restrict__ gain,
                               float* frames, long fr_stride, float* sum, int W, int H, int N,
                               int padX) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= W) return;
  const int pkX = (W + 1) / 2;
  const float g = gain ? gain[(long)y * W + x] : 1.0f;
  const float d = dark ? dark[(long)y * W + x] : 0.0f;
  float s = 0.0f;
  for (int f = 0; f < N; ++f) {
    int b = raw[(long)f * raw_stride + (long)y * pkX + x / 2];
    if (x & 1) b >>= 4;
    float v = (float)(b & 0xf);
    if (dark) v -= d;
    if (gain) v *= g;
    frames[(long)f * fr_stride + (long)y * padX + x] = v;
    s += v;
  }
  if (sum) sum[(long)y * padX + x] = s;
}

int gain_and_sum(const void* raw, int mode, long raw_stride, const float* dark,
                 const float* gain, float* frames, long fr_stride, float* sum, int W, int H, int N,
                 cudaStream_t st) {
  const int padX = 2 * (W / 2 + 1);
  dim3 grid(ceil_div(W, 256), H);
  const double bpp = mode == 101 ? 0.5 : (mode == 0 || mode == 5) ? 1 : (mode == 2 ? 4 : 2);
  prof::Scope ps("k_gain_sum", (double)W * H * (N * (bpp + 4.0) + (gain ? 4.0 : 0.0) + (sum ? 4.0 : 0.0)), st);
  switch (mode) {
    case 101: k_gain_sum_pkd<<<grid, 256, 0, st>>>((const uint8_t*)raw, raw_stride, dark, gain, frames, fr_stride, sum, W, H, N, padX); break;
    case 0: case 5: k_gain_sum<uint8_t><<<grid, 256, 0, st>>>((const uint8_t*)raw, raw_stride, dark, gain, frames, fr_stride, sum, W, H, N, padX); break;
    case 1: k_gain_sum<int16_t><<<grid, 256, 0, st>>>((const int16_t*)raw, raw_stride, dark, gain, frames, fr_stride, sum, W, H, N, padX); break;
    case 2: k_gain_sum<float><<<grid, 256, 0, st>>>((const float*)raw, raw_stride, dark, gain, frames, fr_stride, sum, W, H, N, padX); break;
    case 6: k_gain_sum<uint16_t><<<grid, 256, 0, st>>>((const uint16_t*)raw, raw_stride, dark, gain, frames, fr_stride, sum, W, H, N, padX); break;
    default: return kEUnsupported;
  }
  MC3_CHECK_LAUNCH("k_gain_sum");
  return kOk;
}

// Frame integration fused with the gain pass: rendered frame i is the sum of
// raw frames start[i] .. start[i]+size[i]-1 in 8-bit arithmetic (the
// reference adds raw frames into an unsigned-char rendered frame,
// Util/GAddFrames.cu mGAddUChar, so the sum wraps modulo 256;
// MrcUtil/CLoadCryoEMStack.cpp:184-262), then converted and gain-multiplied
// as an 8-bit frame.  PACKED: 4-bit raw frames (mode 101) unpacked first.
template <bool PACKED>
__global__ void k_gain_sum_int(const uint8_t* __restrict__ raw, long raw_stride,
                               const int* __restrict__ start, const int* __restrict__ size,
                               const float* __restrict__ dark, const float* __restrict__ gain,
                               float* frames, long fr_stride, float* sum, int W, int H, int N,
                               int padX) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= W) return;
  const long off = PACKED ? (long)y * ((W + 1) / 2) + x / 2 : (long)y * W + x;
  const float g = gain ? gain[(long)y * W + x] : 1.0f;
  const float d = dark ? dark[(long)y * W + x] : 0.0f;
  float s = 0.0f;
  for (int f = 0; f < N; ++f) {
    const int r0 = start[f], nr = size[f];
    unsigned acc = 0;
    for (int k = 0; k < nr; ++k) {
      unsigned b = raw[(long)(r0 + k) * raw_stride + off];
      if (PACKED) b = ((x & 1) ? (b >> 4) : b) & 0xfu;
      acc += b;
    }
    float v = (float)(acc & 0xffu);
    if (dark) v -= d;
    if (gain) v *= g;
    frames[(long)f * fr_stride + (long)y * padX + x] = v;
    s += v;
  }
  if (sum) sum[(long)y * padX + x] = s;
}

int gain_and_sum_int(const void* raw, int mode, long raw_stride, const int* start,
                     const int* size, const float* dark, const float* gain, float* frames,
                     long fr_stride, float* sum, int W, int H, int N, cudaStream_t st) {
  const int padX = 2 * (W / 2 + 1);
  dim3 grid(ceil_div(W, 256), H);
  prof::Scope ps("k_gain_sum_int", (double)W * H * N * 4.0, st);  // rendered-frame writes
  switch (mode) {
    case 101:
      k_gain_sum_int<true><<<grid, 256, 0, st>>>((const uint8_t*)raw, raw_stride, start, size, dark,
                                                 gain, frames, fr_stride, sum, W, H, N, padX);
      break;
    case 0: case 5:
      k_gain_sum_int<false><<<grid, 256, 0, st>>>((const uint8_t*)raw, raw_stride, start, size,
                                                  dark, gain, frames, fr_stride, sum, W, H, N, padX);
      break;
    default: return kEUnsupported;
  }
  MC3_CHECK_LAUNCH("k_gain_sum_int");
  return kOk;
}

// Known camera defects added to the detected map: bad |= (defects != 0).
__global__ void k_or_mask(uint8_t* bad, const uint8_t* __restrict__ defects, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && defects[i]) bad[i] = 1;
}

int or_mask(uint8_t* bad, const uint8_t* defects, size_t n, cudaStream_t st) {
  if (n == 0) return kOk;
  k_or_mask<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(bad, defects, n);
  MC3_CHECK_LAUNCH("k_or_mask");
  return kOk;
}

// ---- moments with the reference's reduction order ------------------------
// GCalcMoment2D::DoIt (Util/GCalcMoment2D.cu:10-60, 96-114): grid-stride
// per-thread FP32 sums, shared-memory tree, per-block division by W*H, then
// a one-block tree over the block partials.  The same order gives the same
// FP32 result, so thresholds derived from it match the reference.
__global__ void k_moment_partial(const float* img, int W, int H, long pitch, int iExp, float* part) {
  extern __shared__ float sh[];
  float sum = 0.0f;
  for (int y = blockIdx.x; y < H; y += gridDim.x) {
    const float* ptr = img + (long)y * pitch;
    for (int ix = threadIdx.x; ix < W; ix += blockDim.x) {
      float val = ptr[ix];
      float expval = val;
      for (int i = 1; i < iExp; i++) expval *= val;
      sum += expval;
    }
  }
  sh[threadIdx.x] = sum;
  __syncthreads();
  for (int off = blockDim.x / 2; off > 0; off = off / 2) {
    if (threadIdx.x < off) sh[threadIdx.x] += sh[threadIdx.x + off];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0] / (W * H);
}

__global__ void k_moment_final(float* part, float* out) {
  extern __shared__ float sh[];
  sh[threadIdx.x] = part[threadIdx.x];
  __syncthreads();
  for (int off = blockDim.x / 2; off > 0; off = off / 2) {
    if (threadIdx.x < off) sh[threadIdx.x] += sh[threadIdx.x + off];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

int moment_grid(int W, int H) {
  const long px = (long)W * H;
  const long nb = (px + 511) / 512;
  if (nb >= 512) return 512;
  if (nb >= 128) return 128;
  if (nb >= 64) return 64;
  return 32;
}

int image_moment(const float* img, int W, int H, long pitch, int iExp, float* d_part,
                 float* d_out, cudaStream_t st) {
  const int g = moment_grid(W, H);
  {
  prof::Scope ps("k_moment_partial", (double)W * H * 4.0, st);
  k_moment_partial<<<g, 512, 512 * sizeof(float), st>>>(img, W, H, pitch, iExp, d_part);
  MC3_CHECK_LAUNCH("k_moment_partial");
  }
  prof::Scope ps2("k_moment_final", g * 4.0, st);
  k_moment_final<<<1, g, g * sizeof(float), st>>>(d_part, d_out);
  MC3_CHECK_LAUNCH("k_moment_final");
  return kOk;
}

// ---- hot pixels (BadPixel/GDetectHot.cu:10-57) ----------------------------
// mean/std come from two image_moment() results already on the device.
__global__ void k_detect_hot(const float* sum, long pitch, int W, int H, const float* mom,
                             float thr_sigma, uint8_t* bad) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= W) return;
  const float fMean = mom[0];
  float fStd = mom[1] - fMean * fMean;
  fStd = (float)sqrtf(fmaxf(fStd, 0));
  float fDelta = thr_sigma * fStd;
  if (fDelta < 10) fDelta = 10;
  const float fMax = fMean + fDelta;
  bad[(long)y * W + x] = sum[(long)y * pitch + x] <= fMax ? 0 : 1;
}

// ---- local CC against the ring template (BadPixel/GLocalCC.cu:20-61) -----
__constant__ float c_tpl[64];

__global__ void k_local_cc(const float* img, long pitch, int W, int H, int ms, float* cc) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= W) return;
  const long o = (long)y * pitch + x;
  cc[o] = 0.0f;
  if ((x + ms) >= W) return;
  if ((y + ms) >= H) return;
  const float* src = img + o;
  float fMean = 0.0f, fStd = 0.0f, fCC = 0.0f;
  for (int j = 0; j < ms; j++) {
    for (int i = 0; i < ms; i++) {
      float fImg = src[j * pitch + i];
      float fRef = c_tpl[j * ms + i];
      fMean += fImg;
      fStd += (fImg * fImg);
      fCC += (fRef * fImg);
    }
  }
  int n = ms * ms;
  fCC /= n;
  fMean /= n;
  fStd = fStd / n - fMean * fMean;
  if (fStd < 0) fStd = 0.0f;
  else fStd = sqrtf(fStd);
  if (fStd == 0) cc[o] = 0.0f;
  else cc[o] = fabsf(fCC) / fStd;
}

// GDetectPatch::mUpdateBadMap (BadPixel/GDetectPatch.cu:10-46, 56-104)
__global__ void k_mark_defects(const float* cc, long pitch, int W, int H, const float* mom,
                               float thr_sigma, int ms, uint8_t* bad) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if ((x + ms) >= W) return;
  if ((y + ms) >= H) return;
  const float fMean = mom[0];
  const float fStd = (float)sqrtf(fmaxf(0, mom[1] - fMean * fMean));
  const float thr = fMean + thr_sigma * fStd;
  if (cc[(long)y * pitch + x] <= thr) return;
  for (int j = 0; j < ms; ++j)
    for (int i = 0; i < ms; ++i) bad[(long)(y + j) * W + x + i] = 1;
}

int detect_bad_pixels(const float* sum, int W, int H, float* cc_buf, float* d_part,
                      float* d_mom /*4 floats*/, uint8_t* bad, const float* tpl, int ms,
                      cudaStream_t st, uint8_t* hot_copy) {
  const long pitch = 2 * (W / 2 + 1);
  MC3_TRY(image_moment(sum, W, H, pitch, 1, d_part, d_mom + 0, st));
  MC3_TRY(image_moment(sum, W, H, pitch, 2, d_part, d_mom + 1, st));
  dim3 grid(ceil_div(W, 256), H);
  {
  prof::Scope ps("k_detect_hot", (double)W * H * 5.0, st);
  k_detect_hot<<<grid, 256, 0, st>>>(sum, pitch, W, H, d_mom, 6.0f, bad);
  MC3_CHECK_LAUNCH("k_detect_hot");
  }
  // the hot pixels alone, as CGenStarFile::SetHotPixels lists them (CDetectMain.cpp:66-67)
  if (hot_copy)
    MC3_CUDA(cudaMemcpyAsync(hot_copy, bad, (size_t)W * H, cudaMemcpyDeviceToDevice, st));
  MC3_CUDA(cudaMemcpyToSymbolAsync(c_tpl, tpl, sizeof(float) * ms * ms, 0, cudaMemcpyHostToDevice, st));
  {
  prof::Scope ps("k_local_cc", (double)W * H * 8.0, st);
  k_local_cc<<<grid, 256, 0, st>>>(sum, pitch, W, H, ms, cc_buf);
  MC3_CHECK_LAUNCH("k_local_cc");
  }
  MC3_TRY(image_moment(cc_buf, W, H, pitch, 1, d_part, d_mom + 2, st));
  MC3_TRY(image_moment(cc_buf, W, H, pitch, 2, d_part, d_mom + 3, st));
  prof::Scope ps("k_mark_defects", (double)W * H * 4.0, st);
  k_mark_defects<<<grid, 256, 0, st>>>(cc_buf, pitch, W, H, d_mom + 2, 6.0f, ms, bad);
  MC3_CHECK_LAUNCH("k_mark_defects");
  return kOk;
}

// ---- defect fill (BadPixel/GCorrectBad.cu:44-69, 96-150) ------------------
// The replacement pixel of a bad pixel depends only on its position and on
// the bad-pixel map (the pseudo-random walk below), not on the frame, and
// it is never itself bad.  So the fill is split into: list the bad pixels
// (one pass over the map), pick each one's source once, then copy source
// to destination in every frame.  Fills do not interact, so the list order
// (atomics) does not matter.
__device__ __forceinline__ int bad_source(const uint8_t* bad, int x, int y, int W, int H,
                                          int padX, int win0) {
  const int i = y * padX + x;
  unsigned int next = i * 109 + 619;
  int win = win0;
  for (int j = 0; j < 10; j++) {
    unsigned int nl = next;
    const int w2 = win * win, half = win / 2;
    for (int k = 0; k < 500; k++) {
      nl *= 997;
      int iX = nl % w2;
      int iY = iX / win - half + y;
      if (iY < 0 || iY >= H) continue;
      iX = iX % win - half + x;
      if (iX < 0 || iX >= W) continue;
      if (bad[(long)iY * W + iX] == 1) continue;
      return iY * padX + iX;
    }
    win += 50;
    next *= 997;
  }
  int iX = next % (unsigned int)(W * H);
  int iY = iX / W;
  iX = iX % W;
  return iY * padX + iX;
}

// list[k] = (destination, source) padded offsets of the k-th bad pixel.
__global__ void k_bad_list(const uint8_t* __restrict__ bad, int W, int H, int padX, int win0,
                           int* count, int2* list) {
  const long npx = (long)W * H;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < npx;
       i += (long)gridDim.x * blockDim.x) {
    if (bad[i] == 0) continue;
    const int y = (int)(i / W), x = (int)(i % W);
    const int k = atomicAdd(count, 1);
    list[k] = make_int2(y * padX + x, bad_source(bad, x, y, W, H, padX, win0));
  }
}

__global__ void k_fill_bad(float* frames, long fr_stride, int N, const int* count,
                           const int2* __restrict__ list) {
  const int n = *count;
  const long total = (long)n * N;
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long)gridDim.x * blockDim.x) {
    const int f = (int)(t / n);
    const int2 e = list[t - (long)f * n];
    float* fr = frames + (long)f * fr_stride;
    fr[e.x] = fr[e.y];
  }
}

int correct_bad_pixels(float* frames, long fr_stride, int N, const uint8_t* bad, int W, int H,
                       int* d_count, int2* d_list, cudaStream_t st) {
  const int padX = 2 * (W / 2 + 1);
  MC3_CUDA(cudaMemsetAsync(d_count, 0, sizeof(int), st));
  {
    prof::Scope ps("k_bad_list", (double)W * H, st);
    k_bad_list<<<148 * 8, 256, 0, st>>>(bad, W, H, padX, 31, d_count, d_list);
    MC3_CHECK_LAUNCH("k_bad_list");
  }
  prof::Scope ps("k_fill_bad", 0.0, st);
  k_fill_bad<<<148 * 4, 256, 0, st>>>(frames, fr_stride, N, d_count, d_list);
  MC3_CHECK_LAUNCH("k_fill_bad");
  return kOk;
}

// Synthetic counts 0..3 (a hash of the pixel index) for the autotuner's movie.
__global__ void k_synthetic_counts(float* f, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    unsigned v = (unsigned)i * 2654435761u;
    v ^= v >> 15;
    v *= 2246822519u;
    v ^= v >> 13;
    f[i] = (float)(v & 3u);
  }
}

int synthetic_counts(float* f, long n, cudaStream_t st) {
  k_synthetic_counts<<<1184, 256, 0, st>>>(f, n);
  MC3_CHECK_LAUNCH("k_synthetic_counts");
  return kOk;
}

}  // namespace mc3
