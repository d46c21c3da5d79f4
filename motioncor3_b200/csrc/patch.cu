// Patch-alignment helpers: Fourier cropping and the feature map used to
// place patch centres (Util/GFourierResize2D.cu, Util/GFindMinMax2D.cu,
// Util/GPositivity2D.cu:17-24, Align/GNormByStd2D.cu, Align/CDetectFeatures.cpp:89-119).
#include "kernels.cuh"

namespace mc3 {

// GFourierResize2D::mGResize, copy mode (Util/GFourierResize2D.cu:7-37)
__global__ void k_fourier_crop(const float2* in, int inX, int inY, float2* out, int outX, int outY) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y;
  if (x >= outX) return;
  const long o = (long)y * outX + x;
  if (x >= inX) return;
  if (y > outY / 2) {
    y -= outY;
    if (y <= -inY / 2) return;
    y += inY;
  } else if (y > inY / 2) {
    return;
  }
  out[o] = in[(long)y * inX + x];
}

int fourier_crop(const float2* in, int inX, int inY, float2* out, int outX, int outY,
                 cudaStream_t st) {
  dim3 grid(ceil_div(outX, 128), outY);
  prof::Scope ps("k_fourier_crop", (double)outX * outY * 16.0, st);
  k_fourier_crop<<<grid, 128, 0, st>>>(in, inX, inY, out, outX, outY);
  MC3_CHECK_LAUNCH("k_fourier_crop");
  return kOk;
}

// One-block min over the image (order-free, so any reduction is exact).
__global__ void k_min_add(float* img, int bx, int by, long pitch, float* out_min) {
  __shared__ float sh[256];
  float m = 1e20f;
  for (int i = threadIdx.x; i < bx * by; i += blockDim.x) {
    const int y = i / bx, x = i - y * bx;
    m = fminf(m, img[(long)y * pitch + x]);
  }
  sh[threadIdx.x] = m;
  __syncthreads();
  for (int off = blockDim.x / 2; off > 0; off >>= 1) {
    if (threadIdx.x < off) sh[threadIdx.x] = fminf(sh[threadIdx.x], sh[threadIdx.x + off]);
    __syncthreads();
  }
  const float fVal = 1.0f - sh[0];
  __syncthreads();
  // GPositivity2D::AddVal covers the whole padded buffer.
  for (long i = threadIdx.x; i < pitch * by; i += blockDim.x) img[i] += fVal;
  if (threadIdx.x == 0) *out_min = sh[0];
}

// GNormByStd2D (Align/GNormByStd2D.cu:7-40) with a 5x5 window, reading the
// unmodified input (the reference updates in place while neighbours read).
__global__ void k_norm_by_std(const float* img, float* out, int bx, int by, long pitch, int wx,
                              int wy) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int iy = blockIdx.y;
  if (ix >= bx) return;
  const int ox = ix - wx / 2, oy = iy - wy / 2;
  float fMean = 0.0f, fStd = 0.0f, fVal = 0.0f;
  int iCount = 0;
  for (int j = 0; j < wy; j++) {
    int y = j + oy;
    if (y < 0) continue;
    else if (y >= by) continue;
    for (int i = 0; i < wx; i++) {
      int x = i + ox;
      if (x < 0) continue;
      else if (x >= bx) continue;
      fVal = img[y * pitch + x];
      fMean += fVal;
      fStd += (fVal * fVal);
      iCount += 1;
    }
  }
  fMean /= iCount;
  fStd = fStd / iCount - fMean * fMean;
  const long o = (long)iy * pitch + ix;
  if (fStd < 0) out[o] = 0.0f;
  else out[o] = img[o] / (fStd + (float)1e-20);
}

__global__ void k_copy_unpad(const float* in, long pitch, float* out, int bx, int by) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= bx * by) return;
  const int y = i / bx, x = i - y * bx;
  out[i] = in[(long)y * pitch + x];
}

// d_scal: [0] min, [1] mean, [2] mean of squares.
int feature_map(float* img, int bx, int by, float* tmp, float* d_part, float* d_scal,
                float* map_out, cudaStream_t st) {
  const long pitch = 2 * (bx / 2 + 1);
  {
  prof::Scope ps("k_min_add", (double)pitch * by * 8.0, st);
  k_min_add<<<1, 256, 0, st>>>(img, bx, by, pitch, d_scal);
  MC3_CHECK_LAUNCH("k_min_add");
  }
  dim3 grid(ceil_div(bx, 128), by);
  {
  prof::Scope ps("k_norm_by_std", (double)pitch * by * 8.0, st);
  k_norm_by_std<<<grid, 128, 0, st>>>(img, tmp, bx, by, pitch, 5, 5);
  MC3_CHECK_LAUNCH("k_norm_by_std");
  }
  MC3_TRY(image_moment(tmp, bx, by, pitch, 1, d_part, d_scal + 1, st));
  MC3_TRY(image_moment(tmp, bx, by, pitch, 2, d_part, d_scal + 2, st));
  prof::Scope ps("k_copy_unpad", (double)bx * by * 8.0, st);
  k_copy_unpad<<<ceil_div(bx * by, 256), 256, 0, st>>>(tmp, pitch, map_out, bx, by);
  MC3_CHECK_LAUNCH("k_copy_unpad");
  return kOk;
}

}  // namespace mc3
