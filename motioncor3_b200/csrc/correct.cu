// Correction kernels: dose-weight normalisation, fused shift + dose weight
// + summation over all frames, local-motion gather, output unpadding.
// Restates Correct/GWeightFrame.cu, Correct/CCorrectFullShift.cpp:271-334,
// Correct/GCorrectPatchShift.cu:17-66 and the positivity/unpad steps of
// CCorrectFullShift::mUnpadSums (:146-185).
#include <cstdlib>

#include "kernels.cuh"

namespace mc3 {

// GWeightFrame mGCalcWeight (Correct/GWeightFrame.cu:19-30), split into the
// frame-independent critical dose and the per-frame exponential (the same
// FP32 operations as the reference, with powf evaluated once per frequency).
__device__ __forceinline__ float crit_dose(int x, int y, int cmpX, int cmpY, float kvf, float pix) {
  float fX = (float)x * 0.5f / (float)(unsigned)(cmpX - 1);
  float fY = y / (float)cmpY;
  if (fY >= 0.5f) fY -= 1.0f;
  fX = sqrtf(fX * fX + fY * fY) / pix;
  float fCritDose = 0.24499f * powf(fX, -1.6649f) + 2.8141f;
  fCritDose *= kvf;
  return fCritDose;
}
__device__ __forceinline__ float dose_weight_c(float fCritDose, float fDose) {
  return expf(-0.5f * fDose / fCritDose);
}

// GWeightFrame::BuildWeight: per-frame accumulation of w^2 in frame order,
// then the square root; DC excluded (stays 0).
__global__ void k_dose_norm(const float* acc, int N, int cmpX, int cmpY, float pix, float kvf,
                            float* Wn) {
  const long n = (long)cmpX * cmpY;
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (i == 0) {
    Wn[0] = 0.0f;
    return;
  }
  const int x = (int)(i % cmpX), y = (int)(i / cmpX);
  const float cd = crit_dose(x, y, cmpX, cmpY, kvf, pix);
  float s = 0.0f;
  for (int f = 0; f < N; ++f) {
    const float w = dose_weight_c(cd, acc[f]);
    s += (w * w);
  }
  Wn[i] = sqrtf(s);
}

int dose_norm(const float* acc_dose, int N, int cmpX, int cmpY, float pix, float kvf, float* Wn,
              cudaStream_t st) {
  const long n = (long)cmpX * cmpY;
  prof::Scope ps("k_dose_norm", (double)n * 4.0, st);
  k_dose_norm<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(acc_dose, N, cmpX, cmpY, pix, kvf, Wn);
  MC3_CHECK_LAUNCH("k_dose_norm");
  return kOk;
}

// All sums in one pass over the frames (CCorrectFullShift::mGenSums,
// Correct/CCorrectFullShift.cpp:271-300): sum0 += X; X *= w_f/Wn (DC
// untouched); sum1 += X; sum2 += X when the frame's accumulated dose lies in
// the selected range; with -SplitSum the (weighted) X also goes to the
// "_ODD" sum for even frame indices and to "_EVN" for odd ones.
__global__ void k_frame_sums(const float2* __restrict__ spec, long fr_stride, int N, int cmpX,
                             int cmpY, const float2* __restrict__ ex, const float2* __restrict__ ey,
                             const float* acc, const float* Wn, DoseParams dp, float2* sums,
                             int n_sums) {
  const long n = (long)cmpX * cmpY;
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int x = (int)(k % cmpX), y = (int)(k / cmpX);
  float2 s0 = c2(0.f, 0.f), s1 = c2(0.f, 0.f), s2 = c2(0.f, 0.f);
  float2 so = c2(0.f, 0.f), se = c2(0.f, 0.f);
  const float wn = dp.enabled && k > 0 ? Wn[k] : 1.0f;
  const float cd = dp.enabled && k > 0 ? crit_dose(x, y, cmpX, cmpY, dp.kv_factor, dp.pix_size) : 1.0f;
#pragma unroll 4
  for (int f = 0; f < N; ++f) {
    float2 X = spec[(long)f * fr_stride + k];
    if (ex) {
      const float2 e = cmul(ex[(long)f * cmpX + x], ey[(long)f * cmpY + y]);
      X = c2(e.x * X.x - e.y * X.y, e.x * X.y + e.y * X.x);
    }
    s0 = cadd(X, s0);
    if (dp.enabled) {
      if (k > 0) {
        float fW = dose_weight_c(cd, acc[f]);
        fW = fW / wn;
        X.x *= fW;
        X.y *= fW;
      }
      s1 = cadd(X, s1);
      if (dp.dws && acc[f] >= dp.sum_range[0] && acc[f] <= dp.sum_range[1]) s2 = cadd(X, s2);
    }
    if (dp.split) {
      if (f % 2 == 0) so = cadd(X, so);
      else se = cadd(X, se);
    }
  }
  sums[k] = s0;
  int next = 1;
  if (dp.enabled) {
    sums[n + k] = s1;
    next = 2;
    if (dp.dws) {
      sums[2 * n + k] = s2;
      next = 3;
    }
  }
  if (dp.split) {
    sums[(long)next * n + k] = so;
    sums[(long)(next + 1) * n + k] = se;
  }
}

int frame_sums(const float2* spec, long fr_stride, int N, int cmpX, int cmpY, const float2* ex,
               const float2* ey, const float* acc_dose, const float* Wn, const DoseParams& dp,
               float2* sums, int n_sums, cudaStream_t st) {
  const long n = (long)cmpX * cmpY;
  if (n_sums != 1 + (dp.enabled ? 1 + (dp.dws ? 1 : 0) : 0) + (dp.split ? 2 : 0)) return kEInval;
  prof::Scope ps("k_frame_sums", (double)n * (8.0 * (N + n_sums) + (dp.enabled ? 4.0 : 0.0)), st);
  k_frame_sums<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(spec, fr_stride, N, cmpX, cmpY, ex, ey,
                                                           acc_dose, Wn, dp, sums, n_sums);
  MC3_CHECK_LAUNCH("k_frame_sums");
  return kOk;
}

// mGCorrect3D (Correct/GCorrectPatchShift.cu:17-66) with upsampling 1:
// per-pixel local shift = sum_p w_p s_p / sum_p w_p, w_p = exp(-100 r_p)
// over good patches with normalised distance r_p <= 0.6, then a
// nearest-neighbour (int-truncated) gather; out-of-range sources fold to
// (811*|v|) mod size.
//
// The distance weights do not depend on the frame, so each thread evaluates
// them once for its pixel (held in registers, with a bit mask of the
// patches within 0.6) and then walks all nb frames.  The patches used in a
// frame are that mask minus the frame's bad-patch mask (one 64-bit mask per
// frame); the accumulation runs in patch order exactly as the reference's,
// as predicated adds rather than branches.
// EXACT: P == PMAX; otherwise P < PMAX and reads are clamped to patch P-1.
// Shift = weighted sums / weight total, int-truncated source, fold of
// out-of-range sources (the tail of mGCorrect3D); returns the source offset
// within the padded frame.
__device__ __forceinline__ int gather_src(int W, int H, int padX, int x, int y, float sx, float sy,
                                          float fW) {
  if (fW > 0) {
    sx = sx / fW;
    sy = sy / fW;
  }
  int ix = (int)(((float)(unsigned)x - sx) * 1);
  int iy = (int)((y - sy) * 1);
  if (ix < 0 || iy < 0 || ix >= W || iy >= H) {
    ix = (ix < 0) ? -ix : ix;
    iy = (iy < 0) ? -iy : iy;
    ix = (811 * ix) % W;
    iy = (811 * iy) % H;
    // Only non-finite shifts reach here out of range (the int conversion
    // of NaN/inf); keep the read inside the frame.
    if (ix < 0 || ix >= W) ix = 0;
    if (iy < 0 || iy >= H) iy = 0;
  }
  return iy * padX + ix;
}

template <int PMAX, bool EXACT, int PX>
__global__ void __launch_bounds__(128) k_local_gather(
    const float* __restrict__ in, long in_stride, float* out, long out_stride, int W, int H,
    const float* __restrict__ cent, const float2* __restrict__ sh,
    const unsigned long long* __restrict__ masks, const uint8_t* __restrict__ bad,
    const uint8_t* __restrict__ clean, int P, int nb) {
  // PX pixels per thread, 128 apart in the row: each patch shift read
  // (uniform over the warp) serves PX pixels.
  const int y = blockIdx.y;
  const int xb = blockIdx.x * (128 * PX) + threadIdx.x;
  const float fB = 100.0f;
  float w[PX][PMAX];
  unsigned long long inc[PX];  // patches within r <= 0.6 of each pixel
#pragma unroll
  for (int q = 0; q < PX; ++q) {
    const int x = xb + 128 * q;
    inc[q] = 0ull;
#pragma unroll
    for (int p = 0; p < PMAX; ++p) {
      w[q][p] = 0.0f;
      if (x < W && (EXACT || p < P)) {
        float ax = ((float)(unsigned)x - cent[2 * p]) / (float)(unsigned)W;
        float ay = (y - cent[2 * p + 1]) / H;
        ax = sqrtf(ax * ax + ay * ay);
        if (!(ax > 0.6f)) {
          w[q][p] = expf(-fB * ax);
          inc[q] |= 1ull << p;
        }
      }
    }
  }
  // Sum of the included weights in patch order: the weight total of every
  // frame without bad patches (same additions, same order, same bits).
  float wsum[PX];
#pragma unroll
  for (int q = 0; q < PX; ++q) {
    wsum[q] = 0.0f;
#pragma unroll
    for (int p = 0; p < PMAX; ++p)
      if ((inc[q] >> p) & 1ull) wsum[q] += w[q][p];
  }
  if (xb >= W) return;
  const int padX = (W / 2 + 1) * 2;
  // Frames in groups of FB: the source offsets of the whole group are
  // computed first, then its loads are issued together, then the stores.
  constexpr int FB = 4;
  for (int f0 = 0; f0 < nb; f0 += FB) {
    int src[FB][PX];
#pragma unroll
    for (int b = 0; b < FB; ++b) {
      const int f = f0 + b;
      if (f >= nb) break;
      const float2* s = sh + (long)f * P;
      float fSx[PX], fSy[PX], fW[PX];
      if (clean && clean[f]) {
        // Frame without bad patches and with finite shifts: the excluded
        // patches carry weight 0, and adding 0 * s (s finite) leaves the
        // sums unchanged, so every patch is accumulated without a test.
#pragma unroll
        for (int q = 0; q < PX; ++q) {
          fSx[q] = fSy[q] = 0.0f;
          fW[q] = wsum[q];
        }
#pragma unroll
        for (int p = 0; p < PMAX; ++p) {
          const float2 sp = s[EXACT ? p : (p < P ? p : P - 1)];
#pragma unroll
          for (int q = 0; q < PX; ++q) {
            fSx[q] += sp.x * w[q][p];
            fSy[q] += sp.y * w[q][p];
          }
        }
      } else {
        unsigned long long m = 0ull;
        if (masks) {
          m = masks[f];
        } else if (bad) {
          for (int p = 0; p < P; ++p) m |= (unsigned long long)(bad[(long)f * P + p] != 0) << p;
        }
        unsigned long long use[PX];
#pragma unroll
        for (int q = 0; q < PX; ++q) {
          fSx[q] = fSy[q] = fW[q] = 0.0f;
          use[q] = inc[q] & ~m;
        }
#pragma unroll
        for (int p = 0; p < PMAX; ++p) {
          const float2 sp = s[EXACT ? p : (p < P ? p : P - 1)];
#pragma unroll
          for (int q = 0; q < PX; ++q) {
            if ((use[q] >> p) & 1ull) {
              fW[q] += w[q][p];
              fSx[q] += sp.x * w[q][p];
              fSy[q] += sp.y * w[q][p];
            }
          }
        }
      }
#pragma unroll
      for (int q = 0; q < PX; ++q)
        src[b][q] = gather_src(W, H, padX, xb + 128 * q, y, fSx[q], fSy[q], fW[q]);
    }
    float v[FB][PX];
#pragma unroll
    for (int b = 0; b < FB; ++b)
#pragma unroll
      for (int q = 0; q < PX; ++q)
        if (f0 + b < nb && xb + 128 * q < W) v[b][q] = in[(long)(f0 + b) * in_stride + src[b][q]];
#pragma unroll
    for (int b = 0; b < FB; ++b)
#pragma unroll
      for (int q = 0; q < PX; ++q)
        if (f0 + b < nb && xb + 128 * q < W)
          out[(long)(f0 + b) * out_stride + (long)y * padX + xb + 128 * q] = v[b][q];
  }
}

template <int PMAX, bool EXACT>
static void launch_gather(int W, int H, cudaStream_t st, const float* in, long in_stride,
                          float* out, long out_stride, const float* centers,
                          const float2* shifts, const unsigned long long* masks,
                          const uint8_t* bad, const uint8_t* clean, int P, int nb) {
  // one pixel per thread; MC3_GATHER_PX=2 gives two (up to 36 patches, A/B runs)
  static const bool two = [] {
    const char* e = getenv("MC3_GATHER_PX");
    return e && e[0] == '2';
  }();
  if (PMAX <= 36 && two) {
    dim3 grid(ceil_div(W, 256), H);
    k_local_gather<PMAX, EXACT, 2><<<grid, 128, 0, st>>>(in, in_stride, out, out_stride, W, H,
                                                         centers, shifts, masks, bad, clean, P, nb);
  } else {
    dim3 grid(ceil_div(W, 128), H);
    k_local_gather<PMAX, EXACT, 1><<<grid, 128, 0, st>>>(in, in_stride, out, out_stride, W, H,
                                                         centers, shifts, masks, bad, clean, P, nb);
  }
}

int local_gather(const float* in, long in_stride, float* out, long out_stride, int nb, int W,
                 int H, const float* centers, const float2* shifts,
                 const unsigned long long* masks, const uint8_t* bad, const uint8_t* clean,
                 int P, cudaStream_t st) {
  // `shifts`/`masks`/`bad`/`clean` point at the first frame of the batch.
  if (P < 1 || P > 64) return kEUnsupported;
  prof::Scope ps("k_local_gather", (double)nb * W * H * 8.0, st);
#define MC3_GATHER(PM, EX) \
  launch_gather<PM, EX>(W, H, st, in, in_stride, out, out_stride, centers, shifts, masks, bad, clean, P, nb)
  switch (P) {
    case 4: MC3_GATHER(4, true); break;
    case 9: MC3_GATHER(9, true); break;
    case 16: MC3_GATHER(16, true); break;
    case 25: MC3_GATHER(25, true); break;
    case 35: MC3_GATHER(35, true); break;
    case 36: MC3_GATHER(36, true); break;
    case 49: MC3_GATHER(49, true); break;
    case 64: MC3_GATHER(64, true); break;
    default:
      if (P <= 16) MC3_GATHER(16, false);
      else if (P <= 36) MC3_GATHER(36, false);
      else MC3_GATHER(64, false);
  }
#undef MC3_GATHER
  MC3_CHECK_LAUNCH("k_local_gather");
  return kOk;
}

// Per-frame 64-bit masks of the bad-patch flags [nb][P] (bit p = patch p),
// and clean[f] = 1 when frame f has no bad patch and only finite shifts.
__global__ void k_patch_masks(const uint8_t* bad, const float2* sh, int P, int nb,
                              unsigned long long* masks, uint8_t* clean) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nb) return;
  unsigned long long m = 0ull;
  bool finite = true;
  for (int p = 0; p < P; ++p) {
    m |= (unsigned long long)(bad[(long)f * P + p] != 0) << p;
    const float2 s = sh[(long)f * P + p];
    finite = finite && isfinite(s.x) && isfinite(s.y);
  }
  masks[f] = m;
  clean[f] = (m == 0ull && finite) ? 1 : 0;
}

int patch_masks(const uint8_t* bad, const float2* shifts, int P, int nb,
                unsigned long long* masks, uint8_t* clean, cudaStream_t st) {
  if (P < 1 || P > 64) return kEUnsupported;
  k_patch_masks<<<ceil_div(nb, 128), 128, 0, st>>>(bad, shifts, P, nb, masks, clean);
  MC3_CHECK_LAUNCH("k_patch_masks");
  return kOk;
}

__global__ void k_unpad_positive(const float* in, long pitch, float* out, int W, int H,
                                 long in_stride) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= W) return;
  const int s = blockIdx.z;
  const float v = in[(long)s * in_stride + (long)y * pitch + x];
  out[(long)s * W * H + (long)y * W + x] = fmaxf(0.0f, v);
}

int unpad_positive(const float* in, long pitch, float* out, int W, int H, int n, long in_stride,
                   cudaStream_t st) {
  dim3 grid(ceil_div(W, 256), H, n);
  prof::Scope ps("k_unpad_positive", (double)n * W * H * 8.0, st);
  k_unpad_positive<<<grid, 256, 0, st>>>(in, pitch, out, W, H, in_stride);
  MC3_CHECK_LAUNCH("k_unpad_positive");
  return kOk;
}

}  // namespace mc3
