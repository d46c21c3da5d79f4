// Correction kernels: dose-weight normalisation, fused shift + dose weight
// + summation over all frames, local-motion gather, output unpadding.
// Restates Correct/GWeightFrame.cu, Correct/CCorrectFullShift.cpp:271-334,
// Correct/GCorrectPatchShift.cu:17-66 and the positivity/unpad steps of
// CCorrectFullShift::mUnpadSums (:146-185).
#include <cstdlib>

#include "kernels.cuh"
#include "tuning.h"

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

// Two IEEE fp32 FMAs in one instruction (Blackwell packed f32x2): lane i
// is fmaf(a_i, b_i, c_i), the same rounding as the scalar form.
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) {
  unsigned long long ra, rb, rc, rd;
  asm("mov.b64 %0, {%1, %2};" : "=l"(ra) : "f"(a.x), "f"(a.y));
  asm("mov.b64 %0, {%1, %2};" : "=l"(rb) : "f"(b.x), "f"(b.y));
  asm("mov.b64 %0, {%1, %2};" : "=l"(rc) : "f"(c.x), "f"(c.y));
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(rd) : "l"(ra), "l"(rb), "l"(rc));
  float2 d;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(d.x), "=f"(d.y) : "l"(rd));
  return d;
}

// Weight of one patch for pixel (x, y) as mGCorrect3D computes it: w =
// exp(-100 r), r = distance to the patch centre in units of the frame size;
// false (the patch is skipped) when r > 0.6.
__device__ __forceinline__ bool patch_weight(int x, int y, int W, int H, float cx, float cy,
                                             float* w) {
  float ax = ((float)(unsigned)x - cx) / (float)(unsigned)W;
  float ay = (y - cy) / H;
  ax = sqrtf(ax * ax + ay * ay);
  if (ax > 0.6f) return false;
  *w = expf(-100.0f * ax);
  return true;
}

// The same packed FMA on values kept in 64-bit registers (lane 0 in the low
// half): no packing or unpacking around each instruction.
__device__ __forceinline__ unsigned long long ffma2_b64(unsigned long long a,
                                                        unsigned long long b,
                                                        unsigned long long c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ unsigned long long pack2(float lo, float hi) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ float2 unpack2(unsigned long long v) {
  float2 d;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(d.x), "=f"(d.y) : "l"(v));
  return d;
}

// Per-pixel patch weights of mGCorrect3D: w = exp(-100 r) for patches with
// r <= 0.6 (r = distance to the patch centre in units of the frame size),
// bit p of the returned mask set for those patches; the others weigh 0.
template <int PMAX, bool EXACT>
__device__ __forceinline__ unsigned long long gather_weights(int x, int y, int W, int H,
                                                             const float* __restrict__ cent, int P,
                                                             float (&w)[PMAX]) {
  unsigned long long inc = 0ull;
#pragma unroll
  for (int p = 0; p < PMAX; ++p) {
    w[p] = 0.0f;
    if (x < W && (EXACT || p < P) && patch_weight(x, y, W, H, cent[2 * p], cent[2 * p + 1], &w[p]))
      inc |= 1ull << p;
  }
  return inc;
}

// Local-motion gather (mGCorrect3D): every output pixel of every frame is
// read from the frame at the pixel minus the weighted mean of the patch
// shifts.  One CTA = one row segment; the patch shifts of a chunk of frames
// are staged in shared memory as (sx, sx, sy, sy) so that one 16-byte read
// serves a patch for both pixels of a thread.  PX = 2: the thread's pixels
// are 128 apart in the row and their sums are carried as f32x2 pairs
// (lane q = pixel q), so one packed FMA does the work of two.  PX = 1: one
// pixel, scalar FMAs.  Frames whose patches are all good and whose shifts
// are finite take the branch-free path (excluded patches weigh 0 and the
// weight total is the precomputed sum of the included weights, added in
// patch order); the others test every patch.
template <int PMAX, bool EXACT, int PX>
__global__ void __launch_bounds__(128) k_local_gather(
    const float* __restrict__ in, long in_stride, float* out, long out_stride, int W, int H,
    const float* __restrict__ cent, const float2* __restrict__ sh,
    const unsigned long long* __restrict__ masks, const uint8_t* __restrict__ bad,
    const uint8_t* __restrict__ clean, int P, int nb) {
  static_assert(PX == 1 || PX == 2, "one or two pixels per thread");
  constexpr int FCH = 16;  // frames per shared-memory chunk
  __shared__ float4 s_sh[FCH * PMAX];
  __shared__ int s_clean[FCH];
  const int y = blockIdx.y;
  const int xb = blockIdx.x * (128 * PX) + threadIdx.x;
  float w[PX][PMAX];
  unsigned long long inc[PX];
  float wsum[PX];
#pragma unroll
  for (int q = 0; q < PX; ++q) {
    inc[q] = gather_weights<PMAX, EXACT>(xb + 128 * q, y, W, H, cent, P, w[q]);
    // weight total of a frame without bad patches (same additions, same order)
    wsum[q] = 0.0f;
#pragma unroll
    for (int p = 0; p < PMAX; ++p)
      if ((inc[q] >> p) & 1ull) wsum[q] += w[q][p];
  }
  float2 wp[PMAX];  // (w of pixel 0, w of pixel 1) for the packed FMAs
  unsigned long long wpb[PMAX];  // the same pairs in 64-bit registers
  if constexpr (PX == 2) {
#pragma unroll
    for (int p = 0; p < PMAX; ++p) {
      wp[p] = make_float2(w[0][p], w[1][p]);
      wpb[p] = pack2(w[0][p], w[1][p]);
    }
  }
  const bool act0 = xb < W;
  const int padX = (W / 2 + 1) * 2;
  for (int c0 = 0; c0 < nb; c0 += FCH) {
    const int nc = min(FCH, nb - c0);
    __syncthreads();  // the previous chunk's readers are done
    for (int i = threadIdx.x; i < nc * PMAX; i += 128) {
      const int f = i / PMAX, p = i - f * PMAX;
      float2 v = make_float2(0.0f, 0.0f);  // patches p >= P weigh 0
      if (EXACT || p < P) v = sh[(long)(c0 + f) * P + p];
      s_sh[i] = make_float4(v.x, v.x, v.y, v.y);
    }
    if (threadIdx.x < nc) s_clean[threadIdx.x] = clean ? clean[c0 + threadIdx.x] : 0;
    __syncthreads();
    if (!act0) continue;
    // Frames in groups of FB: source offsets, then loads, then stores.
    constexpr int FB = 4;
    for (int f0 = 0; f0 < nc; f0 += FB) {
      int src[FB][PX];
#pragma unroll
      for (int b = 0; b < FB; ++b) {
        const int fl = f0 + b;
        if (fl >= nc) break;
        const float4* s = s_sh + fl * PMAX;
        float fSx[PX], fSy[PX], fW[PX];
        if (s_clean[fl]) {
          if constexpr (PX == 2) {
            // (sx, sx) and (sy, sy) of each patch come as two 64-bit values.
            // The shared reads need no memory clobber: the chunk's writes
            // are ordered before them by the __syncthreads() above, and the
            // next chunk's writes after them by the one at the loop's top.
            unsigned long long Sx = 0ull, Sy = 0ull;  // (+0, +0)
            const uint32_t sa = (uint32_t)__cvta_generic_to_shared(s);
#pragma unroll
            for (int p = 0; p < PMAX; ++p) {
              unsigned long long sxx, syy;
              asm volatile("ld.shared.v2.u64 {%0, %1}, [%2];" : "=l"(sxx), "=l"(syy) : "r"(sa + 16 * p));
              Sx = ffma2_b64(sxx, wpb[p], Sx);
              Sy = ffma2_b64(syy, wpb[p], Sy);
            }
            const float2 ux = unpack2(Sx), uy = unpack2(Sy);
            fSx[0] = ux.x, fSx[1] = ux.y, fSy[0] = uy.x, fSy[1] = uy.y;
          } else {
            fSx[0] = fSy[0] = 0.0f;
#pragma unroll
            for (int p = 0; p < PMAX; ++p) {
              const float4 sp = s[p];
              fSx[0] += sp.x * w[0][p];
              fSy[0] += sp.z * w[0][p];
            }
          }
#pragma unroll
          for (int q = 0; q < PX; ++q) fW[q] = wsum[q];
        } else {
          const int f = c0 + fl;
          unsigned long long m = 0ull;
          if (masks) {
            m = masks[f];
          } else if (bad) {
            for (int p = 0; p < P; ++p) m |= (unsigned long long)(bad[(long)f * P + p] != 0) << p;
          }
#pragma unroll
          for (int q = 0; q < PX; ++q) {
            const unsigned long long use = inc[q] & ~m;
            fSx[q] = fSy[q] = fW[q] = 0.0f;
#pragma unroll
            for (int p = 0; p < PMAX; ++p) {
              if ((use >> p) & 1ull) {
                const float4 sp = s[p];
                const float wq = PX == 2 ? (q ? wp[p].y : wp[p].x) : w[0][p];
                fW[q] += wq;
                fSx[q] += sp.x * wq;
                fSy[q] += sp.z * wq;
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
          if (f0 + b < nc && xb + 128 * q < W)
            v[b][q] = in[(long)(c0 + f0 + b) * in_stride + src[b][q]];
#pragma unroll
      for (int b = 0; b < FB; ++b)
#pragma unroll
        for (int q = 0; q < PX; ++q)
          if (f0 + b < nc && xb + 128 * q < W)
            out[(long)(c0 + f0 + b) * out_stride + (long)y * padX + xb + 128 * q] = v[b][q];
    }
  }
}

// More than 64 patches (a 64-bit mask per frame no longer covers them):
// patches in chunks of kWideChunk whose weights are held in registers, frames
// in groups of kWideFrames whose running sums carry from chunk to chunk, so
// every (pixel, frame) still adds its good patches in patch order as
// mGCorrect3D does (Correct/GCorrectPatchShift.cu:32-46).  Bad patches come
// from the [nb][P] flags.  Weights are evaluated once per frame group.
constexpr int kWideChunk = 32, kWideFrames = 8;
__global__ void __launch_bounds__(128) k_local_gather_wide(
    const float* __restrict__ in, long in_stride, float* out, long out_stride, int W, int H,
    const float* __restrict__ cent, const float2* __restrict__ sh,
    const uint8_t* __restrict__ bad, int P, int nb) {
  const int y = blockIdx.y;
  const int x = blockIdx.x * 128 + threadIdx.x;
  if (x >= W) return;
  const int padX = (W / 2 + 1) * 2;
  for (int f0 = 0; f0 < nb; f0 += kWideFrames) {
    const int nf = min(kWideFrames, nb - f0);
    float sx[kWideFrames], sy[kWideFrames], sw[kWideFrames];
#pragma unroll
    for (int b = 0; b < kWideFrames; ++b) sx[b] = sy[b] = sw[b] = 0.0f;
    for (int p0 = 0; p0 < P; p0 += kWideChunk) {
      const int np = min(kWideChunk, P - p0);
      float w[kWideChunk];
      unsigned inc = 0u;
#pragma unroll
      for (int i = 0; i < kWideChunk; ++i) {
        w[i] = 0.0f;
        if (i < np && patch_weight(x, y, W, H, cent[2 * (p0 + i)], cent[2 * (p0 + i) + 1], &w[i]))
          inc |= 1u << i;
      }
#pragma unroll
      for (int b = 0; b < kWideFrames; ++b) {
        if (b >= nf) break;
        const long f = f0 + b;
#pragma unroll
        for (int i = 0; i < kWideChunk; ++i) {
          if (((inc >> i) & 1u) && !(bad && bad[f * P + p0 + i])) {
            const float2 s = sh[f * P + p0 + i];
            sw[b] += w[i];
            sx[b] += s.x * w[i];
            sy[b] += s.y * w[i];
          }
        }
      }
    }
#pragma unroll
    for (int b = 0; b < kWideFrames; ++b) {
      if (b >= nf) break;
      const long f = f0 + b;
      const int src = gather_src(W, H, padX, x, y, sx[b], sy[b], sw[b]);
      out[f * out_stride + (long)y * padX + x] = in[f * in_stride + src];
    }
  }
}

template <int PMAX, bool EXACT>
static void launch_gather(int W, int H, cudaStream_t st, const float* in, long in_stride,
                          float* out, long out_stride, const float* centers,
                          const float2* shifts, const unsigned long long* masks,
                          const uint8_t* bad, const uint8_t* clean, int P, int nb) {
  // two pixels per thread up to 36 patches (MC3_GATHER_PX=1 forces one,
  // for A/B runs); one above (register budget of the weights)
  const bool one = active_tuning().gather_px == 1;
  if (PMAX <= 36 && !one) {
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
  if (P < 1) return kEInval;
  if (P > 64) {
    prof::Scope ps("k_local_gather_wide", (double)nb * W * H * 8.0, st);
    dim3 grid(ceil_div(W, 128), H);
    k_local_gather_wide<<<grid, 128, 0, st>>>(in, in_stride, out, out_stride, W, H, centers,
                                              shifts, bad, P, nb);
    MC3_CHECK_LAUNCH("k_local_gather_wide");
    return kOk;
  }
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

// -OutStack frames: GFourierResize2D copy-mode crop (Util/GFourierResize2D.cu:7-37)
// of every frame spectrum, with the frame's phase shift (tables ex [N][inX],
// ey [N][inY], as the column passes apply them) when ex is given.
__global__ void k_crop_frames(const float2* __restrict__ in, int inX, int inY, long in_stride,
                              const float2* __restrict__ ex, const float2* __restrict__ ey,
                              float2* __restrict__ out, int outX, int outY, long out_stride) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int yo = blockIdx.y;
  const int f = blockIdx.z;
  if (x >= outX) return;
  const int yi = yo > outY / 2 ? yo - outY + inY : yo;
  float2 v = in[(long)f * in_stride + (long)yi * inX + x];
  if (ex) v = cmul(v, cmul(ex[(long)f * inX + x], ey[(long)f * inY + yi]));
  out[(long)f * out_stride + (long)yo * outX + x] = v;
}

int crop_frames(const float2* in, int inX, int inY, long in_stride, const float2* ex,
                const float2* ey, float2* out, int outX, int outY, long out_stride, int N,
                cudaStream_t st) {
  if (outX > inX || outY > inY || N < 1 || N > 65535) return kEUnsupported;
  dim3 grid(ceil_div(outX, 128), outY, N);
  prof::Scope ps("k_crop_frames", (double)N * outX * outY * 16.0, st);
  k_crop_frames<<<grid, 128, 0, st>>>(in, inX, inY, in_stride, ex, ey, out, outX, outY,
                                      out_stride);
  MC3_CHECK_LAUNCH("k_crop_frames");
  return kOk;
}

// CZbinStack::mGroup (Align/CZbinStack.cpp:57-71) in place: group g (frames
// grp[g] .. grp[g]+grp[ng+g]-1, consecutive groups) is summed in frame
// order into slot g.  One thread owns one pixel of every frame, and group g
// reads only slots >= its start >= g, so the in-place update is race-free.
__global__ void k_zbin_frames(float* frames, long fr_stride, int pitch, int W, int H,
                              const int* __restrict__ grp, int ng) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= W) return;
  float* p = frames + (long)y * pitch + x;
  for (int g = 0; g < ng; ++g) {
    const int f0 = grp[g], n = grp[ng + g];
    float s = p[(long)f0 * fr_stride];
    for (int i = 1; i < n; ++i) s += p[(long)(f0 + i) * fr_stride];
    p[(long)g * fr_stride] = s;
  }
}

int zbin_frames(float* frames, long fr_stride, int pitch, int W, int H, const int* groups,
                int n_groups, cudaStream_t st) {
  if (n_groups < 1) return kEInval;
  dim3 grid(ceil_div(W, 128), H);
  prof::Scope ps("k_zbin_frames", (double)W * H * 8.0 * n_groups, st);
  k_zbin_frames<<<grid, 128, 0, st>>>(frames, fr_stride, pitch, W, H, groups, n_groups);
  MC3_CHECK_LAUNCH("k_zbin_frames");
  return kOk;
}

// mGStretch (Correct/GStretch.cu:14-44) on n padded real images: the output
// pixel (x, y) of the W x H image reads the input bilinearly at
// m * ((x, y) - c) + c, c = (W/2, H/2), m = [m0 m1; m1 m2]; a source outside
// [1, W-1) x [1, H-1) is folded to (8111 |x| mod (W-1), 8111 |y| mod (H-1)).
// The padding columns of the output are left as they are.
__global__ void k_stretch(const float* __restrict__ in, float* __restrict__ out, int pitch,
                          long stride, int W, int H, float m0, float m1, float m2) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= W) return;
  const float* src = in + (long)blockIdx.z * stride;
  const float cx = 0.5f * W, cy = 0.5f * H;
  const float dx = x - cx, dy = y - cy;
  float ox = dx * m0 + dy * m1 + cx;
  float oy = dx * m1 + dy * m2 + cy;
  if (ox < 1 || oy < 1 || ox >= (W - 1) || oy >= (H - 1)) {
    // the fold in 64-bit arithmetic (the reference's int product is the same
    // for sources within a few image widths, and never negative here)
    const long long ax = (long long)fminf(fabsf(ox), 1.0e9f);
    const long long ay = (long long)fminf(fabsf(oy), 1.0e9f);
    ox = (float)((8111LL * ax) % (W - 1));
    oy = (float)((8111LL * ay) % (H - 1));
  }
  const int ix = (int)ox, iy = (int)oy;
  const float wx = ox - ix, wy = oy - iy;
  const float* p = src + (long)iy * pitch + ix;
  out[(long)blockIdx.z * stride + (long)y * pitch + x] =
      (1 - wx) * (1 - wy) * p[0] + wx * (1 - wy) * p[1] + (1 - wx) * wy * p[pitch] +
      wx * wy * p[pitch + 1];
}

int stretch_images(const float* in, float* out, int pitch, long stride, int W, int H, int n,
                   const float* m, cudaStream_t st) {
  if (W < 3 || H < 3 || n < 1) return kEInval;
  dim3 grid(ceil_div(W, 128), H, n);
  prof::Scope ps("k_stretch", (double)n * W * H * 8.0, st);
  k_stretch<<<grid, 128, 0, st>>>(in, out, pitch, stride, W, H, m[0], m[1], m[2]);
  MC3_CHECK_LAUNCH("k_stretch");
  return kOk;
}

// GMotionWeight::DirWeight (MotionDecon/GMotionWeight.cu:14-36, 56-68,
// 92-107): the spectrum of frame f is multiplied by the sinc of its in-frame
// motion m_f measured along m_f: frequency (x, y) (y signed) lies at distance
// |s x - y| / sqrt(s^2 + 1), s = -m.x / (m.y + 1e-20), from the line through
// the origin perpendicular to m (x itself when |s| > 1e5); with
// d = distance / (2 (cmpX - 1)) the weight is sin(pi |m| d) / (pi |m| d),
// 0 once |m| d > 1, and 1 when the distance is below 0.1.  DC is left alone;
// frames whose |m| is below 0.1 px are skipped (flag 0).
__global__ void k_motion_decon(float2* spec, long fr_stride, int cmpX, int cmpY,
                               const float4* __restrict__ motion) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  const int f = blockIdx.z;
  if (x >= cmpX) return;
  const float4 m = motion[f];  // (m.x, m.y, apply flag, unused)
  if (m.z == 0.0f || (x == 0 && y == 0)) return;
  const float shift = sqrtf(m.x * m.x + m.y * m.y);
  if (shift < 0.1f) return;
  const float slope = -m.x / (m.y + (float)1e-20);
  float dist;
  if (fabsf(slope) > (float)1e5) {
    dist = (float)x;
  } else {
    const int ys = y > cmpY / 2 ? y - cmpY : y;
    dist = fabsf(slope * x - ys) / sqrtf(slope * slope + 1.0f);
  }
  if (dist < 0.1f) return;
  const float pi = 3.141592654f;
  dist = dist / (2 * (cmpX - 1));
  float w;
  if (shift * dist > 1.0f) {
    w = 0.0f;
  } else {
    w = sinf(pi * shift * dist) / (pi * shift * dist);
  }
  float2* p = spec + (long)f * fr_stride + (long)y * cmpX + x;
  float2 v = *p;
  v.x *= w;
  v.y *= w;
  *p = v;
}

int motion_decon(float2* spec, long fr_stride, int cmpX, int cmpY, int N, const float4* motion,
                 cudaStream_t st) {
  if (N < 1 || N > 65535 || cmpX < 2) return kEInval;
  dim3 grid(ceil_div(cmpX, 128), cmpY, N);
  prof::Scope ps("k_motion_decon", (double)N * cmpX * cmpY * 16.0, st);
  k_motion_decon<<<grid, 128, 0, st>>>(spec, fr_stride, cmpX, cmpY, motion);
  MC3_CHECK_LAUNCH("k_motion_decon");
  return kOk;
}

// GCorrLinearInterp mGCorrectCmp (Util/GCorrLinearInterp.cu:7-22): every
// frequency but DC of N frame spectra divided by sinc(pi r)^(1/8),
// r = |(x / (2 (cmpX - 1)), y / cmpY)| with y signed.
__global__ void k_corr_interp(float2* spec, long fr_stride, int cmpX, int cmpY) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= cmpX || (x == 0 && y == 0)) return;
  float fx = x * 0.5f / (cmpX - 1);
  float fy = y / (float)cmpY;
  if (fy > 0.5f) fy -= 1.0f;
  fx = sqrtf(fx * fx + fy * fy) * 3.141592654f;
  fx = sinf(fx) / fx;
  fx = powf(fx, 0.125f);
  float2* p = spec + (long)blockIdx.z * fr_stride + (long)y * cmpX + x;
  float2 v = *p;
  v.x /= fx;
  v.y /= fx;
  *p = v;
}

int corr_interp(float2* spec, long fr_stride, int cmpX, int cmpY, int N, cudaStream_t st) {
  if (N < 1 || N > 65535 || cmpX < 2) return kEInval;
  dim3 grid(ceil_div(cmpX, 128), cmpY, N);
  prof::Scope ps("k_corr_interp", (double)N * cmpX * cmpY * 16.0, st);
  k_corr_interp<<<grid, 128, 0, st>>>(spec, fr_stride, cmpX, cmpY);
  MC3_CHECK_LAUNCH("k_corr_interp");
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
