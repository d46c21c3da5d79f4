// CTF estimation on the motion-corrected sum: the role of FindCtf/
// (CFindCtfMain::DoIt, FindCtf/CFindCtfMain.cpp:49-83), which the reference
// runs on the first (unweighted) sum (Correct/CCorrectFullShift.cpp:129-144,179).
//
// Layout and kernels:
//   * the sum is Fourier-rescaled to a pixel size >= 1.25 A (CRescaleImage)
//     with the row/column FFT passes of fft.cu, into a padded real image;
//   * all 512 x 512 tiles (50 % overlap, CGenAvgSpectrum) are normalised,
//     edge-rounded and transformed in ONE batched R2C; one kernel averages
//     their amplitude spectra in tile order;
//   * background removal (GRmBackground2D), the full-spectrum Gaussian
//     lowpass and the radial average are single launches over the
//     257 x 512 half spectrum;
//   * every sweep of the grid searches (CFindDefocus1D::mBrutalForceSearch,
//     the sweeps of CFindDefocus2D) is one launch that scores all of its
//     candidates at once, one warp (1D) or one CTA (2D) per candidate, over
//     the pixels of the correlation band compacted into a list; the host
//     takes the decisions in the reference's candidate order.  The reference
//     launches and synchronises once per candidate (about 6000 times).
// Reads the reference leaves undefined get the values the oracle uses: the
// Hermitian partner for row 0 of GCalcSpectrum::GenFullSpect and the
// periodic column for the x-Nyquist copy of CGenAvgSpectrum::mLowpass; the
// uninitialised CFindDefocus2D::m_fExtPhase of the first two correlations is 0.
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "fft.cuh"

namespace mc3 {

namespace {

constexpr int kTile = 512;
constexpr int kCX = kTile / 2 + 1;   // 257
constexpr int kTP = 2 * kCX;         // padded tile row (514 floats)
constexpr float kD2R = 0.01745329f;  // FindCtf/CCtfTheory.cpp:8
constexpr float kD2R1 = 0.0174533f;  // FindCtf/CFindDefocus1D.cpp:12

// ---------------------------------------------------------------- kernels

// GPad2D::Pad of the rows that fit the rescaled size (bin 1).
__global__ void k_ctf_pad(const float* __restrict__ img, int nx, float* __restrict__ out, int pitch,
                          int ny) {
  const int y = blockIdx.y;
  if (y >= ny) return;
  for (int x = threadIdx.x + blockIdx.x * blockDim.x; x < pitch; x += blockDim.x * gridDim.x)
    out[(long)y * pitch + x] = x < nx ? img[(long)y * nx + x] : 0.f;
}

// Sum and sum of squares of every 512 x 512 tile (GCalcMoment2D moments 1, 2).
__global__ void __launch_bounds__(256) k_ctf_tile_stats(const float* __restrict__ img, int pitch,
                                                        const int* __restrict__ org, double* stats) {
  const int t = blockIdx.x;
  const int sx = org[2 * t], sy = org[2 * t + 1];
  double a = 0, b = 0;
  for (int i = threadIdx.x; i < kTile * kTile; i += blockDim.x) {
    const float v = img[(long)(sy + i / kTile) * pitch + sx + (i % kTile)];
    a += v;
    b += (double)v * v;
  }
  __shared__ double sa[256], sb[256];
  sa[threadIdx.x] = a;
  sb[threadIdx.x] = b;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      sa[threadIdx.x] += sa[threadIdx.x + o];
      sb[threadIdx.x] += sb[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    stats[2 * t] = sa[0];
    stats[2 * t + 1] = sb[0];
  }
}

// GNormalize2D + GRoundEdge (Util/GNormalize2D.cu, Util/GRoundEdge.cu) into
// the padded tile stack [tiles][512][514]; grid (512 rows, tiles).
__global__ void __launch_bounds__(256) k_ctf_tile_prep(const float* __restrict__ img, int pitch,
                                                       const int* __restrict__ org,
                                                       const double* __restrict__ stats,
                                                       float* __restrict__ tiles) {
  const int y = blockIdx.x, t = blockIdx.y;
  const int sx = org[2 * t], sy = org[2 * t + 1];
  const float mean = (float)(stats[2 * t] / ((double)kTile * kTile));
  float sd = (float)(stats[2 * t + 1] / ((double)kTile * kTile)) - mean * mean;
  sd = sd <= 0 ? 1.0f : sqrtf(sd);
  const float fy = 2 * fabsf(y - kTile * 0.5f) / kTile;
  float* row = tiles + ((long)t * kTile + y) * kTP;
  const float* src = img + (long)(sy + y) * pitch + sx;
  for (int x = threadIdx.x; x < kTP; x += blockDim.x) {
    const float fx = 2 * fabsf(x - kTile * 0.5f) / kTile;
    float r = sqrtf(fx * fx + fy * fy);
    float v = 0.f;
    if (r < 1.0f && x < kTile) {
      v = (src[x] - mean) / sd;
      r = 0.5f * (1 - cosf(3.1415926f * r));
      r = 1.0f - powf(r, 3.0f);
      v = v * r;
    }
    row[x] = v;
  }
}

// Amplitude spectra of the tiles averaged in tile order (GCalcSpectrum::DoIt
// + GAddFrames), DC moved to row 256.
__global__ void k_ctf_amp_avg(const float2* __restrict__ spec, int ntiles, float fac,
                              float* __restrict__ avg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kCX * kTile) return;
  const int y = i / kCX, x = i % kCX;
  float acc = 0.f;
  for (int t = 0; t < ntiles; ++t) {
    const float2 v = spec[(long)t * kCX * kTile + i];
    acc = acc * 1.0f + sqrtf(v.x * v.x + v.y * v.y) * fac;
  }
  avg[((y + kTile / 2) % kTile) * kCX + x] = acc;
}

__global__ void k_ctf_sqrt(const float* __restrict__ in, float* __restrict__ out, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = sqrtf(in[i]);
}

// GRmBackground2D::mGRemove (FindCtf/GRmBackground2D.cu:11-62) with the
// square roots precomputed.
__global__ void k_ctf_rmbg(const float* __restrict__ in, const float* __restrict__ sq, int box,
                           float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kCX * kTile) return;
  const int hx = kCX - 1, hy = kTile / 2, half = box / 2;
  const int x = i % kCX, yc = i / kCX - hy;
  float r = x * 0.5f / (kCX - 1);
  r = sqrtf(r * r + yc * yc / (float)(kTile * kTile));
  if (r < 0.04) {
    out[i] = 0.f;
    return;
  }
  float bg = 0.f;
  for (int k = -half; k <= half; ++k) {
    const int yy = k + yc;
    for (int j = -half; j <= half; ++j) {
      int xx = j + x, ix, iy;
      if (xx >= hx) xx -= 2 * hx;
      if (xx >= 0) {
        ix = xx;
        iy = hy + yy;
      } else {
        ix = -xx;
        iy = hy - yy;
      }
      if (iy < 0) iy += kTile;
      else if (iy >= kTile) iy -= kTile;
      bg += sq[iy * kCX + ix];
    }
  }
  bg /= (box * box);
  bg = bg * bg;
  out[i] = in[i] - bg;
}

// GCalcSpectrum::GenFullSpect (FindCtf/GCalcSpectrum.cu:62-82) into a padded
// [512][514] real image.
__global__ void k_ctf_full(const float* __restrict__ half, float* __restrict__ full) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kTP * kTile) return;
  const int y = i / kTP, x = i % kTP;
  if (x >= kTile) {
    full[i] = 0.f;
    return;
  }
  const int xd = x - (kCX - 1);
  const int xs = xd >= 0 ? xd : -xd;
  const int ys = xd >= 0 ? y : (kTile - y) % kTile;
  full[i] = half[ys * kCX + xs];
}

// GFFTUtil2D::mGLowpass (Util/GFFTUtil2D.cu:51-65).
__global__ void k_ctf_lowpass(float2* spec, float scale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kCX * kTile) return;
  const int x = i % kCX;
  int y = i / kCX;
  if (y > kTile / 2) y -= kTile;
  const float f = expf(scale * (float)(x * x + y * y));
  float2 v = spec[i];
  v.x *= f;
  v.y *= f;
  spec[i] = v;
}

// Right half of the lowpassed full spectrum back into the half spectrum.
__global__ void k_ctf_take_half(const float* __restrict__ full, float* __restrict__ half) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kCX * kTile) return;
  const int y = i / kCX, x = i % kCX;
  half[i] = full[y * kTP + (kCX - 1 + x) % kTile];
}

// GRadialAvg::mGRadAverage (FindCtf/GRadialAvg.cu:11-31).
__global__ void k_ctf_radial(const float* __restrict__ s, float* __restrict__ avg) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= kCX) return;
  int n = (int)(3.1415926f * r + 0.5f);
  if (n < 1) n = 1;
  else if (n > 180) n = 180;
  float sum = 0.f;
  const float step = 180.0f / n;
  for (int i = 0; i < n; ++i) {
    const float rad = (-90.0f + i * step) * 0.017453f;
    int x = (int)(r * cosf(rad) + 0.5f);
    int y = (int)(r * sinf(rad) + kTile / 2 + 0.5f);
    x = min(max(x, 0), kCX - 1);
    y = min(max(y, 0), kTile - 1);
    sum += s[y * kCX + x];
  }
  avg[r] = sum / n;
}

// GCalcCTF1D + GCtfCC1D (B = 0) for a batch of candidates, one warp each:
// cand[c] = (defocus px, added phase rad); out[c] = (sum cs, sum c^2, sum s^2).
__global__ void __launch_bounds__(256) k_ctf_cc1d(const float2* __restrict__ cand, int ncand,
                                                  const float* __restrict__ rad, float wave, float cs,
                                                  float lo, float hi, float4* __restrict__ out) {
  const int c = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (c >= ncand) return;
  const float2 p = cand[c];
  const float w2 = wave * wave;
  float a = 0.f, b = 0.f, d = 0.f;
  for (int x = lane; x < kCX; x += 32) {
    if (!(x >= lo && x < hi)) continue;
    float fs2 = (x * 0.5f) / (kCX - 1.0f);
    fs2 = fs2 * fs2;
    const float ph = p.y + 3.141592654f * wave * fs2 * (p.x - 0.5f * w2 * fs2 * cs);
    const float v = fabsf(-sinf(ph)) - 0.5f;
    const float s = rad[x];
    a += v * s;
    b += v * v;
    d += s * s;
  }
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
    d += __shfl_xor_sync(0xffffffffu, d, o);
  }
  if (lane == 0) out[c] = make_float4(a, b, d, 0.f);
}

// GCalcCTF2D + GCtfCC2D for a batch of candidates, one CTA each, over the
// band pixels (s^2, azimuth, exp(-B s^2), spectrum) = band[k];
// cand[c] = (defocus mean px, half difference px, azimuth rad, added phase rad).
__global__ void __launch_bounds__(256) k_ctf_cc2d(const float4* __restrict__ band, int nb,
                                                  const float4* __restrict__ cand, float wave, float cs,
                                                  float4* __restrict__ out) {
  const float4 p = cand[blockIdx.x];
  const float w2 = wave * wave;
  float a = 0.f, b = 0.f, d = 0.f;
  for (int k = threadIdx.x; k < nb; k += blockDim.x) {
    const float4 e = band[k];
    const float df = p.x + p.y * cosf(2.0f * (e.y - p.z));
    const float v = (fabsf(-sinf(p.w + 3.1415926f * wave * e.x * (df - 0.5f * w2 * e.x * cs))) - 0.5f) * e.z;
    a += v * e.w;
    b += v * v;
    d += e.w * e.w;
  }
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
    d += __shfl_xor_sync(0xffffffffu, d, o);
  }
  __shared__ float sa[8], sb[8], sd[8];
  const int w = threadIdx.x / 32;
  if ((threadIdx.x & 31) == 0) {
    sa[w] = a;
    sb[w] = b;
    sd[w] = d;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float ta = 0.f, tb = 0.f, td = 0.f;
    for (int i = 0; i < (int)(blockDim.x / 32); ++i) {
      ta += sa[i];
      tb += sb[i];
      td += sd[i];
    }
    out[blockIdx.x] = make_float4(ta, tb, td, 0.f);
  }
}

// GCalcCTF2D::mGCalculate (FindCtf/GCalcCTF2D.cu:15-37) on the half grid.
__global__ void k_ctf_model(float wave, float cs, float mean, float sigma, float azim, float add,
                            float* __restrict__ ctf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kCX * kTile) return;
  const int y = i / kCX, x = i % kCX;
  const float fx = x * 0.5f / (kCX - 1);
  const float fy = (y - kTile / 2) / (float)kTile;
  const float s2 = fx * fx + fy * fy, w2 = wave * wave;
  const float ang = atanf(fy / (fx + (float)1e-30));
  const float df = mean + sigma * cosf(2.0f * (ang - azim));
  ctf[i] = -sinf(add + 3.1415926f * wave * s2 * (df - 0.5f * w2 * s2 * cs));
}

// GSpectralCC2D::mGCalc2D (FindCtf/GSpectralCC2D.cu:11-95), width 10: one
// CTA per shell.
__global__ void __launch_bounds__(256) k_ctf_shell_cc(const float* __restrict__ ctf,
                                                      const float* __restrict__ sp, float* __restrict__ cc) {
  const int width = 10, bx = blockIdx.x;
  int lo = bx - width / 2, hi = lo + width;
  if (lo < 0) {
    lo = 0;
    hi = width;
  } else if (hi > kCX) {
    lo = kCX - width;
    hi = kCX;
  }
  double s[6] = {0, 0, 0, 0, 0, 0};  // mc, ms, cs, cc, ss, n
  for (int y = threadIdx.x; y < kTile; y += blockDim.x) {
    const float fy = fabsf(y - kTile * 0.5f);
    if (fy >= hi) continue;
    for (int x = 0; x < kCX && x < hi; ++x) {
      const float r = sqrtf((float)(x * x) + fy * fy);
      if (r < lo || r >= hi) continue;
      const float c = fabsf(ctf[y * kCX + x]) - 0.5f, v = sp[y * kCX + x];
      s[0] += c;
      s[1] += v;
      s[2] += c * v;
      s[3] += c * c;
      s[4] += v * v;
      s[5] += 1;
    }
  }
  __shared__ double sh[6][256];
  for (int k = 0; k < 6; ++k) sh[k][threadIdx.x] = s[k];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int k = 0; k < 6; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x) return;
  const double n = sh[5][0];
  if (n == 0) {
    cc[bx] = 0.f;
    return;
  }
  const double mc = sh[0][0] / n, ms = sh[1][0] / n;
  double cv = sh[2][0] / n, sc = sh[3][0] / n - mc * mc, ss = sh[4][0] / n - ms * ms;
  if (sc <= 0 || ss <= 0) {
    cc[bx] = 0.f;
    return;
  }
  cv -= mc * ms;
  cc[bx] = (float)(cv / sqrt(sc * ss));
}

// GCalcCTF2D::mGEmbedCtf (FindCtf/GCalcCTF2D.cu:49-79) on the unpadded copy
// of the lowpassed full spectrum; grid = 512 rows.
__global__ void k_ctf_embed(const float* __restrict__ full, const float* __restrict__ ctf, float fmin,
                            float fmax, float mean, float gain, float* __restrict__ out) {
  const int y = blockIdx.x, hx = kCX - 1;
  const float fy = (y - kTile * 0.5f) / kTile;
  for (int x = threadIdx.x; x < kTile; x += blockDim.x) {
    float v = full[y * kTP + x];
    if (x < hx) {
      float fx = (x - (float)hx) * 0.5f / hx;
      fx = sqrtf(fx * fx + fy * fy);
      if (!(fx < fmin || fx > fmax)) {
        const int ix = hx - x, iy = (kTile - y) % kTile;
        v = (fabsf(ctf[iy * kCX + ix]) - 0.5f) * gain + mean;
      }
    }
    out[y * kTile + x] = v;
  }
}

// ---------------------------------------------------------------- host side

struct Model {  // CCtfParam (FindCtf/CCtfTheory.cpp:36-60), lengths in pixels
  float wave, cs, amp, pix;
};

Model make_model(float kv, float cs_mm, float ac, float pix) {
  Model m;
  m.cs = (float)(cs_mm * 1e7 / pix);
  m.pix = pix;
  const double wl = 12.26 / std::sqrt((double)(kv * 1000) + 0.9784 * kv * kv);
  m.wave = (float)(wl / pix);
  m.amp = (float)std::atan(ac / std::sqrt(1.0f - ac * ac));
  return m;
}

constexpr int kThreads = 256;
inline int blocks(long n) { return (int)((n + kThreads - 1) / kThreads); }

// Scores candidate lists on the device and returns them to the host.
struct Scorer {
  CtfScratch& s;
  cudaStream_t st;
  Model m;
  float lo1 = 0, hi1 = 0;
  int nb = 0;

  int score1d(const std::vector<float2>& cand, std::vector<float>& cc) {
    const int n = (int)cand.size();
    MC3_TRY(s.cand.ensure(sizeof(float4) * n));
    MC3_TRY(s.res.ensure(sizeof(float4) * n));
    MC3_CUDA(cudaMemcpyAsync(s.cand.p, cand.data(), sizeof(float2) * n, cudaMemcpyHostToDevice, st));
    k_ctf_cc1d<<<ceil_div(n, kThreads / 32), kThreads, 0, st>>>(s.cand.as<float2>(), n, s.rad.as<float>(),
                                                                m.wave, m.cs, lo1, hi1, s.res.as<float4>());
    MC3_CHECK_LAUNCH("k_ctf_cc1d");
    std::vector<float4> r(n);
    MC3_CUDA(cudaMemcpyAsync(r.data(), s.res.p, sizeof(float4) * n, cudaMemcpyDeviceToHost, st));
    MC3_CUDA(cudaStreamSynchronize(st));
    cc.resize(n);
    for (int i = 0; i < n; ++i) {  // GCtfCC1D::DoIt (FindCtf/GCtfCC1D.cu:90-121)
      const double a = r[i].x, b = r[i].y, d = r[i].z;
      cc[i] = (b > 0 && d > 0) ? (float)(a / std::sqrt(b * d)) : 0.f;
    }
    return kOk;
  }

  int score2d(const std::vector<float4>& cand, std::vector<float>& cc) {
    const int n = (int)cand.size();
    cc.clear();
    if (!n) return kOk;
    MC3_TRY(s.cand.ensure(sizeof(float4) * n));
    MC3_TRY(s.res.ensure(sizeof(float4) * n));
    MC3_CUDA(cudaMemcpyAsync(s.cand.p, cand.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, st));
    k_ctf_cc2d<<<n, kThreads, 0, st>>>(s.band.as<float4>(), nb, s.cand.as<float4>(), m.wave, m.cs,
                                       s.res.as<float4>());
    MC3_CHECK_LAUNCH("k_ctf_cc2d");
    std::vector<float4> r(n);
    MC3_CUDA(cudaMemcpyAsync(r.data(), s.res.p, sizeof(float4) * n, cudaMemcpyDeviceToHost, st));
    MC3_CUDA(cudaStreamSynchronize(st));
    cc.resize(n);
    for (int i = 0; i < n; ++i) {  // GCtfCC2D::mGCalc1D (FindCtf/GCtfCC2D.cu:66-92)
      const float sd = sqrtf(r[i].y * r[i].z);
      cc[i] = sd == 0 ? 0.f : r[i].x / sd;
    }
    return kOk;
  }
};

// CFindDefocus1D::mBrutalForceSearch (FindCtf/CFindDefocus1D.cpp:81-123).
int search1d(Scorer& sc, const float* dfr, const float* phr, float* best) {
  int nd = 501;
  const float drange = dfr[1] - dfr[0];
  float dstep = drange / (nd - 1);
  if (dstep < 50) dstep = 50.0f;
  nd = (int)(drange / dstep) / 2 * 2 + 1;
  int np = 37;
  const float prange = phr[1] - phr[0];
  float pstep = prange / (np - 1);
  if (pstep < 2) pstep = 2.0f;
  np = (int)(prange / pstep) / 2 * 2 + 1;
  std::vector<float2> cand((size_t)nd * np);
  for (int i = 0; i < nd * np; ++i) {
    const float df = dfr[0] + (i % nd) * dstep, ph = phr[0] + (i / nd) * pstep;
    cand[i] = make_float2(df / sc.m.pix, sc.m.amp + ph * kD2R1);
  }
  std::vector<float> cc;
  MC3_TRY(sc.score1d(cand, cc));
  best[2] = (float)-1e20;
  for (int i = 0; i < nd * np; ++i)
    if (cc[i] > best[2]) {
      best[0] = dfr[0] + (i % nd) * dstep;
      best[1] = phr[0] + (i / nd) * pstep;
      best[2] = cc[i];
    }
  return kOk;
}

// CFindDefocus2D (FindCtf/CFindDefocus2D.cpp:134-342): the state and the
// sweeps, each sweep scored in one launch.
struct Finder2D {
  Scorer& sc;
  float mean = 0, ast = 0, angle = 0, ext = 0, ccmax = 0;
  float phr[2], dfr[2], astr[2], angr[2];

  float4 cand(float m, float a, float g, float ph) const {
    const float dmin = m * (1.0f - a) / sc.m.pix, dmax = m * (1.0f + a) / sc.m.pix;
    return make_float4(0.5f * (dmin + dmax), 0.5f * (dmax - dmin), g * kD2R, sc.m.amp + ph * kD2R);
  }
  int one(float a, float g, float ph, float* cc) {
    std::vector<float> r;
    MC3_TRY(sc.score2d({cand(mean, a, g, ph)}, r));
    *cc = r[0];
    return kOk;
  }
  int find_astig() {
    const float tiny = (float)1e-20;
    const float ar = astr[1] - astr[0], gr = angr[1] - angr[0];
    if (ar < tiny && gr < tiny) return kOk;
    int na = 51, ng = 51;
    const float as = ar / na, gs = gr / ng;
    if (as < 1e-5) na = 1;
    if (gs < 1e-5) ng = 1;
    if (na == 1 && ng == 1) return kOk;
    std::vector<float4> c;
    for (int j = 0; j < ng; ++j)
      for (int i = 0; i < na; ++i) c.push_back(cand(mean, astr[0] + i * as, angr[0] + j * gs, ext));
    std::vector<float> r;
    MC3_TRY(sc.score2d(c, r));
    float gmax = 0, amax = 0, cmax = (float)-1e20;
    for (int j = 0, k = 0; j < ng; ++j)
      for (int i = 0; i < na; ++i, ++k) {
        if (r[k] <= cmax) continue;
        cmax = r[k];
        gmax = angr[0] + j * gs;
        amax = astr[0] + i * as;
      }
    if (cmax <= ccmax) return kOk;
    ast = amax;
    angle = gmax;
    ccmax = cmax;
    return kOk;
  }
  // A one-parameter sweep: values v[i]; take the best above ccmax.
  template <class MakeF>
  int sweep(const std::vector<float>& v, MakeF make, float* best, bool* took) {
    std::vector<float4> c;
    for (float x : v) c.push_back(make(x));
    std::vector<float> r;
    MC3_TRY(sc.score2d(c, r));
    float cmax = (float)-1e20, b = 0;
    for (size_t i = 0; i < v.size(); ++i) {
      if (r[i] <= cmax) continue;
      cmax = r[i];
      b = v[i];
    }
    *took = !v.empty() && !(cmax <= ccmax);
    if (*took) {
      *best = b;
      ccmax = cmax;
    }
    return kOk;
  }
  int refine_ast(float range) {
    if (range < (float)1e-20) return kOk;
    const float lo = fmaxf(ast - range * 0.5f, astr[0]), hi = fminf(ast + range * 0.5f, astr[1]);
    int n = 21;
    float st = (hi - lo) / (n - 1);
    if (st < 0.001f) st = 0.001f;
    n = (int)((hi - lo) / st) / 2 * 2 + 1;
    if (n == 1) return kOk;
    std::vector<float> v;
    for (int i = 0; i < n; ++i) v.push_back(lo + i * st);
    bool took = false;
    float b = 0;
    MC3_TRY(sweep(v, [&](float x) { return cand(mean, x, angle, ext); }, &b, &took));
    if (took) ast = b;
    return kOk;
  }
  int refine_ang(float range) {
    if (range < (float)1e-20) return kOk;
    const float lo = fmaxf(angle - range * 0.5f, angr[0]), hi = fminf(angle + range * 0.5f, angr[1]);
    int n = 51;
    float st = (hi - lo) / (n - 1);
    if (st < 1.0f) st = 1.0f;
    n = (int)((hi - lo) / st) / 2 * 2 + 1;
    if (n == 1) return kOk;
    std::vector<float> v;
    for (int i = 0; i < n; ++i) v.push_back(lo + i * st);
    bool took = false;
    float b = 0;
    MC3_TRY(sweep(v, [&](float x) { return cand(mean, ast, x, ext); }, &b, &took));
    if (took) angle = b;
    return kOk;
  }
  int refine_df(float range) {
    if (range < (float)1e-30) return kOk;
    int n = 31;
    const float lo = fmaxf(mean - range * 0.5f, dfr[0]), hi = fminf(mean + range * 0.5f, dfr[1]);
    float st = (hi - lo) / n;
    if (st < 20) st = 20.0f;
    n = (int)((hi - lo) / st) / 2 * 2 + 1;
    if (n == 1) return kOk;
    std::vector<float> v;
    for (int i = 0; i < n; ++i) v.push_back(lo + i * st);
    bool took = false;
    float b = 0;
    MC3_TRY(sweep(v, [&](float x) { return cand(x, ast, angle, ext); }, &b, &took));
    if (took) mean = b;
    return kOk;
  }
  int refine_phase(float range) {
    if (range < (float)1e-30) return kOk;
    int n = 61;
    float st = range / n;
    if (st < 0.03f) return kOk;
    if (st > 1.0f) {
      st = 1.0f;
      n = (int)(range / st);
      n = n / 2 * 2 + 1;
    }
    float lo = phr[0] - phr[1] * 0.5f, hi = phr[1] + phr[1] * 0.5f;
    if (lo < 0) lo = 0.0f;
    if (hi > 150) hi = 150.0f;
    std::vector<float> v;
    for (int i = 0; i < n; ++i) {
      const float ph = ext + (i - n / 2) * st;
      if (ph < lo || ph > hi) continue;
      v.push_back(ph);
    }
    bool took = false;
    float b = 0;
    MC3_TRY(sweep(v, [&](float x) { return cand(mean, ast, angle, x); }, &b, &took));
    if (took) ext = b;
    return kOk;
  }
  int iterate() {
    MC3_TRY(one(ast, angle, ext, &ccmax));
    const float old = ccmax;
    MC3_TRY(find_astig());
    if (old > ccmax) return kOk;
    const int iters = 20;
    ext = phr[0];
    const float dr = dfr[1] - dfr[0], ar = astr[1] - astr[0], gr = angr[1] - angr[0];
    for (int i = 1; i < iters; ++i) {
      const float scl = 1.0f - i * 0.5f / iters;
      MC3_TRY(refine_ast(scl * ar));
      if (old > ccmax) return kOk;
      ccmax = old;
      MC3_TRY(refine_ang(scl * gr));
      MC3_TRY(refine_df(scl * dr));
      MC3_TRY(refine_phase(scl * phr[1]));
    }
    return kOk;
  }
};

void df_range(float pix, float init, float range, float* r) {  // CFindCtfBase.cpp:83-95
  const float pix2 = pix * pix;
  float dmin = 1000.0f * pix2;
  const float dmax = 30000.0f * pix2;
  if (dmin < 1000.0f) dmin = 1000.0f;
  r[0] = fmaxf(init - 0.5f * range, dmin);
  r[1] = fminf(r[0] + range, dmax);
}
void phase_range(float init, float range, float* r) {  // CFindCtfBase.cpp:97-106
  r[0] = fmaxf(init - 0.5f * range, 0.0f);
  r[1] = fminf(r[0] + range, 180.0f);
}

}  // namespace

int estimate_ctf(const float* d_img, int nx, int ny, float pix, float kv, float cs, float ac,
                 float ext_phase, float* res6, float* image512, bool image_on_device, CtfScratch& s,
                 cudaStream_t st) {
  if (!d_img || !res6 || nx < 2 || ny < 2 || pix <= 0) return kEInval;
  if ((nx | ny) & 1) return kEUnsupported;  // the FFT passes take even sizes
  // ---- CRescaleImage::DoIt (FindCtf/CRescaleImage.cpp:28-68) ----
  float bin = 1.25f / pix;
  if (bin <= 1) bin = 1.0f;
  const float pixN = pix * bin;
  const int nxN = (int)(nx / bin + 0.5f) / 2 * 2, nyN = (int)(ny / bin + 0.5f) / 2 * 2;
  const int pitch = (nxN / 2 + 1) * 2, cN = nxN / 2 + 1;
  // ---- tile grid (CGenAvgSpectrum::SetSizes, FindCtf/CGenAvgSpectrum.cpp:38-63) ----
  const int overlap = (int)(kTile * 0.50f) / 2 * 2, step = kTile - overlap;
  const int ntx = (nxN - overlap) / step, nty = (nyN - overlap) / step;
  if (ntx < 1 || nty < 1) return kEUnsupported;  // no 512 x 512 tile
  const int ntiles = ntx * nty;
  const int offx = (nxN - ntx * kTile + (ntx - 1) * overlap) / 2;
  const int offy = (nyN - nty * kTile + (nty - 1) * overlap) / 2;
  MC3_TRY(s.img.ensure(sizeof(float) * pitch * (size_t)nyN));
  float* img = s.img.as<float>();
  if (bin == 1) {
    k_ctf_pad<<<dim3(ceil_div(pitch, kThreads), nyN), kThreads, 0, st>>>(d_img, nx, img, pitch, nyN);
    MC3_CHECK_LAUNCH("k_ctf_pad");
  } else {
    const int cX = nx / 2 + 1;
    MC3_TRY(s.spec.ensure(sizeof(float2) * cX * (size_t)ny));
    float2* sp = s.spec.as<float2>();
    Batch b1{1, 1, 0, nullptr, 0};
    MC3_TRY(row_r2c(d_img, nx, sp, cX, nx, ny, b1, 1.0f, st));
    ColOps fwd{};
    fwd.dir = -1;
    fwd.scale = (float)(1.0 / nx / ny);
    MC3_TRY(col_fft(sp, sp, cX, cX, ny, b1, fwd, st));
    float2* cimg = reinterpret_cast<float2*>(img);
    MC3_TRY(fourier_crop(sp, cX, ny, cimg, cN, nyN, st));
    ColOps inv{};
    inv.dir = 1;
    inv.scale = 1.0f;
    MC3_TRY(col_fft(cimg, cimg, cN, cN, nyN, b1, inv, st));
    MC3_TRY(row_c2r(cimg, cN, img, pitch, nxN, nyN, b1, st));
  }
  // ---- tile spectra and their average (CGenAvgSpectrum::mAverage) ----
  std::vector<int> org(2 * ntiles);
  for (int t = 0; t < ntiles; ++t) {
    org[2 * t] = offx + (t % ntx) * step;
    org[2 * t + 1] = offy + (t / ntx) * step;
  }
  const size_t tile_f = (size_t)kTP * kTile;
  MC3_TRY(s.org.ensure(sizeof(int) * 2 * ntiles));
  MC3_TRY(s.stats.ensure(sizeof(double) * 2 * ntiles));
  MC3_TRY(s.tiles.ensure(sizeof(float) * tile_f * ntiles));
  MC3_CUDA(cudaMemcpyAsync(s.org.p, org.data(), sizeof(int) * 2 * ntiles, cudaMemcpyHostToDevice, st));
  k_ctf_tile_stats<<<ntiles, kThreads, 0, st>>>(img, pitch, s.org.as<int>(), s.stats.as<double>());
  MC3_CHECK_LAUNCH("k_ctf_tile_stats");
  k_ctf_tile_prep<<<dim3(kTile, ntiles), kThreads, 0, st>>>(img, pitch, s.org.as<int>(), s.stats.as<double>(),
                                                           s.tiles.as<float>());
  MC3_CHECK_LAUNCH("k_ctf_tile_prep");
  float2* tsp = s.tiles.as<float2>();
  {
    Batch br{ntiles, ntiles, (long)tile_f, nullptr, (long)kCX * kTile};
    MC3_TRY(row_r2c(s.tiles.as<float>(), kTP, tsp, kCX, kTile, kTile, br, 1.0f, st));
    Batch bc{ntiles, ntiles, (long)kCX * kTile, nullptr, (long)kCX * kTile};
    ColOps fwd{};
    fwd.dir = -1;
    fwd.scale = 1.0f;
    MC3_TRY(col_fft(tsp, tsp, kCX, kCX, kTile, bc, fwd, st));
  }
  const int nh = kCX * kTile;
  MC3_TRY(s.half.ensure(sizeof(float) * 3 * nh));
  float* raw = s.half.as<float>();
  float* sq = raw + nh;
  float* half = raw + 2 * nh;
  k_ctf_amp_avg<<<blocks(nh), kThreads, 0, st>>>(tsp, ntiles, 1.0f / ntiles, raw);
  MC3_CHECK_LAUNCH("k_ctf_amp_avg");
  // ---- background (CGenAvgSpectrum::mRmBackground) ----
  int box = (int)(kTile * (1.0f / 30.0f));
  box = box / 2 * 2 + 1;
  if (box < 7) box = 7;
  k_ctf_sqrt<<<blocks(nh), kThreads, 0, st>>>(raw, sq, nh);
  k_ctf_rmbg<<<blocks(nh), kThreads, 0, st>>>(raw, sq, box, half);
  MC3_CHECK_LAUNCH("k_ctf_rmbg");
  // ---- lowpass (CGenAvgSpectrum::mLowpass) ----
  MC3_TRY(s.full.ensure(sizeof(float) * tile_f));
  float* full = s.full.as<float>();
  float2* fsp = s.full.as<float2>();
  k_ctf_full<<<blocks((long)tile_f), kThreads, 0, st>>>(half, full);
  MC3_CHECK_LAUNCH("k_ctf_full");
  {
    Batch b1{1, 1, 0, nullptr, 0};
    MC3_TRY(row_r2c(full, kTP, fsp, kCX, kTile, kTile, b1, 1.0f, st));
    ColOps fwd{};
    fwd.dir = -1;
    fwd.scale = (float)(1.0 / kTile / kTile);
    MC3_TRY(col_fft(fsp, fsp, kCX, kCX, kTile, b1, fwd, st));
    const double tmp = (double)kTile * kTile + (double)kTile * kTile;
    k_ctf_lowpass<<<blocks(nh), kThreads, 0, st>>>(fsp, (float)(-5.0f / tmp));
    MC3_CHECK_LAUNCH("k_ctf_lowpass");
    ColOps inv{};
    inv.dir = 1;
    inv.scale = 1.0f;
    MC3_TRY(col_fft(fsp, fsp, kCX, kCX, kTile, b1, inv, st));
    MC3_TRY(row_c2r(fsp, kCX, full, kTP, kTile, kTile, b1, st));
  }
  k_ctf_take_half<<<blocks(nh), kThreads, 0, st>>>(full, half);
  MC3_CHECK_LAUNCH("k_ctf_take_half");
  // ---- fit (CFindCtfMain::mFindCTF, FindCtf/CFindCtfMain.cpp:96-116) ----
  Scorer sc{s, st, make_model(kv, cs, ac, pixN)};
  const float dfrange = 40000.0f * pixN * pixN;
  const float phrange = fminf(ext_phase * 2.0f, 180.0f);
  float resr[2] = {20.0f * pixN, (2.0f * pixN) / 0.8f};  // CFindCtfBase::Setup2
  if (resr[1] < 3.5f) resr[1] = 3.5f;
  MC3_TRY(s.rad.ensure(sizeof(float) * kCX));
  k_ctf_radial<<<1, 288, 0, st>>>(half, s.rad.as<float>());
  MC3_CHECK_LAUNCH("k_ctf_radial");
  const float res1 = ((kCX - 1) * 2) * pixN;
  sc.lo1 = res1 / resr[0];
  sc.hi1 = res1 / resr[1];
  float dfr[2], phr[2], best[3] = {0, 0, 0};
  df_range(pixN, 0.0f, dfrange, dfr);
  phase_range(0.0f, phrange, phr);
  MC3_TRY(search1d(sc, dfr, phr, best));
  float dfmin_px = best[0] / pixN, ext_rad = best[1] * kD2R;
  df_range(pixN, dfmin_px * pixN, 0.3f * dfrange, dfr);
  phase_range(ext_rad / kD2R, 0.3f * phrange, phr);
  MC3_TRY(search1d(sc, dfr, phr, best));
  dfmin_px = best[0] / pixN;
  ext_rad = best[1] * kD2R;
  // band of the 2D correlation (CFindDefocus2D::Setup2, GCtfCC2D::DoIt)
  std::vector<float> hs(nh);
  MC3_CUDA(cudaMemcpyAsync(hs.data(), half, sizeof(float) * nh, cudaMemcpyDeviceToHost, st));
  MC3_CUDA(cudaStreamSynchronize(st));
  float lo2 = (res1 / resr[0]) / kTile, hi2 = (res1 / resr[1]) / kTile;
  if (hi2 > 0.75f) hi2 = 0.75f;
  lo2 *= lo2;
  hi2 *= hi2;
  std::vector<float4> band;
  for (int y = 0; y < kTile; ++y)
    for (int x = 0; x < kCX; ++x) {
      const float cx = (0.5f * x) / (kCX - 1), cy = (y - kTile * 0.5f) / kTile;
      const float c2 = cx * cx + cy * cy;
      if (c2 < lo2 || c2 > hi2) continue;
      const float fx = x * 0.5f / (kCX - 1), fy = (y - kTile / 2) / (float)kTile;
      band.push_back(make_float4(fx * fx + fy * fy, std::atan(fy / (fx + (float)1e-30)),
                                 std::exp(-16.0f * c2), hs[(size_t)y * kCX + x]));
    }
  sc.nb = (int)band.size();
  MC3_TRY(s.band.ensure(sizeof(float4) * (band.size() + 1)));
  MC3_CUDA(cudaMemcpyAsync(s.band.p, band.data(), sizeof(float4) * band.size(), cudaMemcpyHostToDevice, st));
  Finder2D f{sc};
  f.mean = dfmin_px * pixN;
  f.phr[0] = ext_rad / kD2R;
  f.phr[1] = phrange;
  f.dfr[0] = f.mean * 0.9f;
  f.dfr[1] = f.mean * 1.1f;
  f.astr[0] = 0.0f;
  f.astr[1] = 0.06f;
  f.angr[0] = -90.0f;
  f.angr[1] = 90.0f;
  MC3_TRY(f.iterate());
  // ---- resolution (CFindDefocus2D::mCalcCtfRes) ----
  const float dmin = (f.mean * (1.0f - f.ast)) / pixN, dmax = (f.mean * (1.0f + f.ast)) / pixN;
  const float azim = f.angle * kD2R, ext = f.ext * kD2R;
  MC3_TRY(s.ctf.ensure(sizeof(float) * (nh + kCX)));
  float* ctf = s.ctf.as<float>();
  float* shell_cc = ctf + nh;
  k_ctf_model<<<blocks(nh), kThreads, 0, st>>>(sc.m.wave, sc.m.cs, 0.5f * (dmin + dmax), 0.5f * (dmax - dmin),
                                               azim, sc.m.amp + ext, ctf);
  MC3_CHECK_LAUNCH("k_ctf_model");
  k_ctf_shell_cc<<<kCX, kThreads, 0, st>>>(ctf, half, shell_cc);
  MC3_CHECK_LAUNCH("k_ctf_shell_cc");
  std::vector<float> scc(kCX);
  MC3_CUDA(cudaMemcpyAsync(scc.data(), shell_cc, sizeof(float) * kCX, cudaMemcpyDeviceToHost, st));
  MC3_CUDA(cudaStreamSynchronize(st));
  int imax = 1;  // GSpectralCC2D::DoIt (FindCtf/GSpectralCC2D.cu:137-160)
  float fmx = (float)-1e30;
  for (int i = 1; i < kCX; ++i) {
    if (scc[i] <= fmx) continue;
    fmx = scc[i];
    imax = i;
  }
  int shell = imax;
  if (fmx >= 0.143f)
    for (int i = imax; i < kCX; ++i) {
      if (scc[i] < 0.143f) break;
      shell = i;
    }
  res6[0] = dmax * pixN;
  res6[1] = dmin * pixN;
  res6[2] = azim / kD2R;
  res6[3] = ext / kD2R;
  res6[4] = f.ccmax;
  res6[5] = kTile * pixN / shell;
  if (!image512) return kOk;
  // ---- diagnostic image (CFindCtfMain::mEmbedCTF + mAddSpectrumToPackage) ----
  double m1 = 0, m2 = 0;
  for (float v : hs) {  // the half spectrum the fit used
    m1 += v;
    m2 += (double)v * v;
  }
  const float mean = (float)(m1 / nh);
  float sd = (float)(m2 / nh) - mean * mean;
  sd = sd < 0 ? 0.0f : std::sqrt(sd);
  MC3_TRY(s.out.ensure(sizeof(float) * kTile * kTile));
  k_ctf_embed<<<kTile, kThreads, 0, st>>>(full, ctf, pixN / resr[0], pixN / resr[1], mean, sd * 1.5f,
                                          s.out.as<float>());
  MC3_CHECK_LAUNCH("k_ctf_embed");
  MC3_CUDA(cudaMemcpyAsync(image512, s.out.p, sizeof(float) * kTile * kTile,
                           image_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
  MC3_CUDA(cudaStreamSynchronize(st));
  return kOk;
}

}  // namespace mc3
