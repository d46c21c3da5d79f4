// CTF estimation core shared by the CUDA kernels of ctf.cu and the CPU test
// shim (tests/native/ctf_core_shim.cpp): every per-pixel index map and
// expression of FindCtf/ as __host__ __device__ functions, and the host-side
// search driver (CFindCtf1D / CFindCtf2D / CFindDefocus1D / CFindDefocus2D)
// as a template over the scorer that evaluates a sweep of candidates.
//
// Spectra are 512 x 512 tiles (CFindCtfMain::mGenSpectrums): the half
// spectrum is [512][257] with DC at (0, 256); the full spectrum is a padded
// real image [512][514] with DC at (256, 256).
#pragma once
#include <cuda_runtime.h>
#include <vector_types.h>

#include <cmath>
#include <vector>

#ifndef MC3_HD
#define MC3_HD __host__ __device__ __forceinline__
#endif

namespace mc3 {
namespace ctf {

constexpr int kTile = 512;
constexpr int kCX = kTile / 2 + 1;   // 257
constexpr int kTP = 2 * kCX;         // padded row of the full spectrum
constexpr int kNH = kCX * kTile;     // half-spectrum pixels
constexpr float kD2R = 0.01745329f;  // FindCtf/CCtfTheory.cpp:8, CFindDefocus2D.cpp:13
constexpr float kD2R1 = 0.0174533f;  // FindCtf/CFindDefocus1D.cpp:12

// ---- geometry -----------------------------------------------------------------

// CRescaleImage::DoIt (FindCtf/CRescaleImage.cpp:28-68): the binning that
// brings the pixel size to >= 1.25 A and the even rescaled size.
MC3_HD void rescaled_size(int nx, int ny, float pix, int* nxN, int* nyN, float* pixN, float* bin) {
  float b = 1.25f / pix;
  if (b <= 1) b = 1.0f;
  *bin = b;
  *pixN = pix * b;
  *nxN = (int)(nx / b + 0.5f) / 2 * 2;
  *nyN = (int)(ny / b + 0.5f) / 2 * 2;
}

// CGenAvgSpectrum::SetSizes (FindCtf/CGenAvgSpectrum.cpp:38-63): tiles per
// axis, first-tile offsets and the tile step (50 % overlap).
MC3_HD void tile_grid(int nx, int ny, int* nt, int* off, int* step) {
  const int overlap = (int)(kTile * 0.50f) / 2 * 2;
  *step = kTile - overlap;
  nt[0] = (nx - overlap) / *step;
  nt[1] = (ny - overlap) / *step;
  off[0] = (nx - nt[0] * kTile + (nt[0] - 1) * overlap) / 2;
  off[1] = (ny - nt[1] * kTile + (nt[1] - 1) * overlap) / 2;
}

// ---- spectrum stages ------------------------------------------------------

// GRoundEdge factor at tile pixel (x, y) (Util/GRoundEdge.cu:8-23 with the
// mask of CGenAvgSpectrum::mCalcTileSpectrum): 0 outside the inscribed disc.
MC3_HD float tile_edge(int x, int y) {
  const float fx = 2 * fabsf(x - kTile * 0.5f) / kTile;
  const float fy = 2 * fabsf(y - kTile * 0.5f) / kTile;
  float r = sqrtf(fx * fx + fy * fy);
  if (r >= 1.0f) return 0.0f;
  r = 0.5f * (1 - cosf(3.1415926f * r));
  return 1.0f - powf(r, 3.0f);
}

// Mean and std of a tile from its sum and sum of squares (GCalcMoment2D
// moments 1 and 2, CGenAvgSpectrum.cpp:113-118).
MC3_HD void tile_norm(double m1, double m2, float* mean, float* sd) {
  *mean = (float)(m1 / ((double)kTile * kTile));
  float v = (float)(m2 / ((double)kTile * kTile)) - *mean * *mean;
  *sd = v <= 0 ? 1.0f : sqrtf(v);
}

// Box size of CGenAvgSpectrum::mRmBackground (FindCtf/CGenAvgSpectrum.cpp:148-161).
MC3_HD int background_box() {
  int box = (int)(kTile * (1.0f / 30.0f));
  box = box / 2 * 2 + 1;
  return box < 7 ? 7 : box;
}

// GRmBackground2D::mGRemove (FindCtf/GRmBackground2D.cu:11-62) at half-spectrum
// pixel i; sq holds sqrt(in).
MC3_HD float remove_background_at(const float* in, const float* sq, int box, int i) {
  const int hx = kCX - 1, hy = kTile / 2, half = box / 2;
  const int x = i % kCX, yc = i / kCX - hy;
  float r = x * 0.5f / (kCX - 1);
  r = sqrtf(r * r + yc * yc / (float)(kTile * kTile));
  if (r < 0.04) return 0.0f;
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
  return in[i] - bg;
}

// GCalcSpectrum::GenFullSpect (FindCtf/GCalcSpectrum.cu:62-82): source pixel in
// the half spectrum of full-spectrum element i ([512][514]), -1 for padding.
// Row 0 of the left half takes its Hermitian partner (row 0), where the
// reference reads one row past the half spectrum.
MC3_HD int full_source(int i) {
  const int y = i / kTP, x = i % kTP;
  if (x >= kTile) return -1;
  const int xd = x - (kCX - 1);
  const int xs = xd >= 0 ? xd : -xd;
  const int ys = xd >= 0 ? y : (kTile - y) % kTile;
  return ys * kCX + xs;
}

// GFFTUtil2D::mGLowpass factor (Util/GFFTUtil2D.cu:51-65) of half-spectrum
// element i of the 512^2 transform; scale = -B / (512^2 + 512^2).
MC3_HD float lowpass_factor(int i, float scale) {
  const int x = i % kCX;
  int y = i / kCX;
  if (y > kTile / 2) y -= kTile;
  return expf(scale * (float)(x * x + y * y));
}

// CGenAvgSpectrum::mLowpass copy-back (FindCtf/CGenAvgSpectrum.cpp:177-185):
// full-spectrum element feeding half-spectrum pixel i (the x-Nyquist column
// takes the periodic column 0, not the reference's padding column).
MC3_HD int take_half_source(int i) {
  const int y = i / kCX, x = i % kCX;
  return y * kTP + (kCX - 1 + x) % kTile;
}

// GRadialAvg::mGRadAverage (FindCtf/GRadialAvg.cu:11-31) at radius r; the
// reference reads row 512, past the spectrum, for the last angles of radius
// 256, which is clamped here (no correlation band reaches that radius).
MC3_HD float radial_at(const float* s, int r) {
  int n = (int)(3.1415926f * r + 0.5f);
  if (n < 1) n = 1;
  else if (n > 180) n = 180;
  float sum = 0.f;
  const float step = 180.0f / n;
  for (int i = 0; i < n; ++i) {
    const float rad = (-90.0f + i * step) * 0.017453f;
    int x = (int)(r * cosf(rad) + 0.5f);
    int y = (int)(r * sinf(rad) + kTile / 2 + 0.5f);
    x = x < 0 ? 0 : (x > kCX - 1 ? kCX - 1 : x);
    y = y < 0 ? 0 : (y > kTile - 1 ? kTile - 1 : y);
    sum += s[y * kCX + x];
  }
  return sum / n;
}

// ---- CTF model and scores ---------------------------------------------------

// |CTF| - 0.5 of GCalcCTF1D::mGCalculate (FindCtf/GCalcCTF1D.cu:15-32) at index
// x of the radial average; p = (defocus px, added phase rad).
MC3_HD float ctf1d_term(int x, float2 p, float wave, float cs) {
  float fs2 = (x * 0.5f) / (kCX - 1.0f);
  fs2 = fs2 * fs2;
  const float w2 = wave * wave;
  const float ph = p.y + 3.141592654f * wave * fs2 * (p.x - 0.5f * w2 * fs2 * cs);
  return fabsf(-sinf(ph)) - 0.5f;
}

// Weighted |CTF| - 0.5 of GCalcCTF2D + GCtfCC2D at a band pixel
// e = (s^2, azimuth, exp(-B s^2), spectrum) for p = (mean defocus px, half
// difference px, astigmatism azimuth rad, added phase rad).
MC3_HD float ctf2d_term(float4 e, float4 p, float wave, float cs) {
  const float w2 = wave * wave;
  const float df = p.x + p.y * cosf(2.0f * (e.y - p.z));
  return (fabsf(-sinf(p.w + 3.1415926f * wave * e.x * (df - 0.5f * w2 * e.x * cs))) - 0.5f) * e.z;
}

// GCalcCTF2D::mGCalculate (FindCtf/GCalcCTF2D.cu:15-37) at half-spectrum pixel i.
MC3_HD float ctf_model_at(int i, float wave, float cs, float mean, float sigma, float azim, float add) {
  const int y = i / kCX, x = i % kCX;
  const float fx = x * 0.5f / (kCX - 1);
  const float fy = (y - kTile / 2) / (float)kTile;
  const float s2 = fx * fx + fy * fy, w2 = wave * wave;
  const float ang = atanf(fy / (fx + (float)1e-30));
  const float df = mean + sigma * cosf(2.0f * (ang - azim));
  return -sinf(add + 3.1415926f * wave * s2 * (df - 0.5f * w2 * s2 * cs));
}

// Ring [lo, hi) of shell bx in GSpectralCC2D::mGCalc2D (width 10,
// FindCtf/GSpectralCC2D.cu:22-33).
MC3_HD void shell_ring(int bx, int* lo, int* hi) {
  const int width = 10;
  *lo = bx - width / 2;
  *hi = *lo + width;
  if (*lo < 0) {
    *lo = 0;
    *hi = width;
  } else if (*hi > kCX) {
    *lo = kCX - width;
    *hi = kCX;
  }
}

// Pearson correlation of shell sums s = (sum c, sum s, sum cs, sum c^2,
// sum s^2, n) (FindCtf/GSpectralCC2D.cu:76-95).
MC3_HD float shell_cc(const double* s) {
  const double n = s[5];
  if (n == 0) return 0.f;
  const double mc = s[0] / n, ms = s[1] / n;
  double cv = s[2] / n;
  const double sc = s[3] / n - mc * mc, ss = s[4] / n - ms * ms;
  if (sc <= 0 || ss <= 0) return 0.f;
  cv -= mc * ms;
  return (float)(cv / sqrt(sc * ss));
}

// GCalcCTF2D::mGEmbedCtf (FindCtf/GCalcCTF2D.cu:49-79) at output pixel (x, y) of
// the 512 x 512 diagnostic image: the fitted |CTF| inside [fmin, fmax] on the
// left half, else the lowpassed full spectrum ([512][514]).
MC3_HD float embed_at(const float* full, const float* ctf, int x, int y, float fmin, float fmax,
                      float mean, float gain) {
  const int hx = kCX - 1;
  float v = full[y * kTP + x];
  if (x < hx) {
    const float fy = (y - kTile * 0.5f) / kTile;
    float fx = (x - (float)hx) * 0.5f / hx;
    fx = sqrtf(fx * fx + fy * fy);
    if (!(fx < fmin || fx > fmax)) {
      const int ix = hx - x, iy = (kTile - y) % kTile;
      v = (fabsf(ctf[iy * kCX + ix]) - 0.5f) * gain + mean;
    }
  }
  return v;
}

// ---- host side: parameters and the search ------------------------------------

struct Model {  // CCtfParam (FindCtf/CCtfTheory.cpp:36-60), lengths in pixels
  float wave, cs, amp, pix;
};

inline Model make_model(float kv, float cs_mm, float ac, float pix) {
  Model m;
  m.cs = (float)(cs_mm * 1e7 / pix);
  m.pix = pix;
  const double wl = 12.26 / std::sqrt((double)(kv * 1000) + 0.9784 * kv * kv);
  m.wave = (float)(wl / pix);
  m.amp = (float)std::atan(ac / std::sqrt(1.0f - ac * ac));
  return m;
}

// CFindCtfBase::Setup2 resolution range (FindCtf/CFindCtfBase.cpp:34-48), A.
inline void res_range(float pix, float* r) {
  r[0] = 20.0f * pix;
  r[1] = (2.0f * pix) / 0.8f;
  if (r[1] < 3.5f) r[1] = 3.5f;
}

inline void df_range(float pix, float init, float range, float* r) {  // CFindCtfBase.cpp:83-95
  const float pix2 = pix * pix;
  float dmin = 1000.0f * pix2;
  const float dmax = 30000.0f * pix2;
  if (dmin < 1000.0f) dmin = 1000.0f;
  r[0] = fmaxf(init - 0.5f * range, dmin);
  r[1] = fminf(r[0] + range, dmax);
}

inline void phase_range(float init, float range, float* r) {  // CFindCtfBase.cpp:97-106
  r[0] = fmaxf(init - 0.5f * range, 0.0f);
  r[1] = fminf(r[0] + range, 180.0f);
}

// Band of the 2D correlation (CFindDefocus2D::Setup2, GCtfCC2D::DoIt): the
// half-spectrum pixels with lo2 <= s^2 <= hi2, as (s^2, azimuth, exp(-16 s^2),
// spectrum).
inline void make_band(const float* half, float pix, std::vector<float4>& band) {
  float rr[2];
  res_range(pix, rr);
  const float res1 = kTile * pix;
  float lo2 = (res1 / rr[0]) / kTile, hi2 = (res1 / rr[1]) / kTile;
  if (hi2 > 0.75f) hi2 = 0.75f;
  lo2 *= lo2;
  hi2 *= hi2;
  band.clear();
  for (int y = 0; y < kTile; ++y)
    for (int x = 0; x < kCX; ++x) {
      const float cx = (0.5f * x) / (kCX - 1), cy = (y - kTile * 0.5f) / kTile;
      const float c2 = cx * cx + cy * cy;
      if (c2 < lo2 || c2 > hi2) continue;
      const float fx = x * 0.5f / (kCX - 1), fy = (y - kTile / 2) / (float)kTile;
      float4 e;
      e.x = fx * fx + fy * fy;
      e.y = std::atan(fy / (fx + (float)1e-30));
      e.z = std::exp(-16.0f * c2);
      e.w = half[y * kCX + x];
      band.push_back(e);
    }
}

// GSpectralCC2D::DoIt shell choice (FindCtf/GSpectralCC2D.cu:137-160).
inline int fit_shell(const float* cc) {
  int imax = 1;
  float fmx = (float)-1e30;
  for (int i = 1; i < kCX; ++i) {
    if (cc[i] <= fmx) continue;
    fmx = cc[i];
    imax = i;
  }
  if (fmx < 0.143f) return imax;
  int shell = imax;
  for (int i = imax; i < kCX; ++i) {
    if (cc[i] < 0.143f) break;
    shell = i;
  }
  return shell;
}

struct Fit {  // the final CCtfParam: pixels and radians, and the score
  float dfmin, dfmax, azim, ext, score;
};

// CFindCtf1D::DoIt + CFindCtf2D::DoIt (FindCtf/CFindCtf1D.cpp:53-88,
// CFindCtf2D.cpp:47-84) with the settings of CFindCtfMain::mFindCTF
// (FindCtf/CFindCtfMain.cpp:96-116).  S scores candidate sweeps:
//   int score1d(const std::vector<float2>& cand, std::vector<float>& cc);
//   int score2d(const std::vector<float4>& cand, std::vector<float>& cc);
// (1D: (defocus px, added phase) over the radial average given to
// S::set_radial; 2D: (mean px, half difference px, azimuth rad, added phase)
// over the band given to S::set_band).
template <class S>
struct Search {
  S& sc;
  Model m;

  // CFindDefocus1D::mBrutalForceSearch (FindCtf/CFindDefocus1D.cpp:81-123).
  int brute_1d(const float* dfr, const float* phr, float* best) {
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
      cand[i].x = df / m.pix;
      cand[i].y = m.amp + ph * kD2R1;
    }
    std::vector<float> cc;
    int st = sc.score1d(cand, cc);
    if (st) return st;
    best[2] = (float)-1e20;
    for (int i = 0; i < nd * np; ++i)
      if (cc[i] > best[2]) {
        best[0] = dfr[0] + (i % nd) * dstep;
        best[1] = phr[0] + (i / nd) * pstep;
        best[2] = cc[i];
      }
    return 0;
  }

  // CFindDefocus2D state (FindCtf/CFindDefocus2D.cpp); m_fExtPhase, read
  // before it is set by mIterate, starts at 0.
  float mean = 0, ast = 0, angle = 0, ext = 0, ccmax = 0;
  float phr[2] = {0, 0}, dfr[2] = {0, 0}, astr[2] = {0, 0}, angr[2] = {0, 0};

  float4 cand(float mn, float a, float g, float ph) const {
    const float dmin = mn * (1.0f - a) / m.pix, dmax = mn * (1.0f + a) / m.pix;
    float4 c;
    c.x = 0.5f * (dmin + dmax);
    c.y = 0.5f * (dmax - dmin);
    c.z = g * kD2R;
    c.w = m.amp + ph * kD2R;
    return c;
  }
  // One sweep: the best candidate above ccmax is taken.
  int sweep(const std::vector<float4>& c, int* best) {
    *best = -1;
    if (c.empty()) return 0;
    std::vector<float> r;
    int st = sc.score2d(c, r);
    if (st) return st;
    float cmax = (float)-1e20;
    int b = -1;
    for (size_t i = 0; i < c.size(); ++i) {
      if (r[i] <= cmax) continue;
      cmax = r[i];
      b = (int)i;
    }
    if (!(cmax <= ccmax)) {
      *best = b;
      ccmax = cmax;
    }
    return 0;
  }
  int find_astig() {  // mFindAstig (:167-204)
    const float tiny = (float)1e-20;
    const float ar = astr[1] - astr[0], gr = angr[1] - angr[0];
    if (ar < tiny && gr < tiny) return 0;
    int na = 51, ng = 51;
    const float as = ar / na, gs = gr / ng;
    if (as < 1e-5) na = 1;
    if (gs < 1e-5) ng = 1;
    if (na == 1 && ng == 1) return 0;
    std::vector<float4> c;
    for (int j = 0; j < ng; ++j)
      for (int i = 0; i < na; ++i) c.push_back(cand(mean, astr[0] + i * as, angr[0] + j * gs, ext));
    int b = -1;
    int st = sweep(c, &b);
    if (st || b < 0) return st;
    ast = astr[0] + (b % na) * as;
    angle = angr[0] + (b / na) * gs;
    return 0;
  }
  int refine_ast(float range) {  // mRefineAstMag (:206-236)
    if (range < (float)1e-20) return 0;
    const float lo = fmaxf(ast - range * 0.5f, astr[0]), hi = fminf(ast + range * 0.5f, astr[1]);
    int n = 21;
    float st = (hi - lo) / (n - 1);
    if (st < 0.001f) st = 0.001f;
    n = (int)((hi - lo) / st) / 2 * 2 + 1;
    if (n == 1) return 0;
    std::vector<float4> c;
    for (int i = 0; i < n; ++i) c.push_back(cand(mean, lo + i * st, angle, ext));
    int b = -1;
    int s = sweep(c, &b);
    if (!s && b >= 0) ast = lo + b * st;
    return s;
  }
  int refine_ang(float range) {  // mRefineAstAng (:238-267)
    if (range < (float)1e-20) return 0;
    const float lo = fmaxf(angle - range * 0.5f, angr[0]), hi = fminf(angle + range * 0.5f, angr[1]);
    int n = 51;
    float st = (hi - lo) / (n - 1);
    if (st < 1.0f) st = 1.0f;
    n = (int)((hi - lo) / st) / 2 * 2 + 1;
    if (n == 1) return 0;
    std::vector<float4> c;
    for (int i = 0; i < n; ++i) c.push_back(cand(mean, ast, lo + i * st, ext));
    int b = -1;
    int s = sweep(c, &b);
    if (!s && b >= 0) angle = lo + b * st;
    return s;
  }
  int refine_df(float range) {  // mRefineDfMean (:269-304)
    if (range < (float)1e-30) return 0;
    int n = 31;
    const float lo = fmaxf(mean - range * 0.5f, dfr[0]), hi = fminf(mean + range * 0.5f, dfr[1]);
    float st = (hi - lo) / n;
    if (st < 20) st = 20.0f;
    n = (int)((hi - lo) / st) / 2 * 2 + 1;
    if (n == 1) return 0;
    std::vector<float4> c;
    for (int i = 0; i < n; ++i) c.push_back(cand(lo + i * st, ast, angle, ext));
    int b = -1;
    int s = sweep(c, &b);
    if (!s && b >= 0) mean = lo + b * st;
    return s;
  }
  int refine_phase(float range) {  // mRefinePhase (:306-342)
    if (range < (float)1e-30) return 0;
    int n = 61;
    float st = range / n;
    if (st < 0.03f) return 0;
    if (st > 1.0f) {
      st = 1.0f;
      n = (int)(range / st);
      n = n / 2 * 2 + 1;
    }
    float lo = phr[0] - phr[1] * 0.5f, hi = phr[1] + phr[1] * 0.5f;
    if (lo < 0) lo = 0.0f;
    if (hi > 150) hi = 150.0f;
    std::vector<float4> c;
    std::vector<float> v;
    for (int i = 0; i < n; ++i) {
      const float ph = ext + (i - n / 2) * st;
      if (ph < lo || ph > hi) continue;
      c.push_back(cand(mean, ast, angle, ph));
      v.push_back(ph);
    }
    int b = -1;
    int s = sweep(c, &b);
    if (!s && b >= 0) ext = v[b];
    return s;
  }
  int iterate() {  // mIterate (:134-165)
    std::vector<float> r;
    int st = sc.score2d({cand(mean, ast, angle, ext)}, r);
    if (st) return st;
    ccmax = r[0];
    const float old = ccmax;
    if ((st = find_astig())) return st;
    if (old > ccmax) return 0;
    const int iters = 20;
    ext = phr[0];
    const float dr = dfr[1] - dfr[0], ar = astr[1] - astr[0], gr = angr[1] - angr[0];
    for (int i = 1; i < iters; ++i) {
      const float scl = 1.0f - i * 0.5f / iters;
      if ((st = refine_ast(scl * ar))) return st;
      if (old > ccmax) return 0;
      ccmax = old;
      if ((st = refine_ang(scl * gr))) return st;
      if ((st = refine_df(scl * dr))) return st;
      if ((st = refine_phase(scl * phr[1]))) return st;
    }
    return 0;
  }

  // The whole fit of the half spectrum `half` (host copy).
  int run(const float* half, float ext_phase, Fit* out) {
    const float pix = m.pix;
    const float dfrange = 40000.0f * pix * pix;
    const float phrange = fminf(ext_phase * 2.0f, 180.0f);
    std::vector<float> rad(kCX);
    for (int r = 0; r < kCX; ++r) rad[r] = radial_at(half, r);
    int st = sc.set_radial(rad);
    if (st) return st;
    float d[2], p[2], best[3] = {0, 0, 0};
    df_range(pix, 0.0f, dfrange, d);
    phase_range(0.0f, phrange, p);
    if ((st = brute_1d(d, p, best))) return st;
    float dfmin_px = best[0] / pix, ext_rad = best[1] * kD2R;
    df_range(pix, dfmin_px * pix, 0.3f * dfrange, d);
    phase_range(ext_rad / kD2R, 0.3f * phrange, p);
    if ((st = brute_1d(d, p, best))) return st;
    dfmin_px = best[0] / pix;
    ext_rad = best[1] * kD2R;
    std::vector<float4> band;
    make_band(half, pix, band);
    if ((st = sc.set_band(band))) return st;
    mean = dfmin_px * pix;  // CFindDefocus2D::Setup3 / DoIt (:108-132)
    ast = angle = ext = 0.0f;
    phr[0] = ext_rad / kD2R;
    phr[1] = phrange;
    dfr[0] = mean * 0.9f;
    dfr[1] = mean * 1.1f;
    astr[0] = 0.0f;
    astr[1] = 0.06f;
    angr[0] = -90.0f;
    angr[1] = 90.0f;
    if ((st = iterate())) return st;
    out->dfmin = (mean * (1.0f - ast)) / pix;
    out->dfmax = (mean * (1.0f + ast)) / pix;
    out->azim = angle * kD2R;
    out->ext = this->ext * kD2R;
    out->score = ccmax;
    return 0;
  }
};

// res6 as CSaveSerialCryoEM::mSaveCtfFit prints it.
inline void fit_result(const Fit& f, float pix, int shell, float* res6) {
  res6[0] = f.dfmax * pix;
  res6[1] = f.dfmin * pix;
  res6[2] = f.azim / kD2R;
  res6[3] = f.ext / kD2R;
  res6[4] = f.score;
  res6[5] = kTile * pix / shell;
}

}  // namespace ctf
}  // namespace mc3
