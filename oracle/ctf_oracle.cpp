// CPU restatement of MotionCor3's CTF estimation on the motion-corrected
// sum (FindCtf/, run by CCorrectFullShift::mEstimateCtf on the first,
// unweighted sum: Correct/CCorrectFullShift.cpp:129-144,179).
// TEST INFRASTRUCTURE ONLY: the checker for libmc3's CUDA CTF path; nothing
// in the product links it.
//
// The Fourier transforms run in FP64 (oracle_rfft2 / oracle_irfft2 of
// mc3_oracle.cpp); every step that takes a decision (frequency masks, the
// CTF model, the grid searches and their acceptance rules) follows the
// reference's FP32 expressions.  Two reads the reference leaves undefined are
// given a definite value here:
//   * GCalcSpectrum::GenFullSpect (FindCtf/GCalcSpectrum.cu:62-82) reads row
//     iCmpY - 0 = iCmpY of the half spectrum for the first output row, one
//     row past the buffer; the Hermitian partner (row 0) is used instead;
//   * CGenAvgSpectrum::mLowpass (FindCtf/CGenAvgSpectrum.cpp:177-185) copies
//     the x = Nyquist column from the padding column of the in-place C2R
//     output; the periodic value (column 0 of the full spectrum) is used.
// GRadialAvg (FindCtf/GRadialAvg.cu:11-31) reads row 512, past the half
// spectrum, for the last angles of radius 256; the index is clamped (that
// radius lies outside every correlation band).  CFindDefocus2D::mIterate's
// first two correlations use m_fExtPhase before it is set
// (FindCtf/CFindDefocus2D.cpp:134-141); 0 is used.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <thread>
#include <vector>

extern "C" {
void oracle_rfft2(const double* img, double* spec, int W, int H, int normalise);
void oracle_irfft2(const double* spec, double* img, int W, int H);
}

namespace {

constexpr int kTile = 512;                // CFindCtfMain::mGenSpectrums, tile size
constexpr int kCmpX = kTile / 2 + 1;      // half spectrum [kTile][kCmpX]
constexpr float kD2R = 0.01745329f;       // FindCtf/CCtfTheory.cpp:8, CFindDefocus2D.cpp:13
constexpr float kD2R1 = 0.0174533f;       // FindCtf/CFindDefocus1D.cpp:12

void par_for(long n, const std::function<void(long, long)>& f) {
  unsigned nt = std::thread::hardware_concurrency();
  if (nt < 1) nt = 1;
  if (nt > 16) nt = 16;
  if (n < 64 || nt == 1) {
    f(0, n);
    return;
  }
  std::vector<std::thread> th;
  const long chunk = (n + nt - 1) / nt;
  for (unsigned t = 0; t < nt; ++t) {
    const long a = t * chunk, b = std::min(n, a + chunk);
    if (a < b) th.emplace_back(f, a, b);
  }
  for (auto& t : th) t.join();
}

// CCtfParam::Setup (FindCtf/CCtfTheory.cpp:36-60): lengths in pixels.
struct Param {
  float wave, cs, amp_phase, pix;
  float dfmin = 0, dfmax = 0, ast = 0, ext = 0;  // pixels, radians
};

Param make_param(float kv, float cs_mm, float ac, float pix) {
  Param p;
  p.cs = (float)(cs_mm * 1e7 / pix);
  p.pix = pix;
  const double wl = 12.26 / std::sqrt((double)(kv * 1000) + 0.9784 * kv * kv);
  p.wave = (float)(wl / pix);
  const float ac2 = ac * ac;
  p.amp_phase = (float)std::atan(ac / std::sqrt(1.0f - ac2));
  return p;
}

// ---- spectrum (CRescaleImage, CGenAvgSpectrum) --------------------------

// GFourierResize2D::mGResize copy mode (Util/GFourierResize2D.cu:7-37).
void crop_spec(const std::vector<double>& in, int inX, int inY, std::vector<double>& out, int outX,
               int outY) {
  out.assign((size_t)2 * outX * outY, 0.0);
  for (int yo = 0; yo < outY; ++yo) {
    int y = yo;
    bool ok = true;
    if (y > outY / 2) {
      y -= outY;
      if (y <= -inY / 2) ok = false;
      else y += inY;
    } else if (y > inY / 2) {
      ok = false;
    }
    if (!ok) continue;
    for (int x = 0; x < outX && x < inX; ++x) {
      out[2 * ((size_t)yo * outX + x)] = in[2 * ((size_t)y * inX + x)];
      out[2 * ((size_t)yo * outX + x) + 1] = in[2 * ((size_t)y * inX + x) + 1];
    }
  }
}

struct Spectrum {
  float pixN = 0;
  int imgN[2] = {0, 0};
  std::vector<float> avg;   // [kTile][kCmpX], DC at (0, kTile/2)
  std::vector<float> full;  // [kTile][kTile], DC at (kTile/2, kTile/2)
};

// CRescaleImage::DoIt (FindCtf/CRescaleImage.cpp:28-68): returns the image
// at pixel size pixN as rows of pitch (nxN/2+1)*2 (only nxN used).
std::vector<float> rescale(const float* img, int nx, int ny, float pix, Spectrum& s, int* pitch) {
  float bin = 1.25f / pix;
  if (bin <= 1) bin = 1.0f;
  s.pixN = pix * bin;
  int nxN = (int)(nx / bin + 0.5f), nyN = (int)(ny / bin + 0.5f);
  nxN = nxN / 2 * 2;
  nyN = nyN / 2 * 2;
  s.imgN[0] = nxN;
  s.imgN[1] = nyN;
  *pitch = (nxN / 2 + 1) * 2;
  std::vector<float> out((size_t)*pitch * nyN, 0.f);
  if (bin == 1) {  // GPad2D::Pad of the rows that fit
    for (int y = 0; y < nyN; ++y)
      for (int x = 0; x < nx && x < *pitch; ++x) out[(size_t)y * *pitch + x] = img[(size_t)y * nx + x];
    return out;
  }
  std::vector<double> d((size_t)nx * ny), spec((size_t)2 * (nx / 2 + 1) * ny), crop;
  for (size_t i = 0; i < d.size(); ++i) d[i] = img[i];
  oracle_rfft2(d.data(), spec.data(), nx, ny, 1);
  crop_spec(spec, nx / 2 + 1, ny, crop, nxN / 2 + 1, nyN);
  std::vector<double> r((size_t)nxN * nyN);
  oracle_irfft2(crop.data(), r.data(), nxN, nyN);
  for (int y = 0; y < nyN; ++y)
    for (int x = 0; x < nxN; ++x) out[(size_t)y * *pitch + x] = (float)r[(size_t)y * nxN + x];
  return out;
}

// CGenAvgSpectrum::SetSizes (FindCtf/CGenAvgSpectrum.cpp:38-63).
void tile_grid(int nx, int ny, int* nt, int* off) {
  const int overlap = (int)(kTile * 0.50f) / 2 * 2;
  const int step = kTile - overlap;
  const int n[2] = {nx, ny};
  for (int a = 0; a < 2; ++a) {
    nt[a] = (n[a] - overlap) / step;
    off[a] = (n[a] - nt[a] * kTile + (nt[a] - 1) * overlap) / 2;
  }
}

// CGenAvgSpectrum::mAverage / mCalcTileSpectrum (FindCtf/CGenAvgSpectrum.cpp:83-146):
// each tile normalised by its mean and std, edge-rounded (Util/GRoundEdge.cu),
// amplitude spectrum of the unnormalised R2C with DC moved to row kTile/2
// (FindCtf/GCalcSpectrum.cu:15-32), averaged with factor 1/n per tile.
bool average_spectrum(const std::vector<float>& img, int pitch, int nx, int ny, std::vector<float>& avg) {
  int nt[2], off[2];
  tile_grid(nx, ny, nt, off);
  const int ntiles = nt[0] * nt[1];
  if (nt[0] < 1 || nt[1] < 1) return false;
  const float fac = 1.0f / ntiles;
  avg.assign((size_t)kCmpX * kTile, 0.f);
  std::vector<std::vector<float>> amp(ntiles);
  const int step = kTile - (int)(kTile * 0.50f) / 2 * 2;
  par_for(ntiles, [&](long t0, long t1) {
    std::vector<double> tile((size_t)kTile * kTile), spec((size_t)2 * kCmpX * kTile);
    for (long t = t0; t < t1; ++t) {
      const int tx = (int)(t % nt[0]), ty = (int)(t / nt[0]);
      const int sx = off[0] + tx * step, sy = off[1] + ty * step;
      double m1 = 0, m2 = 0;
      for (int y = 0; y < kTile; ++y)
        for (int x = 0; x < kTile; ++x) {
          const double v = img[(size_t)(sy + y) * pitch + sx + x];
          tile[(size_t)y * kTile + x] = v;
          m1 += v;
          m2 += v * v;
        }
      const float mean = (float)(m1 / ((double)kTile * kTile));
      float sd = (float)(m2 / ((double)kTile * kTile)) - mean * mean;
      sd = sd <= 0 ? 1.0f : std::sqrt(sd);
      for (int y = 0; y < kTile; ++y)
        for (int x = 0; x < kTile; ++x) {
          float v = ((float)tile[(size_t)y * kTile + x] - mean) / sd;
          const float fx = 2 * std::fabs(x - kTile * 0.5f) / kTile;
          const float fy = 2 * std::fabs(y - kTile * 0.5f) / kTile;
          float r = std::sqrt(fx * fx + fy * fy);
          if (r >= 1.0f) {
            v = 0.f;
          } else {
            r = 0.5f * (1 - std::cos(3.1415926f * r));
            r = 1.0f - std::pow(r, 3.0f);
            v = v * r;
          }
          tile[(size_t)y * kTile + x] = v;
        }
      oracle_rfft2(tile.data(), spec.data(), kTile, kTile, 0);
      std::vector<float>& a = amp[t];
      a.resize((size_t)kCmpX * kTile);
      for (int y = 0; y < kTile; ++y) {
        const int yd = (y + kTile / 2) % kTile;
        for (int x = 0; x < kCmpX; ++x) {
          const double re = spec[2 * ((size_t)y * kCmpX + x)], im = spec[2 * ((size_t)y * kCmpX + x) + 1];
          a[(size_t)yd * kCmpX + x] = (float)std::sqrt(re * re + im * im);
        }
      }
    }
  });
  for (int t = 0; t < ntiles; ++t)  // GAddFrames, tile order
    for (size_t i = 0; i < avg.size(); ++i) avg[i] = avg[i] * 1.0f + amp[t][i] * fac;
  return true;
}

// GRmBackground2D (FindCtf/GRmBackground2D.cu:11-62) with the box of
// CGenAvgSpectrum::mRmBackground (FindCtf/CGenAvgSpectrum.cpp:148-161).
void remove_background(const std::vector<float>& in, std::vector<float>& out) {
  int box = (int)(kTile * (1.0f / 30.0f));
  box = box / 2 * 2 + 1;
  if (box < 7) box = 7;
  const int half = box / 2, hx = kCmpX - 1, hy = kTile / 2;
  out.assign(in.size(), 0.f);
  par_for(kTile, [&](long y0, long y1) {
    for (long y = y0; y < y1; ++y)
      for (int x = 0; x < kCmpX; ++x) {
        const int yc = (int)y - hy;
        float r = x * 0.5f / (kCmpX - 1);
        r = std::sqrt(r * r + yc * yc / (float)(kTile * kTile));
        const size_t i = (size_t)y * kCmpX + x;
        if (r < 0.04) {
          out[i] = 0.f;
          continue;
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
            bg += std::sqrt(in[(size_t)iy * kCmpX + ix]);
          }
        }
        bg /= (box * box);
        bg = bg * bg;
        out[i] = in[i] - bg;
      }
  });
}

// CGenAvgSpectrum::mLowpass (FindCtf/CGenAvgSpectrum.cpp:163-186): full
// spectrum (GCalcSpectrum::GenFullSpect), normalised R2C, Gaussian lowpass
// (Util/GFFTUtil2D.cu:51-65,137-153 with B = 5), C2R; the right half goes back
// into the half spectrum.
void lowpass(std::vector<float>& avg, std::vector<float>& full) {
  const int hx = kCmpX - 1;
  std::vector<double> f((size_t)kTile * kTile), spec((size_t)2 * kCmpX * kTile);
  for (int y = 0; y < kTile; ++y)
    for (int x = 0; x < kTile; ++x) {
      const int xd = x - hx;
      int xs, ys;
      if (xd >= 0) {
        xs = xd;
        ys = y;
      } else {
        xs = -xd;
        ys = (kTile - y) % kTile;
      }
      f[(size_t)y * kTile + x] = avg[(size_t)ys * kCmpX + xs];
    }
  oracle_rfft2(f.data(), spec.data(), kTile, kTile, 1);
  const double tmp = (double)kTile * kTile + (double)kTile * kTile;
  const float scale = (float)(-5.0f / tmp);
  for (int y = 0; y < kTile; ++y) {
    const int yy = y > kTile / 2 ? y - kTile : y;
    for (int x = 0; x < kCmpX; ++x) {
      const float filt = std::exp(scale * (float)(x * x + yy * yy));
      spec[2 * ((size_t)y * kCmpX + x)] *= filt;
      spec[2 * ((size_t)y * kCmpX + x) + 1] *= filt;
    }
  }
  oracle_irfft2(spec.data(), f.data(), kTile, kTile);
  full.resize((size_t)kTile * kTile);
  for (size_t i = 0; i < full.size(); ++i) full[i] = (float)f[i];
  for (int y = 0; y < kTile; ++y)
    for (int x = 0; x < kCmpX; ++x)
      avg[(size_t)y * kCmpX + x] = full[(size_t)y * kTile + (hx + x) % kTile];
}

// ---- CTF model and scores ------------------------------------------------

// GRadialAvg (FindCtf/GRadialAvg.cu:11-31).
void radial_average(const std::vector<float>& s, std::vector<float>& avg) {
  avg.assign(kCmpX, 0.f);
  for (int r = 0; r < kCmpX; ++r) {
    int n = (int)(3.1415926f * r + 0.5f);
    if (n < 1) n = 1;
    else if (n > 180) n = 180;
    float sum = 0.f;
    const float step = 180.0f / n;
    for (int i = 0; i < n; ++i) {
      const float rad = (-90.0f + i * step) * 0.017453f;
      int x = (int)(r * std::cos(rad) + 0.5f);
      int y = (int)(r * std::sin(rad) + kTile / 2 + 0.5f);
      x = std::min(std::max(x, 0), kCmpX - 1);  // r = 256 reaches row 512 near 90 degrees
      y = std::min(std::max(y, 0), kTile - 1);
      sum += s[(size_t)y * kCmpX + x];
    }
    avg[r] = sum / n;
  }
}

// GCalcCTF1D::mGCalculate + GCtfCC1D (FindCtf/GCalcCTF1D.cu:15-32,
// GCtfCC1D.cu:15-59,90-121) with B = 0.
float cc1d(const Param& p, float df_pix, float add_phase, const std::vector<float>& rad, float lo,
           float hi) {
  double cc = 0, s1 = 0, s2 = 0;
  const float w2 = p.wave * p.wave;
  for (int x = 0; x < kCmpX; ++x) {
    if (!(x >= lo && x < hi)) continue;
    float fs2 = (x * 0.5f) / (kCmpX - 1.0f);
    fs2 = fs2 * fs2;
    const float ph = add_phase + 3.141592654f * p.wave * fs2 * (df_pix - 0.5f * w2 * fs2 * p.cs);
    const float c = std::fabs(-std::sin(ph)) - 0.5f;
    const float s = rad[x];
    cc += c * s;
    s1 += c * c;
    s2 += s * s;
  }
  if (s1 > 0 && s2 > 0) return (float)(cc / std::sqrt(s1 * s2));
  return 0.f;
}

// Pixels of the half spectrum with their frequency terms (GCalcCTF2D.cu:15-37,
// GCtfCC2D.cu:15-63).
struct Grid2D {
  std::vector<float> s2, ang, spect;   // all pixels
  std::vector<int> band;               // indices inside the CC band
  std::vector<float> wband;            // exp(-B s^2) there
};

Grid2D make_grid(const std::vector<float>& spect, float lo2, float hi2, float bfac) {
  Grid2D g;
  const size_t n = (size_t)kCmpX * kTile;
  g.s2.resize(n);
  g.ang.resize(n);
  g.spect = spect;
  for (int y = 0; y < kTile; ++y)
    for (int x = 0; x < kCmpX; ++x) {
      const size_t i = (size_t)y * kCmpX + x;
      float fx = x * 0.5f / (kCmpX - 1);
      const float fy = (y - kTile / 2) / (float)kTile;
      g.s2[i] = fx * fx + fy * fy;
      g.ang[i] = std::atan(fy / (fx + (float)1e-30));
      const float cx = (0.5f * x) / (kCmpX - 1), cy = (y - kTile * 0.5f) / kTile;
      const float c2 = cx * cx + cy * cy;
      if (c2 < lo2 || c2 > hi2) continue;
      g.band.push_back((int)i);
      g.wband.push_back(std::exp(-bfac * c2));
    }
  return g;
}

inline float ctf2d(const Param& p, float s2, float ang, float mean, float sigma, float azim, float add) {
  const float w2 = p.wave * p.wave;
  const float df = mean + sigma * std::cos(2.0f * (ang - azim));
  return -std::sin(add + 3.1415926f * p.wave * s2 * (df - 0.5f * w2 * s2 * p.cs));
}

float cc2d(const Param& p, const Grid2D& g, float dfmin, float dfmax, float azim, float ext) {
  const float mean = 0.5f * (dfmin + dfmax), sigma = 0.5f * (dfmax - dfmin);
  const float add = p.amp_phase + ext;
  const long nb = (long)g.band.size();
  const int nt = 16;
  std::vector<double> part(3 * nt, 0.0);
  par_for(nt, [&](long t0, long t1) {
    for (long t = t0; t < t1; ++t) {
      double a = 0, b = 0, c = 0;
      for (long k = t * nb / nt; k < (t + 1) * nb / nt; ++k) {
        const int i = g.band[k];
        const float cv = (std::fabs(ctf2d(p, g.s2[i], g.ang[i], mean, sigma, azim, add)) - 0.5f) * g.wband[k];
        const float sv = g.spect[i];
        a += cv * sv;
        b += cv * cv;
        c += sv * sv;
      }
      part[3 * t] = a;
      part[3 * t + 1] = b;
      part[3 * t + 2] = c;
    }
  });
  double a = 0, b = 0, c = 0;
  for (int t = 0; t < nt; ++t) {
    a += part[3 * t];
    b += part[3 * t + 1];
    c += part[3 * t + 2];
  }
  const float sd = std::sqrt((float)b * (float)c);
  return sd == 0 ? 0.f : (float)a / sd;
}

// ---- searches ------------------------------------------------------------

// CFindCtfBase::mGetDfRange / mGetPhaseRange (FindCtf/CFindCtfBase.cpp:83-106).
void df_range(float pix, float init, float range, float* r) {
  const float pix2 = pix * pix;
  float dmin = 1000.0f * pix2;
  const float dmax = 30000.0f * pix2;
  if (dmin < 1000.0f) dmin = 1000.0f;
  r[0] = std::fmax(init - 0.5f * range, dmin);
  r[1] = std::fmin(r[0] + range, dmax);
}
void phase_range(float init, float range, float* r) {
  r[0] = std::fmax(init - 0.5f * range, 0.0f);
  r[1] = std::fmin(r[0] + range, 180.0f);
}

// CFindDefocus1D::mBrutalForceSearch (FindCtf/CFindDefocus1D.cpp:81-123).
void search1d(const Param& p, const std::vector<float>& rad, const float* res, const float* dfr,
              const float* phr, float* best) {
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
  const float res1 = ((kCmpX - 1) * 2) * p.pix;
  const float lo = res1 / res[0], hi = res1 / res[1];
  const int npts = nd * np;
  std::vector<float> cc(npts);
  par_for(npts, [&](long a, long b) {
    for (long i = a; i < b; ++i) {
      const float df = dfr[0] + (i % nd) * dstep;
      const float ph = phr[0] + (i / nd) * pstep;
      cc[i] = cc1d(p, df / p.pix, p.amp_phase + ph * kD2R1, rad, lo, hi);
    }
  });
  best[2] = (float)-1e20;
  for (int i = 0; i < npts; ++i)
    if (cc[i] > best[2]) {
      best[0] = dfr[0] + (i % nd) * dstep;
      best[1] = phr[0] + (i / nd) * pstep;
      best[2] = cc[i];
    }
}

// CFindDefocus2D (FindCtf/CFindDefocus2D.cpp): state and sweeps.
struct Finder2D {
  const Param& p;
  const Grid2D& g;
  float mean, ast, angle, ext, ccmax, ctfres;
  float phr[2], dfr[2], astr[2], angr[2];

  float corr(float a, float ang, float ph) const {
    const float phr_ = ph * kD2R, angr_ = ang * kD2R;
    const float dmin = mean * (1.0f - a) / p.pix, dmax = mean * (1.0f + a) / p.pix;
    return cc2d(p, g, dmin, dmax, angr_, phr_);
  }
  void find_astig() {  // mFindAstig (:167-204)
    const float tiny = (float)1e-20;
    const float ar = astr[1] - astr[0], gr = angr[1] - angr[0];
    if (ar < tiny && gr < tiny) return;
    int na = 51, ng = 51;
    const float as = ar / na, gs = gr / ng;
    if (as < 1e-5) na = 1;
    if (gs < 1e-5) ng = 1;
    if (na == 1 && ng == 1) return;
    float gmax = 0, amax = 0, cmax = (float)-1e20;
    for (int j = 0; j < ng; ++j) {
      const float gv = angr[0] + j * gs;
      for (int i = 0; i < na; ++i) {
        const float av = astr[0] + i * as;
        const float c = corr(av, gv, ext);
        if (c <= cmax) continue;
        cmax = c;
        gmax = gv;
        amax = av;
      }
    }
    if (cmax <= ccmax) return;
    ast = amax;
    angle = gmax;
    ccmax = cmax;
  }
  void refine_ast(float range) {  // mRefineAstMag (:206-236)
    if (range < (float)1e-20) return;
    const float lo = std::fmax(ast - range * 0.5f, astr[0]);
    const float hi = std::fmin(ast + range * 0.5f, astr[1]);
    int n = 21;
    float st = (hi - lo) / (n - 1);
    if (st < 0.001f) st = 0.001f;
    n = (int)((hi - lo) / st) / 2 * 2 + 1;
    if (n == 1) return;
    float best = 0, cmax = (float)-1e20;
    for (int i = 0; i < n; ++i) {
      const float a = lo + i * st;
      const float c = corr(a, angle, ext);
      if (c <= cmax) continue;
      cmax = c;
      best = a;
    }
    if (cmax <= ccmax) return;
    ast = best;
    ccmax = cmax;
  }
  void refine_ang(float range) {  // mRefineAstAng (:238-267)
    if (range < (float)1e-20) return;
    const float lo = std::fmax(angle - range * 0.5f, angr[0]);
    const float hi = std::fmin(angle + range * 0.5f, angr[1]);
    int n = 51;
    float st = (hi - lo) / (n - 1);
    if (st < 1.0f) st = 1.0f;
    n = (int)((hi - lo) / st) / 2 * 2 + 1;
    if (n == 1) return;
    float best = 0, cmax = (float)-1e20;
    for (int i = 0; i < n; ++i) {
      const float a = lo + i * st;
      const float c = corr(ast, a, ext);
      if (c <= cmax) continue;
      cmax = c;
      best = a;
    }
    if (cmax <= ccmax) return;
    angle = best;
    ccmax = cmax;
  }
  void refine_df(float range) {  // mRefineDfMean (:269-304)
    if (range < (float)1e-30) return;
    const float old = mean;
    int n = 31;
    const float lo = std::fmax(mean - range * 0.5f, dfr[0]);
    const float hi = std::fmin(mean + range * 0.5f, dfr[1]);
    float st = (hi - lo) / n;
    if (st < 20) st = 20.0f;
    n = (int)((hi - lo) / st) / 2 * 2 + 1;
    if (n == 1) return;
    float best = 0, cmax = (float)-1e20;
    for (int i = 0; i < n; ++i) {
      mean = lo + i * st;
      const float c = corr(ast, angle, ext);
      if (c <= cmax) continue;
      best = mean;
      cmax = c;
    }
    if (cmax <= ccmax) {
      mean = old;
      return;
    }
    mean = best;
    ccmax = cmax;
  }
  void refine_phase(float range) {  // mRefinePhase (:306-342)
    if (range < (float)1e-30) return;
    int n = 61;
    float st = range / n;
    if (st < 0.03f) return;
    if (st > 1.0f) {
      st = 1.0f;
      n = (int)(range / st);
      n = n / 2 * 2 + 1;
    }
    float lo = phr[0] - phr[1] * 0.5f, hi = phr[1] + phr[1] * 0.5f;
    if (lo < 0) lo = 0.0f;
    if (hi > 150) hi = 150.0f;
    float cmax = (float)-1e20, best = 0;
    for (int i = 0; i < n; ++i) {
      const float ph = ext + (i - n / 2) * st;
      if (ph < lo || ph > hi) continue;
      const float c = corr(ast, angle, ph);
      if (c <= cmax) continue;
      best = ph;
      cmax = c;
    }
    if (cmax <= ccmax) return;
    ext = best;
    ccmax = cmax;
  }
  void iterate() {  // mIterate (:134-165)
    ccmax = corr(ast, angle, ext);
    const float old = ccmax;
    find_astig();
    if (old > ccmax) return;
    const int iters = 20;
    ext = phr[0];
    const float dr = dfr[1] - dfr[0], ar = astr[1] - astr[0], gr = angr[1] - angr[0];
    for (int i = 1; i < iters; ++i) {
      const float sc = 1.0f - i * 0.5f / iters;
      refine_ast(sc * ar);
      if (old > ccmax) return;
      ccmax = old;
      refine_ang(sc * gr);
      refine_df(sc * dr);
      refine_phase(sc * phr[1]);
    }
  }
};

// GSpectralCC2D (FindCtf/GSpectralCC2D.cu:11-160) with width 10, and
// CFindDefocus2D::mCalcCtfRes (FindCtf/CFindDefocus2D.cpp:362-383).
int spectral_shell(const std::vector<float>& ctf, const std::vector<float>& sp) {
  const int width = 10;
  std::vector<float> cc(kCmpX);
  for (int b = 0; b < kCmpX; ++b) {
    int lo = b - width / 2, hi = lo + width;
    if (lo < 0) {
      lo = 0;
      hi = width;
    } else if (hi > kCmpX) {
      lo = kCmpX - width;
      hi = kCmpX;
    }
    double cs = 0, mc = 0, ms = 0, sc = 0, ss = 0, n = 0;
    for (int y = 0; y < kTile; ++y) {
      const float fy = std::fabs(y - kTile * 0.5f);
      if (fy >= hi) continue;
      for (int x = 0; x < kCmpX && x < hi; ++x) {
        const float r = std::sqrt((float)(x * x) + fy * fy);
        if (r < lo || r >= hi) continue;
        const size_t i = (size_t)y * kCmpX + x;
        const float c = std::fabs(ctf[i]) - 0.5f, s = sp[i];
        mc += c;
        ms += s;
        cs += c * s;
        sc += c * c;
        ss += s * s;
        n += 1;
      }
    }
    if (n == 0) {
      cc[b] = 0;
      continue;
    }
    mc /= n;
    ms /= n;
    cs /= n;
    sc /= n;
    ss /= n;
    sc -= mc * mc;
    ss -= ms * ms;
    if (sc <= 0 || ss <= 0) {
      cc[b] = 0;
      continue;
    }
    cs -= mc * ms;
    cc[b] = (float)(cs / std::sqrt(sc * ss));
  }
  int imax = 1;
  float fmax = (float)-1e30;
  for (int i = 1; i < kCmpX; ++i) {
    if (cc[i] <= fmax) continue;
    fmax = cc[i];
    imax = i;
  }
  if (fmax < 0.143f) return imax;
  int shell = imax;
  for (int i = imax; i < kCmpX; ++i) {
    if (cc[i] < 0.143f) break;
    shell = i;
  }
  return shell;
}

void ctf_image(const Param& p, float dfmin, float dfmax, float azim, float ext, std::vector<float>& out) {
  out.resize((size_t)kCmpX * kTile);
  const float mean = 0.5f * (dfmin + dfmax), sigma = 0.5f * (dfmax - dfmin);
  for (int y = 0; y < kTile; ++y)
    for (int x = 0; x < kCmpX; ++x) {
      const float fx = x * 0.5f / (kCmpX - 1);
      const float fy = (y - kTile / 2) / (float)kTile;
      const float s2 = fx * fx + fy * fy;
      const float ang = std::atan(fy / (fx + (float)1e-30));
      out[(size_t)y * kCmpX + x] = ctf2d(p, s2, ang, mean, sigma, azim, p.amp_phase + ext);
    }
}

// CFindCtf1D::DoIt + CFindCtf2D::DoIt + mGetResults (FindCtf/CFindCtf1D.cpp:53-88,
// CFindCtf2D.cpp:47-84) with the settings of CFindCtfMain::mFindCTF
// (FindCtf/CFindCtfMain.cpp:96-116).  res: dfmax, dfmin (A), azimuth (deg),
// phase (deg), score, resolution (A).
void search(const std::vector<float>& spect, float pixN, float kv, float cs, float ac, float ext_phase,
            Param* out, float* res6) {
  Param p = make_param(kv, cs, ac, pixN);
  const float dfrange = 40000.0f * pixN * pixN;
  const float phrange = std::fmin(ext_phase * 2.0f, 180.0f);
  float resr[2] = {20.0f * pixN, (2.0f * pixN) / 0.8f};  // CFindCtfBase::Setup2 (:34-48)
  if (resr[1] < 3.5f) resr[1] = 3.5f;
  std::vector<float> rad;
  radial_average(spect, rad);
  float dfr[2], phr[2], best[3] = {0, 0, 0};
  df_range(p.pix, 0.0f * p.pix, dfrange, dfr);
  phase_range(0.0f / kD2R, phrange, phr);
  search1d(p, rad, resr, dfr, phr, best);
  float dfmin_px = best[0] / p.pix, ext_rad = best[1] * kD2R;
  df_range(p.pix, dfmin_px * p.pix, 0.3f * dfrange, dfr);
  phase_range(ext_rad / kD2R, 0.3f * phrange, phr);
  search1d(p, rad, resr, dfr, phr, best);
  dfmin_px = best[0] / p.pix;
  ext_rad = best[1] * kD2R;
  // CFindDefocus2D::Setup2 / Setup3 / DoIt (:86-132)
  const float res1 = kTile * p.pix;
  float lo = res1 / resr[0], hi = res1 / resr[1];
  float lo2 = lo / kTile, hi2 = hi / kTile;
  if (hi2 > 0.75f) hi2 = 0.75f;
  lo2 *= lo2;
  hi2 *= hi2;
  Grid2D g = make_grid(spect, lo2, hi2, 16.0f);
  Finder2D f{p, g};
  f.mean = dfmin_px * p.pix;
  f.ast = 0.0f;
  f.angle = 0.0f;
  f.ext = 0.0f;
  f.phr[0] = ext_rad / kD2R;
  f.phr[1] = phrange;
  f.dfr[0] = f.mean * 0.9f;
  f.dfr[1] = f.mean * 1.1f;
  f.astr[0] = 0.0f;
  f.astr[1] = 0.06f;
  f.angr[0] = -90.0f;
  f.angr[1] = 90.0f;
  f.iterate();
  std::vector<float> ctf;
  ctf_image(p, f.mean * (1.0f - f.ast) / p.pix, f.mean * (1.0f + f.ast) / p.pix, f.angle * kD2R,
            f.ext * kD2R, ctf);
  const int shell = spectral_shell(ctf, spect);
  f.ctfres = kTile * p.pix / shell;
  p.dfmin = (f.mean * (1.0f - f.ast)) / p.pix;
  p.dfmax = (f.mean * (1.0f + f.ast)) / p.pix;
  p.ast = f.angle * kD2R;
  p.ext = f.ext * kD2R;
  *out = p;
  res6[0] = p.dfmax * p.pix;
  res6[1] = p.dfmin * p.pix;
  res6[2] = p.ast / kD2R;
  res6[3] = p.ext / kD2R;
  res6[4] = f.ccmax;
  res6[5] = f.ctfres;
}

// CFindCtfMain::mEmbedCTF + mAddSpectrumToPackage (FindCtf/CFindCtfMain.cpp:118-161)
// with GCalcCTF2D::EmbedCtf (FindCtf/GCalcCTF2D.cu:49-79).
void embed(const Param& p, const std::vector<float>& avg, const std::vector<float>& full, float pixN,
           std::vector<float>& out) {
  double m1 = 0, m2 = 0;
  for (float v : avg) {
    m1 += v;
    m2 += (double)v * v;
  }
  const float mean = (float)(m1 / avg.size());
  float sd = (float)(m2 / avg.size()) - mean * mean;
  sd = sd < 0 ? 0.0f : std::sqrt(sd);
  const float gain = sd * 1.5f;
  float resr[2] = {20.0f * pixN, (2.0f * pixN) / 0.8f};
  if (resr[1] < 3.5f) resr[1] = 3.5f;
  const float fmin = pixN / resr[0], fmax = pixN / resr[1];
  std::vector<float> ctf;
  ctf_image(p, p.dfmin, p.dfmax, p.ast, p.ext, ctf);
  out = full;
  const int hx = kCmpX - 1;
  for (int y = 0; y < kTile; ++y)
    for (int x = 0; x < hx; ++x) {
      const float fy = (y - kTile * 0.5f) / kTile;
      float fx = (x - (float)hx) * 0.5f / hx;
      fx = std::sqrt(fx * fx + fy * fy);
      if (fx < fmin || fx > fmax) continue;
      const int ix = hx - x, iy = (kTile - y) % kTile;
      const float v = std::fabs(ctf[(size_t)iy * kCmpX + ix]);
      out[(size_t)y * kTile + x] = (v - 0.5f) * gain + mean;
    }
}

}  // namespace

extern "C" {

// The half spectrum the CTF is fitted to, [512][257] with DC at (0, 256),
// the lowpassed full spectrum [512][512], and the pixel size it refers to.
// Returns 0, or 1 when the rescaled image holds no 512 x 512 tile.
int oracle_ctf_spectrum(const float* img, int nx, int ny, float pix, float* avg_out, float* full_out,
                        float* pix_n) {
  Spectrum s;
  int pitch = 0;
  std::vector<float> r = rescale(img, nx, ny, pix, s, &pitch);
  std::vector<float> raw, bg;
  if (!average_spectrum(r, pitch, s.imgN[0], s.imgN[1], raw)) return 1;
  remove_background(raw, bg);
  std::vector<float> full;
  lowpass(bg, full);
  std::memcpy(avg_out, bg.data(), sizeof(float) * bg.size());
  if (full_out) std::memcpy(full_out, full.data(), sizeof(float) * full.size());
  *pix_n = s.pixN;
  return 0;
}

// The stages of oracle_ctf_spectrum: the averaged amplitude spectrum before
// (raw) and after (bg) background removal, the lowpassed half spectrum and
// full spectrum.  Returns 0, or 1 when no tile fits.
int oracle_ctf_stages(const float* img, int nx, int ny, float pix, float* raw_out, float* bg_out,
                      float* half_out, float* full_out, float* pix_n) {
  Spectrum s;
  int pitch = 0;
  std::vector<float> r = rescale(img, nx, ny, pix, s, &pitch);
  std::vector<float> raw, bg;
  if (!average_spectrum(r, pitch, s.imgN[0], s.imgN[1], raw)) return 1;
  remove_background(raw, bg);
  std::memcpy(raw_out, raw.data(), sizeof(float) * raw.size());
  std::memcpy(bg_out, bg.data(), sizeof(float) * bg.size());
  std::vector<float> full;
  lowpass(bg, full);
  std::memcpy(half_out, bg.data(), sizeof(float) * bg.size());
  std::memcpy(full_out, full.data(), sizeof(float) * full.size());
  *pix_n = s.pixN;
  return 0;
}

// Fit of a [512][257] half spectrum: res6 as CSaveSerialCryoEM::mSaveCtfFit
// prints it (dfmax, dfmin [A], azimuth [deg], phase [deg], score, res [A]).
void oracle_ctf_search(const float* avg, float pix_n, float kv, float cs, float ac, float ext_phase,
                       float* res6) {
  std::vector<float> s(avg, avg + (size_t)kCmpX * kTile);
  Param p;
  search(s, pix_n, kv, cs, ac, ext_phase, &p, res6);
}

// Whole estimate: res6 as above and the 512 x 512 diagnostic image written
// as <stem>_Ctf.mrc (may be NULL).
int oracle_find_ctf(const float* img, int nx, int ny, float pix, float kv, float cs, float ac,
                    float ext_phase, float* res6, float* image512) {
  std::vector<float> avg((size_t)kCmpX * kTile), full((size_t)kTile * kTile);
  float pixN = 0;
  if (oracle_ctf_spectrum(img, nx, ny, pix, avg.data(), full.data(), &pixN)) return 1;
  Param p;
  search(avg, pixN, kv, cs, ac, ext_phase, &p, res6);
  if (image512) {
    std::vector<float> out;
    embed(p, avg, full, pixN, out);
    std::memcpy(image512, out.data(), sizeof(float) * out.size());
  }
  return 0;
}

// CCtfParam::Setup values: wavelength and Cs in pixels, amplitude phase.
void oracle_ctf_param(float kv, float cs, float ac, float pix, float* out3) {
  const Param p = make_param(kv, cs, ac, pix);
  out3[0] = p.wave;
  out3[1] = p.cs;
  out3[2] = p.amp_phase;
}

// GCalcCTF2D::mGCalculate on the half-spectrum grid (defocus in pixels).
void oracle_ctf_model(float kv, float cs, float ac, float pix, float dfmin, float dfmax, float azim_rad,
                      float ext_rad, float* out) {
  const Param p = make_param(kv, cs, ac, pix);
  std::vector<float> c;
  ctf_image(p, dfmin, dfmax, azim_rad, ext_rad, c);
  std::memcpy(out, c.data(), sizeof(float) * c.size());
}

}  // extern "C"
