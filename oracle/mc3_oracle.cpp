// FP64 CPU oracle for the MotionCor3 hot path -- TEST INFRASTRUCTURE ONLY.
// See mc3_oracle.h.  Every function cites the reference file:line it
// restates (paths relative to the reference project root).
#include "mc3_oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <map>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

typedef std::complex<double> cd;

namespace {

// Parallel loop over [0, n) on all host cores (std::thread; no OpenMP so
// the oracle builds with any C++17 compiler).
int g_threads = 0;
int n_threads() {
  if (g_threads <= 0) {
    unsigned h = std::thread::hardware_concurrency();
    g_threads = h ? (int)h : 1;
  }
  return g_threads;
}
void parallel_for(long n, const std::function<void(long, long)>& body) {
  int T = n_threads();
  if (T <= 1 || n < 2) { body(0, n); return; }
  if (T > n) T = (int)n;
  std::vector<std::thread> th;
  long chunk = (n + T - 1) / T;
  for (int t = 0; t < T; ++t) {
    long a = t * chunk, b = std::min(n, a + chunk);
    if (a >= b) break;
    th.emplace_back(body, a, b);
  }
  for (auto& x : th) x.join();
}

// ======================================================================
// FFT: recursive mixed-radix decimation in time, FP64, any length.
// Independent of the product's Stockham kernels on purpose.
// ======================================================================
struct Plan {
  int n;
  std::vector<int> fac;
  std::vector<cd> w;  // w[k] = exp(-2 pi i k / n)
  int maxp;
};

std::mutex g_plan_mu;
std::map<int, Plan*> g_plans;

const Plan* get_plan(int n) {
  std::lock_guard<std::mutex> lk(g_plan_mu);
  auto it = g_plans.find(n);
  if (it != g_plans.end()) return it->second;
  Plan* p = new Plan;
  p->n = n;
  int m = n;
  while (m % 4 == 0) { p->fac.push_back(4); m /= 4; }
  while (m % 2 == 0) { p->fac.push_back(2); m /= 2; }
  for (int q = 3; m > 1; q += 2) {
    while (m % q == 0) { p->fac.push_back(q); m /= q; }
    if ((long)q * q > m && m > 1) { p->fac.push_back(m); m = 1; }
  }
  p->fac.push_back(1);
  p->maxp = 1;
  for (int f : p->fac) p->maxp = std::max(p->maxp, f);
  p->w.resize(n);
  for (int k = 0; k < n; ++k) {
    double a = -2.0 * M_PI * (double)k / (double)n;
    p->w[k] = cd(std::cos(a), std::sin(a));
  }
  g_plans[n] = p;
  return p;
}

void fft_rec(const cd* x, long xs, cd* y, int n, const Plan* P, int level, int dir,
             cd* scratch) {
  if (n == 1) { y[0] = x[0]; return; }
  const int p = P->fac[level];
  const int m = n / p;
  for (int q = 0; q < p; ++q) fft_rec(x + q * xs, xs * p, y + q * m, m, P, level + 1, dir, scratch);
  const long stride = P->n / n;
  for (int k = 0; k < m; ++k) {
    for (int q = 0; q < p; ++q) scratch[q] = y[q * m + k];
    for (int r = 0; r < p; ++r) {
      const long e0 = k + (long)r * m;
      cd acc = 0.0;
      for (int q = 0; q < p; ++q) {
        const long e = ((long)q * e0) % n;
        cd w = P->w[e * stride];
        if (dir > 0) w = std::conj(w);
        acc += scratch[q] * w;
      }
      y[k + (long)r * m] = acc;
    }
  }
}

// y = DFT(x) of length n; dir -1 forward, +1 inverse (unnormalised).
void fft1(const cd* x, cd* y, int n, int dir) {
  const Plan* P = get_plan(n);
  std::vector<cd> scratch(P->maxp);
  fft_rec(x, 1, y, n, P, 0, dir, scratch.data());
}

// Normalised (optionally) R2C, layout [H][W/2+1]; cuFFT semantics of
// Util/CCufft2D.cpp:65-80 (forward, then x 1/(Nx*Ny) when bNorm).
void rfft2(const double* img, cd* spec, int W, int H, bool norm) {
  const int M = W / 2 + 1;
  get_plan(W);
  get_plan(H);
  parallel_for(H, [&](long y0, long y1) {
    std::vector<cd> a(W), b(W);
    for (long y = y0; y < y1; ++y) {
      for (int x = 0; x < W; ++x) a[x] = cd(img[y * W + x], 0.0);
      fft1(a.data(), b.data(), W, -1);
      for (int k = 0; k < M; ++k) spec[y * M + k] = b[k];
    }
  });
  const double s = norm ? 1.0 / ((double)W * (double)H) : 1.0;
  parallel_for(M, [&](long k0, long k1) {
    std::vector<cd> a(H), b(H);
    for (long k = k0; k < k1; ++k) {
      for (int y = 0; y < H; ++y) a[y] = spec[(long)y * M + k];
      fft1(a.data(), b.data(), H, -1);
      for (int y = 0; y < H; ++y) spec[(long)y * M + k] = b[y] * s;
    }
  });
}

// Whether cuFFT's single-image 2D C2R plan (Util/CCufft2D.cpp:39-53,
// cufftPlan2d) keeps the imaginary parts of each row's DC and Nyquist terms
// for a W x H image: they then add -(b0 + bM) to every even sample and
// b0 - bM to every odd sample of the row (measured by probing the library
// with single imaginary DC / Nyquist terms).
bool c2r_keeps_edge_imag(int W, int H) {
  // probed sizes: kept for 2048^2, 4096^2, 4096 x 2048, 2048 x 4096,
  // 1024 x 2048; dropped for 64^2 .. 1536^2, 384 x 320, 192 x 160, 408^2,
  // 410 x 408, 2882 x 2048, 5760 x 4092, 2048 x 1024
  auto pow2 = [](int n) { return n > 0 && (n & (n - 1)) == 0; };
  return pow2(W) && pow2(H) && H >= 2048;
}

// Unnormalised C2R [H][W/2+1] -> [H][W]: complex inverse along y for every
// kx column, then a real inverse along x that uses only the real parts of
// the DC and Nyquist terms (Util/CCufft2D.cpp:105-120 semantics), plus the
// rows' DC / Nyquist imaginary parts where cuFFT keeps them.
void irfft2(const cd* spec, double* img, int W, int H) {
  const bool keep = c2r_keeps_edge_imag(W, H);
  const int M = W / 2 + 1;
  std::vector<cd> tmp((long)H * M);
  get_plan(W);
  get_plan(H);
  parallel_for(M, [&](long k0, long k1) {
    std::vector<cd> a(H), b(H);
    for (long k = k0; k < k1; ++k) {
      for (int y = 0; y < H; ++y) a[y] = spec[(long)y * M + k];
      fft1(a.data(), b.data(), H, +1);
      for (int y = 0; y < H; ++y) tmp[(long)y * M + k] = b[y];
    }
  });
  parallel_for(H, [&](long y0, long y1) {
    std::vector<cd> a(W), b(W);
    for (long y = y0; y < y1; ++y) {
      const cd* r = &tmp[y * M];
      a[0] = cd(r[0].real(), 0.0);
      a[W / 2] = cd(r[W / 2].real(), 0.0);
      for (int k = 1; k < W / 2; ++k) {
        a[k] = r[k];
        a[W - k] = std::conj(r[k]);
      }
      fft1(a.data(), b.data(), W, +1);
      const double b0 = keep ? r[0].imag() : 0.0, bm = keep ? r[W / 2].imag() : 0.0;
      for (int x = 0; x < W; ++x)
        img[y * W + x] = b[x].real() + ((x & 1) ? (b0 - bm) : -(b0 + bm));
    }
  });
}

// ======================================================================
// Geometry (CBufferPool.cpp:185-270, Util/GFourierResize2D.cu:49-80)
// ======================================================================
struct Geo {
  int W, H, N;
  int cmpX, cmpY;
  int xcfCmpX, xcfCmpY;
  float xcfBin[2];
  bool patch;
  int patCmpX, patCmpY;  // pat buffer (CBufferPool.cpp:244-262)
  int patSizeX, patSizeY;  // CPatchCenters patch size (CPatchCenters.cpp:50-51)
  int Px, Py;
};

Geo make_geo(int W, int H, int N, const oracle_params* p) {
  Geo g;
  g.W = W; g.H = H; g.N = N;
  g.cmpX = W / 2 + 1;
  g.cmpY = H;
  // CBufferPool::mCreateXcfBuffer (CBufferPool.cpp:220-242)
  float fBinX = W / 2048.0f;
  float fBinY = H / 2048.0f;
  float fBin = (float)std::fmin(fBinX, fBinY);
  if (fBin < 1) fBin = 1.0f;
  int iXcfX = (int)(W / fBin + 0.5f);
  int iXcfY = (int)(H / fBin + 0.5f);
  g.xcfCmpX = iXcfX / 2 + 1;
  g.xcfCmpY = iXcfY / 2 * 2;
  g.xcfBin[0] = (g.cmpX - 1.0f) / (g.xcfCmpX - 1.0f);
  g.xcfBin[1] = g.cmpY * 1.0f / g.xcfCmpY;
  // CBufferPool::mCreatePatBuffer (CBufferPool.cpp:244-262)
  g.Px = p->patch[0];
  g.Py = p->patch[1];
  g.patch = false;
  g.patCmpX = g.patCmpY = g.patSizeX = g.patSizeY = 0;
  if (g.Px > 1 && g.Py > 1) {
    int iX = (g.xcfCmpX - 1) * 2, iY = g.xcfCmpY;
    int iPatX = iX / g.Px, iPatY = iY / g.Py;
    if (iPatX <= iX / 2 && iPatY <= iY / 2) {
      g.patch = true;
      g.patCmpX = iPatX / 2 + 1;
      g.patCmpY = iPatY / 2 * 2;
      g.patSizeX = iX / g.Px / 2 * 2;
      g.patSizeY = iY / g.Py / 2 * 2;
    }
  }
  return g;
}

// ======================================================================
// Frame integration / groups (DataUtil/CFmIntParam.cpp:260-278, 423-429;
// DataUtil/CFmGroupParam.cpp:26-78, 115-123) without -FmIntFile/-Throw.
// ======================================================================
struct Groups {
  std::vector<int> start, size;
  std::vector<float> center;     // group centres
  std::vector<float> fm_center;  // rendered-frame time stamps
  int binZ;
};

// CFmGroupParam::Setup (DataUtil/CFmGroupParam.cpp:26-78) over rendered
// frames of int_size raw frames each (all 1 when int_size is NULL), whose
// time stamps are start + 0.5*(size-1) (CFmIntParam.cpp:276-283).
Groups make_groups(int N, int binZ, const int* int_size = nullptr) {
  Groups G;
  G.binZ = binZ;
  std::vector<int> sz(N, 1);
  if (int_size) sz.assign(int_size, int_size + N);
  G.fm_center.resize(N);
  int raw0 = 0, minRaw = sz.empty() ? 1 : sz[0];
  for (int i = 0; i < N; ++i) {
    G.fm_center[i] = raw0 + 0.5f * (sz[i] - 1.0f);
    raw0 += sz[i];
    minRaw = std::min(minRaw, sz[i]);
  }
  const int maxRaw = binZ * minRaw;
  int f = 0;
  while (f < N) {
    G.start.push_back(f);
    int n = 0, raw = 0;
    while (true) {
      raw += sz[f];
      n += 1;
      f += 1;
      if (f >= N) break;
      if (raw >= maxRaw) break;
    }
    G.size.push_back(n);
  }
  for (size_t g = 0; g < G.start.size(); ++g) {
    float s = 0.0f;
    for (int i = 0; i < G.size[g]; ++i) s += G.fm_center[G.start[g] + i];
    G.center.push_back(s / G.size[g]);
  }
  return G;
}

// ======================================================================
// Shift bookkeeping in FP32 (Align/CStackShift.cpp, CInterpolateShift.cpp,
// Util/CRemoveSpikes1D.cpp, Util/CSplineFit1D.cpp, LibSrc/Util/Util_LinEqs.cpp)
// ======================================================================
struct Shifts {  // [X...][Y...] like CStackShift
  int n;
  std::vector<float> v;
  explicit Shifts(int n_ = 0) : n(n_), v(2 * (size_t)n_, 0.0f) {}
  float& x(int i) { return v[i]; }
  float& y(int i) { return v[n + i]; }
};

// Util_LinEqs::DoIt (LibSrc/Util/Util_LinEqs.cpp:19-41): Gauss-Jordan with
// full pivot search, FP32 matrix, FP64 pivot normalisation.
bool lin_eqs(float* A, float* b, int dim) {
  std::vector<int> colIdx(dim), rowIdx(dim), piv(dim, 0);
  for (int ip = 0; ip < dim; ++ip) {
    int iX = 0, iY = 0;
    bool found = false;
    float fMax = 0.0f;
    for (int y = 0; y < dim; ++y) {
      if (piv[y] == 1) continue;
      for (int x = 0; x < dim; ++x) {
        if (piv[x] == 1) continue;
        float c = (float)std::fabs(A[y * dim + x]);
        if (c <= fMax) continue;
        fMax = c; iX = x; iY = y; found = true;
      }
    }
    if (!found) return false;
    piv[iX] += 1;
    colIdx[ip] = iX;
    rowIdx[ip] = iY;
    if (A[iY * dim + iX] == 0.0f) return false;
    // swap rows colIdx <-> rowIdx (:88-110)
    int r1 = colIdx[ip], r2 = rowIdx[ip];
    if (r1 != r2) {
      for (int x = 0; x < dim; ++x) std::swap(A[r1 * dim + x], A[r2 * dim + x]);
      std::swap(b[r1], b[r2]);
    }
    // normalise (:112-128)
    int col = colIdx[ip];
    double inv = 1.0 / (A[col * dim + col] + 1e-30);
    for (int x = 0; x < dim; ++x) A[col * dim + x] = (float)(A[col * dim + x] * inv);
    b[col] = (float)(b[col] * inv);
    // reduce (:130-148)
    for (int y = 0; y < dim; ++y) {
      if (y == col) continue;
      float d = A[y * dim + col];
      for (int x = 0; x < dim; ++x) A[y * dim + x] -= (A[col * dim + x] * d);
      b[y] -= (b[col] * d);
    }
  }
  return true;
}

// CSplineFit1D (Util/CSplineFit1D.cpp:43-115)
struct Spline {
  int nk, dim;
  const float* knots;
  std::vector<float> terms, cur, coeff, mat;
  void setup(int n, const float* k) {
    nk = n; dim = n + 3; knots = k;
    terms.assign(dim, 0.f); cur.assign(dim, 0.f); coeff.assign(dim, 0.f); mat.assign(dim * dim, 0.f);
  }
  void calc_terms(float x) {
    terms[0] = 1;
    for (int i = 1; i < 3; ++i) terms[i] = terms[i - 1] * x;
    for (int i = 0; i < nk; ++i) terms[i + 3] = 0.f;
    for (int i = 0; i < nk; ++i) {
      if (x < knots[i]) break;
      float v = x - knots[i];
      terms[i + 3] = v * v;
    }
  }
  void calc_cur(float x) {
    for (int i = 0; i < dim; ++i) cur[i] = 0.f;
    cur[1] = 1.0f;
    cur[2] = 2.0f * x;
    for (int i = 0; i < nk; ++i) {
      float v = x - knots[i];
      if (v > 0) break;
      cur[i + 3] = 2.0f * v;
    }
  }
  bool fit(const float* X, const float* Y, const bool* bad, int n, float* out, float reg) {
    std::fill(mat.begin(), mat.end(), 0.f);
    std::fill(coeff.begin(), coeff.end(), 0.f);
    std::fill(terms.begin(), terms.end(), 0.f);
    std::fill(cur.begin(), cur.end(), 0.f);
    for (int i = 0; i < n; ++i) {
      if (bad && bad[i]) continue;
      calc_terms(X[i]);
      if (reg != 0.0f) calc_cur(X[i]);
      for (int r = 0; r < dim; ++r) {
        for (int c = 0; c < dim; ++c) {
          float p1 = terms[r] * terms[c];
          float p2 = reg * cur[r] * cur[c];
          mat[r * dim + c] += (p1 + p2);
        }
        coeff[r] += (terms[r] * Y[i]);
      }
    }
    if (!lin_eqs(mat.data(), coeff.data(), dim)) return false;
    for (int i = 0; i < n; ++i) {
      calc_terms(X[i]);
      float f = 0.0f;
      for (int k = 0; k < dim; ++k) f += coeff[k] * terms[k];
      out[i] = f;
    }
    return true;
  }
};

// CRemoveSpikes1D::mRemoveSingle (Util/CRemoveSpikes1D.cpp:127-148)
void remove_single(float* raw, int n, float* buf) {
  std::memcpy(buf, raw, sizeof(float) * n);
  float tol = 5.0f;
  int end = n - 1;
  for (int i = 1; i < end; ++i) {
    if (std::fabs(buf[i] - buf[i - 1]) < tol) continue;
    if (std::fabs(buf[i] - buf[i + 1]) < tol) continue;
    raw[i] = (buf[i - 1] + buf[i + 1]) / 2.0f;
  }
  tol = 10.0f;
  if (std::fabs(buf[0] - buf[1]) > tol && std::fabs(buf[0]) > std::fabs(buf[1]))
    raw[0] = 2.0f * buf[1] - buf[2];
  if (std::fabs(buf[end] - buf[end - 1]) > tol && std::fabs(buf[end]) > std::fabs(buf[end - 1]))
    raw[end] = 2.0f * buf[end - 1] - buf[end - 2];
}

// CRemoveSpikes1D::SetDataSize + DoIt(bSingle=false) (:31-105, 107-125)
void remove_spikes(float* sx, float* sy, int n) {
  std::vector<float> time(n), buf(n), fitX(n, 0.f), fitY(n, 0.f);
  std::vector<bool> badv(n, false);
  bool* bad = new bool[n];
  float fact = 1.0f / n;
  for (int i = 0; i < n; ++i) time[i] = (float)std::sqrt(i * fact);
  const int kd = 15;
  int nk = (n - 2 * kd) / kd;
  if (nk < 0) nk = 0;
  else if (nk > 6) nk = 6;
  if (nk == 0 && n >= 2 * kd) nk = 1;
  std::vector<float> knots(nk);
  for (int i = 0; i < nk; ++i) knots[i] = time[(i + 1) * kd];
  Spline sp;
  sp.setup(nk, knots.data());
  for (int i = 0; i < 2; ++i) {
    remove_single(sx, n, buf.data());
    remove_single(sy, n, buf.data());
  }
  for (int i = 0; i < n; ++i) bad[i] = false;
  const float reg = (float)1e-20;
  sp.fit(time.data(), sx, bad, n, fitX.data(), reg);
  sp.fit(time.data(), sy, bad, n, fitY.data(), reg);
  auto find_bad = [&](float* raw, float* fit, float tol) {
    bool has = false;
    for (int i = 0; i < n; ++i) bad[i] = false;
    for (int i = 0; i < n; ++i) {
      if (std::fabs(fit[i] - raw[i]) > tol) {
        if (std::fabs(raw[i]) > std::fabs(fit[i])) { raw[i] = fit[i]; has = true; }
      }
    }
    return has;
  };
  std::memcpy(buf.data(), sx, sizeof(float) * n);
  if (find_bad(buf.data(), fitX.data(), 3.0f)) sp.fit(time.data(), buf.data(), bad, n, fitX.data(), reg);
  std::memcpy(buf.data(), sy, sizeof(float) * n);
  // The y refit reads the unmodified y shifts (CRemoveSpikes1D.cpp:88).
  if (find_bad(buf.data(), fitY.data(), 3.0f)) sp.fit(time.data(), sy, bad, n, fitY.data(), reg);
  for (int i = 0; i < n; ++i) {
    float tol = 5.0f;
    if (i > 20) tol = 4.0f;
    if (i < 50) tol = 3.0f;
    float dx = fitX[i] - sx[i];
    float dy = fitY[i] - sy[i];
    if (std::fabs(dx) > tol) sx[i] = fitX[i];
    if (std::fabs(dy) > tol) sy[i] = fitY[i];
  }
  delete[] bad;
}

// CStackShift::Smooth (Align/CStackShift.cpp:180-198)
void smooth(Shifts& s, float w) {
  if (w >= 1) return;
  const int n = s.n;
  std::vector<float> o = s.v;
  float w2 = 0.5f * (1.0f - w);
  for (int i = 1; i < n - 1; ++i) {
    o[i] = w * s.v[i] + w2 * (s.v[i - 1] + s.v[i + 1]);
    o[n + i] = w * s.v[n + i] + w2 * (s.v[n + i - 1] + s.v[n + i + 1]);
  }
  s.v = o;
}

// CInterpolateShift::DoIt (Align/CInterpolateShift.cpp:36-143)
Shifts interpolate(Shifts& grp, const Groups& G, int nFrames, bool nearest) {
  Shifts out(nFrames);
  const int nG = grp.n;
  if (nFrames == nG) { out.v = grp.v; return out; }
  if (nearest) {
    for (int g = 0; g < nG; ++g)
      for (int i = 0; i < G.size[g]; ++i) {
        out.x(G.start[g] + i) = grp.x(g);
        out.y(G.start[g] + i) = grp.y(g);
      }
    return out;
  }
  for (int i = 0; i < nFrames; ++i) {
    const float fc = G.fm_center[i];  // frame time stamps (CFmIntParam.cpp:276-283)
    int g;
    if (fc <= G.center[0]) g = 1;
    else {
      g = nG - 1;
      for (int k = 1; k < nG; ++k)
        if (fc < G.center[k]) { g = k; break; }
    }
    int f = g - 1;
    float difG = G.center[g] - G.center[f];
    float difF = fc - G.center[f];
    float slx = (grp.x(g) - grp.x(f)) / difG;
    float sly = (grp.y(g) - grp.y(f)) / difG;
    out.x(i) = grp.x(f) + slx * difF;
    out.y(i) = grp.y(f) + sly * difF;
  }
  return out;
}

// CPeak2D::DoIt (Align/CPeak2D.cpp:39-109)
void peak2d(const float* img, int sx, int sy, float* shift) {
  int n = sx * sy;
  float pk = img[0];
  int ip = 0;
  for (int i = 1; i < n; ++i) {
    if (pk >= img[i]) continue;
    pk = img[i];
    ip = i;
  }
  int px = ip % sx, py = ip / sx;
  if (px == 0) px = 1;
  if (py == 0) py = 1;
  if (px == sx - 1) px -= 1;
  if (py == sy - 1) py -= 1;
  int ic = py * sx + px;
  double a = (img[ic + 1] + img[ic - 1]) * 0.5 - img[ic];
  double b = (img[ic + 1] - img[ic - 1]) * 0.5;
  double c = (img[ic + sx] + img[ic - sx]) * 0.5f - img[ic];
  double d = (img[ic + sx] - img[ic - sx]) * 0.5;
  double cx = -b / (2 * a + 1e-30);
  double cy = -d / (2 * c + 1e-30);
  if (std::fabs(cx) > 1) cx = 0;
  if (std::fabs(cy) > 1) cy = 0;
  float fx = (float)(px + cx), fy = (float)(py + cy);
  shift[0] = fx - sx / 2;
  shift[1] = fy - sy / 2;
}

// ======================================================================
// Spectral operations
// ======================================================================
// GPhaseShift2D::mGShiftFrame (Util/GPhaseShift2D.cu:12-38): multiply by
// exp(i*phi), phi = 2 pi (kx*sx/Nx + ky*sy/Ny), ky wrapped to (-Ny/2, Ny/2].
void phase_shift(const cd* in, cd* out, int cmpX, int cmpY, double sx, double sy, bool add) {
  const int Nx = (cmpX - 1) * 2;
  const int Ny = cmpY;
  for (int y = 0; y < cmpY; ++y) {
    int yy = y > cmpY / 2 ? y - cmpY : y;
    const double py = 2.0 * M_PI * yy * sy / Ny;
    for (int x = 0; x < cmpX; ++x) {
      double phi = 2.0 * M_PI * x * sx / Nx + py;
      cd v = in[(long)y * cmpX + x] * cd(std::cos(phi), std::sin(phi));
      if (add) out[(long)y * cmpX + x] += v;
      else out[(long)y * cmpX + x] = v;
    }
  }
}

// GFourierResize2D::mGResize (Util/GFourierResize2D.cu:7-37), copy mode.
void fourier_resize(const cd* in, int inX, int inY, cd* out, int outX, int outY) {
  for (int yo = 0; yo < outY; ++yo) {
    for (int x = 0; x < outX; ++x) {
      cd v = 0.0;
      bool ok = x < inX;
      int y = yo;
      if (ok) {
        if (y > outY / 2) {
          y -= outY;
          if (y <= -inY / 2) ok = false;
          else y += inY;
        } else if (y > inY / 2) ok = false;
      }
      if (ok) v = in[(long)y * inX + x];
      // The reference leaves skipped outputs untouched; its output buffers
      // are only ever read where they were written for these sizes.
      out[(long)yo * outX + x] = v;
    }
  }
}

// GCorrelateSum2D::DoIt (Align/GCorrelateSum2D.cu:108-140) + window copy.
void correlate_window(const cd* grp, const cd* sum, int cmpX, int cmpY, float bf, bool phaseOnly,
                      int sx, int sy, float* win) {
  const long n = (long)cmpX * cmpY;
  std::vector<cd> c(n);
  const double filt0 = -0.25 * (double)bf / ((double)(cmpX - 1) * cmpY);
  for (int y = 0; y < cmpY; ++y) {
    int yy = y > cmpY / 2 ? y - cmpY : y;
    for (int x = 0; x < cmpX; ++x) {
      long i = (long)y * cmpX + x;
      cd g = grp[i];
      cd s = sum[i] - g;  // mGConv with bSubtract
      cd v(g.real() * s.real() + g.imag() * s.imag(), g.real() * s.imag() - g.imag() * s.real());
      double f = std::exp(filt0 * ((double)x * x + (double)yy * yy));
      if (phaseOnly) f = f / (std::abs(v) + 1e-20);
      if (i > 0) v *= f;
      else v = 0.0;  // mGLowpass DC (:54-61)
      if ((x + y) % 2) v = -v;  // mGCenterOrigin
      c[i] = v;
    }
  }
  const int Nx = (cmpX - 1) * 2, Ny = cmpY;
  std::vector<double> img((long)Nx * Ny);
  irfft2(c.data(), img.data(), Nx, Ny);
  const int x0 = (Nx - sx) / 2, y0 = (cmpY - sy) / 2;
  for (int j = 0; j < sy; ++j)
    for (int i = 0; i < sx; ++i) win[j * sx + i] = (float)img[(long)(y0 + j) * Nx + x0 + i];
}

// ======================================================================
// Iterative alignment (Align/CIterativeAlign.cpp:55-156,
// Align/CAlignStack.cpp:82-215, Align/CAlignedSum.cpp:25-126)
// ======================================================================
struct AlignResult {
  Shifts shifts;
  int iterations;
};

// init (may be NULL): a first iterate of the per-frame shifts (the learned
// proposal's warm start); the group totals start at their frames' mean.
AlignResult iterative_align(const cd* spec, int cmpX, int cmpY, int N, const Groups& G,
                            int maxIter, float tol, float bfactor, bool phaseOnly,
                            const float* init = nullptr) {
  const long n = (long)cmpX * cmpY;
  const int nG = (int)G.start.size();
  const int imgX = (cmpX - 1) * 2;
  const int seaX = 64 < imgX ? 64 : imgX;
  const int seaY = 64 < cmpY ? 64 : cmpY;
  Shifts tmp(N), grpS(nG), total(nG);
  float bf = bfactor;
  float maxErr = 0.0f;
  int iters = 0;
  std::vector<cd> sum(n), gsum(n);
  std::vector<float> win(seaX * seaY);
  if (init) {
    for (int f = 0; f < N; ++f) {
      tmp.x(f) = init[2 * f];
      tmp.y(f) = init[2 * f + 1];
    }
    for (int g = 0; g < nG; ++g) {
      double sx = 0, sy = 0;
      for (int i = 0; i < G.size[g]; ++i) {
        sx += init[2 * (G.start[g] + i)];
        sy += init[2 * (G.start[g] + i) + 1];
      }
      total.x(g) = (float)(sx / G.size[g]);
      total.y(g) = (float)(sy / G.size[g]);
    }
  }
  for (int it = 0; it < maxIter; ++it) {
    // CAlignedSum: sum of all frames shifted by -tmp
    std::fill(sum.begin(), sum.end(), cd(0.0));
    for (int f = 0; f < N; ++f)
      phase_shift(spec + f * n, sum.data(), cmpX, cmpY, -(double)tmp.x(f), -(double)tmp.y(f), true);
    maxErr = 0.0f;
    for (int g = 0; g < nG; ++g) {
      for (int i = 0; i < G.size[g]; ++i) {
        int f = G.start[g] + i;
        phase_shift(spec + f * n, gsum.data(), cmpX, cmpY, -(double)tmp.x(f), -(double)tmp.y(f), i > 0);
      }
      correlate_window(gsum.data(), sum.data(), cmpX, cmpY, bf, phaseOnly, seaX, seaY, win.data());
      float sh[2];
      peak2d(win.data(), seaX, seaY, sh);
      grpS.x(g) = sh[0];
      grpS.y(g) = sh[1];
      // CAlignStack::mUpdateError (Align/CAlignStack.cpp:211-215)
      double dS = (double)std::sqrt((float)(sh[0] * sh[0] + sh[1] * sh[1]));
      if (maxErr < dS) maxErr = (float)dS;
    }
    bf -= 2;
    if (bf < 20) bf = 20.0f;
    for (int i = 0; i < 2 * nG; ++i) total.v[i] += grpS.v[i];
    Shifts ip = interpolate(grpS, G, N, true);
    for (int i = 0; i < 2 * N; ++i) tmp.v[i] += ip.v[i];
    iters += 1;
    if (maxErr < tol && it > 0) break;
  }
  Shifts res = interpolate(total, G, N, false);
  remove_spikes(res.v.data(), res.v.data() + N, N);
  smooth(res, 0.5f);
  // CIterativeAlign::DoIt (:72-81): second smoothing with 0.3 + 0.1*binZ
  float w = 0.3f + 0.1f * G.binZ;
  if (w > 0.9f) w = 0.9f;
  smooth(res, w);
  AlignResult R;
  R.shifts = res;
  R.iterations = iters;
  return R;
}

// ======================================================================
// Bad pixels (BadPixel/CDetectMain.cpp:54-123, GDetectHot.cu, GLocalCC.cu,
// CTemplate.cpp, GDetectPatch.cu, GCorrectBad.cu)
// ======================================================================
void moments(const double* img, long n, double* mean, double* std) {
  double s = 0, s2 = 0;
  for (long i = 0; i < n; ++i) { s += img[i]; s2 += img[i] * img[i]; }
  *mean = s / n;
  double v = s2 / n - (*mean) * (*mean);
  *std = std::sqrt(std::max(v, 0.0));
}

void detect_bad(const double* sum, int W, int H, unsigned char* bad) {
  const long n = (long)W * H;
  double mean, sd;
  moments(sum, n, &mean, &sd);
  double delta = 6.0 * sd;  // GDetectHot::DoIt (GDetectHot.cu:33-50)
  if (delta < 10) delta = 10;
  const double thr = mean + delta;
  for (long i = 0; i < n; ++i) bad[i] = sum[i] <= thr ? 0 : 1;
  // Local CC against a 6x6 ring template (CTemplate.cpp:20-57, GLocalCC.cu:20-61)
  const int ms = 6;
  double tpl[36];
  double tm = 0, ts = 0;
  for (int i = 0; i < 36; ++i) {
    int x = i % ms, y = i / ms;
    tpl[i] = (x == 0 || x == ms - 1 || y == 0 || y == ms - 1) ? -1.0 : 1.0;
    tm += tpl[i];
    ts += tpl[i] * tpl[i];
  }
  double fm = tm / 36.0;
  double fs = std::sqrt(std::max(ts / 36.0 - fm * fm, 0.0)) + 1e-30;
  for (int i = 0; i < 36; ++i) tpl[i] = (tpl[i] - fm) / fs;
  std::vector<double> cc(n, 0.0);
  parallel_for(H, [&](long y0, long y1) {
  for (int y = (int)y0; y < (int)y1; ++y) {
    for (int x = 0; x < W; ++x) {
      if (x + ms >= W || y + ms >= H) continue;
      double m = 0, s = 0, c = 0;
      for (int j = 0; j < ms; ++j)
        for (int i = 0; i < ms; ++i) {
          double v = sum[(long)(y + j) * W + x + i];
          m += v; s += v * v; c += tpl[j * ms + i] * v;
        }
      c /= 36.0; m /= 36.0;
      s = s / 36.0 - m * m;
      s = s < 0 ? 0.0 : std::sqrt(s);
      cc[(long)y * W + x] = s == 0 ? 0.0 : std::fabs(c) / s;
    }
  }
  });
  double cm, csd;
  moments(cc.data(), n, &cm, &csd);
  const double cthr = cm + 6.0 * csd;  // GDetectPatch::DoIt (GDetectPatch.cu:56-82)
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      if (x + ms >= W || y + ms >= H) continue;
      if (!(cc[(long)y * W + x] > cthr)) continue;
      for (int j = 0; j < ms; ++j)
        for (int i = 0; i < ms; ++i) bad[(long)(y + j) * W + x + i] = 1;
    }
}

// GCorrectBad mGCorrect/mGFindGood (GCorrectBad.cu:96-150), window 31.
void correct_bad(double* fr, const unsigned char* bad, int W, int H) {
  const int padX = (W / 2 + 1) * 2;
  std::vector<double> src(fr, fr + (long)W * H);
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      if (!bad[(long)y * W + x]) continue;
      const int i = y * padX + x;
      uint32_t next = (uint32_t)i * 109u + 619u;
      int win = 31;
      bool done = false;
      for (int j = 0; j < 10 && !done; ++j) {
        uint32_t nl = next;
        const int w2 = win * win, half = win / 2;
        for (int k = 0; k < 500; ++k) {
          nl *= 997u;
          int iX = (int)(nl % (uint32_t)w2);
          int iY = iX / win - half + y;
          if (iY < 0 || iY >= H) continue;
          iX = iX % win - half + x;
          if (iX < 0 || iX >= W) continue;
          if (bad[(long)iY * W + iX] == 1) continue;
          fr[(long)y * W + x] = src[(long)iY * W + iX];
          done = true;
          break;
        }
        if (done) break;
        win += 50;
        next *= 997u;
      }
      if (!done) {
        int iX = (int)(next % (uint32_t)(W * H));
        int iY = iX / W;
        iX = iX % W;
        fr[(long)y * W + x] = src[(long)iY * W + iX];
      }
    }
}

// ======================================================================
// Patch features and centres (Align/CDetectFeatures.cpp, CPatchCenters.cpp,
// Align/GNormByStd2D.cu, Util/GCalcMoment2D.cu)
// ======================================================================
struct Features {
  int B[2] = {128, 128};
  int P[2];
  float patSize[2];
  int sea[4];
  std::vector<unsigned char> feat, used;
  std::vector<float> centers;  // [P][3]
  int check_range(int s, int sz, const int* r) {
    if (s < r[0]) return r[0];
    if (s + sz > r[1]) return r[1] - sz;
    return s;
  }
  void set_used(float cx, float cy) {
    int wx = (int)(patSize[0] * 0.8f), wy = (int)(patSize[1] * 0.8f);
    int sx = (int)(cx - wx / 2), sy = (int)(cy - wy / 2);
    sx = check_range(sx, wx, &sea[0]);
    sy = check_range(sy, wy, &sea[2]);
    for (int y = 0; y < wy; ++y)
      for (int x = 0; x < wx; ++x) used[(sy + y) * B[0] + sx + x] = 1;
  }
  bool check_feature(float cx, float cy) {
    int ix = (int)cx, iy = (int)cy;
    if (ix < sea[0] || ix > sea[1]) return false;
    if (iy < sea[2] || iy > sea[3]) return false;
    return feat[iy * B[0] + ix];
  }
  void find_center(float* c) {
    int wx = B[0] / 3, wy = B[1] / 3;
    int sx = (int)(c[0] - wx * 0.5f + 0.5f);
    int sy = (int)(c[1] - wy * 0.5f + 0.5f);
    sx = check_range(sx, wx, &sea[0]);
    sy = check_range(sy, wy, &sea[2]);
    float minR = (float)1e20;
    float ac[2] = {-1.0f, 0.0f};
    for (int y = 0; y < wy; ++y)
      for (int x = 0; x < wx; ++x) {
        int j = (sy + y) * B[0] + sx + x;
        if (used[j]) continue;
        if (!feat[j]) continue;
        float fx = x + sx + 0.5f, fy = y + sy + 0.5f;
        float dx = fx - c[0], dy = fy - c[1];
        float r = (float)std::sqrt(dx * dx + dy * dy);
        if (r >= minR) continue;
        minR = r; ac[0] = fx; ac[1] = fy;
      }
    if (ac[0] > 0) { c[0] = ac[0]; c[1] = ac[1]; }
    set_used(c[0], c[1]);
  }
};

// CDetectFeatures::DoIt (Align/CDetectFeatures.cpp:58-181) on the aligned
// xcf sum; the local-variance normalisation reads unmodified input values
// (Align/GNormByStd2D.cu updates in place while neighbouring threads still
// read, a race whose outcome depends on scheduling).
Features detect_features(const cd* xsum, int xcfCmpX, int xcfCmpY, int Px, int Py) {
  Features F;
  F.P[0] = Px; F.P[1] = Py;
  F.patSize[0] = F.B[0] * 1.0f / Px;
  F.patSize[1] = F.B[1] * 1.0f / Py;
  F.sea[0] = (int)(F.patSize[0] * 0.5f - 0.5f);
  if (F.sea[0] < 4) F.sea[0] = 4;
  F.sea[1] = F.B[0] - F.sea[0];
  F.sea[2] = (int)(F.patSize[1] * 0.5f - 0.5f);
  if (F.sea[2] < 4) F.sea[2] = 4;
  F.sea[3] = F.B[1] - F.sea[2];
  const int bx = F.B[0], by = F.B[1];
  const int bcx = bx / 2 + 1;
  std::vector<cd> crop((long)bcx * by);
  fourier_resize(xsum, xcfCmpX, xcfCmpY, crop.data(), bcx, by);
  std::vector<double> img((long)bx * by);
  irfft2(crop.data(), img.data(), bx, by);
  double mn = img[0];
  for (double v : img) mn = std::min(mn, v);
  for (double& v : img) v += 1.0 - mn;
  std::vector<double> nrm(img.size());
  for (int y = 0; y < by; ++y)
    for (int x = 0; x < bx; ++x) {
      double m = 0, s = 0;
      int cnt = 0;
      for (int j = 0; j < 5; ++j) {
        int yy = y - 2 + j;
        if (yy < 0 || yy >= by) continue;
        for (int i = 0; i < 5; ++i) {
          int xx = x - 2 + i;
          if (xx < 0 || xx >= bx) continue;
          double v = img[yy * bx + xx];
          m += v; s += v * v; cnt++;
        }
      }
      m /= cnt;
      s = s / cnt - m * m;
      nrm[y * bx + x] = s < 0 ? 0.0 : img[y * bx + x] / (s + 1e-20);
    }
  double mean = 0, m2 = 0;
  for (double v : nrm) { mean += v; m2 += v * v; }
  mean /= nrm.size();
  m2 /= nrm.size();
  double sd = m2 - mean * mean;
  sd = sd < 0 ? 0.0 : std::sqrt(sd);
  std::vector<float> bs(nrm.size());
  for (size_t i = 0; i < nrm.size(); ++i) bs[i] = (float)nrm[i];
  float fMin = (float)(mean - 4.0 * sd), fMax = (float)(mean + 4.0 * sd);
  double dm = 0, ds = 0;
  int cnt = 0;
  for (float v : bs) {
    if (v < fMin || v > fMax) continue;
    dm += v; ds += (double)(v * v); cnt++;
  }
  dm /= (cnt + 1e-30);
  ds = ds / (cnt + 1e-30) - dm * dm;
  ds = ds < 0 ? 0.0 : (double)std::sqrt((float)ds);
  fMin = (float)(dm - 4.0 * ds);
  fMax = (float)(dm - 0.08f * ds);
  F.feat.assign(bs.size(), 0);
  for (size_t i = 0; i < bs.size(); ++i) F.feat[i] = (bs[i] < fMin || bs[i] > fMax) ? 0 : 1;
  F.used.assign(bs.size(), 0);
  // mFindCenters (:273-313); the early return is an assignment and never
  // taken, so every patch without a feature is relocated.
  const int np = Px * Py;
  F.centers.assign(3 * np, 0.f);
  for (int i = 0; i < np; ++i) {
    int x = i % Px, y = i / Px;
    float cx = (x + 0.5f) * F.patSize[0], cy = (y + 0.5f) * F.patSize[1];
    bool has = F.check_feature(cx, cy);
    F.centers[3 * i] = cx;
    F.centers[3 * i + 1] = cy;
    if (has) { F.centers[3 * i + 2] = 1.0f; F.set_used(cx, cy); }
    else F.centers[3 * i + 2] = -1.0f;
  }
  for (int i = 0; i < np; ++i) {
    float* c = &F.centers[3 * i];
    if (c[2] > 0) continue;
    F.find_center(c);
  }
  return F;
}

// CPatchShifts::MakeRelative (Align/CPatchShifts.cpp:263-286).  `shifts`
// has one extra zero float after [N][P][2]: the reference reads one element
// past the last patch of the reference frame (the first x of the next
// frame, or the zero-initialised flag array after the last frame).
void patch_make_relative(float* s, int N, int P) {
  float fMin = (float)1e20;
  int iRef = 0;
  for (int i = 1; i < N; ++i) {
    const float* ps = s + (long)i * P * 2;
    float mx = 0.f, my = 0.f;
    for (int j = 0; j < P; ++j) { mx += ps[2 * j]; my += ps[2 * j + 1]; }
    mx /= P; my /= P;
    float sd = 0.f;
    for (int j = 0; j < P; ++j) {
      float dx = ps[2 * j] - mx, dy = ps[2 * j + 1] - my;
      sd += (dx * dx + dy * dy);
    }
    sd = (float)std::sqrt(sd / P);
    float m = (float)std::sqrt(mx * mx + my * my);
    float v = m + sd;
    if (v > fMin) continue;
    fMin = v;
    iRef = i;
  }
  float* ref = s + (long)iRef * P * 2;
  for (int i = 0; i < N; ++i) {
    float* ps = s + (long)i * P * 2;
    for (int j = 0; j < P; ++j) {
      int k = 2 * j;
      ps[k] -= ref[k];
      ps[k + 1] -= ref[k + 2];
    }
  }
}

// CPatchShifts::DetectBads / mCalcLocalRms (:288-355)
void patch_detect_bads(const float* s, const float* cent, int N, int P, int W, int H,
                       unsigned char* bad) {
  for (int f = 0; f < N; ++f) {
    const float* ps = s + (long)f * P * 2;
    for (int i = 0; i < P; ++i) {
      float sx = ps[2 * i], sy = ps[2 * i + 1];
      double dS = std::sqrt(sx * sx + sy * sy);
      double rms = 0, sw = 0;
      for (int k = 0; k < P; ++k) {
        if (k == i) continue;
        float fx = (cent[2 * k] - cent[2 * i]) / W;
        float fy = (cent[2 * k + 1] - cent[2 * i + 1]) / H;
        double w = (double)expf((float)(-100.0 * (double)(fx * fx + fy * fy)));
        float ax = ps[2 * k], ay = ps[2 * k + 1];
        rms += (w * (ax * ax + ay * ay));
        sw += w;
      }
      float lr = (float)(double)std::sqrt((float)(rms / sw));
      if (lr < 2) lr = 2.0f;
      bad[(long)f * P + i] = dS > (1 * lr) ? 1 : 0;
    }
  }
}

// mGCorrect3D (Correct/GCorrectPatchShift.cu:17-66), upsampling 1.
void local_gather(const double* in, double* out, int W, int H, const float* cent,
                  const float* sh, const unsigned char* bad, int P) {
  parallel_for(H, [&](long y0, long y1) {
  for (int y = (int)y0; y < (int)y1; ++y) {
    for (int x = 0; x < W; ++x) {
      float fSx = 0.f, fSy = 0.f, fW = 0.f;
      for (int p = 0; p < P; ++p) {
        if (bad && bad[p]) continue;
        float ax = (x - cent[2 * p]) / (float)W;
        float ay = (y - cent[2 * p + 1]) / (float)H;
        float r = std::sqrt(ax * ax + ay * ay);
        if (r > 0.6f) continue;
        float w = std::exp(-100.0f * r);
        fW += w;
        fSx += sh[2 * p] * w;
        fSy += sh[2 * p + 1] * w;
      }
      if (fW > 0) { fSx = fSx / fW; fSy = fSy / fW; }
      int ix = (int)((x - fSx) * 1);
      int iy = (int)((y - fSy) * 1);
      if (ix < 0 || iy < 0 || ix >= W || iy >= H) {
        ix = ix < 0 ? -ix : ix;
        iy = iy < 0 ? -iy : iy;
        ix = (811 * ix) % W;
        iy = (811 * iy) % H;
        if (ix < 0 || ix >= W) ix = 0;  // non-finite shifts only
        if (iy < 0 || iy >= H) iy = 0;
      }
      out[(long)y * W + x] = in[(long)iy * W + ix];
    }
  }
  });
}

// GWeightFrame (Correct/GWeightFrame.cu:19-71, 90-135)
double kv_factor(int kv) {
  float f = 1.0f;
  if (kv >= 300) f = 1.0f;
  else if (kv < 300 && kv >= 200) f = 0.002f * (kv - 200) + 0.8f;
  else if (kv < 200 && kv >= 120) f = 0.004375f * (kv - 120) + 0.45f;
  else f = 0.45f;
  return f;
}

double dose_weight(int x, int y, int cmpX, int cmpY, double dose, double pix, double kvf) {
  double fx = x * 0.5 / (cmpX - 1);
  double fy = y / (double)cmpY;
  if (fy >= 0.5) fy -= 1.0;
  double k = std::sqrt(fx * fx + fy * fy) / pix;
  double crit = (0.24499 * std::pow(k, -1.6649) + 2.8141) * kvf;
  return std::exp(-0.5 * dose / crit);
}

void dose_weights(const float* acc, int nF, int frame, int cmpX, int cmpY, float pix, int kv,
                  double* out) {
  const double kvf = kv_factor(kv);
  for (int y = 0; y < cmpY; ++y)
    for (int x = 0; x < cmpX; ++x) {
      long i = (long)y * cmpX + x;
      if (i == 0) { out[0] = 1.0; continue; }
      double s = 0;
      for (int f = 0; f < nF; ++f) {
        double w = dose_weight(x, y, cmpX, cmpY, acc[f], pix, kvf);
        s += w * w;
      }
      out[i] = dose_weight(x, y, cmpX, cmpY, acc[frame], pix, kvf) / std::sqrt(s);
    }
}

}  // namespace

// ======================================================================
// C API
// ======================================================================
extern "C" {

void oracle_default_params(oracle_params* p) {
  // CInput::CInput defaults (CInput.cpp:82-127)
  p->patch[0] = p->patch[1] = 0;
  p->iter = 15;
  p->tol = 0.1f;
  p->bft[0] = 500.0f;
  p->bft[1] = 100.0f;
  p->phase_only = 0;
  p->fm_dose = 0.0f;
  p->pix_size = 0.0f;
  p->kv = 300;
  p->group[0] = 1;
  p->group[1] = 4;
  p->fm_ref = -1;
  p->sum_range[0] = 3.0f;
  p->sum_range[1] = 25.0f;
  p->correct_bad = 1;
  p->split_sum = 0;
  p->ft_bin = 1.0f;
  p->out_stack[0] = 0;
  p->out_stack[1] = 1;
  p->int_size = nullptr;
  p->acc_dose = nullptr;
  p->dose_weight = 0;
  p->dark = nullptr;
  p->mag[0] = p->mag[1] = 1.0f;
  p->mag[2] = 0.0f;
  p->in_fm_motion = 0;
  p->corr_interp = 0;
  p->defects = nullptr;
}

void oracle_rfft2(const double* img, double* spec, int W, int H, int normalise) {
  rfft2(img, reinterpret_cast<cd*>(spec), W, H, normalise != 0);
}

void oracle_irfft2(const double* spec, double* img, int W, int H) {
  irfft2(reinterpret_cast<const cd*>(spec), img, W, H);
}

void oracle_cfft(const double* in, double* out, int n, int dir) {
  fft1(reinterpret_cast<const cd*>(in), reinterpret_cast<cd*>(out), n, dir);
}

void oracle_detect_bad(const double* sum, int W, int H, unsigned char* bad) { detect_bad(sum, W, H, bad); }

void oracle_correct_bad(double* frame, const unsigned char* bad, int W, int H) {
  correct_bad(frame, bad, W, H);
}

void oracle_correlate_window(const double* grp, const double* sum, int cmpX, int cmpY,
                             float bfactor, int phase_only, int sx, int sy, float* win) {
  correlate_window(reinterpret_cast<const cd*>(grp), reinterpret_cast<const cd*>(sum), cmpX, cmpY,
                   bfactor, phase_only != 0, sx, sy, win);
}

void oracle_peak2d(const float* win, int sx, int sy, float* shift) { peak2d(win, sx, sy, shift); }

void oracle_remove_spikes(float* sx, float* sy, int n) { remove_spikes(sx, sy, n); }

void oracle_smooth(float* sx, float* sy, int n, float w) {
  Shifts s(n);
  std::memcpy(s.v.data(), sx, sizeof(float) * n);
  std::memcpy(s.v.data() + n, sy, sizeof(float) * n);
  smooth(s, w);
  std::memcpy(sx, s.v.data(), sizeof(float) * n);
  std::memcpy(sy, s.v.data() + n, sizeof(float) * n);
}

int oracle_lin_eqs(float* coeff, float* vals, int dim) { return lin_eqs(coeff, vals, dim) ? 1 : 0; }

void oracle_patch_make_relative(float* shifts, int n_frames, int n_patches) {
  std::vector<float> s((size_t)n_frames * n_patches * 2 + 1, 0.0f);
  std::memcpy(s.data(), shifts, sizeof(float) * n_frames * n_patches * 2);
  patch_make_relative(s.data(), n_frames, n_patches);
  std::memcpy(shifts, s.data(), sizeof(float) * n_frames * n_patches * 2);
}

void oracle_patch_detect_bads(const float* shifts, const float* centers, int n_frames,
                              int n_patches, int W, int H, unsigned char* bad) {
  patch_detect_bads(shifts, centers, n_frames, n_patches, W, H, bad);
}

void oracle_dose_weights(const float* acc_dose, int n_frames, int frame, int cmpX, int cmpY,
                         float pix_size, int kv, double* out) {
  dose_weights(acc_dose, n_frames, frame, cmpX, cmpY, pix_size, kv, out);
}

void oracle_local_gather(const double* in, double* out, int W, int H, const float* centers,
                         const float* shifts, const unsigned char* bad, int n_patches) {
  local_gather(in, out, W, H, centers, shifts, bad, n_patches);
}

int oracle_iterative_align(const double* spec, int cmpX, int cmpY, int N, int group_size,
                           int max_iter, float tol, float bfactor, int phase_only, float* shifts) {
  return oracle_iterative_align_warm(spec, cmpX, cmpY, N, group_size, max_iter, tol, bfactor,
                                     phase_only, nullptr, shifts);
}

// The same with a first iterate init[N][2] (NULL: start from zero).
int oracle_iterative_align_warm(const double* spec, int cmpX, int cmpY, int N, int group_size,
                                int max_iter, float tol, float bfactor, int phase_only,
                                const float* init, float* shifts) {
  Groups G = make_groups(N, group_size);
  AlignResult r = iterative_align(reinterpret_cast<const cd*>(spec), cmpX, cmpY, N, G, max_iter,
                                  tol, bfactor, phase_only != 0, init);
  for (int i = 0; i < N; ++i) {
    shifts[2 * i] = r.shifts.v[i];
    shifts[2 * i + 1] = r.shifts.v[N + i];
  }
  return r.iterations;
}

int oracle_process_movie(const oracle_params* p, const float* frames, int W, int H, int N,
                         const float* gain, oracle_result* out) {
  if (W < 16 || H < 16 || N < 3 || (W % 2) || (H % 2)) return -1;
  Geo g = make_geo(W, H, N, p);
  const long npx = (long)W * H;
  // ---- gain (MrcUtil/GApplyRefsToFrame.cu:56-72) ----
  std::vector<double> fr((long)N * npx);
  for (long i = 0; i < (long)N * npx; ++i) {
    double v = frames[i];
    if (p->dark) v -= p->dark[i % npx];
    if (gain) v *= gain[i % npx];
    fr[i] = v;
  }
  // ---- bad pixels (CProcessThread.cpp:94-99) ----
  std::vector<unsigned char> bad(npx, 0);
  if (p->correct_bad) {
    std::vector<double> sum(npx, 0.0);
    for (int f = 0; f < N; ++f)
      for (long i = 0; i < npx; ++i) sum[i] += fr[(long)f * npx + i];
    detect_bad(sum.data(), W, H, bad.data());
    // CDetectMain::mLoadDefectFile / mLoadDefectMap (BadPixel/CDetectMain.cpp:146-260)
    if (p->defects)
      for (long i = 0; i < npx; ++i)
        if (p->defects[i]) bad[i] = 1;
    parallel_for(N, [&](long f0, long f1) {
      for (long f = f0; f < f1; ++f) correct_bad(&fr[f * npx], bad.data(), W, H);
    });
  }
  if (out->bad_map) std::memcpy(out->bad_map, bad.data(), npx);
  // ---- forward FFT, normalised (Align/CTransformStack.cpp:59-136) ----
  const long ncmp = (long)g.cmpX * g.cmpY;
  std::vector<cd> spec((long)N * ncmp);
  for (int f = 0; f < N; ++f) rfft2(&fr[(long)f * npx], &spec[(long)f * ncmp], W, H, true);
  fr.clear();
  fr.shrink_to_fit();
  // ---- xcf stack (Align/CGenXcfStack.cpp:72-108) ----
  const long nx = (long)g.xcfCmpX * g.xcfCmpY;
  std::vector<cd> xcf((long)N * nx);
  for (int f = 0; f < N; ++f)
    fourier_resize(&spec[(long)f * ncmp], g.cmpX, g.cmpY, &xcf[(long)f * nx], g.xcfCmpX, g.xcfCmpY);
  // ---- global alignment (Align/CFullAlign.cpp:70-164) ----
  const bool forced = out->use_global_shifts != nullptr;
  const float bin = std::fmax(g.xcfBin[0], g.xcfBin[1]);
  const float tol = p->tol / bin;
  Groups G0 = make_groups(N, p->group[0], p->int_size);
  Shifts xs(N);  // xcf units
  if (!forced) {
    AlignResult ga = iterative_align(xcf.data(), g.xcfCmpX, g.xcfCmpY, N, G0, p->iter, tol,
                                     p->bft[0], p->phase_only != 0);
    xs = ga.shifts;
    if (out->iterations) out->iterations[0] = ga.iterations;
  }

  const bool patchMode = g.patch;
  std::vector<float> patCent, patShift;
  std::vector<unsigned char> patBad;
  const int P = patchMode ? g.Px * g.Py : 0;
  std::vector<double> xreal;
  std::vector<int> patStart;
  if (patchMode && !forced) {
    // CDetectFeatures::DoIt on the aligned xcf sum (CFullAlign.cpp:147-159)
    std::vector<cd> xsum(nx, cd(0.0));
    for (int f = 0; f < N; ++f)
      phase_shift(&xcf[(long)f * nx], xsum.data(), g.xcfCmpX, g.xcfCmpY, -(double)xs.x(f),
                  -(double)xs.y(f), true);
    Features F = detect_features(xsum.data(), g.xcfCmpX, g.xcfCmpY, g.Px, g.Py);
    // CPatchCenters::Calculate (Align/CPatchCenters.cpp:42-84)
    const int xcfX = (g.xcfCmpX - 1) * 2, xcfY = g.xcfCmpY;
    patStart.resize(2 * P);
    for (int i = 0; i < P; ++i) {
      float binX = xcfX * 1.0f / F.B[0], binY = xcfY * 1.0f / F.B[1];
      float cx = F.centers[3 * i] * binX, cy = F.centers[3 * i + 1] * binY;
      auto calc = [](float c, int ps, int xs_) {
        int s = (int)(c - ps / 2);
        if (s < 0) s = 0;
        else if (s + ps > xs_) s = xs_ - ps;
        return s;
      };
      patStart[2 * i] = calc(cx, g.patSizeX, xcfX);
      patStart[2 * i + 1] = calc(cy, g.patSizeY, xcfY);
    }
    // CGenRealStack on xcf with the xcf-unit shifts (Correct/CGenRealStack.cpp:136-206)
    xreal.resize((long)N * xcfX * xcfY);
    for (int f = 0; f < N; ++f) {
      std::vector<cd> t(&xcf[(long)f * nx], &xcf[(long)f * nx] + nx);
      float s[2] = {-xs.x(f), -xs.y(f)};
      double d = (double)std::sqrt((float)(s[0] * s[0] + s[1] * s[1]));
      if (!(d < 0.1)) phase_shift(t.data(), t.data(), g.xcfCmpX, g.xcfCmpY, s[0], s[1], false);
      irfft2(t.data(), &xreal[(long)f * xcfX * xcfY], xcfX, xcfY);
    }
  }
  // shifts to full-frame pixels, then 0.01 px truncation (CFullAlign.cpp:96,163)
  Shifts fs = xs;
  for (int i = 0; i < N; ++i) {
    fs.x(i) *= g.xcfBin[0];
    fs.y(i) *= g.xcfBin[1];
  }
  for (int i = 0; i < 2 * N; ++i) fs.v[i] = 0.01f * (int)(fs.v[i] * 100);

  if (forced) {
    for (int i = 0; i < N; ++i) {
      fs.x(i) = out->use_global_shifts[2 * i];
      fs.y(i) = out->use_global_shifts[2 * i + 1];
    }
    if (patchMode) {
      // CPatchAlign::mCorrectFullShift makes loaded shifts relative too
      // (Align/CPatchAlign.cpp:47-52); shifts already relative are unchanged
      int ref = p->fm_ref < 0 ? N / 2 : std::min(std::max(p->fm_ref - 1, 0), N - 1);
      float rx = fs.x(ref), ry = fs.y(ref);
      for (int i = 0; i < N; ++i) { fs.x(i) -= rx; fs.y(i) -= ry; }
      patShift.assign(out->use_patch_shifts, out->use_patch_shifts + (size_t)N * P * 2);
      patCent.assign(out->use_patch_centers, out->use_patch_centers + (size_t)P * 2);
      patBad.assign(out->use_patch_bad, out->use_patch_bad + (size_t)N * P);
    }
  } else if (patchMode) {
    // CPatchAlign::mCorrectFullShift (Align/CPatchAlign.cpp:47-65)
    int ref = p->fm_ref < 0 ? N / 2 : std::min(std::max(p->fm_ref - 1, 0), N - 1);
    float rx = fs.x(ref), ry = fs.y(ref);
    for (int i = 0; i < N; ++i) { fs.x(i) -= rx; fs.y(i) -= ry; }
    // CMeasurePatches::DoIt (Align/CMeasurePatches.cpp:22-84)
    const int xcfX = (g.xcfCmpX - 1) * 2, xcfY = g.xcfCmpY;
    const int pw = (g.patCmpX - 1) * 2, ph = g.patCmpY;
    const long npat = (long)g.patCmpX * g.patCmpY;
    patShift.assign((size_t)N * P * 2, 0.f);
    patCent.assign((size_t)P * 2, 0.f);
    Groups G1 = make_groups(N, p->group[1], p->int_size);
    for (int pi = 0; pi < P; ++pi) {
      std::vector<cd> pspec((long)N * npat);
      std::vector<double> win((long)pw * ph);
      for (int f = 0; f < N; ++f) {
        const double* src = &xreal[(long)f * xcfX * xcfY];
        for (int y = 0; y < ph; ++y)
          for (int x = 0; x < pw; ++x)
            win[(long)y * pw + x] = src[(long)(patStart[2 * pi + 1] + y) * xcfX + patStart[2 * pi] + x];
        rfft2(win.data(), &pspec[(long)f * npat], pw, ph, false);
      }
      AlignResult pr = iterative_align(pspec.data(), g.patCmpX, g.patCmpY, N, G1, p->iter, tol,
                                       p->bft[1], p->phase_only != 0);
      if (out->iterations) out->iterations[1 + pi] = pr.iterations;
      int cx = patStart[2 * pi] + g.patSizeX / 2, cy = patStart[2 * pi + 1] + g.patSizeY / 2;
      patCent[2 * pi] = cx * g.xcfBin[0];
      patCent[2 * pi + 1] = cy * g.xcfBin[1];
      for (int f = 0; f < N; ++f) {
        patShift[((long)f * P + pi) * 2] = pr.shifts.x(f) * g.xcfBin[0];
        patShift[((long)f * P + pi) * 2 + 1] = pr.shifts.y(f) * g.xcfBin[1];
      }
    }
    std::vector<float> ext(patShift.size() + 1, 0.f);
    std::memcpy(ext.data(), patShift.data(), sizeof(float) * patShift.size());
    patch_make_relative(ext.data(), N, P);
    std::memcpy(patShift.data(), ext.data(), sizeof(float) * patShift.size());
    patBad.assign((size_t)N * P, 0);
    patch_detect_bads(patShift.data(), patCent.data(), N, P, W, H, patBad.data());
  }

  // ---- correction and sums (Correct/CCorrectFullShift.cpp,
  //      Correct/GCorrectPatchShift.cu) ----
  const bool dw = !(p->kv < 80 || p->kv > 300) && p->pix_size > 0 &&
                  (p->fm_dose > 0 || p->dose_weight);
  const bool dws = dw && p->sum_range[0] >= 0 && p->sum_range[1] > 0 &&
                   (p->sum_range[1] - p->sum_range[0]) > 1.0f;
  const int nBase = 1 + (dw ? 1 : 0) + (dws ? 1 : 0);
  const int nSums = nBase + (p->split_sum ? 2 : 0);
  std::vector<float> acc(N);
  for (int i = 0; i < N; ++i) acc[i] = p->acc_dose ? p->acc_dose[i] : p->fm_dose * (i + 1);
  std::vector<double> wsum;
  double kvf = kv_factor(p->kv);
  if (dw) {
    wsum.assign(ncmp, 0.0);
    for (int y = 0; y < g.cmpY; ++y)
      for (int x = 0; x < g.cmpX; ++x) {
        long i = (long)y * g.cmpX + x;
        if (i == 0) continue;
        double s = 0;
        for (int f = 0; f < N; ++f) {
          double w = dose_weight(x, y, g.cmpX, g.cmpY, acc[f], p->pix_size, kvf);
          s += w * w;
        }
        wsum[i] = std::sqrt(s);
      }
  }
  // output size of -FtBin (CInput::GetBinnedSize, CInput.cpp:678-688)
  int oW = W, oH = H;
  if (p->ft_bin > 0) {
    oW = (int)(W / p->ft_bin + 0.5f) / 2 * 2;
    oH = (int)(H / p->ft_bin + 0.5f) / 2 * 2;
  }
  const int ocX = oW / 2 + 1;
  const long opx = (long)oW * oH;
  // GFourierResize2D copy-mode crop (Util/GFourierResize2D.cu:7-37)
  auto crop_to_out = [&](const cd* S, cd* dst) {
    for (int yo = 0; yo < oH; ++yo) {
      const int yi = yo > oH / 2 ? yo - oH + H : yo;
      for (int x = 0; x < ocX; ++x) dst[(long)yo * ocX + x] = S[(long)yi * g.cmpX + x];
    }
  };
  const bool want_stack = p->out_stack[0] != 0 && out->stack != nullptr;
  std::vector<cd> stk_crop(want_stack ? (long)ocX * oH : 0);
  std::vector<double> stk_img(want_stack ? opx : 0);
  std::vector<cd> sums((long)nSums * ncmp, cd(0.0));
  std::vector<double> realf, gath;
  if (patchMode) { realf.resize(npx); gath.resize(npx); }
  for (int f = 0; f < N; ++f) {
    cd* X = &spec[(long)f * ncmp];
    float s[2] = {-fs.x(f), -fs.y(f)};
    double d = (double)std::sqrt((float)(s[0] * s[0] + s[1] * s[1]));
    if (!(d < 0.1)) phase_shift(X, X, g.cmpX, g.cmpY, s[0], s[1], false);
    // CInFrameMotion::GetFullMotion + GMotionWeight::DirWeight
    // (MotionDecon/CInFrameMotion.cpp:78-97, MotionDecon/GMotionWeight.cu:14-36)
    auto motion_weight = [&](cd* X) {
      const int f1 = f == N - 1 ? f - 1 : f, f2 = f == N - 1 ? f : f + 1;
      const float mx = fs.x(f2) - fs.x(f1), my = fs.y(f2) - fs.y(f1);
      const double mot = std::sqrt((float)(mx * mx + my * my));
      if (!(mot < 0.1)) {
        const float shift = std::sqrt(mx * mx + my * my);
        const float slope = -mx / (my + (float)1e-20);
        for (int y = 0; y < g.cmpY; ++y)
          for (int x = 0; x < g.cmpX; ++x) {
            if (x == 0 && y == 0) continue;
            float dist;
            if (std::fabs(slope) > (float)1e5) {
              dist = (float)x;
            } else {
              const int ys = y > g.cmpY / 2 ? y - g.cmpY : y;
              dist = std::fabs(slope * x - ys) / std::sqrt(slope * slope + 1.0f);
            }
            if (dist < 0.1f) continue;
            dist = dist / (2 * (g.cmpX - 1));
            const double a = 3.141592654 * shift * dist;
            const double w = (shift * dist > 1.0f) ? 0.0 : std::sin(a) / a;
            X[(long)y * g.cmpX + x] *= w;
          }
      }
    };
    if (patchMode && p->corr_interp) {
      // CGenRealStack::mCorrectBilinear (GCorrLinearInterp, Util/GCorrLinearInterp.cu:7-22)
      for (int y = 0; y < g.cmpY; ++y)
        for (int x = 0; x < g.cmpX; ++x) {
          if (x == 0 && y == 0) continue;
          float fx = x * 0.5f / (g.cmpX - 1), fy = y / (float)g.cmpY;
          if (fy > 0.5f) fy -= 1.0f;
          const double r = std::sqrt((double)fx * fx + (double)fy * fy) * 3.141592654;
          X[(long)y * g.cmpX + x] /= std::pow(std::sin(r) / r, 0.125);
        }
    }
    if (p->in_fm_motion) motion_weight(X);
    if (patchMode) {
      irfft2(X, realf.data(), W, H);
      local_gather(realf.data(), gath.data(), W, H, patCent.data(), &patShift[(long)f * P * 2],
                   &patBad[(long)f * P], P);
      rfft2(gath.data(), X, W, H, true);
      // the reference's non-virtual CCorrectFullShift::mMotionDecon runs again
      // in mGenSums on the locally corrected frame (Correct/CCorrectInc.h:115)
      if (p->in_fm_motion) motion_weight(X);
    }
    cd* s0 = &sums[0];
    for (long i = 0; i < ncmp; ++i) s0[i] += X[i];
    if (want_stack) {
      // CCorrectFullShift::mCropFrame (Correct/CCorrectFullShift.cpp:336-356)
      crop_to_out(X, stk_crop.data());
      irfft2(stk_crop.data(), stk_img.data(), oW, oH);
      for (long i = 0; i < opx; ++i) out->stack[(long)f * opx + i] = (float)stk_img[i];
    }
    // CCorrectFullShift::mGenSums (Correct/CCorrectFullShift.cpp:271-300):
    // the odd/even split sums take the frame after dose weighting
    cd* split = p->split_sum ? &sums[(long)(nBase + (f % 2)) * ncmp] : nullptr;
    if (dw) {
      const bool inRange = acc[f] >= p->sum_range[0] && acc[f] <= p->sum_range[1];
      for (int y = 0; y < g.cmpY; ++y)
        for (int x = 0; x < g.cmpX; ++x) {
          long i = (long)y * g.cmpX + x;
          cd v = X[i];
          if (i > 0) v *= dose_weight(x, y, g.cmpX, g.cmpY, acc[f], p->pix_size, kvf) / wsum[i];
          sums[ncmp + i] += v;
          if (dws && inRange) sums[2 * ncmp + i] += v;
          if (split) split[i] += v;
        }
    } else if (split) {
      for (long i = 0; i < ncmp; ++i) split[i] += X[i];
    }
  }
  // CCorrectFullShift::mCorrectMag (Correct/CCorrectFullShift.cpp:94-127):
  // each sum to real space, stretched (Correct/GStretch.cu), forward again
  {
    const float stretch = p->mag[0] / p->mag[1], axis = -1.0f * p->mag[2];
    if (!(std::fabs(stretch - 1) < 1e-5)) {
      const double t2 = 2 * axis * 3.1416 / 180;
      const double dp = 0.5 * (stretch + 1), dm = 0.5 * (stretch - 1);
      const float a0 = (float)(dp + dm * std::cos(t2)), a1 = (float)(dm * std::sin(t2));
      const float a2 = (float)(dp - dm * std::cos(t2));
      const float det = a0 * a2 - a1 * a1;
      const float m0 = a2 / det, m1 = -a1 / det, m2 = a0 / det;
      std::vector<double> img(npx), out(npx);
      for (int s = 0; s < nSums; ++s) {
        cd* S = &sums[(long)s * ncmp];
        irfft2(S, img.data(), W, H);
        const float cx = 0.5f * W, cy = 0.5f * H;
        for (int y = 0; y < H; ++y)
          for (int x = 0; x < W; ++x) {
            const float dx = x - cx, dy = y - cy;
            float ox = dx * m0 + dy * m1 + cx, oy = dx * m1 + dy * m2 + cy;
            if (ox < 1 || oy < 1 || ox >= W - 1 || oy >= H - 1) {
              ox = (float)((8111LL * (long long)std::fabs(ox)) % (W - 1));
              oy = (float)((8111LL * (long long)std::fabs(oy)) % (H - 1));
            }
            const int ix = (int)ox, iy = (int)oy;
            const double wx = ox - ix, wy = oy - iy;
            const double* q = &img[(long)iy * W + ix];
            out[(long)y * W + x] = (1 - wx) * (1 - wy) * q[0] + wx * (1 - wy) * q[1] +
                                   (1 - wx) * wy * q[W] + wx * wy * q[W + 1];
          }
        rfft2(out.data(), S, W, H, true);
      }
    }
  }
  // mUnpadSums (CCorrectFullShift.cpp:146-185): Fourier crop to the -FtBin
  // size (CInput::GetBinnedSize, CInput.cpp:678-688; GFourierResize2D copy
  // mode, Util/GFourierResize2D.cu:7-37), C2R, positivity
  std::vector<double> img(opx);
  std::vector<cd> crop((long)ocX * oH);
  for (int s = 0; s < nSums; ++s) {
    crop_to_out(&sums[(long)s * ncmp], crop.data());
    irfft2(crop.data(), img.data(), oW, oH);
    for (long i = 0; i < opx; ++i) out->sums[(long)s * opx + i] = (float)std::max(0.0, img[i]);
  }
  out->n_sums = nSums;
  out->stack_frames = 0;
  if (want_stack) {
    // CZbinStack::DoIt (Align/CZbinStack.cpp:27-71): FP32 sums in frame
    // order, groups of out_stack[1] frames, the last one shorter
    const int zb = p->out_stack[1] > 1 ? p->out_stack[1] : 1;
    Groups Z = make_groups(N, zb, p->int_size);
    int ng = 0;
    for (; ng < (int)Z.start.size(); ++ng) {
      const int f0 = Z.start[ng], n = Z.size[ng];
      float* dst = out->stack + (long)ng * opx;
      for (long i = 0; i < opx; ++i) {
        float v = out->stack[(long)f0 * opx + i];
        for (int k = 1; k < n; ++k) v += out->stack[(long)(f0 + k) * opx + i];
        dst[i] = v;
      }
    }
    out->stack_frames = ng;
  }
  // logged full-frame shifts: absolute (global mode) or relative (patch mode)
  for (int i = 0; i < N; ++i) {
    out->global_shifts[2 * i] = fs.x(i);
    out->global_shifts[2 * i + 1] = fs.y(i);
  }
  out->n_patches = P;
  if (P) {
    if (out->patch_shifts) std::memcpy(out->patch_shifts, patShift.data(), sizeof(float) * patShift.size());
    if (out->patch_centers) std::memcpy(out->patch_centers, patCent.data(), sizeof(float) * patCent.size());
    if (out->patch_bad) std::memcpy(out->patch_bad, patBad.data(), patBad.size());
  }
  return 0;
}

}  // extern "C"
