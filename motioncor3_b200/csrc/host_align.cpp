// Host-side FP32 shift bookkeeping (see host_align.h).
#include "host_align.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <math.h>

namespace mc3 {
namespace host {

// ---- Correct/GStretch.cu:53-72, Align/CAlignParam.cpp:55-72 ------------------
bool mag_matrix(const float mag[3], float m[3]) {
  if (!(mag[0] > 0 && mag[1] > 0)) return false;  // no meaningful stretch
  const float stretch = mag[0] / mag[1];
  const float axis = -1.0f * mag[2];
  if (std::fabs(stretch - 1) < 1e-5) return false;
  const double t2 = 2 * axis * 3.1416 / 180;  // the reference's value of pi
  const double s2 = std::sin(t2), c2 = std::cos(t2);
  const double dp = 0.5 * (stretch + 1), dm = 0.5 * (stretch - 1);
  const float a0 = (float)(dp + dm * c2), a1 = (float)(1 * dm * s2), a2 = (float)(dp - dm * c2);
  const float det = a0 * a2 - a1 * a1;
  m[0] = a2 / det;
  m[1] = -a1 / det;
  m[2] = a0 / det;
  return true;
}

// ---- DataUtil/CFmIntParam.cpp ------------------------------------------------
void FmInt::plain(int n_raw, float fm_dose) {
  start.resize(n_raw);
  size.assign(n_raw, 1);
  dose.assign(n_raw, fm_dose);
  acc.resize(n_raw);
  for (int i = 0; i < n_raw; ++i) {
    start[i] = i;
    acc[i] = fm_dose * (i + 1);
  }
  centers();
}

void FmInt::integrate(const std::vector<int>& gsz_in, const std::vector<int>& isz, float raw_dose,
                      int n_raw) {
  const int ne = (int)gsz_in.size();
  std::vector<int> gsz(gsz_in), nint(ne, 0);
  int count = 0;
  for (int i = 0; i < ne; ++i) count += gsz[i];
  // more frames in the file than in the movie: take them off the last
  // entries first; fewer: the last entry gets the rest (:150-161)
  int extra = count - n_raw;
  const int last = ne - 1;
  if (extra > 0) {
    for (int i = last; i >= 0; --i) {
      const int g = gsz[i];
      gsz[i] -= extra;
      if (gsz[i] <= 0) gsz[i] = 0;
      else extra = extra - g;
      if (extra <= 0) break;
    }
  } else if (extra < 0) {
    gsz[last] -= extra;
  }
  // leftovers of an entry move to the next one (:165-173)
  for (int i = 0; i < last; ++i) {
    nint[i] = gsz[i] / isz[i];
    gsz[i + 1] += gsz[i] % isz[i];
  }
  extra = gsz[last] % isz[last];
  nint[last] = gsz[last] / isz[last];
  int n = 0;
  for (int i = 0; i < ne; ++i) n += nint[i];
  size.assign(n, 0);
  start.assign(n, 0);
  int c = 0;
  for (int i = 0; i < ne; ++i)
    for (int k = 0; k < nint[i]; ++k) size[c++] = isz[i];
  // the last rendered frames take one leftover raw frame each (:189-193)
  for (int i = 0; i < extra; ++i) size[n - 1 - i] += 1;
  for (int i = 1; i < n; ++i) start[i] = start[i - 1] + size[i - 1];
  dose.resize(n);
  acc.resize(n);
  for (int i = 0; i < n; ++i) dose[i] = size[i] * raw_dose;
  if (n > 0) acc[0] = dose[0];
  for (int i = 1; i < n; ++i) acc[i] = acc[i - 1] + dose[i];
  centers();
}

bool FmInt::drop(int t0, int t1) {
  if (t0 + t1 <= 0) return true;
  const int keep = count() - t0 - t1;
  if (keep <= 5) return false;
  start.erase(start.begin(), start.begin() + t0);
  size.erase(size.begin(), size.begin() + t0);
  dose.erase(dose.begin(), dose.begin() + t0);
  acc.erase(acc.begin(), acc.begin() + t0);
  start.resize(keep);
  size.resize(keep);
  dose.resize(keep);
  acc.resize(keep);
  centers();
  return true;
}

void FmInt::centers() {
  center.resize(start.size());
  for (size_t i = 0; i < start.size(); ++i) center[i] = start[i] + 0.5f * (size[i] - 1.0f);
}

bool read_fmint_file(const char* path, float cli_fm_dose, std::vector<int>& gs,
                     std::vector<int>& is, std::vector<float>& ds) {
  gs.clear();
  is.clear();
  ds.clear();
  FILE* f = std::fopen(path, "rt");
  if (!f) return false;
  char buf[256] = {0};
  int g = 0, n = 0;
  float d = 0.0f;
  if (!std::fgets(buf, sizeof(buf), f)) buf[0] = 0;
  int items = std::sscanf(buf, "%d  %d  %f", &g, &n, &d);
  bool ok = items >= 2;
  const bool two = items == 2;
  if (two) d = cli_fm_dose;
  while (ok) {
    gs.push_back(g);
    is.push_back(n);
    ds.push_back(d);
    if (std::feof(f)) break;
    if (!std::fgets(buf, sizeof(buf), f)) break;
    if (two) {
      if (std::sscanf(buf, "%d  %d", &g, &n) != 2) continue;
    } else {
      // the reference compares (==) instead of assigning here, so a line
      // that does not scan leaves the previous values, which are pushed again
      std::sscanf(buf, "%d  %d  %f", &g, &n, &d);
      if (d < 0) ok = false;
    }
  }
  std::fclose(f);
  for (size_t i = 1; i < ds.size(); ++i)
    if (ds[i] != ds[0]) {  // various frame doses: no integration (:160-169)
      gs.clear();
      is.clear();
      ds.clear();
      break;
    }
  return true;
}

// ---- DataUtil/CFmGroupParam.cpp:26-78 ----------------------------------------
void FrameGroups::setup(int n_frames, int bin_z) {
  FmInt fi;
  fi.plain(n_frames, 0.0f);
  setup(fi, bin_z);
}

void FrameGroups::setup(const FmInt& fi, int bin_z) {
  binZ = bin_z;
  start.clear();
  size.clear();
  center.clear();
  fm_center = fi.center;
  const int n = fi.count();
  int min_raw = 2147483647;  // (int)1e20 in the reference, which g++ folds to INT_MAX
  for (int i = 0; i < n; ++i) min_raw = fi.size[i] < min_raw ? fi.size[i] : min_raw;
  const int max_raw = bin_z * min_raw;  // mFindMaxGroupRawFms
  int f = 0;
  while (f < n) {  // mGroupByRawSize
    start.push_back(f);
    int sz = 0, raw = 0;
    for (;;) {
      raw += fi.size[f];
      sz += 1;
      f += 1;
      if (f >= n || raw >= max_raw) break;
    }
    size.push_back(sz);
  }
  for (size_t g = 0; g < start.size(); ++g) {
    float acc = 0.0f;
    for (int i = 0; i < size[g]; ++i) acc += fi.center[start[g] + i];
    center.push_back(acc / size[g]);
  }
}

// ---- Align/CStackShift.cpp ------------------------------------------------
void StackShift::add(const StackShift& d) {
  for (int i = 0; i < n; ++i) {
    v[i] += d.v[i];
    v[n + i] += d.v[n + i];
  }
}

void StackShift::multiply(float fx, float fy) {
  for (int i = 0; i < n; ++i) {
    v[i] *= fx;
    v[n + i] *= fy;
  }
}

void StackShift::truncate_decimal() {
  for (int i = 0; i < 2 * n; ++i) v[i] = 0.01f * (int)(v[i] * 100);
}

void StackShift::make_relative(int ref) {
  const float rx = v[ref], ry = v[n + ref];
  for (int i = 0; i < n; ++i) {
    v[i] -= rx;
    v[n + i] -= ry;
  }
}

void StackShift::smooth(float w) {
  if (w >= 1) return;
  std::vector<float> o(v);
  const float w2 = 0.5f * (1.0f - w);
  for (int i = 1; i < n - 1; ++i) {
    o[i] = w * v[i] + w2 * (v[i - 1] + v[i + 1]);
    o[n + i] = w * v[n + i] + w2 * (v[n + i - 1] + v[n + i + 1]);
  }
  v.swap(o);
}

void StackShift::remove_spikes() { host::remove_spikes(v.data(), v.data() + n, n); }

// ---- Align/CInterpolateShift.cpp:36-143 -----------------------------------
StackShift interpolate(const StackShift& grp, const FrameGroups& g, int n_frames, bool nearest) {
  StackShift out;
  out.setup(n_frames);
  const int ng = grp.n;
  if (n_frames == ng) {
    out.v = grp.v;
    return out;
  }
  if (nearest) {
    for (int k = 0; k < ng; ++k)
      for (int i = 0; i < g.size[k]; ++i) {
        out.x(g.start[k] + i) = grp.x(k);
        out.y(g.start[k] + i) = grp.y(k);
      }
    return out;
  }
  for (int i = 0; i < n_frames; ++i) {
    const float fc = g.fm_center[i];  // CFmIntParam::m_pfIntFmCents
    int k = ng - 1;
    if (fc <= g.center[0]) {
      k = 1;
    } else {
      for (int j = 1; j < ng; ++j)
        if (fc < g.center[j]) {
          k = j;
          break;
        }
    }
    const int f = k - 1;
    const float dg = g.center[k] - g.center[f];
    const float df = fc - g.center[f];
    const float sx = (grp.x(k) - grp.x(f)) / dg;
    const float sy = (grp.y(k) - grp.y(f)) / dg;
    out.x(i) = grp.x(f) + sx * df;
    out.y(i) = grp.y(f) + sy * df;
  }
  return out;
}

// ---- LibSrc/Util/Util_LinEqs.cpp:19-148 -----------------------------------
bool lin_eqs(float* a, float* b, int dim) {
  std::vector<int> col(dim), row(dim), piv(dim, 0);
  for (int ip = 0; ip < dim; ++ip) {
    int cx = 0, cy = 0;
    bool found = false;
    float big = 0.0f;
    for (int y = 0; y < dim; ++y) {
      if (piv[y] == 1) continue;
      for (int x = 0; x < dim; ++x) {
        if (piv[x] == 1) continue;
        const float c = (float)fabs(a[y * dim + x]);
        if (c <= big) continue;
        big = c;
        cx = x;
        cy = y;
        found = true;
      }
    }
    if (!found) return false;
    piv[cx] += 1;
    col[ip] = cx;
    row[ip] = cy;
    if (a[cy * dim + cx] == 0.0f) return false;
    const int r1 = col[ip], r2 = row[ip];
    if (r1 != r2) {
      for (int x = 0; x < dim; ++x) {
        float t = a[r1 * dim + x];
        a[r1 * dim + x] = a[r2 * dim + x];
        a[r2 * dim + x] = t;
      }
      float t = b[r1];
      b[r1] = b[r2];
      b[r2] = t;
    }
    const int c = col[ip];
    const double inv = 1.0 / (a[c * dim + c] + 1e-30);
    for (int x = 0; x < dim; ++x) a[c * dim + x] = (float)(a[c * dim + x] * inv);
    b[c] = (float)(b[c] * inv);
    for (int y = 0; y < dim; ++y) {
      if (y == c) continue;
      const float d = a[y * dim + c];
      for (int x = 0; x < dim; ++x) a[y * dim + x] -= (a[c * dim + x] * d);
      b[y] -= (b[c] * d);
    }
  }
  return true;
}

// ---- Util/CSplineFit1D.cpp:43-115 -----------------------------------------
namespace {
struct SplineFit {
  int nk = 0, dim = 3;
  const float* knots = nullptr;
  std::vector<float> t, cur, coef, mat;
  void setup(int n, const float* k) {
    nk = n;
    dim = n + 3;
    knots = k;
    t.assign(dim, 0.f);
    cur.assign(dim, 0.f);
    coef.assign(dim, 0.f);
    mat.assign((size_t)dim * dim, 0.f);
  }
  void terms(float x) {
    t[0] = 1;
    for (int i = 1; i < 3; ++i) t[i] = t[i - 1] * x;
    for (int i = 0; i < nk; ++i) t[i + 3] = 0.0f;
    for (int i = 0; i < nk; ++i) {
      if (x < knots[i]) break;
      const float d = x - knots[i];
      t[i + 3] = d * d;
    }
  }
  void cur_terms(float x) {
    for (int i = 0; i < dim; ++i) cur[i] = 0.0f;
    cur[1] = 1.0f;
    cur[2] = 2.0f * x;
    for (int i = 0; i < nk; ++i) {
      const float d = x - knots[i];
      if (d > 0) break;
      cur[i + 3] = 2.0f * d;
    }
  }
  bool fit(const float* X, const float* Y, int n, float* out, float reg) {
    for (auto& m : mat) m = 0.0f;
    for (auto& c : coef) c = 0.0f;
    for (auto& c : t) c = 0.0f;
    for (auto& c : cur) c = 0.0f;
    for (int i = 0; i < n; ++i) {
      terms(X[i]);
      if (reg != 0.0f) cur_terms(X[i]);
      for (int r = 0; r < dim; ++r) {
        for (int c = 0; c < dim; ++c) {
          const float p = t[r] * t[c];
          const float q = reg * cur[r] * cur[c];
          mat[r * dim + c] += (p + q);
        }
        coef[r] += (t[r] * Y[i]);
      }
    }
    if (!lin_eqs(mat.data(), coef.data(), dim)) return false;
    for (int i = 0; i < n; ++i) {
      terms(X[i]);
      float v = 0.0f;
      for (int k = 0; k < dim; ++k) v += coef[k] * t[k];
      out[i] = v;
    }
    return true;
  }
};

// CRemoveSpikes1D::mRemoveSingle (Util/CRemoveSpikes1D.cpp:127-148)
void remove_single(float* s, int n, float* buf) {
  std::memcpy(buf, s, sizeof(float) * n);
  const int e = n - 1;
  for (int i = 1; i < e; ++i) {
    if (fabs(buf[i] - buf[i - 1]) < 5.0f) continue;
    if (fabs(buf[i] - buf[i + 1]) < 5.0f) continue;
    s[i] = (buf[i - 1] + buf[i + 1]) / 2.0f;
  }
  if (fabs(buf[0] - buf[1]) > 10.0f && fabs(buf[0]) > fabs(buf[1])) s[0] = 2.0f * buf[1] - buf[2];
  if (fabs(buf[e] - buf[e - 1]) > 10.0f && fabs(buf[e]) > fabs(buf[e - 1]))
    s[e] = 2.0f * buf[e - 1] - buf[e - 2];
}

// CRemoveSpikes1D::mFindBad (:107-125): replaces outliers in `raw` by the fit.
bool find_bad(float* raw, const float* fit, int n, float tol) {
  bool has = false;
  for (int i = 0; i < n; ++i) {
    if (fabs(fit[i] - raw[i]) > tol && fabs(raw[i]) > fabs(fit[i])) {
      raw[i] = fit[i];
      has = true;
    }
  }
  return has;
}
}  // namespace

// CRemoveSpikes1D::SetDataSize + DoIt(bSingle = false) (:31-105)
void remove_spikes(float* sx, float* sy, int n) {
  if (n < 3) return;
  std::vector<float> tm(n), buf(n), fx(n, 0.0f), fy(n, 0.0f);
  const float fact = 1.0f / n;
  for (int i = 0; i < n; ++i) tm[i] = (float)sqrt(i * fact);
  const int kd = 15;
  int nk = (n - 2 * kd) / kd;
  if (nk < 0) nk = 0;
  else if (nk > 6) nk = 6;
  if (nk == 0 && n >= 2 * kd) nk = 1;
  std::vector<float> knots(nk > 0 ? nk : 1);
  for (int i = 0; i < nk; ++i) knots[i] = tm[(i + 1) * kd];
  SplineFit sp;
  sp.setup(nk, knots.data());
  for (int r = 0; r < 2; ++r) {
    remove_single(sx, n, buf.data());
    remove_single(sy, n, buf.data());
  }
  const float reg = (float)1e-20;
  sp.fit(tm.data(), sx, n, fx.data(), reg);
  sp.fit(tm.data(), sy, n, fy.data(), reg);
  std::memcpy(buf.data(), sx, sizeof(float) * n);
  if (find_bad(buf.data(), fx.data(), n, 3.0f)) sp.fit(tm.data(), buf.data(), n, fx.data(), reg);
  std::memcpy(buf.data(), sy, sizeof(float) * n);
  // The y refit uses the y shifts as given, not the cleaned copy
  // (CRemoveSpikes1D.cpp:83-90).
  if (find_bad(buf.data(), fy.data(), n, 3.0f)) sp.fit(tm.data(), sy, n, fy.data(), reg);
  for (int i = 0; i < n; ++i) {
    float tol = 5.0f;
    if (i > 20) tol = 4.0f;
    if (i < 50) tol = 3.0f;
    const float dx = fx[i] - sx[i];
    const float dy = fy[i] - sy[i];
    if (fabs(dx) > tol) sx[i] = fx[i];
    if (fabs(dy) > tol) sy[i] = fy[i];
  }
}

// ---- Align/CPeak2D.cpp:39-109 ---------------------------------------------
void peak2d(const float* img, int sx, int sy, float* shift) {
  const int n = sx * sy;
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
  const int ic = py * sx + px;
  const double a = (img[ic + 1] + img[ic - 1]) * 0.5 - img[ic];
  const double b = (img[ic + 1] - img[ic - 1]) * 0.5;
  const double c = (img[ic + sx] + img[ic - sx]) * 0.5f - img[ic];
  const double d = (img[ic + sx] - img[ic - sx]) * 0.5;
  double cx = -b / (2 * a + 1e-30);
  double cy = -d / (2 * c + 1e-30);
  if (fabs(cx) > 1) cx = 0;
  if (fabs(cy) > 1) cy = 0;
  const float fx = (float)(px + cx), fy = (float)(py + cy);
  shift[0] = fx - sx / 2;
  shift[1] = fy - sy / 2;
}

// ---- Align/CIterativeAlign.cpp:99-156 -------------------------------------
void IterState::start(int n_frames, int n_groups, float bf) {
  tmp.setup(n_frames);
  grp.setup(n_groups);
  total.setup(n_groups);
  bfactor = bf;
  max_err = 0.0f;
  iterations = 0;
  done = false;
  errors.clear();
}

void IterState::start_from(const float* init, const FrameGroups& g, int n_frames, float bf) {
  start(n_frames, g.count(), bf);
  for (int f = 0; f < n_frames; ++f) {
    tmp.x(f) = init[2 * f];
    tmp.y(f) = init[2 * f + 1];
  }
  for (int k = 0; k < g.count(); ++k) {
    double sx = 0.0, sy = 0.0;
    for (int i = 0; i < g.size[k]; ++i) {
      sx += init[2 * (g.start[k] + i)];
      sy += init[2 * (g.start[k] + i) + 1];
    }
    total.x(k) = (float)(sx / g.size[k]);
    total.y(k) = (float)(sy / g.size[k]);
  }
}

bool IterState::step(const float* gxy, const FrameGroups& g, int it, int max_iter, float tol) {
  const int ng = grp.n;
  max_err = 0.0f;
  for (int k = 0; k < ng; ++k) {
    const float sx = gxy[2 * k], sy = gxy[2 * k + 1];
    grp.x(k) = sx;
    grp.y(k) = sy;
    // CAlignStack::mUpdateError (Align/CAlignStack.cpp:211-215)
    const double d = sqrtf(sx * sx + sy * sy);
    if (max_err < d) max_err = (float)d;
  }
  bfactor -= 2;
  if (bfactor < 20) bfactor = 20.0f;
  total.add(grp);
  StackShift ip = interpolate(grp, g, tmp.n, true);
  tmp.add(ip);
  errors.push_back(max_err);
  iterations += 1;
  if ((max_err < tol && it > 0) || it + 1 >= max_iter) done = true;
  return done;
}

StackShift IterState::finish(const FrameGroups& g, int n_frames) const {
  StackShift r = interpolate(total, g, n_frames, false);
  r.remove_spikes();
  r.smooth(0.5f);
  // CIterativeAlign::DoIt (:72-81)
  float w = 0.3f + 0.1f * g.binZ;
  if (w > 0.9f) w = 0.9f;
  r.smooth(w);
  return r;
}

// ---- Align/CPatchShifts.cpp:263-355 ---------------------------------------
void patch_make_relative(std::vector<float>& s, int N, int P) {
  // One zero float after the table: for the last patch of the reference
  // frame the reference reads one element past the frame's row.
  std::vector<float> e(s.size() + 1, 0.0f);
  std::memcpy(e.data(), s.data(), sizeof(float) * s.size());
  float fmin = (float)1e20;
  int ref = 0;
  for (int i = 1; i < N; ++i) {
    const float* p = e.data() + (long)i * P * 2;
    float mx = 0.0f, my = 0.0f;
    for (int j = 0; j < P; ++j) {
      mx += p[2 * j];
      my += p[2 * j + 1];
    }
    mx /= P;
    my /= P;
    float sd = 0.0f;
    for (int j = 0; j < P; ++j) {
      const float dx = p[2 * j] - mx, dy = p[2 * j + 1] - my;
      sd += (dx * dx + dy * dy);
    }
    sd = (float)sqrt(sd / P);
    const float m = (float)sqrt(mx * mx + my * my);
    const float val = m + sd;
    if (val > fmin) continue;
    fmin = val;
    ref = i;
  }
  float* r = e.data() + (long)ref * P * 2;
  for (int i = 0; i < N; ++i) {
    float* p = e.data() + (long)i * P * 2;
    for (int j = 0; j < P; ++j) {
      const int k = 2 * j;
      p[k] -= r[k];
      p[k + 1] -= r[k + 2];
    }
  }
  std::memcpy(s.data(), e.data(), sizeof(float) * s.size());
}

void patch_detect_bads(const float* s, const float* cent, int N, int P, int W, int H,
                       unsigned char* bad) {
  for (int f = 0; f < N; ++f) {
    const float* p = s + (long)f * P * 2;
    for (int i = 0; i < P; ++i) {
      const float sx = p[2 * i], sy = p[2 * i + 1];
      const double dS = sqrt(sx * sx + sy * sy);
      double rms = 0, sw = 0;
      for (int k = 0; k < P; ++k) {
        if (k == i) continue;
        float fx = (cent[2 * k] - cent[2 * i]) / W;
        float fy = (cent[2 * k + 1] - cent[2 * i + 1]) / H;
        const double w = expf(-100.0 * (fx * fx + fy * fy));
        fx = p[2 * k];
        fy = p[2 * k + 1];
        rms += (w * (fx * fx + fy * fy));
        sw += w;
      }
      rms = sqrtf(rms / sw);
      float lr = (float)rms;
      if (lr < 2) lr = 2.0f;
      bad[(long)f * P + i] = (dS > (1 * lr)) ? 1 : 0;
    }
  }
}

// ---- Align/CDetectFeatures.cpp:58-181, 273-396; CPatchCenters.cpp:42-106 --
namespace {
struct FeatureSearch {
  int B[2];
  float pat[2];
  int sea[4];
  std::vector<unsigned char> feat, used;
  int range(int s, int sz, const int* r) const {
    if (s < r[0]) return r[0];
    if ((s + sz) > r[1]) return r[1] - sz;
    return s;
  }
  void set_used(float cx, float cy) {
    const int wx = (int)(pat[0] * 0.8f), wy = (int)(pat[1] * 0.8f);
    int sx = (int)(cx - wx / 2), sy = (int)(cy - wy / 2);
    sx = range(sx, wx, &sea[0]);
    sy = range(sy, wy, &sea[2]);
    for (int y = 0; y < wy; ++y)
      for (int x = 0; x < wx; ++x) used[(sy + y) * B[0] + sx + x] = 1;
  }
  bool has_feature(float cx, float cy) const {
    const int ix = (int)cx, iy = (int)cy;
    if (ix < sea[0] || ix > sea[1]) return false;
    if (iy < sea[2] || iy > sea[3]) return false;
    return feat[iy * B[0] + ix] != 0;
  }
  void relocate(float* c) {
    const int wx = B[0] / 3, wy = B[1] / 3;
    int sx = (int)(c[0] - wx * 0.5f + 0.5f);
    int sy = (int)(c[1] - wy * 0.5f + 0.5f);
    sx = range(sx, wx, &sea[0]);
    sy = range(sy, wy, &sea[2]);
    float best = (float)1e20;
    float found[2] = {-1.0f, 0.0f};
    for (int y = 0; y < wy; ++y)
      for (int x = 0; x < wx; ++x) {
        const int j = (sy + y) * B[0] + sx + x;
        if (used[j] || !feat[j]) continue;
        const float fx = x + sx + 0.5f, fy = y + sy + 0.5f;
        const float dx = fx - c[0], dy = fy - c[1];
        const float r = (float)sqrtf(dx * dx + dy * dy);
        if (r >= best) continue;
        best = r;
        found[0] = fx;
        found[1] = fy;
      }
    if (found[0] > 0) {
      c[0] = found[0];
      c[1] = found[1];
    }
    set_used(c[0], c[1]);
  }
};
}  // namespace

void patch_starts(const float* map, int bx, int by, float fMean, float m2, int px, int py,
                  int xcf_x, int xcf_y, int pat_x, int pat_y, std::vector<int>& starts) {
  FeatureSearch F;
  F.B[0] = bx;
  F.B[1] = by;
  F.pat[0] = bx * 1.0f / px;
  F.pat[1] = by * 1.0f / py;
  F.sea[0] = (int)(F.pat[0] * 0.5f - 0.5f);
  if (F.sea[0] < 4) F.sea[0] = 4;
  F.sea[1] = bx - F.sea[0];
  F.sea[2] = (int)(F.pat[1] * 0.5f - 0.5f);
  if (F.sea[2] < 4) F.sea[2] = 4;
  F.sea[3] = by - F.sea[2];
  float fStd = m2 - fMean * fMean;
  if (fStd < 0) fStd = 0.0f;
  else fStd = (float)sqrtf(fStd);
  const int n = bx * by;
  float lo = fMean - 4.0f * fStd, hi = fMean + 4.0f * fStd;
  double dm = 0, ds = 0;
  int cnt = 0;
  for (int i = 0; i < n; ++i) {
    if (map[i] < lo) continue;
    if (map[i] > hi) continue;
    dm += map[i];
    ds += (map[i] * map[i]);
    cnt += 1;
  }
  dm /= (cnt + 1e-30);
  ds = ds / (cnt + 1e-30) - dm * dm;
  if (ds < 0) ds = 0;
  else ds = sqrtf(ds);
  lo = (float)(dm - 4.0 * ds);
  hi = (float)(dm - 0.08f * ds);
  F.feat.assign(n, 0);
  F.used.assign(n, 0);
  for (int i = 0; i < n; ++i) F.feat[i] = (map[i] < lo || map[i] > hi) ? 0 : 1;
  // mFindCenters: the "no feature" early return never triggers (it is an
  // assignment in the reference), so featureless patches are relocated.
  const int np = px * py;
  std::vector<float> cen(3 * (size_t)np, 0.0f);
  for (int i = 0; i < np; ++i) {
    const int x = i % px, y = i / px;
    const float cx = (x + 0.5f) * F.pat[0], cy = (y + 0.5f) * F.pat[1];
    const bool has = F.has_feature(cx, cy);
    cen[3 * i] = cx;
    cen[3 * i + 1] = cy;
    if (has) {
      cen[3 * i + 2] = 1.0f;
      F.set_used(cx, cy);
    } else {
      cen[3 * i + 2] = -1.0f;
    }
  }
  for (int i = 0; i < np; ++i) {
    float* c = &cen[3 * i];
    if (c[2] > 0) continue;
    F.relocate(c);
  }
  // CDetectFeatures::GetCenter + CPatchCenters::mCalcStart
  starts.assign(2 * (size_t)np, 0);
  const float binx = xcf_x * 1.0f / bx, biny = xcf_y * 1.0f / by;
  for (int i = 0; i < np; ++i) {
    const float c[2] = {cen[3 * i] * binx, cen[3 * i + 1] * biny};
    const int ps[2] = {pat_x, pat_y};
    const int xs[2] = {xcf_x, xcf_y};
    for (int d = 0; d < 2; ++d) {
      int s = (int)(c[d] - ps[d] / 2);
      if (s < 0) s = 0;
      else if ((s + ps[d]) > xs[d]) s = xs[d] - ps[d];
      starts[2 * i + d] = s;
    }
  }
}

void defect_template(int ms, float* tpl) {
  const int n = ms * ms;
  const int ex = ms - 1, ey = ms - 1;
  for (int i = 0; i < n; ++i) {
    const int x = i % ms, y = i / ms;
    if (x == 0 || x == ex) tpl[i] = -1.0f;
    else if (y == 0 || y == ey) tpl[i] = -1.0f;
    else tpl[i] = 1.0f;
  }
  double dm = 0, ds = 0;
  for (int i = 0; i < n; ++i) {
    dm += tpl[i];
    ds += (tpl[i] * tpl[i]);
  }
  const float fm = (float)(dm / n);
  ds = ds / n - fm * fm;
  float fs = (ds <= 0) ? 0.0f : (float)sqrt(ds);
  fs += (float)(1e-30);
  for (int i = 0; i < n; ++i) tpl[i] = (tpl[i] - fm) / fs;
}

float kv_factor(int kv) {
  float f = 1.0f;
  if (kv >= 300) f = 1.0f;
  else if (kv < 300 && kv >= 200) f = 0.002f * (kv - 200) + 0.8f;
  else if (kv < 200 && kv >= 120) f = 0.004375f * (kv - 120) + 0.45f;
  else f = 0.45f;
  return f;
}

void patch_starts_from_centers(const float* centers, int n_patches, float bin_x, float bin_y,
                               int xcf_x, int xcf_y, int pat_x, int pat_y,
                               std::vector<int>& starts) {
  starts.assign(2 * (size_t)n_patches, 0);
  for (int p = 0; p < n_patches; ++p) {
    const int cx = (int)lrintf(centers[2 * p] / bin_x);
    const int cy = (int)lrintf(centers[2 * p + 1] / bin_y);
    starts[2 * p] = std::min(std::max(cx - pat_x / 2, 0), xcf_x - pat_x);
    starts[2 * p + 1] = std::min(std::max(cy - pat_y / 2, 0), xcf_y - pat_y);
  }
}

}  // namespace host
}  // namespace mc3
