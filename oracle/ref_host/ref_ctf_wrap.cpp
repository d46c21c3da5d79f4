// Test harness: the reference's CTF fitting drivers (CCtfParam, CFindCtfBase,
// CFindCtf1D, CFindCtf2D, CFindDefocus1D, CFindDefocus2D, CFindCtfHelp),
// compiled unmodified from the reference sources, driven through a C API so
// the CPU tests can pin the oracle's search (its step sizes, sweep order and
// acceptance rules) against them.  The GPU kernel classes these drivers call
// are given host stand-ins below that evaluate the same expressions as the
// kernels (FindCtf/GRadialAvg.cu, GCalcCTF1D.cu, GCtfCC1D.cu, GCalcCTF2D.cu,
// GCtfCC2D.cu, GSpectralCC2D.cu) with double accumulation.
// TEST INFRASTRUCTURE ONLY -- never linked into the product.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>
#include <cuda_runtime.h>

#define private public
#include "FindCtf/CFindCtfInc.h"
#undef private

using namespace MotionCor2::FindCtf;

// ---- host memory behind the CUDA runtime calls of the drivers ----
extern "C" cudaError_t cudaMalloc(void** p, size_t n) {
  *p = std::calloc(n ? n : 1, 1);
  return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
extern "C" cudaError_t cudaFree(void* p) {
  std::free(p);
  return cudaSuccess;
}
extern "C" cudaError_t cudaMemcpy(void* d, const void* s, size_t n, cudaMemcpyKind) {
  std::memcpy(d, s, n);
  return cudaSuccess;
}
extern "C" cudaError_t cudaMemset(void* d, int v, size_t n) {
  std::memset(d, v, n);
  return cudaSuccess;
}

namespace {
float g_ctf1d[2], g_ctf2d[2];  // the kernels' __constant__ (wavelength, Cs) pairs
}

// ---- GRadialAvg (FindCtf/GRadialAvg.cu:11-31) ----
GRadialAvg::GRadialAvg(void) {}
GRadialAvg::~GRadialAvg(void) {}
void GRadialAvg::DoIt(float* s, float* avg, int* cmp) {
  for (int r = 0; r < cmp[0]; ++r) {
    int n = (int)(3.1415926f * r + 0.5f);
    if (n < 1) n = 1;
    else if (n > 180) n = 180;
    float sum = 0.f;
    const float step = 180.0f / n;
    for (int i = 0; i < n; ++i) {
      const float rad = (-90.0f + i * step) * 0.017453f;
      int x = (int)(r * cosf(rad) + 0.5f);
      int y = (int)(r * sinf(rad) + cmp[1] / 2 + 0.5f);
      if (y > cmp[1] - 1) y = cmp[1] - 1;  // the kernel reads past the spectrum at r = 256
      if (x > cmp[0] - 1) x = cmp[0] - 1;
      sum += s[y * cmp[0] + x];
    }
    avg[r] = sum / n;
  }
}

// ---- GCalcCTF1D (FindCtf/GCalcCTF1D.cu) ----
GCalcCTF1D::GCalcCTF1D(void) {}
GCalcCTF1D::~GCalcCTF1D(void) {}
void GCalcCTF1D::SetParam(CCtfParam* p) {
  g_ctf1d[0] = p->m_fWaveLen;
  g_ctf1d[1] = p->m_fCs;
  m_fAmpPhase = p->m_fAmpPhaseShift;
}
void GCalcCTF1D::DoIt(float df, float ext, float* ctf, int n) {
  const float add = m_fAmpPhase + ext;
  for (int i = 0; i < n; ++i) {
    float fs2 = (i * 0.5f) / (n - 1.0f);
    fs2 = fs2 * fs2;
    const float fw2 = g_ctf1d[0] * g_ctf1d[0];
    const float ph = add + 3.141592654f * g_ctf1d[0] * fs2 * (df - 0.5f * fw2 * fs2 * g_ctf1d[1]);
    ctf[i] = -sinf(ph);
  }
}

// ---- GCtfCC1D (FindCtf/GCtfCC1D.cu) ----
GCtfCC1D::GCtfCC1D(void) : m_gfRes(nullptr), m_fBFactor(1.0f) {}
GCtfCC1D::~GCtfCC1D(void) {}
void GCtfCC1D::SetSize(int n) { m_iSize = n; }
void GCtfCC1D::Setup(float lo, float hi, float b) {
  m_fFreqLow = lo;
  m_fFreqHigh = hi;
  m_fBFactor = b;
}
float GCtfCC1D::DoIt(float* ctf, float* sp) {
  double cc = 0, s1 = 0, s2 = 0;
  for (int x = 0; x < m_iSize; ++x) {
    if (!(x >= m_fFreqLow && x < m_fFreqHigh)) continue;
    float f = x * 0.5f / (m_iSize - 1);
    const float c = (fabsf(ctf[x]) - 0.5f) * expf(-m_fBFactor * f * f);
    const float s = sp[x];
    cc += c * s;
    s1 += c * c;
    s2 += s * s;
  }
  if (s1 > 0 && s2 > 0) cc /= sqrt(s1 * s2);
  else cc = 0.0;
  return (float)cc;
}

// ---- GCalcCTF2D (FindCtf/GCalcCTF2D.cu:15-37) ----
GCalcCTF2D::GCalcCTF2D(void) {}
GCalcCTF2D::~GCalcCTF2D(void) {}
void GCalcCTF2D::SetParam(CCtfParam* p) {
  g_ctf2d[0] = p->m_fWaveLen;
  g_ctf2d[1] = p->m_fCs;
  m_fAmpPhase = p->m_fAmpPhaseShift;
}
void GCalcCTF2D::DoIt(float dfmin, float dfmax, float azim, float ext, float* ctf, int* cmp) {
  const float mean = 0.5f * (dfmin + dfmax), sigma = 0.5f * (dfmax - dfmin);
  const float add = m_fAmpPhase + ext;
  // one pixel per kernel thread: rows split over host threads
  const int nt = 8, rows = cmp[1];
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t)
    th.emplace_back([=] {
  for (int y = t * rows / nt; y < (t + 1) * rows / nt; ++y)
    for (int x = 0; x < cmp[0]; ++x) {
      float fx = x * 0.5f / (cmp[0] - 1);
      const float fy = (y - cmp[1] / 2) / (float)cmp[1];
      const float s2 = fx * fx + fy * fy, w2 = g_ctf2d[0] * g_ctf2d[0];
      fx = atanf(fy / (fx + (float)1e-30));
      fx = mean + sigma * cosf(2.0f * (fx - azim));
      ctf[y * cmp[0] + x] = -sinf(add + 3.1415926f * g_ctf2d[0] * s2 * (fx - 0.5f * w2 * s2 * g_ctf2d[1]));
    }
    });
  for (auto& t : th) t.join();
}

// ---- GCtfCC2D (FindCtf/GCtfCC2D.cu) ----
GCtfCC2D::GCtfCC2D(void) : m_fBFactor(1.0f), m_gfRes(nullptr) {}
GCtfCC2D::~GCtfCC2D(void) {}
void GCtfCC2D::Setup(float lo, float hi, float b) {
  m_fFreqLow = lo;
  m_fFreqHigh = hi;
  m_fBFactor = b;
}
void GCtfCC2D::SetSize(int* cmp) {
  m_aiCmpSize[0] = cmp[0];
  m_aiCmpSize[1] = cmp[1];
}
float GCtfCC2D::DoIt(float* ctf, float* sp) {
  float lo2 = m_fFreqLow / m_aiCmpSize[1], hi2 = m_fFreqHigh / m_aiCmpSize[1];
  if (hi2 > 0.75f) hi2 = 0.75f;
  lo2 *= lo2;
  hi2 *= hi2;
  double a = 0, b = 0, c = 0;
  for (int y = 0; y < m_aiCmpSize[1]; ++y) {
    const float fy = (y - m_aiCmpSize[1] * 0.5f) / m_aiCmpSize[1];
    for (int x = 0; x < m_aiCmpSize[0]; ++x) {
      float fx = (0.5f * x) / (m_aiCmpSize[0] - 1);
      fx = fx * fx + fy * fy;
      if (fx < lo2 || fx > hi2) continue;
      const int i = y * m_aiCmpSize[0] + x;
      const float cv = (fabsf(ctf[i]) - 0.5f) * expf(-m_fBFactor * fx);
      const float sv = sp[i];
      a += cv * sv;
      b += cv * cv;
      c += sv * sv;
    }
  }
  const float sd = sqrtf((float)b * (float)c);
  return sd == 0 ? 0.0f : (float)a / sd;
}

// ---- GSpectralCC2D (FindCtf/GSpectralCC2D.cu) ----
GSpectralCC2D::GSpectralCC2D(void) : m_gfCC(nullptr), m_pfCC(nullptr) {
  m_aiSpectSize[0] = m_aiSpectSize[1] = 0;
}
GSpectralCC2D::~GSpectralCC2D(void) {}
void GSpectralCC2D::SetSize(int* s) {
  m_aiSpectSize[0] = s[0];
  m_aiSpectSize[1] = s[1];
}
int GSpectralCC2D::DoIt(float* ctf, float* sp) {
  const int X = m_aiSpectSize[0], Y = m_aiSpectSize[1], width = 10;
  std::vector<float> cc(X);
  for (int bx = 0; bx < X; ++bx) {
    int lo = bx - width / 2, hi = lo + width;
    if (lo < 0) {
      lo = 0;
      hi = width;
    } else if (hi > X) {
      lo = X - width;
      hi = X;
    }
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int y = 0; y < Y; ++y) {
      const float fy = fabsf(y - Y * 0.5f);
      if (fy >= hi) continue;
      for (int x = 0; x < X; ++x) {
        if (x >= hi) continue;
        const float r = sqrtf(x * x + fy * fy);
        if (r < lo || r >= hi) continue;
        const float c = fabsf(ctf[y * X + x]) - 0.5f, v = sp[y * X + x];
        s[0] += c;
        s[1] += v;
        s[2] += c * v;
        s[3] += c * c;
        s[4] += v * v;
        s[5] += 1;
      }
    }
    if (s[5] == 0) {
      cc[bx] = 0;
      continue;
    }
    const double mc = s[0] / s[5], ms = s[1] / s[5];
    double cv = s[2] / s[5], sc = s[3] / s[5] - mc * mc, ss = s[4] / s[5] - ms * ms;
    if (sc <= 0 || ss <= 0) {
      cc[bx] = 0;
      continue;
    }
    cv -= mc * ms;
    cc[bx] = (float)(cv / sqrt(sc * ss));
  }
  int imax = 1;
  float fmax = (float)-1e30;
  for (int i = 1; i < X; ++i) {
    if (cc[i] <= fmax) continue;
    fmax = cc[i];
    imax = i;
  }
  if (fmax < 0.143f) return imax;
  int shell = imax;
  for (int i = imax; i < X; ++i) {
    if (cc[i] < 0.143f) break;
    shell = i;
  }
  return shell;
}

extern "C" {

// CCtfParam::Setup: wavelength and Cs in pixels, amplitude phase.
void ref_ctf_param(float kv, float cs, float ac, float pix, float* out3) {
  CCtfParam p;
  p.Setup(kv, cs, ac, pix);
  out3[0] = p.m_fWaveLen;
  out3[1] = p.m_fCs;
  out3[2] = p.m_fAmpPhaseShift;
}

// CFindCtfMain::mFindCTF (FindCtf/CFindCtfMain.cpp:96-116) on a [512][257]
// half spectrum; res6 as CSaveSerialCryoEM::mSaveCtfFit prints it.
void ref_ctf_search(const float* spect, float pix_n, float kv, float cs, float ac, float ext_phase,
                    float* res6) {
  CCtfParam param;
  param.Setup(kv, cs, ac, pix_n);
  const float df_range = 40000.0f * pix_n * pix_n;
  const float ph_range = fminf(ext_phase * 2.0f, 180.0f);
  int size[2] = {257, 512};
  CFindCtf2D* f = new CFindCtf2D;
  f->Setup1(size);
  f->Setup2(&param);
  f->SetDfRange(df_range);
  f->SetAstRange(0.10f);
  f->SetAngRange(180.0f);
  f->SetPhaseRange(ph_range);
  f->m_pFindDefocus2D->m_fExtPhase = 0.0f;  // read before it is set (mIterate)
  std::vector<float> s(spect, spect + 257 * 512);
  f->DoIt(s.data());
  CCtfParam* r = f->GetResult();
  res6[0] = r->GetDfMax(true);
  res6[1] = r->GetDfMin(true);
  res6[2] = r->GetAstAng(true);
  res6[3] = r->GetExtPhase(true);
  res6[4] = r->m_fScore;
  res6[5] = r->m_fCtfRes;
  delete r;
  delete f;
}

}  // extern "C"
