// Test harness: exposes the reference's own host-side shift bookkeeping
// classes, compiled unmodified from the reference sources, through a C API
// so the CPU tests can pin libmc3's host code and the oracle against them.
// TEST INFRASTRUCTURE ONLY -- never linked into the product.
#include <cstdlib>
#include <cstring>
#include <cstdio>
#include <cmath>
#include <new>
#include <vector>
#include <cuda_runtime.h>

// Private members of the reference classes are reached from this harness
// only to construct inputs and read results.
#define private public
#include "Align/CAlignInc.h"
#include "CMainInc.h"
#include "DataUtil/CDataUtilInc.h"
#include "EerUtil/CEerUtilInc.h"
#include "Util/CUtilInc.h"
#include <Util/Util_LinEqs.h>
#undef private

using namespace MotionCor2;

// ---- host-memory stand-ins for the few CUDA runtime calls CPatchShifts
// makes on pinned host buffers (no GPU is needed for this code path) ----
extern "C" cudaError_t cudaMallocHost(void** p, size_t n) {
  *p = std::calloc(n ? n : 1, 1);
  return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
extern "C" cudaError_t cudaHostAlloc(void** p, size_t n, unsigned int) { return cudaMallocHost(p, n); }
extern "C" cudaError_t cudaFreeHost(void* p) { std::free(p); return cudaSuccess; }
extern "C" cudaError_t cudaMemcpy(void* d, const void* s, size_t n, cudaMemcpyKind) {
  std::memcpy(d, s, n);
  return cudaSuccess;
}

// CInput, CParseArgs and CReadFmIntFile are compiled from the reference too:
// the frame-integration tables below are set up through the reference's own
// singletons with the command-line values written into CInput.

extern "C" {

void ref_peak2d(float* win, int sx, int sy, float* shift) {
  Align::CPeak2D p;
  int sz[2] = {sx, sy};
  p.DoIt(win, sz);
  shift[0] = p.m_afShift[0];
  shift[1] = p.m_afShift[1];
}

void ref_remove_spikes(float* x, float* y, int n) {
  Util::CRemoveSpikes1D r;
  r.SetDataSize(n);
  r.DoIt(x, y, false);
}

int ref_lin_eqs(float* a, float* b, int dim) {
  Util_LinEqs e;
  return e.DoIt(a, b, dim) ? 1 : 0;
}

void ref_smooth(float* x, float* y, int n, float w) {
  Align::CStackShift s;
  s.Setup(n);
  std::memcpy(s.m_pfShiftXs, x, sizeof(float) * n);
  std::memcpy(s.m_pfShiftYs, y, sizeof(float) * n);
  s.Smooth(w);
  std::memcpy(x, s.m_pfShiftXs, sizeof(float) * n);
  std::memcpy(y, s.m_pfShiftYs, sizeof(float) * n);
}

void ref_truncate(float* x, float* y, int n) {
  Align::CStackShift s;
  s.Setup(n);
  std::memcpy(s.m_pfShiftXs, x, sizeof(float) * n);
  std::memcpy(s.m_pfShiftYs, y, sizeof(float) * n);
  s.TruncateDecimal();
  std::memcpy(x, s.m_pfShiftXs, sizeof(float) * n);
  std::memcpy(y, s.m_pfShiftYs, sizeof(float) * n);
}

// CInterpolateShift::DoIt for n frames grouped by binZ (one raw frame per
// integrated frame).  grp: [ng][2] in, out: [n][2].
int ref_interpolate(const float* grp, int n, int binZ, int nearest, float* out) {
  DataUtil::CFmIntParam ip;
  ip.m_iNumIntFms = n;
  ip.m_iNumRawFms = n;
  ip.mAllocate();
  for (int i = 0; i < n; ++i) {
    ip.m_piIntFmStart[i] = i;
    ip.m_piIntFmSize[i] = 1;
    ip.m_pfIntFmDose[i] = 1.0f;
    ip.m_pfAccFmDose[i] = (float)(i + 1);
  }
  ip.mCalcIntFmCenters();
  DataUtil::CFmGroupParam gp;
  gp.Setup(binZ, &ip);
  const int ng = gp.m_iNumGroups;
  Align::CStackShift g;
  g.Setup(ng);
  for (int k = 0; k < ng; ++k) {
    g.m_pfShiftXs[k] = grp[2 * k];
    g.m_pfShiftYs[k] = grp[2 * k + 1];
  }
  Align::CInterpolateShift is;
  Align::CStackShift* r = is.DoIt(&g, &gp, &ip, nearest != 0);
  for (int i = 0; i < n; ++i) {
    out[2 * i] = r->m_pfShiftXs[i];
    out[2 * i + 1] = r->m_pfShiftYs[i];
  }
  delete r;
  return ng;
}

// CPatchShifts::MakeRelative + DetectBads on raw per-patch shifts.
// raw: [P][N][2] per patch trajectories, centres [P][2];
// out_shifts [N][P][2], out_bad [N][P].
void ref_patch_shifts(const float* raw, const float* centres, int N, int P, int W, int H,
                      float* out_shifts, unsigned char* out_bad) {
  Align::CPatchShifts ps;
  int full[3] = {W, H, N};
  ps.Setup(P, full);
  for (int p = 0; p < P; ++p) {
    Align::CStackShift s;
    s.Setup(N);
    for (int f = 0; f < N; ++f) {
      s.m_pfShiftXs[f] = raw[((size_t)p * N + f) * 2];
      s.m_pfShiftYs[f] = raw[((size_t)p * N + f) * 2 + 1];
    }
    s.SetCenter(centres[2 * p], centres[2 * p + 1]);
    ps.SetRawShift(&s, p);
  }
  ps.MakeRelative();
  ps.DetectBads();
  for (int f = 0; f < N; ++f)
    for (int p = 0; p < P; ++p) {
      float v[2];
      ps.GetLocalShift(f, p, v);
      out_shifts[((size_t)f * P + p) * 2] = v[0];
      out_shifts[((size_t)f * P + p) * 2 + 1] = v[1];
      out_bad[(size_t)f * P + p] = ps.m_pbBadShifts[(size_t)f * P + p] ? 1 : 0;
    }
}

// CReadFmIntFile::DoIt, CFmIntParam::Setup and CFmGroupParam::Setup of the
// reference for n_raw raw frames, with -FmIntFile path (NULL or "" for
// none), -FmDose and -Throw / -Trunc; tables truncated to max_n entries.
int ref_fmint(const char* path, float fm_dose, int throw0, int throw1, int n_raw, int bin_z,
              int max_n, int* n_int, int* start, int* size, float* acc, float* cent,
              int* n_groups, int* g_start, int* g_size, float* g_cent, int* has_dose) {
  CInput* in = CInput::GetInstance();
  std::snprintf(in->m_acFmIntFile, sizeof(in->m_acFmIntFile), "%s", path ? path : "");
  in->m_fFmDose = fm_dose;
  in->m_aiThrow[0] = throw0;
  in->m_aiThrow[1] = throw1;
  DataUtil::CReadFmIntFile* rf = DataUtil::CReadFmIntFile::GetInstance();
  rf->DoIt();
  *has_dose = rf->HasDose() ? 1 : 0;
  DataUtil::CFmIntParam ip;
  ip.Setup(n_raw, 0);
  *n_int = ip.m_iNumIntFms;
  for (int i = 0; i < ip.m_iNumIntFms && i < max_n; ++i) {
    start[i] = ip.m_piIntFmStart[i];
    size[i] = ip.m_piIntFmSize[i];
    acc[i] = ip.m_pfAccFmDose[i];
    cent[i] = ip.m_pfIntFmCents[i];
  }
  DataUtil::CFmGroupParam gp;
  gp.Setup(bin_z, &ip);
  *n_groups = gp.m_iNumGroups;
  for (int g = 0; g < gp.m_iNumGroups && g < max_n; ++g) {
    g_start[g] = gp.m_piGroupStart[g];
    g_size[g] = gp.m_piGroupSize[g];
    g_cent[g] = gp.m_pfGroupCenters[g];
  }
  return 0;
}

// EerUtil::CDecodeEerFrame of the reference on one EER frame (its electrons
// are added to `frame`, cam x cam y times the sampling factor squared); the
// buffer is padded because the 7-bit decoder reads whole 32-bit words.
void ref_eer_decode(const unsigned char* data, int nbytes, int cam_x, int cam_y, int sampling,
                    int bits, unsigned char* frame) {
  EerUtil::CDecodeEerFrame d;
  int cam[2] = {cam_x, cam_y};
  d.Setup(cam, sampling);
  std::vector<unsigned char> buf(data, data + nbytes);
  buf.resize((size_t)nbytes + 8, 0);
  if (bits == 7) d.Do7Bits(buf.data(), nbytes, frame);
  else d.Do8Bits(buf.data(), nbytes, frame);
}

}  // extern "C"
