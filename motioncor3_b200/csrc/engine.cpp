// Processing engine: the single-movie path of CProcessThread::mProcess
// (CProcessThread.cpp:82-107) on one GPU stream.
#include "engine.h"

#include "dft_gemm.cuh"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <math.h>

namespace mc3 {

int cuda_status(cudaError_t e, const char* where) {
  (void)where;
  if (e == cudaSuccess) return kOk;
  if (e == cudaErrorMemoryAllocation) return kENoMem;
  return kECuda;
}

int last_cuda_status(const char* where) { return cuda_status(cudaGetLastError(), where); }

int DevBuf::ensure(size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (bytes <= cap) return kOk;
  release();
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    p = nullptr;
    cudaGetLastError();
    return kENoMem;
  }
  cap = bytes;
  return kOk;
}

void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
}

// ---------------------------------------------------------------------------
int Geometry::compute(int w, int h, int n, const mc3_params& p, bool file_dose) {
  if (w < 16 || h < 16 || n < 3 || (w & 1) || (h & 1)) return kEInval;
  W = w;
  H = h;
  N = n;
  cmpX = W / 2 + 1;
  cmpY = H;
  padX = 2 * cmpX;
  // CBufferPool::mCreateXcfBuffer (CBufferPool.cpp:220-242)
  const float fBinX = W / 2048.0f;
  const float fBinY = H / 2048.0f;
  float fBin = (float)fmin(fBinX, fBinY);
  if (fBin < 1) fBin = 1.0f;
  const int iXcfX = (int)(W / fBin + 0.5f);
  const int iXcfY = (int)(H / fBin + 0.5f);
  xcfCmpX = iXcfX / 2 + 1;
  xcfCmpY = iXcfY / 2 * 2;
  xcfBin[0] = (cmpX - 1.0f) / (xcfCmpX - 1.0f);
  xcfBin[1] = cmpY * 1.0f / xcfCmpY;
  // CBufferPool::mCreatePatBuffer (CBufferPool.cpp:244-262),
  // CPatchCenters::Calculate patch size (Align/CPatchCenters.cpp:48-51)
  Px = p.patch[0] > 1 ? p.patch[0] : 0;
  Py = p.patch[1] > 1 ? p.patch[1] : 0;
  patch = false;
  P = 0;
  if (Px > 1 && Py > 1) {
    const int ix = (xcfCmpX - 1) * 2, iy = xcfCmpY;
    const int ipx = ix / Px, ipy = iy / Py;
    if (ipx <= ix / 2 && ipy <= iy / 2) {
      patch = true;
      P = Px * Py;
      patCmpX = ipx / 2 + 1;
      patCmpY = ipy / 2 * 2;
      patSizeX = ix / Px / 2 * 2;
      patSizeY = iy / Py / 2 * 2;
    }
  }
  // CFmIntParam::bDoseWeight / bDWSelectedSum (DataUtil/CFmIntParam.cpp:222-247)
  dw = !(p.kv < 80 || p.kv > 300) && p.pix_size > 0 && (p.fm_dose > 0 || file_dose);
  dws = dw && p.sum_range[0] >= 0 && p.sum_range[1] > 0 &&
        (p.sum_range[1] - p.sum_range[0]) > 1.0f;
  nSums = 1 + (dw ? 1 : 0) + (dws ? 1 : 0) + (p.split_sum ? 2 : 0);
  // CInput::GetBinnedSize (CInput.cpp:678-688): output sums binned by -FtBin
  outW = W;
  outH = H;
  if (p.ft_bin > 0) {
    outW = (int)(W / p.ft_bin + 0.5f) / 2 * 2;
    outH = (int)(H / p.ft_bin + 0.5f) / 2 * 2;
  }
  if (outW < 2 || outH < 2 || outW > W || outH > H) return kEUnsupported;
  return kOk;
}

// ---------------------------------------------------------------------------
Engine::Engine(const mc3_params& p) : prm(p) { device = p.gpu; }

Engine::~Engine() {
  if (device >= 0) cudaSetDevice(device);
  if (copy_stream) cudaStreamSynchronize(copy_stream);
  if (copy_stream2) cudaStreamSynchronize(copy_stream2);
  if (half_done) cudaEventDestroy(half_done);
  if (copy_stream2) cudaStreamDestroy(copy_stream2);
  for (int i = 0; i < 2; ++i) {
    if (slot_loaded[i]) cudaEventDestroy(slot_loaded[i]);
    if (slot_free[i]) cudaEventDestroy(slot_free[i]);
  }
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  if (copy_stream) cudaStreamDestroy(copy_stream);
  if (own_stream) cudaStreamDestroy(own_stream);
}

int Engine::init() {
  MC3_CUDA(cudaSetDevice(device));
  MC3_CUDA(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking));
  MC3_CUDA(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking));
  MC3_CUDA(cudaStreamCreateWithFlags(&copy_stream2, cudaStreamNonBlocking));
  MC3_CUDA(cudaEventCreateWithFlags(&half_done, cudaEventDisableTiming));
  stream = own_stream;
  MC3_CUDA(cudaEventCreate(&ev0));
  MC3_CUDA(cudaEventCreate(&ev1));
  for (int i = 0; i < 2; ++i) {
    MC3_CUDA(cudaEventCreateWithFlags(&slot_loaded[i], cudaEventDisableTiming));
    MC3_CUDA(cudaEventCreateWithFlags(&slot_free[i], cudaEventDisableTiming));
  }
  return kOk;
}

namespace {
// Bytes of one raw frame in MRC mode `mode` (0 when unsupported); mode 101
// packs two 4-bit pixels per byte in rows of (nx+1)/2 bytes
// (LibSrc/Mrcfile/Image/C4BitImage.cpp:15-40).
size_t raw_frame_bytes(int mode, int nx, int ny) {
  switch (mode) {
    case 0: case 5: return (size_t)nx * ny;
    case 1: case 6: return (size_t)nx * ny * 2;
    case 2: return (size_t)nx * ny * 4;
    case 101: return (size_t)((nx + 1) / 2) * ny;
    default: return 0;
  }
}
}  // namespace

// The reference overlaps loading the next movie with processing the
// current one through its loader thread and pinned frame buffers
// (MrcUtil/CLoadCryoEMStack.cpp:130-180, CGpuBuffer.cpp:156-175).  Here the
// raw frames of a later movie are copied on a second stream into one of two
// device slots while the caller's stream works on the current movie.
int Engine::prefetch(const mc3_movie& mv) {
  MC3_CUDA(cudaSetDevice(device));
  if (!mv.frames || mv.nx < 1 || mv.ny < 1 || mv.nz < 1) return kEInval;
  const size_t fbytes = raw_frame_bytes(mv.mode, mv.nx, mv.ny);
  if (!fbytes) return kEUnsupported;
  if (mv.on_device) return kOk;  // nothing to copy
  if (n_pending >= 2) {
    last_error = "two movies are already prefetched; process one first";
    return kEInval;
  }
  const size_t bytes = fbytes * mv.nz;
  const int slot = next_slot;
  if (d_rawslot[slot].cap < bytes) {
    // growing the slot frees it: wait for its last reader first
    MC3_CUDA(cudaEventSynchronize(slot_free[slot]));
    MC3_TRY(d_rawslot[slot].ensure(bytes));
  }
  MC3_CUDA(cudaStreamWaitEvent(copy_stream, slot_free[slot], 0));
  // MC3_H2D_SPLIT=1 copies in two halves on two streams (A/B runs: whether
  // two copy engines move more than one over the host link).
  static const bool split = [] {
    const char* e = getenv("MC3_H2D_SPLIT");
    return e && e[0] == '1';
  }();
  if (split && bytes >= (size_t)1 << 24) {
    const size_t h = bytes / 2 / 256 * 256;
    MC3_CUDA(cudaStreamWaitEvent(copy_stream2, slot_free[slot], 0));
    MC3_CUDA(cudaMemcpyAsync(d_rawslot[slot].p, mv.frames, h, cudaMemcpyHostToDevice, copy_stream));
    MC3_CUDA(cudaMemcpyAsync(static_cast<char*>(d_rawslot[slot].p) + h,
                             static_cast<const char*>(mv.frames) + h, bytes - h,
                             cudaMemcpyHostToDevice, copy_stream2));
    MC3_CUDA(cudaEventRecord(half_done, copy_stream2));
    MC3_CUDA(cudaStreamWaitEvent(copy_stream, half_done, 0));
  } else {
    MC3_CUDA(cudaMemcpyAsync(d_rawslot[slot].p, mv.frames, bytes, cudaMemcpyHostToDevice, copy_stream));
  }
  MC3_CUDA(cudaEventRecord(slot_loaded[slot], copy_stream));
  pending[n_pending++] = Pending{mv.frames, bytes, slot};
  next_slot ^= 1;
  return kOk;
}

void Engine::drop_prefetched() {
  cudaSetDevice(device);
  cudaStreamSynchronize(copy_stream);
  cudaStreamSynchronize(copy_stream2);
  for (int i = 0; i < 2; ++i) cudaEventRecord(slot_free[i], copy_stream);
  n_pending = 0;
}

int Engine::set_stream(cudaStream_t s) {
  stream = s ? s : own_stream;
  return kOk;
}

int Engine::set_gain(const float* gain, int w, int h, bool on_device) {
  MC3_CUDA(cudaSetDevice(device));
  if (!gain) {
    has_gain = false;
    return kOk;
  }
  if (w <= 0 || h <= 0) return kEInval;
  MC3_TRY(d_gain.ensure(sizeof(float) * (size_t)w * h));
  MC3_CUDA(cudaMemcpyAsync(d_gain.p, gain, sizeof(float) * (size_t)w * h,
                           on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, stream));
  MC3_CUDA(cudaStreamSynchronize(stream));
  has_gain = true;
  gain_w = w;
  gain_h = h;
  return kOk;
}

int Engine::set_dark(const float* dark, int w, int h, bool on_device) {
  MC3_CUDA(cudaSetDevice(device));
  if (!dark) {
    has_dark = false;
    return kOk;
  }
  if (w <= 0 || h <= 0) return kEInval;
  MC3_TRY(d_dark.ensure(sizeof(float) * (size_t)w * h));
  MC3_CUDA(cudaMemcpyAsync(d_dark.p, dark, sizeof(float) * (size_t)w * h,
                           on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, stream));
  MC3_CUDA(cudaStreamSynchronize(stream));
  has_dark = true;
  dark_w = w;
  dark_h = h;
  return kOk;
}

int Engine::set_defects(const unsigned char* mask, int w, int h) {
  MC3_CUDA(cudaSetDevice(device));
  if (!mask) {
    has_defects = false;
    return kOk;
  }
  if (w <= 0 || h <= 0) return kEInval;
  MC3_TRY(d_defects.ensure((size_t)w * h));
  MC3_CUDA(cudaMemcpyAsync(d_defects.p, mask, (size_t)w * h, cudaMemcpyHostToDevice, stream));
  MC3_CUDA(cudaStreamSynchronize(stream));
  has_defects = true;
  defects_w = w;
  defects_h = h;
  return kOk;
}

int Engine::plan(int w, int h, int n, mc3_plan_info* info) {
  Geometry g;
  MC3_TRY(geometry(w, h, n, info, &g));
  // Reserve the large per-movie buffers now, as the reference creates its
  // buffer pool before processing (CMain::mCreateBufferPool, CMain.cpp:400-427);
  // process() reuses them (grow-only, same sizes).
  MC3_CUDA(cudaSetDevice(device));
  const size_t ncmp = (size_t)g.cmpX * g.cmpY;
  const size_t nxcf = (size_t)g.xcfCmpX * g.xcfCmpY;
  MC3_TRY(d_frames.ensure(sizeof(float2) * ncmp * g.N));
  MC3_TRY(d_sum.ensure(sizeof(float) * (size_t)g.padX * g.H));
  if (prm.correct_bad) {
    MC3_TRY(d_cc.ensure(sizeof(float) * (size_t)g.padX * g.H));
    MC3_TRY(d_bad.ensure((size_t)g.W * g.H));
  }
  MC3_TRY(d_xcf.ensure(sizeof(float2) * nxcf * g.N));
  if (prm.correct_bad) {
    MC3_TRY(d_badn.ensure(sizeof(int)));
    MC3_TRY(d_badlist.ensure(sizeof(int2) * (size_t)g.W * g.H));
  }
  MC3_TRY(d_sums.ensure(sizeof(float2) * ncmp * g.nSums));
  MC3_TRY(d_Wn.ensure(sizeof(float) * ncmp));
  if (g.patch) {
    MC3_TRY(d_pat.ensure(sizeof(float2) * (size_t)g.patCmpX * g.patCmpY * g.N * g.P));
    MC3_TRY(d_gath.ensure(sizeof(float2) * ncmp * g.N));
  }
  return kOk;
}

int Engine::geometry(int w, int h, int n, mc3_plan_info* info, Geometry* out) const {
  Geometry g;
  if (fmint && n != (fmint_rendered ? fmint_tab.count() : fmint_raw)) return kEInval;
  MC3_TRY(g.compute(w, h, fmint ? fmint_tab.count() : n, prm, fmint && fmint_dose));
  info->n_sums = g.nSums;
  info->n_patches = g.P;
  info->xcf_size[0] = (g.xcfCmpX - 1) * 2;
  info->xcf_size[1] = g.xcfCmpY;
  info->patch_size[0] = g.patch ? (g.patCmpX - 1) * 2 : 0;
  info->patch_size[1] = g.patch ? g.patCmpY : 0;
  info->xcf_bin[0] = g.xcfBin[0];
  info->xcf_bin[1] = g.xcfBin[1];
  info->out_size[0] = g.outW;
  info->out_size[1] = g.outH;
  info->n_frames = g.N;
  size_t cmp = (size_t)g.cmpX * g.cmpY * sizeof(float2);
  size_t xcf = (size_t)g.xcfCmpX * g.xcfCmpY * sizeof(float2);
  size_t bytes = cmp * g.N + xcf * g.N + cmp * (g.nSums + 2) + (size_t)g.W * g.H * 4 * g.N;
  if (g.patch) bytes += (size_t)g.P * g.N * g.patCmpX * g.patCmpY * sizeof(float2) + 2 * cmp * 32;
  info->device_bytes = bytes;
  if (out) *out = g;
  return kOk;
}

// ---------------------------------------------------------------------------
// Batched CIterativeAlign::mAlignStack (Align/CIterativeAlign.cpp:99-156).
int Engine::align_stacks(const float2* spec, long stack_stride, int nstack, int cmpX, int cmpY,
                         int N, const host::FrameGroups& grp, float bf0, float tol,
                         std::vector<host::StackShift>& shifts, std::vector<int>& iters,
                         std::vector<std::vector<float>>& errors, const float* init,
                         int max_iter_init, bool* converged) {
  const int G = grp.count();
  const int imgX = (cmpX - 1) * 2;
  AlignDims d;
  d.cmpX = cmpX;
  d.cmpY = cmpY;
  d.N = N;
  d.stack_stride = stack_stride;
  d.G = G;
  d.seaX = 64 < imgX ? 64 : imgX;   // CAlignStack::Set2 (Align/CAlignStack.cpp:58-61)
  d.seaY = 64 < cmpY ? 64 : cmpY;
  const size_t nel = (size_t)cmpX * cmpY;
  MC3_TRY(d_sh.ensure(sizeof(float2) * (size_t)nstack * N));
  MC3_TRY(d_ex.ensure(sizeof(float2) * (size_t)nstack * N * cmpX));
  MC3_TRY(d_ey.ensure(sizeof(float2) * (size_t)nstack * N * cmpY));
  MC3_TRY(d_S.ensure(sizeof(float2) * (size_t)nstack * nel));
  MC3_TRY(d_T.ensure(sizeof(float2) * (size_t)nstack * G * d.seaY * cmpX));
  MC3_TRY(d_win.ensure(sizeof(float) * (size_t)nstack * G * d.seaY * d.seaX));
  MC3_TRY(d_gsh.ensure(sizeof(float2) * (size_t)nstack * G));
  MC3_TRY(d_act.ensure(sizeof(int) * (size_t)nstack));
  MC3_TRY(d_gstart.ensure(sizeof(int) * (size_t)G));
  MC3_TRY(d_gsize.ensure(sizeof(int) * (size_t)G));
  MC3_CUDA(cudaMemcpyAsync(d_gstart.p, grp.start.data(), sizeof(int) * G, cudaMemcpyHostToDevice, stream));
  MC3_CUDA(cudaMemcpyAsync(d_gsize.p, grp.size.data(), sizeof(int) * G, cudaMemcpyHostToDevice, stream));

  std::vector<host::IterState> st(nstack);
  for (auto& s : st) s.start(N, G, bf0);
  // a warm start (the learned proposal's first iterate) caps the iterations
  const int max_iter = init ? std::min(max_iter_init, prm.iter) : prm.iter;
  if (init) st[0].start_from(init, grp, N, bf0);
  std::vector<int> active(nstack);
  for (int i = 0; i < nstack; ++i) active[i] = i;
  std::vector<float2> hsh((size_t)nstack * N);
  std::vector<float2> hg((size_t)nstack * G);
  for (int it = 0; it < max_iter && !active.empty(); ++it) {
    const int A = (int)active.size();
    d.A = A;
    for (int a = 0; a < A; ++a) {
      const host::StackShift& t = st[active[a]].tmp;
      for (int f = 0; f < N; ++f) {
        // CAlignedSum / CAlignStack apply GetShift(f, -1): the negated shift
        hsh[(size_t)a * N + f].x = t.x(f) * -1.0f;
        hsh[(size_t)a * N + f].y = t.y(f) * -1.0f;
      }
    }
    MC3_CUDA(cudaMemcpyAsync(d_act.p, active.data(), sizeof(int) * A, cudaMemcpyHostToDevice, stream));
    MC3_CUDA(cudaMemcpyAsync(d_sh.p, hsh.data(), sizeof(float2) * (size_t)A * N, cudaMemcpyHostToDevice, stream));
    MC3_TRY(phase_tables(d_sh.as<float2>(), A * N, cmpX, cmpY, d_ex.as<float2>(), d_ey.as<float2>(), false, stream));
    MC3_TRY(aligned_sum(spec, d_act.as<int>(), d_ex.as<float2>(), d_ey.as<float2>(), d_S.as<float2>(), d, stream));
    const float bf = st[active[0]].bfactor;
    MC3_TRY(corr_cols(spec, d_act.as<int>(), d_ex.as<float2>(), d_ey.as<float2>(), d_S.as<float2>(),
                      d_gstart.as<int>(), d_gsize.as<int>(), bf, prm.phase_only, d_T.as<float2>(), d, stream));
    MC3_TRY(corr_rows(d_T.as<float2>(), d_win.as<float>(), d, stream));
    MC3_TRY(peak_search(d_win.as<float>(), d_gsh.as<float2>(), d, stream));
    MC3_CUDA(cudaMemcpyAsync(hg.data(), d_gsh.p, sizeof(float2) * (size_t)A * G, cudaMemcpyDeviceToHost, stream));
    MC3_CUDA(cudaStreamSynchronize(stream));
    std::vector<int> next;
    for (int a = 0; a < A; ++a) {
      host::IterState& s = st[active[a]];
      const bool fin = s.step(reinterpret_cast<const float*>(&hg[(size_t)a * G]), grp, it, max_iter, tol);
      if (!fin) next.push_back(active[a]);
    }
    active.swap(next);
  }
  if (converged) *converged = st[0].max_err < tol && st[0].iterations > 1;
  shifts.resize(nstack);
  iters.resize(nstack);
  errors.resize(nstack);
  for (int s = 0; s < nstack; ++s) {
    shifts[s] = st[s].finish(grp, N);
    iters[s] = st[s].iterations;
    errors[s] = st[s].errors;
  }
  return kOk;
}

// ---------------------------------------------------------------------------
int Engine::global_sums(const float2* spec, int N, const host::StackShift& fs, const Geometry& g) {
  MC3_TRY(d_sh.ensure(sizeof(float2) * (size_t)N));
  MC3_TRY(d_fex.ensure(sizeof(float2) * (size_t)N * g.cmpX));
  MC3_TRY(d_fey.ensure(sizeof(float2) * (size_t)N * g.cmpY));
  std::vector<float2> hsh(N);
  for (int f = 0; f < N; ++f) {
    hsh[f].x = fs.x(f) * -1.0f;
    hsh[f].y = fs.y(f) * -1.0f;
  }
  MC3_CUDA(cudaMemcpyAsync(d_sh.p, hsh.data(), sizeof(float2) * N, cudaMemcpyHostToDevice, stream));
  // in-place GPhaseShift2D::DoIt skips |s| < 0.1 px (Util/GPhaseShift2D.cu:68-79)
  MC3_TRY(phase_tables(d_sh.as<float2>(), N, g.cmpX, g.cmpY, d_fex.as<float2>(), d_fey.as<float2>(), true, stream));
  return kOk;
}

// ---------------------------------------------------------------------------
// Align/CLoadAlign.cpp:52-250: the loaded tables replace the measured ones.
int Engine::set_alignment(const mc3_alignment* aln) {
  if (!aln) {
    aln_loaded = false;
    aln_global.clear();
    aln_patch.clear();
    aln_centers.clear();
    return kOk;
  }
  if (aln->nz < 1 || !aln->global_shifts || aln->n_patches < 0)
    return kEInval;
  if (aln->n_patches > 0 && (!aln->patch_shifts || !aln->patch_centers)) return kEInval;
  aln_nz = aln->nz;
  aln_P = aln->n_patches;
  aln_global.assign(aln->global_shifts, aln->global_shifts + 2 * (size_t)aln->nz);
  if (aln_P > 0) {
    aln_patch.assign(aln->patch_shifts, aln->patch_shifts + 2 * (size_t)aln->nz * aln_P);
    aln_centers.assign(aln->patch_centers, aln->patch_centers + 2 * (size_t)aln_P);
  } else {
    aln_patch.clear();
    aln_centers.clear();
  }
  aln_loaded = true;
  return kOk;
}

int Engine::set_frame_integration(const mc3_frame_integration* fi) {
  if (!fi) {
    fmint = false;
    fmint_tab = host::FmInt();
    return kOk;
  }
  if (fi->n_raw < 1 || fi->n_int < 1 || !fi->start || !fi->size || !fi->acc_dose) return kEInval;
  host::FmInt t;
  t.start.assign(fi->start, fi->start + fi->n_int);
  t.size.assign(fi->size, fi->size + fi->n_int);
  t.acc.assign(fi->acc_dose, fi->acc_dose + fi->n_int);
  t.dose.assign(fi->n_int, 0.0f);
  for (int i = 0; i < fi->n_int; ++i)
    if (t.size[i] < 1 || t.start[i] < 0 || t.start[i] + t.size[i] > fi->n_raw) return kEInval;
  t.centers();
  fmint_tab = t;
  fmint_raw = fi->n_raw;
  fmint_dose = fi->dose_weight != 0;
  fmint_rendered = fi->rendered != 0;
  fmint = true;
  return kOk;
}

host::FmInt Engine::frame_tables(int n_raw) const {
  if (fmint) return fmint_tab;
  host::FmInt t;
  t.plain(n_raw, prm.fm_dose);  // CFmIntParam::mSetup
  return t;
}

// CCorrectFullShift::mCropFrame (Correct/CCorrectFullShift.cpp:336-356) for
// all frames at once, then CZbinStack::DoIt (Align/CZbinStack.cpp:27-71):
// the (shifted) normalised spectra are cropped to the output size, brought
// to real space by an unnormalised C2R and, with a z-bin above 1, summed in
// groups of out_stack[1] frames (the last group takes what is left).
int Engine::write_stack(float2* spec, bool phase, const Geometry& g, const host::FmInt& fi,
                        mc3_result* out) {
  const int N = g.N, oW = g.outW, oH = g.outH, ocX = oW / 2 + 1;
  const size_t ncmp = (size_t)g.cmpX * g.cmpY, ocmp = (size_t)ocX * oH;
  cudaStream_t st = stream;
  float2* s = spec;
  const bool crop = oW != g.W || oH != g.H;
  if (crop) {
    MC3_TRY(d_stk.ensure(sizeof(float2) * ocmp * N));
    s = d_stk.as<float2>();
    MC3_TRY(crop_frames(spec, g.cmpX, g.cmpY, (long)ncmp, phase ? d_fex.as<float2>() : nullptr,
                        phase ? d_fey.as<float2>() : nullptr, s, ocX, oH, (long)ocmp, N, st));
  }
  Batch bi{N, N, (long)ocmp, nullptr, (long)ocmp};
  ColOps inv{};
  inv.dir = 1;
  inv.scale = 1.0f;
  if (phase && !crop) {
    inv.ex = d_fex.as<float2>();
    inv.ey = d_fey.as<float2>();
  }
  MC3_TRY(col_fft(s, s, ocX, ocX, oH, bi, inv, st));
  Batch br{N, N, (long)ocmp, nullptr, (long)ocmp * 2};
  float* real = reinterpret_cast<float*>(s);
  MC3_TRY(row_c2r(s, ocX, real, 2 * ocX, oW, oH, br, st));
  int nf = N;
  if (prm.out_stack[1] > 1) {
    host::FrameGroups G;  // CFmGroupParam::Setup(OutStack[1], FmIntParam)
    G.setup(fi, prm.out_stack[1]);
    nf = G.count();
    MC3_TRY(d_zgrp.ensure(sizeof(int) * 2 * nf));
    std::vector<int> tab(G.start);
    tab.insert(tab.end(), G.size.begin(), G.size.end());
    MC3_CUDA(cudaMemcpyAsync(d_zgrp.p, tab.data(), sizeof(int) * 2 * nf, cudaMemcpyHostToDevice, st));
    MC3_TRY(zbin_frames(real, (long)ocmp * 2, 2 * ocX, oW, oH, d_zgrp.as<int>(), nf, st));
  }
  // every row of every frame lies 2*ocX floats after the previous one
  MC3_CUDA(cudaMemcpy2DAsync(out->stack, sizeof(float) * oW, real, sizeof(float) * 2 * ocX,
                             sizeof(float) * oW, (size_t)nf * oH,
                             out->stack_on_device ? cudaMemcpyDeviceToDevice
                                                  : cudaMemcpyDeviceToHost,
                             st));
  out->stack_frames = nf;
  return kOk;
}

// ---------------------------------------------------------------------------
Tuning Engine::tuning_for(int w, int h, int n) const {
  // same frame size and patch grid; the nearest frame count
  const TuningEntry* best = nullptr;
  for (const TuningEntry& e : tuning_table)
    if (e.nx == w && e.ny == h && e.px == prm.patch[0] && e.py == prm.patch[1] &&
        (!best || std::abs(e.nz - n) < std::abs(best->nz - n)))
      best = &e;
  return best ? best->best : default_tuning();
}

int Engine::autotune(int w, int h, int n, TuningEntry* out) {
  MC3_CUDA(cudaSetDevice(device));
  mc3_plan_info info;
  MC3_TRY(plan(w, h, n, &info));
  DevBuf frames, sums;
  MC3_TRY(frames.ensure(sizeof(float) * (size_t)w * h * n));
  MC3_TRY(sums.ensure(sizeof(float) * (size_t)info.out_size[0] * info.out_size[1] * info.n_sums));
  MC3_TRY(synthetic_counts(frames.as<float>(), (long)w * h * n, stream));
  mc3_movie mv{frames.p, 2, w, h, n, 1};
  mc3_result r;
  std::memset(&r, 0, sizeof(r));
  r.sums = sums.as<float>();
  r.sums_on_device = 1;
  const bool had_gain = has_gain;
  has_gain = false;  // the tuner's frames need no gain
  TuningEntry e;
  e.nx = w;
  e.ny = h;
  e.nz = n;
  e.px = prm.patch[0];
  e.py = prm.patch[1];
  int st = kOk;
  for (const Tuning& t : tuning_candidates()) {
    TuningScope scope(t);
    double best = 1e30;
    for (int rep = 0; rep < 3 && st == kOk; ++rep) {  // first run: warm-up
      st = process_with(mv, &r, t);
      if (rep > 0 && r.time_ms < best) best = r.time_ms;
    }
    if (st != kOk) break;
    e.cand.push_back(t);
    e.cand_ms.push_back(best);
    if (e.cand.size() == 1 || best < e.best_ms) {
      e.best = t;
      e.best_ms = best;
    }
  }
  has_gain = had_gain;
  if (st != kOk) return st;
  for (auto it = tuning_table.begin(); it != tuning_table.end();)
    it = (it->nx == w && it->ny == h && it->nz == n && it->px == e.px && it->py == e.py)
             ? tuning_table.erase(it)
             : it + 1;
  tuning_table.push_back(e);
  if (out) *out = e;
  return kOk;
}

int Engine::process(const mc3_movie& mv, mc3_result* out) {
  Geometry g0;
  mc3_plan_info info;
  const Tuning t = geometry(mv.nx, mv.ny, mv.nz, &info, &g0) == kOk
                       ? tuning_for(mv.nx, mv.ny, mv.nz)
                       : default_tuning();
  return process_with(mv, out, t);
}

int Engine::process_with(const mc3_movie& mv, mc3_result* out, const Tuning& tune) {
  TuningScope scope(tune);
  MC3_CUDA(cudaSetDevice(device));
  if (prm.align == 0) return kEUnsupported;
  if (!mv.frames) return kEInval;
  const size_t fbytes = raw_frame_bytes(mv.mode, mv.nx, mv.ny);
  if (!fbytes) return kEUnsupported;
  Geometry g;
  const int expect_nz = fmint ? (fmint_rendered ? fmint_tab.count() : fmint_raw) : mv.nz;
  if (mv.nz != expect_nz) {
    last_error = "movie frame count differs from the frame-integration table";
    return kEInval;
  }
  const host::FmInt fi = frame_tables(mv.nz);
  MC3_TRY(g.compute(mv.nx, mv.ny, fi.count(), prm, fmint && fmint_dose));
  const int Nraw = mv.nz;
  bool render = false;  // some rendered frame sums several raw frames
  long first_raw = 0;   // one raw frame per frame from here on (-Throw)
  if (fmint && !fmint_rendered) {
    for (int i = 0; i < fi.count(); ++i) render = render || fi.size[i] != 1;
    first_raw = fi.start[0];
    for (int i = 0; !render && i < fi.count(); ++i) render = fi.start[i] != first_raw + i;
    if (render) first_raw = 0;
  }
  if (render && !(mv.mode == 0 || mv.mode == 5 || mv.mode == 101)) {
    // the reference renders integrated frames as 8-bit (CLoadCryoEMStack::OpenFile)
    last_error = "frame integration needs an 8-bit or 4-bit movie";
    return kEUnsupported;
  }
  if (has_gain && (gain_w != g.W || gain_h != g.H)) return kEInval;  // CProcessThread::mCheckGain
  if (has_dark && (dark_w != g.W || dark_h != g.H)) return kEInval;
  if (has_defects && (defects_w != g.W || defects_h != g.H)) return kEInval;
  const float* dark = has_dark ? d_dark.as<float>() : nullptr;
  const bool loaded = aln_loaded;
  if (loaded && (aln_nz != g.N || aln_P != g.P)) {
    last_error = "loaded alignment does not match the movie (frames or patches)";
    return kEInval;
  }
  const bool want_stack = prm.out_stack[0] != 0 && out && out->stack;
  const int W = g.W, H = g.H, N = g.N;
  const size_t npx = (size_t)W * H;
  const size_t ncmp = (size_t)g.cmpX * g.cmpY;
  const size_t nxcf = (size_t)g.xcfCmpX * g.xcfCmpY;
  cudaStream_t st = stream;

  MC3_CUDA(cudaEventRecord(ev0, st));
  // ---- 1. raw frames on the device ----
  const void* raw = mv.frames;
  int used_slot = -1;
  if (!mv.on_device && n_pending > 0) {
    // the oldest prefetched movie must be this one
    const Pending pf = pending[0];
    if (pf.host != mv.frames || pf.bytes != fbytes * Nraw) {
      last_error = "movie differs from the oldest prefetched movie";
      return kEInval;
    }
    pending[0] = pending[1];
    --n_pending;
    MC3_CUDA(cudaStreamWaitEvent(st, slot_loaded[pf.slot], 0));
    raw = d_rawslot[pf.slot].p;
    used_slot = pf.slot;
  } else if (!mv.on_device) {
    MC3_TRY(d_raw.ensure(fbytes * Nraw));
    MC3_CUDA(cudaMemcpyAsync(d_raw.p, mv.frames, fbytes * Nraw, cudaMemcpyHostToDevice, st));
    raw = d_raw.p;
  }
  // ---- 2. gain + frame sum (MrcUtil/CApplyRefs.cpp:36-212, CSumFFTStack) ----
  MC3_TRY(d_frames.ensure(sizeof(float2) * ncmp * N));
  MC3_TRY(d_sum.ensure(sizeof(float) * (size_t)g.padX * H));
  float* frames = d_frames.as<float>();
  const long fr_stride_f = (long)g.padX * H;
  // raw frame stride in elements of the mode's type (bytes for packed 4-bit)
  const long raw_stride = mv.mode == 101 ? (long)fbytes : (long)npx;
  if (render) {
    // CLoadCryoEMStack::mLoadInt / mLoadInt4Bits (MrcUtil/CLoadCryoEMStack.cpp:184-262)
    // fused with the gain pass
    MC3_TRY(d_istart.ensure(sizeof(int) * N));
    MC3_TRY(d_isize.ensure(sizeof(int) * N));
    MC3_CUDA(cudaMemcpyAsync(d_istart.p, fi.start.data(), sizeof(int) * N, cudaMemcpyHostToDevice, st));
    MC3_CUDA(cudaMemcpyAsync(d_isize.p, fi.size.data(), sizeof(int) * N, cudaMemcpyHostToDevice, st));
    MC3_TRY(gain_and_sum_int(raw, mv.mode, raw_stride, d_istart.as<int>(), d_isize.as<int>(),
                             dark, has_gain ? d_gain.as<float>() : nullptr, frames, fr_stride_f,
                             prm.correct_bad ? d_sum.as<float>() : nullptr, W, H, N, st));
  } else {
    if (first_raw) raw = static_cast<const char*>(raw) + (size_t)first_raw * fbytes;
    MC3_TRY(gain_and_sum(raw, mv.mode, raw_stride, dark, has_gain ? d_gain.as<float>() : nullptr, frames,
                         fr_stride_f, prm.correct_bad ? d_sum.as<float>() : nullptr, W, H, N, st));
  }
  if (used_slot >= 0) MC3_CUDA(cudaEventRecord(slot_free[used_slot], st));  // raw is read only above
  // ---- 3. hot pixels and defects (BadPixel/CDetectMain.cpp, CCorrectMain.cpp) ----
  if (prm.correct_bad) {
    MC3_TRY(d_cc.ensure(sizeof(float) * (size_t)g.padX * H));
    MC3_TRY(d_bad.ensure(npx));
    MC3_TRY(d_part.ensure(sizeof(float) * 1024));
    MC3_TRY(d_mom.ensure(sizeof(float) * 16));
    float tpl[36];
    host::defect_template(6, tpl);
    const bool want_hot = out && out->hot_map;
    if (want_hot) MC3_TRY(d_hot.ensure(npx));
    MC3_TRY(detect_bad_pixels(d_sum.as<float>(), W, H, d_cc.as<float>(), d_part.as<float>(),
                              d_mom.as<float>(), d_bad.as<uint8_t>(), tpl, 6, st,
                              want_hot ? d_hot.as<uint8_t>() : nullptr));
    if (want_hot)
      MC3_CUDA(cudaMemcpyAsync(out->hot_map, d_hot.p, npx, cudaMemcpyDeviceToHost, st));
    // CDetectMain::mLoadDefectFile / mLoadDefectMap (BadPixel/CDetectMain.cpp:146-260)
    if (has_defects) MC3_TRY(or_mask(d_bad.as<uint8_t>(), d_defects.as<uint8_t>(), npx, st));
    MC3_TRY(d_badn.ensure(sizeof(int)));
    MC3_TRY(d_badlist.ensure(sizeof(int2) * npx));
    MC3_TRY(correct_bad_pixels(frames, fr_stride_f, N, d_bad.as<uint8_t>(), W, H, d_badn.as<int>(),
                               d_badlist.as<int2>(), st));
  }
  // ---- 4. forward FFT, normalised, + xcf crop (CTransformStack, CGenXcfStack) ----
  MC3_TRY(d_xcf.ensure(sizeof(float2) * nxcf * N));
  float2* spec = d_frames.as<float2>();
  {
    Batch b{N, N, fr_stride_f, nullptr, (long)ncmp};
    MC3_TRY(row_r2c(frames, g.padX, spec, g.cmpX, W, H, b, 1.0f, st));
    Batch bc{N, N, (long)ncmp, nullptr, (long)ncmp};
    ColOps ops{};
    ops.dir = -1;
    ops.scale = (float)(1.0 / W / H);
    if (!loaded) {  // a loaded alignment needs no alignment stack
      ops.crop = d_xcf.as<float2>();
      ops.crop_x = g.xcfCmpX;
      ops.crop_y = g.xcfCmpY;
    }
    MC3_TRY(col_fft(spec, spec, g.cmpX, g.cmpX, H, bc, ops, st));
  }
  // ---- 5. full-frame alignment (Align/CFullAlign.cpp:127-164) ----
  const float bin = fmaxf(g.xcfBin[0], g.xcfBin[1]);
  const float tol = prm.tol / bin;
  host::FrameGroups G0, G1;
  G0.setup(fi, prm.group[0]);
  std::vector<host::StackShift> xs;
  std::vector<int> it0;
  std::vector<std::vector<float>> err0;
  if (loaded) {  // CFullAlign::Align with CLoadAlign loaded (Align/CFullAlign.cpp:85-89)
    xs.resize(1);
    xs[0].setup(N);
    it0.assign(1, 0);
    err0.assign(1, std::vector<float>());
  } else if ((int)first_iterate.size() == 2 * N) {
    // Warm start from a first iterate (full-frame pixels -> alignment pixels),
    // at most first_iterate_max iterations.  The plain aligner judges it: its
    // first correlation measures the first iterate's error, and the warm
    // result is kept only when that error is below 1 px of the alignment
    // image and the iterations converged; otherwise the plain aligner runs
    // from zero (the fallback).
    std::vector<float> init(2 * N);
    for (int f = 0; f < N; ++f) {
      init[2 * f] = first_iterate[2 * f] / g.xcfBin[0];
      init[2 * f + 1] = first_iterate[2 * f + 1] / g.xcfBin[1];
    }
    first_iterate.clear();
    bool conv = false;
    MC3_TRY(align_stacks(d_xcf.as<float2>(), (long)nxcf * N, 1, g.xcfCmpX, g.xcfCmpY, N, G0,
                         prm.bft[0], tol, xs, it0, err0, init.data(), first_iterate_max, &conv));
    first_iterate_used = 1;
    const bool judged_ok = !err0[0].empty() && err0[0][0] < 1.0f;
    if (!conv || !judged_ok) {
      const int warm_iters = it0[0];
      MC3_TRY(align_stacks(d_xcf.as<float2>(), (long)nxcf * N, 1, g.xcfCmpX, g.xcfCmpY, N, G0,
                           prm.bft[0], tol, xs, it0, err0));
      it0[0] += warm_iters;  // every iteration run counts
      first_iterate_used = 2;
    }
  } else {
    first_iterate_used = 0;
    first_iterate.clear();
    MC3_TRY(align_stacks(d_xcf.as<float2>(), (long)nxcf * N, 1, g.xcfCmpX, g.xcfCmpY, N, G0,
                         prm.bft[0], tol, xs, it0, err0));
  }
  host::StackShift xsh = xs[0];  // xcf pixels

  std::vector<float> patShift, patCent;
  std::vector<unsigned char> patBad;
  std::vector<int> patIters;
  std::vector<std::vector<float>> patErr;
  if (g.patch && loaded) {
    // CPatchAlign::mCalcPatchShifts with CLoadAlign loaded
    // (Align/CPatchAlign.cpp:67-96): tables as read, no bad flags
    patShift = aln_patch;
    patCent = aln_centers;
    patBad.assign((size_t)N * g.P, 0);
    patIters.assign(g.P, 0);
    patErr.assign(g.P, std::vector<float>());
  } else if (g.patch) {
    const int xcfX = (g.xcfCmpX - 1) * 2, xcfY = g.xcfCmpY;
    // ---- 6a. features on the aligned xcf sum (Align/CDetectFeatures.cpp:58-181) ----
    {
      MC3_TRY(d_sh.ensure(sizeof(float2) * N));
      MC3_TRY(d_ex.ensure(sizeof(float2) * (size_t)N * g.xcfCmpX));
      MC3_TRY(d_ey.ensure(sizeof(float2) * (size_t)N * g.xcfCmpY));
      MC3_TRY(d_S.ensure(sizeof(float2) * nxcf));
      MC3_TRY(d_act.ensure(sizeof(int)));
      std::vector<float2> hsh(N);
      for (int f = 0; f < N; ++f) {
        hsh[f].x = xsh.x(f) * -1.0f;
        hsh[f].y = xsh.y(f) * -1.0f;
      }
      int zero = 0;
      MC3_CUDA(cudaMemcpyAsync(d_act.p, &zero, sizeof(int), cudaMemcpyHostToDevice, st));
      MC3_CUDA(cudaMemcpyAsync(d_sh.p, hsh.data(), sizeof(float2) * N, cudaMemcpyHostToDevice, st));
      MC3_TRY(phase_tables(d_sh.as<float2>(), N, g.xcfCmpX, g.xcfCmpY, d_ex.as<float2>(), d_ey.as<float2>(), false, st));
      AlignDims d{};
      d.cmpX = g.xcfCmpX;
      d.cmpY = g.xcfCmpY;
      d.N = N;
      d.stack_stride = (long)nxcf * N;
      d.A = 1;
      MC3_TRY(aligned_sum(d_xcf.as<float2>(), d_act.as<int>(), d_ex.as<float2>(), d_ey.as<float2>(), d_S.as<float2>(), d, st));
      const int bx = 128, by = 128, bcx = bx / 2 + 1;
      MC3_TRY(d_bsum.ensure(sizeof(float2) * bcx * by));
      MC3_TRY(d_btmp.ensure(sizeof(float2) * bcx * by));
      MC3_TRY(d_bmap.ensure(sizeof(float) * bx * by));
      MC3_TRY(d_scal.ensure(sizeof(float) * 8));
      MC3_TRY(d_part.ensure(sizeof(float) * 1024));
      MC3_TRY(fourier_crop(d_S.as<float2>(), g.xcfCmpX, g.xcfCmpY, d_bsum.as<float2>(), bcx, by, st));
      Batch b1{1, 1, 0, nullptr, 0};
      ColOps ops{};
      ops.dir = 1;
      ops.scale = 1.0f;
      MC3_TRY(col_fft(d_bsum.as<float2>(), d_bsum.as<float2>(), bcx, bcx, by, b1, ops, st));
      MC3_TRY(row_c2r(d_bsum.as<float2>(), bcx, d_bsum.as<float>(), 2 * bcx, bx, by, b1, st));
      MC3_TRY(feature_map(d_bsum.as<float>(), bx, by, d_btmp.as<float>(), d_part.as<float>(), d_scal.as<float>(), d_bmap.as<float>(), st));
      std::vector<float> map((size_t)bx * by);
      float scal[3];
      MC3_CUDA(cudaMemcpyAsync(map.data(), d_bmap.p, sizeof(float) * bx * by, cudaMemcpyDeviceToHost, st));
      MC3_CUDA(cudaMemcpyAsync(scal, d_scal.p, sizeof(float) * 3, cudaMemcpyDeviceToHost, st));
      MC3_CUDA(cudaStreamSynchronize(st));
      std::vector<int> starts;
      host::patch_starts(map.data(), bx, by, scal[1], scal[2], g.Px, g.Py, xcfX, xcfY,
                         g.patSizeX, g.patSizeY, starts);
      if (patch_centers_given.size() == 2 * (size_t)g.P)  // the caller's centres
        host::patch_starts_from_centers(patch_centers_given.data(), g.P, g.xcfBin[0],
                                        g.xcfBin[1], xcfX, xcfY, g.patSizeX, g.patSizeY, starts);
      // ---- 6b. xcf frames to real space (Correct/CGenRealStack.cpp) ----
      MC3_TRY(phase_tables(d_sh.as<float2>(), N, g.xcfCmpX, g.xcfCmpY, d_ex.as<float2>(), d_ey.as<float2>(), true, st));
      Batch bn{N, N, (long)nxcf, nullptr, (long)nxcf};
      ColOps inv{};
      inv.dir = 1;
      inv.scale = 1.0f;
      inv.ex = d_ex.as<float2>();
      inv.ey = d_ey.as<float2>();
      MC3_TRY(col_fft(d_xcf.as<float2>(), d_xcf.as<float2>(), g.xcfCmpX, g.xcfCmpX, xcfY, bn, inv, st));
      Batch br{N, N, (long)nxcf, nullptr, (long)nxcf * 2};
      MC3_TRY(row_c2r(d_xcf.as<float2>(), g.xcfCmpX, d_xcf.as<float>(), 2 * g.xcfCmpX, xcfX, xcfY, br, st));
      // ---- 6c. patch extraction + unnormalised R2C (CExtractPatch, CTransformStack) ----
      const int P = g.P;
      const size_t npat = (size_t)g.patCmpX * g.patCmpY;
      MC3_TRY(d_pat.ensure(sizeof(float2) * npat * N * P));
      MC3_TRY(d_patoff.ensure(sizeof(long) * P));
      std::vector<long> off(P);
      for (int p = 0; p < P; ++p) off[p] = (long)starts[2 * p + 1] * (2 * g.xcfCmpX) + starts[2 * p];
      MC3_CUDA(cudaMemcpyAsync(d_patoff.p, off.data(), sizeof(long) * P, cudaMemcpyHostToDevice, st));
      const int pw = (g.patCmpX - 1) * 2, ph = g.patCmpY;
      Batch bp{P * N, N, (long)nxcf * 2, d_patoff.as<long>(), (long)npat};
      if (prm.dft_gemm && dft_rows_supported(pw))  // split-BF16 DFT GEMM on the tensor cores
        MC3_TRY(dft_rows_r2c(d_xcf.as<float>(), 2 * g.xcfCmpX, d_pat.as<float2>(), g.patCmpX, pw,
                             ph, bp, 1.0f, st));
      else
        MC3_TRY(row_r2c(d_xcf.as<float>(), 2 * g.xcfCmpX, d_pat.as<float2>(), g.patCmpX, pw, ph,
                        bp, 1.0f, st));
      Batch bpc{P * N, P * N, (long)npat, nullptr, (long)npat};
      ColOps fwd{};
      fwd.dir = -1;
      fwd.scale = 1.0f;
      MC3_TRY(col_fft(d_pat.as<float2>(), d_pat.as<float2>(), g.patCmpX, g.patCmpX, ph, bpc, fwd, st));
      // ---- 6d. all patch stacks aligned together (Align/CMeasurePatches.cpp:22-84) ----
      G1.setup(fi, prm.group[1]);
      std::vector<host::StackShift> ps;
      MC3_TRY(align_stacks(d_pat.as<float2>(), (long)npat * N, P, g.patCmpX, g.patCmpY, N, G1,
                           prm.bft[1], tol, ps, patIters, patErr));
      if (prm.dft_gemm) {  // the stream was synchronised by the alignment
        int flag = 0;
        MC3_TRY(dft_gemm_error(true, &flag));
        if (flag) {
          last_error = "a bounded wait of the DFT-GEMM kernel gave up";
          return kETimeout;
        }
      }
      patShift.assign((size_t)N * P * 2, 0.0f);
      patCent.assign((size_t)P * 2, 0.0f);
      for (int p = 0; p < P; ++p) {
        const int cx = starts[2 * p] + g.patSizeX / 2, cy = starts[2 * p + 1] + g.patSizeY / 2;
        patCent[2 * p] = cx * g.xcfBin[0];
        patCent[2 * p + 1] = cy * g.xcfBin[1];
        host::StackShift s = ps[p];
        s.multiply(g.xcfBin[0], g.xcfBin[1]);
        for (int f = 0; f < N; ++f) {
          patShift[((size_t)f * P + p) * 2] = s.x(f);
          patShift[((size_t)f * P + p) * 2 + 1] = s.y(f);
        }
      }
      host::patch_make_relative(patShift, N, P);
      patBad.assign((size_t)N * P, 0);
      host::patch_detect_bads(patShift.data(), patCent.data(), N, P, W, H, patBad.data());
    }
  }
  // full-frame pixels + 0.01 px truncation (CFullAlign.cpp:96, 163)
  host::StackShift fs = xsh;
  fs.multiply(g.xcfBin[0], g.xcfBin[1]);
  fs.truncate_decimal();
  if (loaded)
    for (int f = 0; f < N; ++f) {
      fs.x(f) = aln_global[2 * f];
      fs.y(f) = aln_global[2 * f + 1];
    }
  if (g.patch) {
    // CPatchAlign::mCorrectFullShift (Align/CPatchAlign.cpp:47-65)
    int ref = N / 2;
    if (prm.fm_ref >= 0) {
      ref = prm.fm_ref - 1;
      if (ref < 0) ref = 0;
      else if (ref >= N) ref = N - 1;
    }
    fs.make_relative(ref);
  }

  // ---- 7. correction + sums ----
  MC3_TRY(d_sums.ensure(sizeof(float2) * ncmp * g.nSums));
  MC3_TRY(d_acc.ensure(sizeof(float) * N));
  MC3_TRY(d_Wn.ensure(sizeof(float) * ncmp));
  std::vector<float> acc(N);
  for (int i = 0; i < N; ++i) acc[i] = fi.acc[i];  // CFmIntParam::m_pfAccFmDose
  MC3_CUDA(cudaMemcpyAsync(d_acc.p, acc.data(), sizeof(float) * N, cudaMemcpyHostToDevice, st));
  DoseParams dp{};
  dp.enabled = g.dw ? 1 : 0;
  dp.dws = g.dws ? 1 : 0;
  dp.split = prm.split_sum ? 1 : 0;
  dp.pix_size = prm.pix_size;
  dp.kv_factor = host::kv_factor(prm.kv);
  dp.sum_range[0] = prm.sum_range[0];
  dp.sum_range[1] = prm.sum_range[1];
  if (g.dw) {
    // The normalisation depends only on the geometry and the dose options,
    // so it is rebuilt only when they change between movies.
    double acc_key = 0.0;  // the dose table enters through the accumulated doses
    for (int i = 0; i < N; ++i) acc_key += (double)acc[i] * (i + 1);
    const double key[6] = {(double)g.cmpX, (double)g.cmpY, (double)N, acc_key, dp.pix_size,
                           dp.kv_factor};
    if (!wn_valid || std::memcmp(key, wn_key, sizeof(key)) != 0 || d_Wn.cap < sizeof(float) * ncmp) {
      MC3_TRY(dose_norm(d_acc.as<float>(), N, g.cmpX, g.cmpY, dp.pix_size, dp.kv_factor,
                        d_Wn.as<float>(), st));
      std::memcpy(wn_key, key, sizeof(key));
      wn_valid = true;
    }
  }
  MC3_TRY(global_sums(spec, N, fs, g));
  if (g.patch && prm.corr_interp) {
    // -CorrInterp: CGenRealStack::mCorrectBilinear on the frames of
    // CPatchAlign::mCorrectFullShift (Align/CPatchAlign.cpp:52-61), before the
    // in-frame motion weighting
    MC3_TRY(corr_interp(spec, (long)ncmp, g.cmpX, g.cmpY, N, st));
  }
  if (prm.in_fm_motion) {
    // -InFmMotion: CCorrectFullShift::mMotionDecon (Correct/CCorrectFullShift.cpp:309-318)
    // in global mode, CGenRealStack::mMotionDecon (Correct/CGenRealStack.cpp:156-166)
    // on the globally corrected frames in patch mode; motion of frame f =
    // s(f+1) - s(f), of the last frame s(N-1) - s(N-2) (CInFrameMotion::GetFullMotion)
    std::vector<float4> mo(N);
    for (int f = 0; f < N; ++f) {
      const int f1 = f == N - 1 ? f - 1 : f, f2 = f == N - 1 ? f : f + 1;
      const float mx = fs.x(f2) - fs.x(f1), my = fs.y(f2) - fs.y(f1);
      const double d = sqrtf(mx * mx + my * my);  // GMotionWeight::DirWeight skip test
      mo[f] = make_float4(mx, my, d < 0.1 ? 0.0f : 1.0f, 0.0f);
    }
    MC3_TRY(d_motion.ensure(sizeof(float4) * N));
    MC3_CUDA(cudaMemcpyAsync(d_motion.p, mo.data(), sizeof(float4) * N, cudaMemcpyHostToDevice, st));
    MC3_TRY(motion_decon(spec, (long)ncmp, g.cmpX, g.cmpY, N, d_motion.as<float4>(), st));
  }
  if (!g.patch) {
    MC3_TRY(frame_sums(spec, (long)ncmp, N, g.cmpX, g.cmpY, d_fex.as<float2>(), d_fey.as<float2>(),
                       d_acc.as<float>(), d_Wn.as<float>(), dp, d_sums.as<float2>(), g.nSums, st));
    if (want_stack) MC3_TRY(write_stack(spec, true, g, fi, out));  // spectra are not needed after
  } else {
    // Correct/GCorrectPatchShift.cu:97-285: per frame C2R -> gather -> R2C
    const int P = g.P;
    MC3_TRY(d_pcent.ensure(sizeof(float) * 2 * P));
    MC3_TRY(d_pshift.ensure(sizeof(float) * 2 * (size_t)P * N));
    MC3_TRY(d_pbad.ensure((size_t)P * N));
    MC3_CUDA(cudaMemcpyAsync(d_pcent.p, patCent.data(), sizeof(float) * 2 * P, cudaMemcpyHostToDevice, st));
    MC3_CUDA(cudaMemcpyAsync(d_pshift.p, patShift.data(), sizeof(float) * 2 * (size_t)P * N, cudaMemcpyHostToDevice, st));
    MC3_CUDA(cudaMemcpyAsync(d_pbad.p, patBad.data(), (size_t)P * N, cudaMemcpyHostToDevice, st));
    // All frames at once: the spectra are shifted and inverted in place, the
    // gather writes a second frame stack, and the forward transform of the
    // gathered frames lands back in the spectrum buffer.  Patch weights are
    // then evaluated once per pixel for the whole movie.
    MC3_TRY(d_gath.ensure(sizeof(float2) * ncmp * N));
    {
      Batch bi{N, N, (long)ncmp, nullptr, (long)ncmp};
      ColOps inv{};
      inv.dir = 1;
      inv.scale = 1.0f;
      inv.ex = d_fex.as<float2>();
      inv.ey = d_fey.as<float2>();
      MC3_TRY(col_fft(spec, spec, g.cmpX, g.cmpX, H, bi, inv, st));
      Batch br{N, N, (long)ncmp, nullptr, (long)ncmp * 2};
      MC3_TRY(row_c2r(spec, g.cmpX, frames, g.padX, W, H, br, st));
      if (P <= 64) {
        MC3_TRY(d_pmask.ensure(sizeof(unsigned long long) * N + N));
        unsigned long long* masks = d_pmask.as<unsigned long long>();
        uint8_t* clean = reinterpret_cast<uint8_t*>(masks + N);
        MC3_TRY(patch_masks(d_pbad.as<uint8_t>(), d_pshift.as<float2>(), P, N, masks, clean, st));
        MC3_TRY(local_gather(frames, (long)ncmp * 2, d_gath.as<float>(), (long)ncmp * 2, N, W, H,
                             d_pcent.as<float>(), d_pshift.as<float2>(), masks, nullptr, clean,
                             P, st));
      } else {  // bad-patch flags read directly (no 64-bit masks)
        MC3_TRY(local_gather(frames, (long)ncmp * 2, d_gath.as<float>(), (long)ncmp * 2, N, W, H,
                             d_pcent.as<float>(), d_pshift.as<float2>(), nullptr,
                             d_pbad.as<uint8_t>(), nullptr, P, st));
      }
      Batch bf{N, N, (long)ncmp * 2, nullptr, (long)ncmp};
      MC3_TRY(row_r2c(d_gath.as<float>(), g.padX, spec, g.cmpX, W, H, bf, 1.0f, st));
      ColOps fwd{};
      fwd.dir = -1;
      fwd.scale = (float)(1.0 / W / H);
      MC3_TRY(col_fft(spec, spec, g.cmpX, g.cmpX, H, bi, fwd, st));
      // CCorrectFullShift::mGenSums calls its own (non-virtual) mMotionDecon
      // on the locally corrected frames too (Correct/CCorrectInc.h:115,
      // Correct/CCorrectFullShift.cpp:271-274), so in patch mode the weight is
      // applied a second time
      if (prm.in_fm_motion)
        MC3_TRY(motion_decon(spec, (long)ncmp, g.cmpX, g.cmpY, N, d_motion.as<float4>(), st));
    }
    MC3_TRY(frame_sums(spec, (long)ncmp, N, g.cmpX, g.cmpY, nullptr, nullptr, d_acc.as<float>(),
                       d_Wn.as<float>(), dp, d_sums.as<float2>(), g.nSums, st));
    if (want_stack) MC3_TRY(write_stack(spec, false, g, fi, out));
  }
  if (out && !want_stack) out->stack_frames = 0;
  // ---- 7b. CCorrectFullShift::mCorrectMag (Correct/CCorrectFullShift.cpp:94-127):
  //      every sum to real space (unnormalised), stretched, forward again ----
  float mm[3];
  if (host::mag_matrix(prm.mag, mm)) {
    const int n = g.nSums;
    MC3_TRY(d_mag.ensure(sizeof(float2) * ncmp * n));
    float2* S = d_sums.as<float2>();
    Batch b{n, n, (long)ncmp, nullptr, (long)ncmp};
    ColOps inv{};
    inv.dir = 1;
    inv.scale = 1.0f;
    MC3_TRY(col_fft(S, S, g.cmpX, g.cmpX, H, b, inv, st));
    Batch br{n, n, (long)ncmp, nullptr, (long)ncmp * 2};
    MC3_TRY(row_c2r(S, g.cmpX, reinterpret_cast<float*>(S), g.padX, W, H, br, st));
    MC3_TRY(stretch_images(reinterpret_cast<float*>(S), d_mag.as<float>(), g.padX, (long)ncmp * 2,
                           W, H, n, mm, st));
    Batch bf{n, n, (long)ncmp * 2, nullptr, (long)ncmp};
    MC3_TRY(row_r2c(d_mag.as<float>(), g.padX, S, g.cmpX, W, H, bf, 1.0f, st));
    ColOps fwd{};
    fwd.dir = -1;
    fwd.scale = (float)(1.0 / W / H);
    MC3_TRY(col_fft(S, S, g.cmpX, g.cmpX, H, b, fwd, st));
  }
  // ---- 8. sums to real space (CCorrectFullShift::mUnpadSums,
  //      Correct/CCorrectFullShift.cpp:146-185): Fourier crop to the -FtBin
  //      output size, C2R, positivity, unpad ----
  const float* sum0 = nullptr;  // first output sum, device
  {
    const int oW = g.outW, oH = g.outH;
    const int ocX = oW / 2 + 1;
    const size_t ocmp = (size_t)ocX * oH;
    float2* osum = d_sums.as<float2>();
    if (oW != W || oH != H) {
      MC3_TRY(d_bsums.ensure(sizeof(float2) * ocmp * g.nSums));
      osum = d_bsums.as<float2>();
      for (int sidx = 0; sidx < g.nSums; ++sidx)
        MC3_TRY(fourier_crop(d_sums.as<float2>() + ncmp * sidx, g.cmpX, g.cmpY, osum + ocmp * sidx,
                             ocX, oH, st));
    }
    Batch bs{g.nSums, g.nSums, (long)ocmp, nullptr, (long)ocmp};
    ColOps inv{};
    inv.dir = 1;
    inv.scale = 1.0f;
    MC3_TRY(col_fft(osum, osum, ocX, ocX, oH, bs, inv, st));
    Batch br{g.nSums, g.nSums, (long)ocmp, nullptr, (long)ocmp * 2};
    MC3_TRY(row_c2r(osum, ocX, reinterpret_cast<float*>(osum), 2 * ocX, oW, oH, br, st));
    const size_t opx = (size_t)oW * oH;
    float* dst = nullptr;
    if (out && out->sums && out->sums_on_device) {
      dst = out->sums;
    } else {
      MC3_TRY(d_out.ensure(sizeof(float) * opx * g.nSums));
      dst = d_out.as<float>();
    }
    MC3_TRY(unpad_positive(reinterpret_cast<float*>(osum), 2 * ocX, dst, oW, oH, g.nSums,
                           (long)ocmp * 2, st));
    sum0 = dst;
    if (out && out->sums && !out->sums_on_device)
      MC3_CUDA(cudaMemcpyAsync(out->sums, dst, sizeof(float) * opx * g.nSums, cudaMemcpyDeviceToHost, st));
  }
  MC3_CUDA(cudaEventRecord(ev1, st));
  MC3_CUDA(cudaStreamSynchronize(st));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ev0, ev1);
  // ---- 8b. CTF of the first sum, outside the timed region
  //      (CCorrectFullShift::mEstimateCtf, Correct/CCorrectFullShift.cpp:129-144,179,
  //      gated as CFindCtfMain::bEstimate, FindCtf/CFindCtfMain.cpp:26-40; pixel
  //      size CInput::GetFinalPixelSize, CInput.cpp:709-715) ----
  if (out) out->ctf_done = 0;
  if (out && prm.cs > 0.001f && prm.kv != 0 && prm.pix_size != 0) {
    const float pixf = prm.pix_size * prm.ft_bin / (prm.mag[0] > prm.mag[1] ? prm.mag[0] : prm.mag[1]);
    const int cst = estimate_ctf(sum0, g.outW, g.outH, pixf, (float)prm.kv, prm.cs, prm.amp_cont,
                                 prm.ext_phase, out->ctf, out->ctf_spectrum,
                                 out->ctf_spectrum_on_device != 0, ctf, st);
    if (cst == kOk) out->ctf_done = 1;
    else if (cst != kEUnsupported) return cst;  // too small for a 512 x 512 tile: no estimate
  }
  if (active_tuning().row_pipe) {  // a pipelined pass that gave up waiting for its copies
    int flag = 0;
    MC3_TRY(fft_pipe_error(true, &flag));
    if (flag) {
      last_error = "a pipelined FFT pass timed out waiting for its bulk copies";
      return kECuda;
    }
  }
  // ---- 9. result tables ----
  if (out) {
    out->n_sums = g.nSums;
    out->n_patches = g.P;
    out->first_iterate = first_iterate_used;
    out->time_ms = ms;
    if (out->global_shifts)
      for (int f = 0; f < N; ++f) {
        out->global_shifts[2 * f] = fs.x(f);
        out->global_shifts[2 * f + 1] = fs.y(f);
      }
    if (g.patch) {
      if (out->patch_shifts) std::memcpy(out->patch_shifts, patShift.data(), sizeof(float) * patShift.size());
      if (out->patch_centers) std::memcpy(out->patch_centers, patCent.data(), sizeof(float) * patCent.size());
      if (out->patch_bad) std::memcpy(out->patch_bad, patBad.data(), patBad.size());
    }
    if (out->iterations) {
      out->iterations[0] = it0[0];
      for (int p = 0; p < g.P; ++p) out->iterations[1 + p] = patIters[p];
    }
    if (out->errors) {
      const int I = prm.iter;
      for (int s = 0; s < 1 + g.P; ++s) {
        const std::vector<float>& e = s == 0 ? err0[0] : patErr[s - 1];
        for (int i = 0; i < I; ++i) out->errors[(size_t)s * I + i] = i < (int)e.size() ? e[i] * bin : 0.0f;
      }
    }
  }
  return kOk;
}

}  // namespace mc3
