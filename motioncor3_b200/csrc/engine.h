// The per-context processing engine behind the C ABI: owns device buffers
// sized for the current movie geometry and runs the whole path on one
// stream.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/mc3.h"
#include "host_align.h"
#include "kernels.cuh"
#include "tuning.h"

namespace mc3 {

// Grows-only device allocation reused across movies.
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  int ensure(size_t bytes);
  void release();
  template <typename T>
  T* as() const { return reinterpret_cast<T*>(p); }
  ~DevBuf() { release(); }
};

// Buffer geometry of one movie (CBufferPool.cpp:185-270).
struct Geometry {
  int W = 0, H = 0, N = 0;
  int cmpX = 0, cmpY = 0, padX = 0;
  int xcfCmpX = 0, xcfCmpY = 0;
  float xcfBin[2] = {1.f, 1.f};
  bool patch = false;
  int Px = 0, Py = 0, P = 0;
  int patCmpX = 0, patCmpY = 0;
  int patSizeX = 0, patSizeY = 0;
  bool dw = false, dws = false;
  int nSums = 1;
  int outW = 0, outH = 0;  // output sum size after -FtBin
  // n: rendered frames; file_dose: a frame-integration file gave a dose
  int compute(int w, int h, int n, const mc3_params& p, bool file_dose = false);
};

// Device scratch of the CTF estimate (ctf.cu), grown on demand.
struct CtfScratch {
  DevBuf img, spec, org, stats, tiles, half, full, rad, cand, res, band, ctf, out;
};

// CTF estimate of the device image d_img [ny][nx] (even sizes) as
// FindCtf::CFindCtfMain::DoIt makes it: res6 = defocus max, min (A),
// astigmatism azimuth (deg), extra phase (deg), score, fit resolution (A);
// image512 (optional, host or device) = the 512 x 512 diagnostic spectrum.
int estimate_ctf(const float* d_img, int nx, int ny, float pix, float kv, float cs, float ac,
                 float ext_phase, float* res6, float* image512, bool image_on_device, CtfScratch& s,
                 cudaStream_t st);

class Engine {
 public:
  explicit Engine(const mc3_params& p);
  ~Engine();
  int init();
  int set_stream(cudaStream_t s);
  int set_gain(const float* gain, int w, int h, bool on_device);
  int set_dark(const float* dark, int w, int h, bool on_device);
  int set_defects(const unsigned char* mask, int w, int h);
  int plan(int w, int h, int n, mc3_plan_info* info);
  // Autotuner: times every kernel variant on a synthetic movie of this size
  // with the context's options, keeps the fastest in the table.
  int autotune(int w, int h, int n, TuningEntry* out);
  // The table's choice for a movie size: the entry of the same frame size
  // and patch grid with the nearest frame count (the defaults when absent).
  Tuning tuning_for(int w, int h, int n) const;
  std::vector<TuningEntry> tuning_table;
  // Sizes of a movie (no allocation, no device work).
  int geometry(int w, int h, int n, mc3_plan_info* info, Geometry* g = nullptr) const;
  int process(const mc3_movie& mv, mc3_result* out);
  // process() with the given kernel variants active.
  int process_with(const mc3_movie& mv, mc3_result* out, const Tuning& t);
  // Starts the host->device copy of a later movie's raw frames on the copy
  // stream (at most two outstanding); process() consumes them in order.
  int prefetch(const mc3_movie& mv);
  // Waits for the outstanding prefetch copies and forgets them.
  void drop_prefetched();
  // Known alignment used instead of measuring (NULL clears it).
  int set_alignment(const mc3_alignment* aln);
  int set_frame_integration(const mc3_frame_integration* fi);
  // Rendered-frame tables of a movie of n_raw raw frames.
  host::FmInt frame_tables(int n_raw) const;
  // -OutStack: the corrected frames (spectra `spec`, phase tables when
  // `phase`) cropped to the output size, to real space, z-binned, copied to
  // out->stack.
  int write_stack(float2* spec, bool phase, const Geometry& g, const host::FmInt& fi,
                  mc3_result* out);

  // Batched CIterativeAlign over `nstack` stacks of N spectra each.  init
  // (optional): a first iterate [N][2] of the first stack's shifts, and
  // max_iter_init its iteration cap.
  int align_stacks(const float2* spec, long stack_stride, int nstack, int cmpX, int cmpY, int N,
                   const host::FrameGroups& grp, float bf0, float tol,
                   std::vector<host::StackShift>& shifts, std::vector<int>& iters,
                   std::vector<std::vector<float>>& errors, const float* init = nullptr,
                   int max_iter_init = 0, bool* converged = nullptr);
  // Patch centres given by the caller (mc3_set_patch_centers): [P][2]
  // full-frame pixels replacing the feature-based placement; empty: detect.
  std::vector<float> patch_centers_given;
  // First iterate of the next movie's full-frame alignment (mc3_set_first_iterate).
  std::vector<float> first_iterate;  // [nz][2] full-frame pixels; empty: cold start
  int first_iterate_max = 3;
  int first_iterate_used = 0;        // last movie: 1 warm start kept, 2 fell back to cold
  // Sums of spectra shifted by -shifts (global correction) into d_sums_.
  int global_sums(const float2* spec, int N, const host::StackShift& fs, const Geometry& g);

  mc3_params prm;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;

  // Movie prefetch: two raw-frame slots filled on copy_stream.
  struct Pending {
    const void* host;
    size_t bytes;
    int slot;
  };
  cudaStream_t copy_stream = nullptr;
  cudaStream_t copy_stream2 = nullptr;  // second half of a split copy
  cudaEvent_t half_done = nullptr;
  cudaEvent_t slot_loaded[2] = {nullptr, nullptr};  // copy into the slot finished
  cudaEvent_t slot_free[2] = {nullptr, nullptr};    // last read of the slot finished
  DevBuf d_rawslot[2];
  Pending pending[2];
  int n_pending = 0;
  int next_slot = 0;
  std::string last_error;

  // device buffers
  DevBuf d_gain, d_raw, d_frames, d_sum, d_cc, d_bad, d_part, d_mom, d_badn, d_badlist;
  DevBuf d_xcf, d_sh, d_ex, d_ey, d_S, d_T, d_win, d_gsh, d_act, d_gstart, d_gsize;
  DevBuf d_pat, d_patoff, d_bsum, d_bimg, d_btmp, d_bmap, d_scal;
  DevBuf d_fex, d_fey, d_Wn, d_acc, d_sums, d_real, d_gath, d_pcent, d_pshift, d_pbad, d_pmask, d_out, d_bsums;
  DevBuf d_stk, d_zgrp, d_mag, d_motion, d_defects, d_hot;
  bool has_defects = false;
  int defects_w = 0, defects_h = 0;
  // loaded alignment (mc3_set_alignment)
  bool aln_loaded = false;
  int aln_nz = 0, aln_P = 0;
  std::vector<float> aln_global, aln_patch, aln_centers;
  // frame integration (mc3_set_frame_integration)
  bool fmint = false;
  int fmint_raw = 0;
  bool fmint_dose = false;
  bool fmint_rendered = false;  // the movie holds the rendered frames already
  host::FmInt fmint_tab;
  DevBuf d_istart, d_isize;
  DevBuf d_dark;
  CtfScratch ctf;
  bool has_dark = false;
  int dark_w = 0, dark_h = 0;
  bool has_gain = false;
  double wn_key[6] = {0, 0, 0, 0, 0, 0};  // geometry and dose options of d_Wn
  bool wn_valid = false;
  int gain_w = 0, gain_h = 0;
};

}  // namespace mc3
