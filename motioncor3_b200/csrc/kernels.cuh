// Launch wrappers for every libmc3 kernel.  All take device pointers and a
// stream, return a Status code and never synchronise unless stated.
#pragma once
#include "common.cuh"
#include "fft.cuh"

namespace mc3 {

// ---- prep.cu ----
// mode: MRC pixel mode (0 u8, 1 i16, 2 f32, 6 u16).  frames: padded stack.
int gain_and_sum(const void* raw, int mode, long raw_stride, const float* dark,
                 const float* gain, float* frames, long fr_stride, float* sum, int W, int H, int N,
                 cudaStream_t st);
// The same with frame integration (modes 0, 5, 101): rendered frame f sums
// raw frames start[f] .. start[f]+size[f]-1 modulo 256 (device tables).
int gain_and_sum_int(const void* raw, int mode, long raw_stride, const int* start,
                     const int* size, const float* dark, const float* gain, float* frames,
                     long fr_stride, float* sum, int W, int H, int N, cudaStream_t st);
// bad[i] = 1 where defects[i] != 0 (device, n pixels).
int or_mask(uint8_t* bad, const uint8_t* defects, size_t n, cudaStream_t st);
int moment_grid(int W, int H);
int image_moment(const float* img, int W, int H, long pitch, int iExp, float* d_part,
                 float* d_out, cudaStream_t st);
// hot_copy (optional, device W*H): receives the hot-pixel map before the
// defect patches are added.
int detect_bad_pixels(const float* sum, int W, int H, float* cc_buf, float* d_part,
                      float* d_mom, uint8_t* bad, const float* tpl, int ms, cudaStream_t st,
                      uint8_t* hot_copy = nullptr);
// d_count: 1 int, d_list: W*H int2 of device scratch (bad-pixel list).
int correct_bad_pixels(float* frames, long fr_stride, int N, const uint8_t* bad, int W, int H,
                       int* d_count, int2* d_list, cudaStream_t st);

// Synthetic counts 0..3 (pixel-index hash) for the autotuner's movie.
int synthetic_counts(float* f, long n, cudaStream_t st);

// ---- align.cu ----
// Separable phase tables for shifts sh[item] = (sx, sy) in pixels of an
// Nx x Ny image: ex[item][kx] = e^{i 2 pi kx sx / Nx}, ey[item][ky] =
// e^{i 2 pi ky' sy / Ny} (ky' wrapped); with skip_small, items whose
// |s| < 0.1 px get unit tables (GPhaseShift2D.cu:68-79).
int phase_tables(const float2* sh, int items, int cmpX, int cmpY, float2* ex, float2* ey,
                 bool skip_small, cudaStream_t st);

// out (+)= in * ex[kx] * ey[ky] for one spectrum.
int phase_apply(const float2* in, float2* out, int cmpX, int cmpY, const float2* ex,
                const float2* ey, bool accumulate, cudaStream_t st);

struct AlignDims {
  int cmpX, cmpY;      // stack spectrum size
  int N;               // frames per stack
  long stack_stride;   // complex elements between stacks
  int G;               // groups
  int seaX, seaY;      // search window
  int A;               // active stacks in this launch
};

// S[a] = sum_f X[act[a]][f] * ex * ey  (CAlignedSum with even/odd partials)
int aligned_sum(const float2* spec, const int* act, const float2* ex, const float2* ey,
                float2* S, const AlignDims& d, cudaStream_t st);
// Correlation of every group with (S - group), B-factor filter, centring,
// inverse column FFT; keeps the seaY central rows: T[a][g][seaY][cmpX].
int corr_cols(const float2* spec, const int* act, const float2* ex, const float2* ey,
              const float2* S, const int* gstart, const int* gsize, float bfactor,
              int phase_only, float2* T, const AlignDims& d, cudaStream_t st);
// Real inverse of each kept row; keeps the seaX central columns:
// win[a][g][seaY][seaX].
int corr_rows(const float2* T, float* win, const AlignDims& d, cudaStream_t st);
// CPeak2D on every window: out[a][g] = shift.
int peak_search(const float* win, float2* out, const AlignDims& d, cudaStream_t st);

// ---- correct.cu ----
struct DoseParams {
  int enabled;
  int dws;
  float pix_size;
  float kv_factor;
  float sum_range[2];
  int split;  // odd/even sums of the (weighted) frames after the others
};
// Wn[k] = sqrt(sum_f w_f(k)^2) (GWeightFrame::BuildWeight)
int dose_norm(const float* acc_dose, int N, int cmpX, int cmpY, float pix, float kvf, float* Wn,
              cudaStream_t st);
// sums[s][k] over frames, with optional phase tables (identity when null).
int frame_sums(const float2* spec, long fr_stride, int N, int cmpX, int cmpY, const float2* ex,
               const float2* ey, const float* acc_dose, const float* Wn, const DoseParams& dp,
               float2* sums, int n_sums, cudaStream_t st);
// mGCorrect3D per frame of a batch.  Bad patches come as per-frame 64-bit
// masks (patch_masks) or, when masks is null, as [nb][P] flags; clean[f]
// (optional) marks frames without bad patches and with finite shifts.
int local_gather(const float* in, long in_stride, float* out, long out_stride, int nb, int W,
                 int H, const float* centers, const float2* shifts,
                 const unsigned long long* masks, const uint8_t* bad, const uint8_t* clean,
                 int P, cudaStream_t st);
int patch_masks(const uint8_t* bad, const float2* shifts, int P, int nb,
                unsigned long long* masks, uint8_t* clean, cudaStream_t st);
// Fourier crop of N frame spectra, with their phase shift when ex/ey are given.
int crop_frames(const float2* in, int inX, int inY, long in_stride, const float2* ex,
                const float2* ey, float2* out, int outX, int outY, long out_stride, int N,
                cudaStream_t st);
// In-place group sums of real frames into the first n_groups frames;
// groups: device [2][n_groups] (starts, then sizes) of consecutive groups.
int zbin_frames(float* frames, long fr_stride, int pitch, int W, int H, const int* groups,
                int n_groups, cudaStream_t st);
// Bilinear anisotropic stretch of n padded real images (GStretch); m: the
// three entries of the symmetric inverse stretch matrix.
int stretch_images(const float* in, float* out, int pitch, long stride, int W, int H, int n,
                   const float* m, cudaStream_t st);
// In-frame motion weighting of N frame spectra; motion[f] = (m.x, m.y,
// apply, 0) per frame.
int motion_decon(float2* spec, long fr_stride, int cmpX, int cmpY, int N, const float4* motion,
                 cudaStream_t st);
// Linear-interpolation correction (-CorrInterp) of N frame spectra.
int corr_interp(float2* spec, long fr_stride, int cmpX, int cmpY, int N, cudaStream_t st);
// out[y*W+x] = max(0, in[y*pitch+x])
int unpad_positive(const float* in, long pitch, float* out, int W, int H, int n,
                   long in_stride, cudaStream_t st);

// ---- patch.cu ----
int fourier_crop(const float2* in, int inX, int inY, float2* out, int outX, int outY,
                 cudaStream_t st);
// Feature map of the binned sum (CDetectFeatures.cpp:94-119): returns on
// the device the normalised map [by][bx] (unpadded) and its moments.
int feature_map(float* img_padded, int bx, int by, float* tmp, float* d_part, float* d_scal,
                float* map_out, cudaStream_t st);

}  // namespace mc3
