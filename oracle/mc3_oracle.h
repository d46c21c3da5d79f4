/*
 * FP64 CPU oracle for the MotionCor3 motion-correction hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker used by tests/,
 * by __graft_entry__.smoke() and by the CPU-baseline leg of bench.py.  It is
 * never linked into, loaded by or called from the product library (libmc3)
 * or its command-line front end.
 *
 * It restates, step by step, the algorithm of the reference (MotionCor3
 * 1.2.1) for the in-scope path: gain application, hot-pixel / defect
 * detection and correction, normalised forward FFT, Fourier cropping to the
 * alignment size, the iterative B-factor-weighted cross-correlation
 * alignment with its shift bookkeeping, patch alignment, local-motion
 * correction, dose weighting and summation.  Image and spectrum arithmetic
 * is FP64 with an independent FFT; the host-side shift bookkeeping runs in
 * FP32 exactly as the reference's host code does, so its discontinuous
 * steps (0.01 px truncation, int-truncated gathers, tolerance tests) are
 * comparable bit for bit.  Each function cites the reference file:line it
 * follows.
 */
#ifndef MC3_ORACLE_H
#define MC3_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int patch[2];       /* -Patch: patches in x, y (<=1 means none)        */
  int iter;           /* -Iter                                            */
  float tol;          /* -Tol (pixels)                                    */
  float bft[2];       /* -Bft global, patch                               */
  int phase_only;     /* -PhaseOnly                                       */
  float fm_dose;      /* -FmDose (e/A^2 per frame)                        */
  float pix_size;     /* -PixSize (A)                                     */
  int kv;             /* -kV                                              */
  int group[2];       /* -Group global, patch                             */
  int fm_ref;         /* -FmRef (<0: central frame)                       */
  float sum_range[2]; /* -SumRange (e/A^2)                                */
  int correct_bad;    /* run hot-pixel/defect detection and correction     */
  int split_sum;      /* -SplitSum: odd and even frame sums after the others */
  float ft_bin;       /* -FtBin: Fourier binning of the output sums        */
  int out_stack[2];   /* -OutStack: aligned frames wanted, z-bin            */
  /* Rendered frames of a frame-integration file (NULL: one raw frame per
   * frame): raw frames per rendered frame [N] and the accumulated dose [N];
   * dose_weight turns dose weighting on without fm_dose. */
  const int* int_size;
  const float* acc_dose;
  int dose_weight;
  const float* dark;  /* [H][W] dark reference subtracted before the gain, or NULL */
  float mag[3];       /* -Mag major minor angle (1 1 0 = none)             */
  int in_fm_motion;   /* -InFmMotion: in-frame motion weighting            */
  int corr_interp;    /* -CorrInterp: interpolation correction (patch mode) */
  const unsigned char* defects;  /* [H][W] known camera defects, or NULL */
} oracle_params;

typedef struct {
  int n_sums;             /* 1 (plain), +1 DW, +1 DWS, +2 odd/even         */
  float* sums;            /* [n_sums][Hb][Wb] caller-allocated (-FtBin size) */
  float* global_shifts;   /* [N][2] final full-frame shifts (log values)  */
  int n_patches;          /* P (0 in global mode)                         */
  float* patch_shifts;    /* [N][P][2] relative local shifts              */
  float* patch_centers;   /* [P][2]                                       */
  unsigned char* patch_bad; /* [N][P]                                     */
  int* iterations;        /* [1 + P] iterations run (global, each patch)  */
  unsigned char* bad_map; /* [H][W] detected bad pixels, may be NULL      */
  /* Optional inputs: when use_global_shifts is set, alignment is skipped and
   * the movie is corrected with these shifts (as logged: absolute in global
   * mode, relative to the reference frame in patch mode) and, in patch
   * mode, with the given local shifts, centres and bad flags. */
  const float* use_global_shifts;     /* [N][2]    */
  const float* use_patch_shifts;      /* [N][P][2] */
  const float* use_patch_centers;     /* [P][2]    */
  const unsigned char* use_patch_bad; /* [N][P]    */
  /* -OutStack output (when out_stack[0] and stack are set): the corrected
   * frames before dose weighting, -FtBin-cropped, C2R, unclamped, z-binned
   * into the first stack_frames slots; [N][Hb][Wb] caller-allocated. */
  float* stack;
  int stack_frames;       /* out */
} oracle_result;

void oracle_default_params(oracle_params* p);

/* Full single-movie path.  frames: [N][H][W] float32 raw values; gain:
 * [H][W] or NULL.  Returns 0 on success. */
int oracle_process_movie(const oracle_params* p, const float* frames, int W, int H, int N,
                         const float* gain, oracle_result* out);

/* ---- component entry points (targeted parity tests) ---- */
/* Normalised 2D R2C: img [H][W] -> spec [H][W/2+1] complex (interleaved). */
void oracle_rfft2(const double* img, double* spec, int W, int H, int normalise);
/* Unnormalised 2D C2R: spec [H][W/2+1] -> img [H][W]. */
void oracle_irfft2(const double* spec, double* img, int W, int H);
/* Complex 1D FFT, dir -1 forward / +1 inverse, unnormalised. */
void oracle_cfft(const double* in, double* out, int n, int dir);

/* Hot/defect pixel map of a frame sum [H][W] (BadPixel/CDetectMain.cpp). */
void oracle_detect_bad(const double* sum, int W, int H, unsigned char* bad);
/* Defect fill of one frame in place (BadPixel/GCorrectBad.cu). */
void oracle_correct_bad(double* frame, const unsigned char* bad, int W, int H);

/* Correlation window of one group against the sum (Align/GCorrelateSum2D.cu)
 * grp, sum: [cmpY][cmpX] complex.  win: [sy][sx] float. */
void oracle_correlate_window(const double* grp, const double* sum, int cmpX, int cmpY,
                             float bfactor, int phase_only, int sx, int sy, float* win);
/* CPeak2D::DoIt on a float window -> shift[2] (Align/CPeak2D.cpp:39). */
void oracle_peak2d(const float* win, int sx, int sy, float* shift);

/* Host shift bookkeeping, FP32 as in the reference. */
void oracle_remove_spikes(float* sx, float* sy, int n);             /* CRemoveSpikes1D::DoIt(...,false) */
void oracle_smooth(float* sx, float* sy, int n, float w);           /* CStackShift::Smooth */
int oracle_lin_eqs(float* coeff, float* vals, int dim);             /* Util_LinEqs::DoIt */
void oracle_patch_make_relative(float* shifts, int n_frames, int n_patches); /* CPatchShifts::MakeRelative */
void oracle_patch_detect_bads(const float* shifts, const float* centers, int n_frames,
                              int n_patches, int W, int H, unsigned char* bad); /* CPatchShifts::DetectBads */

/* Dose-weight factor w_f(k)/sqrt(sum_f w_f(k)^2) table for one frame
 * (Correct/GWeightFrame.cu): out [cmpY][cmpX]. */
void oracle_dose_weights(const float* acc_dose, int n_frames, int frame, int cmpX, int cmpY,
                         float pix_size, int kv, double* out);

/* Local-motion gather of one real frame (Correct/GCorrectPatchShift.cu:17). */
void oracle_local_gather(const double* in, double* out, int W, int H, const float* centers,
                         const float* shifts, const unsigned char* bad, int n_patches);

/* Iterative alignment of a stack of spectra (Align/CIterativeAlign.cpp):
 * spec [N][cmpY][cmpX] complex; group_size = -Group value; out shifts [N][2]
 * in the stack's own pixel units; returns iterations run. */
int oracle_iterative_align(const double* spec, int cmpX, int cmpY, int N, int group_size,
                           int max_iter, float tol, float bfactor, int phase_only,
                           float* shifts);
/* oracle_iterative_align with a first iterate init[N][2] (NULL: from zero). */
int oracle_iterative_align_warm(const double* spec, int cmpX, int cmpY, int N, int group_size,
                                int max_iter, float tol, float bfactor, int phase_only,
                                const float* init, float* shifts);

#ifdef __cplusplus
}
#endif
#endif
