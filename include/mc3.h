/*
 * libmc3 -- B200-native motion correction of cryo-EM movie stacks.
 *
 * C ABI of the MotionCor3 hot path: gain application, hot-pixel / defect
 * correction, iterative full-frame alignment, patch alignment, local-motion
 * correction, dose weighting and summation.  Plain pointers and sizes
 * only; device pointers are CUDA device addresses on the context's GPU and
 * `stream` arguments are cudaStream_t values passed as void*.
 *
 * Every entry point returns an mc3 status code (MC3_OK on success) and
 * never aborts the process or resets the device.  A context is
 * thread-compatible: one host thread at a time per context.
 *
 * Each declaration names the reference (MotionCor3 1.2.1) interface it
 * replaces, as path:line within the reference project.
 */
#ifndef MC3_H
#define MC3_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MC3_OK 0
#define MC3_EINVAL 1      /* bad argument or unsupported size */
#define MC3_ENOMEM 2      /* device or host allocation failed */
#define MC3_ECUDA 3       /* CUDA runtime error (sticky errors included) */
#define MC3_ETIMEOUT 4    /* a bounded device wait gave up */
#define MC3_EIO 5         /* file could not be read or written */
#define MC3_EUNSUPPORTED 6 /* option or size outside the implemented path */
#define MC3_ETOOBIG 7     /* size above the fixed scratch of a no-allocation entry point */

typedef struct mc3_ctx mc3_ctx;

/* Options of the in-scope command-line tags; defaults as CInput::CInput
 * (CInput.cpp:82-127). */
typedef struct {
  int patch[3];        /* -Patch nx ny overlap; patch alignment needs nx,ny > 1 */
  int iter;            /* -Iter (15)                                           */
  float tol;           /* -Tol (0.1 px)                                        */
  float bft[2];        /* -Bft global, patch (500, 100)                        */
  int phase_only;      /* -PhaseOnly (0)                                       */
  float ft_bin;        /* -FtBin (1): Fourier binning of the output sums       */
  float init_dose;     /* -InitDose (accepted, unused by the reference path)  */
  float fm_dose;       /* -FmDose e/A^2 per frame (0 = no dose weighting)      */
  float pix_size;      /* -PixSize A (0)                                       */
  int kv;              /* -kV (300)                                            */
  int group[2];        /* -Group global, patch (1, 4)                          */
  int fm_ref;          /* -FmRef, 1-based; <0 = central frame (-1)             */
  float sum_range[2];  /* -SumRange e/A^2 (3, 25)                              */
  int align;           /* -Align (1; 0 = simple sum is not implemented)        */
  int correct_bad;     /* hot-pixel / defect detection + fill (1, as the
                          reference's CProcessThread.cpp:94-99 always runs)    */
  int gpu;             /* CUDA device ordinal (-Gpu first entry)               */
  int split_sum;       /* -SplitSum (0): also sum odd and even frames           */
  int out_stack[2];    /* -OutStack (0 1): 1 = also return the aligned frames;
                          second value: sum them in groups of this many frames
                          (CZbinStack, Align/CZbinStack.cpp:27-71)              */
  float mag[3];        /* -Mag major minor angle (1 1 0): anisotropic
                          magnification corrected on the sums
                          (CCorrectFullShift::mCorrectMag,
                          Correct/CCorrectFullShift.cpp:94-127)               */
  int in_fm_motion;    /* -InFmMotion (0): weight each aligned frame by the
                          directional sinc of its in-frame motion
                          (MotionDecon/GMotionWeight.cu, CInFrameMotion)      */
  int corr_interp;     /* -CorrInterp (0): in patch mode divide each globally
                          corrected frame spectrum by sinc(pi r)^(1/8)
                          (Util/GCorrLinearInterp.cu)                         */
  float cs;            /* -Cs mm: spherical aberration.  The CTF of the first
                          sum is estimated when cs > 0.001, kv != 0 and
                          pix_size != 0 (CFindCtfMain::bEstimate,
                          FindCtf/CFindCtfMain.cpp:26-40).  Library default 0
                          (no estimate); the command line's default is the
                          reference's 2.7                                     */
  float amp_cont;      /* -AmpCont (0.07): amplitude contrast                 */
  float ext_phase;     /* -ExtPhase deg (0): the extra phase searched spans
                          [0, min(2 ext_phase, 180)]                          */
  int dft_gemm;        /* 1: the row transforms of the patch stacks (the
                          patch pass of CTransformStack,
                          Align/CMeasurePatches.cpp:55) run as split-
                          precision BF16 DFT GEMMs on the tensor cores
                          (hi*hi + hi*lo + lo*hi, FP32 accumulation;
                          ~1e-5 relative error against 1e-7 for the FP32
                          FFT).  0 (default): the FP32 FFT                  */
} mc3_params;

/* Sizes a movie will use (CBufferPool::CreateBuffers, CBufferPool.cpp:95-270). */
typedef struct {
  int n_sums;          /* 1 + DW + DWS + 2*SplitSum                           */
  int n_patches;       /* px*py in patch mode, else 0                         */
  int xcf_size[2];     /* alignment (Fourier-binned) image size               */
  int patch_size[2];   /* patch image size (0 in global mode)                 */
  float xcf_bin[2];    /* binning factors of the alignment image             */
  size_t device_bytes; /* device memory the context holds for this movie     */
  int out_size[2];     /* size of each output sum (binned by -FtBin)          */
  int n_frames;        /* rendered frames (nz unless frame integration is set) */
} mc3_plan_info;

typedef struct {
  const void* frames;  /* [nz][ny][nx] pixels, MRC mode `mode`               */
  int mode;            /* 0 and 5 uint8, 1 int16, 2 float32, 6 uint16, 101
                          4-bit packed (rows of (nx+1)/2 bytes, even pixel in
                          the low nibble; MrcUtil/GApplyRefsToFrame.cu:30-53) */
  int nx, ny, nz;
  int on_device;       /* 1: frames is a device pointer                       */
} mc3_movie;

/* Caller-allocated outputs; any pointer may be NULL to skip it. */
typedef struct {
  float* sums;             /* [n_sums][out_size[1]][out_size[0]]: plain, DW, DWS,
                              ODD, EVN as enabled (out_size from mc3_plan) */
  int sums_on_device;      /* 1: `sums` is a device pointer                   */
  float* global_shifts;    /* [nz][2]: full-frame shifts as logged            */
  float* patch_shifts;     /* [nz][n_patches][2]                              */
  float* patch_centers;    /* [n_patches][2]                                  */
  unsigned char* patch_bad;/* [nz][n_patches]                                 */
  int* iterations;         /* [1 + n_patches]: global, then per patch         */
  float* errors;           /* [iter * (1 + n_patches)] max group shift per iteration */
  int n_sums;              /* out                                             */
  int n_patches;           /* out                                             */
  double time_ms;          /* out: device time of the call                    */
  float* stack;            /* -OutStack: [nz][out_size[1]][out_size[0]] aligned
                              (and locally corrected) frames before dose
                              weighting, -FtBin-binned, unclamped
                              (CCorrectFullShift::mCropFrame,
                              Correct/CCorrectFullShift.cpp:336-356); with
                              out_stack[1] > 1 the group sums fill the first
                              stack_frames slots                               */
  int stack_on_device;     /* 1: `stack` is a device pointer                   */
  int stack_frames;        /* out: frames written to `stack`                   */
  unsigned char* hot_map;  /* [ny][nx] host: the detected hot pixels (before the
                              defect patches), as -OutStar lists them
                              (CGenStarFile::SetHotPixels)                      */
  float ctf[6];            /* out when ctf_done: defocus max, defocus min (A),
                              astigmatism azimuth (deg), extra phase (deg),
                              score, fit resolution (A), as the _Ctf.txt line
                              (CSaveSerialCryoEM::mSaveCtfFit)                 */
  int ctf_done;            /* out: 1 when the CTF was estimated                */
  float* ctf_spectrum;     /* [512][512]: the averaged spectrum with the fitted
                              CTF drawn in (<stem>_Ctf.mrc)                    */
  int ctf_spectrum_on_device; /* 1: `ctf_spectrum` is a device pointer         */
  int first_iterate;       /* out: 0 cold start; 1 the first iterate set by
                              mc3_set_first_iterate converged within its cap;
                              2 it did not and the plain aligner ran from zero */
} mc3_result;

/* A known alignment (the -InAln file of Align/CLoadAlign.cpp:118-250): the
 * movie is corrected with these shifts and not aligned. */
typedef struct {
  int nz;                     /* frames the tables cover (must equal the movie's) */
  const float* global_shifts; /* [nz][2] full-frame shifts as in the file     */
  int n_patches;              /* 0: full-frame correction only                */
  const float* patch_shifts;  /* [nz][n_patches][2] local shifts              */
  const float* patch_centers; /* [n_patches][2]                               */
} mc3_alignment;

/* Frame integration (-FmIntFile; DataUtil/CFmIntParam.cpp:29-283 and
 * MrcUtil/CLoadCryoEMStack.cpp:184-262): the movie's n_raw raw frames are
 * rendered into n_int frames, frame i the sum of raw frames start[i] ..
 * start[i]+size[i]-1 taken modulo 256 as the reference's 8-bit rendered
 * stack holds it (modes 0, 5 and 101 only).  acc_dose[i] is the dose
 * accumulated at the end of rendered frame i; dose_weight asks for dose
 * weighting even when -FmDose is 0 (the file gave a dose). */
typedef struct {
  int n_raw;              /* raw frames (mc3_movie.nz)                         */
  int n_int;              /* rendered frames                                   */
  const int* start;       /* [n_int]                                           */
  const int* size;        /* [n_int]                                           */
  const float* acc_dose;  /* [n_int] e/A^2                                     */
  int dose_weight;
  int rendered;           /* 1: movies already hold the n_int rendered frames
                             (EER, rendered by mc3_eer_render); the tables then
                             only give doses, groups and time stamps          */
} mc3_frame_integration;

/* ---- library ---- */
const char* mc3_version(void);
const char* mc3_strerror(int code);
/* CInput::CInput defaults (CInput.cpp:82-127). */
void mc3_params_default(mc3_params* p);

/* ---- context ---- */
/* Replaces the CInput/CBufferPool/CAlignParam singletons set up in
 * CMain::DoIt (CMain.cpp:37-91) and CMain::mCreateBufferPool (:400-427). */
int mc3_create(const mc3_params* p, mc3_ctx** out);
int mc3_destroy(mc3_ctx* ctx);
/* Work stream (cudaStream_t); NULL = the context's own stream. */
int mc3_set_stream(mc3_ctx* ctx, void* stream);
/* Buffer geometry for a movie size (CBufferPool.cpp:185-270); also reserves
 * the context's device buffers for that size (CBufferPool::CreateBuffers,
 * CBufferPool.cpp:95-183), so the first mc3_process_movie does not pay for
 * the allocation. */
int mc3_plan(mc3_ctx* ctx, int nx, int ny, int nz, mc3_plan_info* info);
/* Page-locked host memory for movies and sums (the reference keeps frames
 * that do not fit on the GPU in cudaMallocHost buffers,
 * CGpuBuffer.cpp:156-175, and reads raw frames over the link from pinned
 * memory, MrcUtil/GApplyRefsToFrame.cu:129): copies from it run at full link
 * speed and can overlap kernels. */
int mc3_host_alloc(size_t bytes, void** ptr);
int mc3_host_free(void* ptr);
/* Gain reference [ny][nx] float (CLoadRefs::LoadGain, CLoadRefs.cpp:82-95);
 * NULL clears it. */
int mc3_set_gain(mc3_ctx* ctx, const float* gain, int nx, int ny, int on_device);
/* Dark reference [ny][nx] float (CLoadRefs::LoadDark, CLoadRefs.cpp:161-202),
 * subtracted before the gain multiplication (GApplyRefsToFrame,
 * MrcUtil/GApplyRefsToFrame.cu:56-72); NULL clears it. */
int mc3_set_dark(mc3_ctx* ctx, const float* dark, int nx, int ny, int on_device);
/* Camera defects known in advance (-DefectFile rectangles, -DefectMap image;
 * BadPixel/CDetectMain.cpp:146-260): a host [ny][nx] mask whose nonzero
 * pixels are added to the detected bad pixels before they are filled; NULL
 * clears it. */
int mc3_set_defects(mc3_ctx* ctx, const unsigned char* mask, int nx, int ny);

/* ---- whole path ---- */
/* One movie from raw frames to sums and shift tables: replaces
 * CProcessThread::mProcess from mApplyRefs through mAlignStack
 * (CProcessThread.cpp:82-107, 136-182), i.e. CApplyRefs::DoIt,
 * BadPixel::CDetectMain::DoIt, BadPixel::CCorrectMain::DoIt and
 * Align::CAlignMain::DoIt (Align/CAlignMain.cpp:39-75). */
int mc3_process_movie(mc3_ctx* ctx, const mc3_movie* movie, mc3_result* out);
/* Movie queue: the reference's processing thread and its package queue
 * (CProcessThread::ThreadMain, CProcessThread.cpp:39-80), with the loader
 * thread's overlap (MrcUtil/CLoadCryoEMStack.cpp:104-152).  mc3_submit
 * hands a movie to the context's worker thread and returns its ticket at
 * once; movies are processed in submission order, each one's raw frames
 * copied to the device while the one before it is processed (pinned host
 * frames overlap fully).  Movies of any size and frame count may follow one
 * another.  The movie's frames and the result's buffers must stay valid and
 * unchanged until mc3_wait has returned for its ticket, and while tickets
 * are outstanding mc3_process_movie and mc3_prefetch_movie return
 * MC3_EINVAL (the other entry points of the context must not be called).
 * mc3_destroy finishes the queued movies first. */
int mc3_submit(mc3_ctx* ctx, const mc3_movie* movie, mc3_result* out, int* ticket);
/* Blocks until the movie of `ticket` is done and returns its status (as
 * mc3_process_movie would); latency_ms (may be NULL) receives the time from
 * its mc3_submit to the end of its processing.  Each ticket is waited for
 * once. */
int mc3_wait(mc3_ctx* ctx, int ticket, double* latency_ms);
/* Autotuner (no counterpart in the reference, whose launch shapes are
 * fixed): times every variant of the tunable kernel families -- radix-16 or
 * radix-8 register FFT passes for power-of-two lengths, two or four columns
 * per CTA in the 4096-point column pass, one or two pixels per thread in
 * the local-motion gather -- on a synthetic movie of nx x ny x nz with the
 * context's options (its device time per movie, best of two runs after a
 * warm-up), and keeps the fastest for movies of that size and patch grid on
 * this context.  With json_path the choice (and every candidate's time) is
 * also written to that JSON file, replacing an earlier entry for the same
 * size and keeping the others; ms_best (may be NULL) receives the winner's
 * time.  Takes a few seconds per size. */
int mc3_autotune(mc3_ctx* ctx, int nx, int ny, int nz, const char* json_path, double* ms_best);
/* Reads the choices of a file written by mc3_autotune into the context.
 * MC3_EIO when the file is missing or not such a file. */
int mc3_load_tuning(mc3_ctx* ctx, const char* json_path);
/* CTF estimate of one image [ny][nx] (even sizes) at pixel size pix_size A:
 * the role of FindCtf::CFindCtfMain::DoIt (FindCtf/CFindCtfMain.cpp:49-83),
 * which the reference runs on the first sum of every movie
 * (Correct/CCorrectFullShift.cpp:129-144).  result6 as mc3_result::ctf;
 * spectrum512 (may be NULL) on the host, or on the device when on_device.
 * MC3_EUNSUPPORTED when the image, rescaled to >= 1.25 A pixels, holds no
 * 512 x 512 tile. */
int mc3_estimate_ctf(mc3_ctx* ctx, const float* image, int nx, int ny, int on_device,
                     float pix_size, float kv, float cs, float amp_cont, float ext_phase,
                     float* result6, float* spectrum512);
/* Loading the next movie while the current one is processed, as the
 * reference's loader thread does (MrcUtil/CLoadCryoEMStack.cpp:130-180):
 * starts the host->device copy of `movie`'s raw frames on the context's
 * copy stream and returns.  The following mc3_process_movie calls must
 * pass the prefetched movies in the same order (same frames pointer and
 * size; MC3_EINVAL otherwise); at most two may be outstanding.  The host
 * frames must stay valid and unchanged until their mc3_process_movie
 * returns, and must be pinned (mc3_host_alloc, cudaHostAlloc or
 * cudaHostRegister) for the copy to overlap.  Device-resident movies need
 * no prefetch (no-op). */
int mc3_prefetch_movie(mc3_ctx* ctx, const mc3_movie* movie);
/* Align::CLoadAlign (Align/CLoadAlign.cpp:52-250; used by
 * CFullAlign::Align, Align/CFullAlign.cpp:85-89, and
 * CPatchAlign::mCalcPatchShifts, Align/CPatchAlign.cpp:67-96): the tables
 * are copied and used, instead of measuring, by every following
 * mc3_process_movie until cleared with NULL.  As in the reference, patch
 * mode makes the full-frame shifts relative to the reference frame
 * (-FmRef) and treats every loaded patch shift as good.  n_patches must
 * match the context's -Patch grid (MC3_EINVAL otherwise). */
int mc3_set_alignment(mc3_ctx* ctx, const mc3_alignment* aln);
/* Warm start of the next movie's full-frame alignment: CIterativeAlign::DoIt
 * (Align/CIterativeAlign.cpp:55-97) begins from these per-frame shifts
 * global_xy [nz][2] (full-frame pixels, as mc3_result.global_shifts) instead
 * of zero -- each frame group's running total starts at its frames' mean --
 * and runs at most max_iter iterations (<= 0: 3).  The plain aligner judges
 * the first iterate: when its first correlation finds the first iterate more
 * than 1 pixel of the alignment image off, or the iterations have not
 * converged to -Tol, the plain aligner runs from zero with the full -Iter
 * budget and its result is used (mc3_result.first_iterate tells which).
 * Consumed by the next mc3_process_movie; NULL clears it.  This is the entry
 * of the learned proposal (mc3_proposal_*). */
int mc3_set_first_iterate(mc3_ctx* ctx, const float* global_xy, int nz, int max_iter);
/* Patch centres of the following movies, centers_xy [n_patches][2] in
 * full-frame pixels (as mc3_result.patch_centers), instead of the placement
 * from the feature map (Align/CDetectFeatures.cpp:58-181, CPatchAlign's
 * centre search): each patch is cut around the given centre, kept inside the
 * alignment image.  Used to reproduce another run's patch layout -- for
 * instance a run of the reference program, whose in-place feature-map
 * normalisation (Align/GNormByStd2D.cu:7-40) can move its centres -- so that
 * patch shifts and sums can be compared patch for patch.  Applies while
 * n_patches equals the movie's patch count; NULL clears it.  No counterpart
 * option in the reference. */
int mc3_set_patch_centers(mc3_ctx* ctx, const float* centers_xy, int n_patches);
/* CFmIntParam / CFmGroupParam set up from a frame-integration table: the
 * following movies (nz = n_raw) are rendered, dose-weighted with acc_dose
 * and grouped by raw-frame counts (CFmGroupParam::mGroupByRawSize,
 * DataUtil/CFmGroupParam.cpp:60-78); NULL clears it. */
int mc3_set_frame_integration(mc3_ctx* ctx, const mc3_frame_integration* fi);

/* ---- components (device pointers unless stated) ---- */
/* Util::CCufft2D::Forward (Util/CCufft2D.cpp:65-87): in-place R2C of nz
 * padded real frames [nz][ny][2*(nx/2+1)], optionally x 1/(nx*ny). */
int mc3_fft_forward(float* frames, int nx, int ny, int nz, int normalise, void* stream);
/* The row pass of Util::CCufft2D::Forward (Util/CCufft2D.cpp:65-78): real
 * DFT of each of n_rows rows of nx floats (row pitch in_pitch floats) into
 * nx/2+1 complex values per row (row pitch out_pitch complex), not
 * normalised.  method 0: the FP32 FFT; 1: the split-precision BF16 DFT GEMM
 * on the tensor cores (even nx <= 414).  Not in place. */
int mc3_rfft_rows(const float* in, int in_pitch, float* out, int out_pitch, int nx, int n_rows,
                  int method, void* stream);
/* Util::CCufft2D::Inverse (Util/CCufft2D.cpp:105-120): in-place,
 * unnormalised C2R of nz half spectra [nz][ny][nx/2+1] complex. */
int mc3_fft_inverse(float* frames, int nx, int ny, int nz, void* stream);
/* Util::GPhaseShift2D::DoIt (Util/GPhaseShift2D.cu:48-66): out (+)= in *
 * e^{i 2pi (kx sx/Nx + ky sy/Ny)} on a [cmp_y][cmp_x] half spectrum. */
int mc3_phase_shift(const float* in, float* out, int cmp_x, int cmp_y, float sx, float sy,
                    int accumulate, void* stream);
/* No counterpart in the reference.  The same phase shift as mc3_phase_shift,
 * for callers that cannot allocate device memory while they run (an
 * application that owns a fixed memory pool or budget, or a latency-bound
 * path where cudaMalloc/cudaFree would stall the device): it calls no
 * cudaMalloc, cudaFree or allocating library routine.  Its scratch is a
 * fixed device array of 197,120 bytes inside libmc3, so cmp_x may be at most
 * MC3_NOALLOC_MAX_CMP_X and cmp_y at most MC3_NOALLOC_MAX_CMP_Y; larger sizes
 * return MC3_ETOOBIG.  The first call on a device looks up that array's
 * address (once per device, the device current); make that first call before
 * any stream capture.  The address is kept for the life of the process, so
 * after a cudaDeviceReset of a device this entry point must not be called on
 * it again.  Every call on a device shares the one array, so calls that
 * overlap on the GPU (other streams, other host threads) race; calls in one
 * stream are ordered.  The shift reaches the device as a kernel argument (no
 * host memory is read); the call only enqueues work on `stream` and returns
 * without waiting for it, unlike mc3_phase_shift, which synchronises. */
#define MC3_NOALLOC_MAX_CMP_X 8193
#define MC3_NOALLOC_MAX_CMP_Y 16384
int mc3_phase_shift_noalloc(const float* in, float* out, int cmp_x, int cmp_y, float sx,
                            float sy, int accumulate, void* stream);
/* Util::GFourierResize2D::DoIt (Util/GFourierResize2D.cu:110-126), copy mode. */
int mc3_fourier_crop(const float* in, int in_cmp_x, int in_cmp_y, float* out, int out_cmp_x,
                     int out_cmp_y, void* stream);
/* Align::GCorrelateSum2D::DoIt + Align::CPeak2D::DoIt
 * (Align/GCorrelateSum2D.cu:108-140, Align/CPeak2D.cpp:39-109): correlation
 * window [sea_y][sea_x] of a group spectrum against (sum - group) and its
 * sub-pixel peak (host float[2]). */
int mc3_correlate(const float* group, const float* sum, int cmp_x, int cmp_y, float bfactor,
                  int phase_only, int sea_x, int sea_y, float* window, float* shift_host,
                  void* stream);
/* Align::CIterativeAlign::DoIt (Align/CIterativeAlign.cpp:55-156) on a
 * device stack of n half spectra [n][cmp_y][cmp_x]; shifts_host [n][2];
 * returns iterations through *iters. */
int mc3_iterative_align(mc3_ctx* ctx, const float* stack, int cmp_x, int cmp_y, int n,
                        int group, int max_iter, float tol, float bfactor, int phase_only,
                        float* shifts_host, int* iters);
/* BadPixel::CDetectMain::DoIt detection part (BadPixel/CDetectMain.cpp:54-123)
 * on a padded frame sum [ny][2*(nx/2+1)] -> bad map [ny][nx] (device). */
int mc3_detect_bad_pixels(const float* sum, int nx, int ny, unsigned char* bad, void* stream);
/* BadPixel::GCorrectBad::GDoIt (BadPixel/GCorrectBad.cu:167-185) on nz
 * padded frames. */
int mc3_correct_bad_pixels(float* frames, int nx, int ny, int nz, const unsigned char* bad,
                           void* stream);
/* Correct::mGCorrect3D (Correct/GCorrectPatchShift.cu:17-66) on one padded
 * real frame; centers [P][2], shifts [P][2], bad [P] (device, bad may be NULL). */
int mc3_local_gather(const float* in, float* out, int nx, int ny, const float* centers,
                     const float* shifts, const unsigned char* bad, int n_patches, void* stream);
/* Correct::GWeightFrame (Correct/GWeightFrame.cu:90-147) + the sums of
 * CCorrectFullShift::mGenSums (Correct/CCorrectFullShift.cpp:271-300):
 * sums of nz half spectra after the phase shift by -shifts (host [nz][2],
 * |s| < 0.1 px skipped) with dose weighting when fm_dose > 0. */
int mc3_dose_weighted_sums(mc3_ctx* ctx, const float* spectra, int nx, int ny, int nz,
                           const float* shifts_host, float* sums, int* n_sums);

/* ---- learned shift proposal (no counterpart in the reference) ----
 * A small convolutional network (strided convolutions + ReLU, global
 * average pool, linear head) that maps a binned frame pair [2][h][w] to a
 * first iterate of that frame's shift, trained on the GPU by the library's
 * own forward and backward kernels (FP32, Adam) on shifts that the plain
 * aligner measured, and used through mc3_set_first_iterate, where the plain
 * aligner decides whether the warm result is kept and remains the fallback. */
typedef struct mc3_proposal mc3_proposal;
/* spec: n_layers groups of (cin, cout, k, stride, pad), the first cin = 2;
 * nout outputs; weights He-initialised from seed, on device `gpu`. */
int mc3_proposal_create(const int* spec, int n_layers, int nout, unsigned seed, int gpu,
                        mc3_proposal** out);
int mc3_proposal_destroy(mc3_proposal* p);
int mc3_proposal_num_params(mc3_proposal* p, long* n);
/* Parameters in the order: per layer weights [cout][cin][k][k] then biases,
 * then the head's weights [nout][cout_last] then biases (host floats). */
int mc3_proposal_get_params(mc3_proposal* p, float* params);
int mc3_proposal_set_params(mc3_proposal* p, const float* params);
/* Forward and backward of a batch x [batch][2][h][w] against target
 * [batch][nout] (host arrays): loss = sum over the batch of
 * 0.5 |out - target|^2, grad (may be NULL) = its gradient summed over the
 * batch, out (may be NULL) = the outputs. */
int mc3_proposal_loss_grad(mc3_proposal* p, const float* x, int batch, int h, int w,
                           const float* target, double* loss, float* grad, float* out);
/* One Adam step (learning rate lr) on a batch; x and target on the device
 * when on_device; *loss receives the batch's mean loss. */
int mc3_proposal_train_step(mc3_proposal* p, const float* x, const float* target, int batch,
                            int h, int w, int on_device, float lr, double* loss);
/* Outputs [batch][nout] (host) for inputs x [batch][2][h][w]. */
int mc3_proposal_predict(mc3_proposal* p, const float* x, int batch, int h, int w, int on_device,
                         float* out);
/* Inputs of n frame pairs from a device movie frames [nz][ny][nx] (float):
 * pairs [n][2] (host) frame indices, each pair binned by `bin` and normalised
 * by its mean and standard deviation into x [n][2][ny/bin][nx/bin] (device). */
int mc3_proposal_pair_inputs(const float* frames, int nx, int ny, int nz, const int* pairs, int n,
                             int bin, float* x, void* stream);

/* ---- diagnostics (no counterpart in the reference, which reports NVTX
 * ranges and wall-clock prints instead, e.g. CProcessThread.cpp:103-104) ---- */
/* Per-kernel timing with CUDA events around every launch (process-wide). */
void mc3_profile_enable(int on);
/* Writes {"kernel": [launches, total_ms, algorithmic_bytes], ...} as JSON. */
int mc3_profile_read(char* buf, size_t len, int reset);
/* Kernel launches issued by this library since it was loaded. */
unsigned long long mc3_kernel_launches(void);

/* ---- movie files (host) ---- */
/* TiffUtil/CLoadTiffHeader.cpp (size = first directory, frames = number of
 * directories, mode from bits per sample and sample format: 8 -> 0, 16 -> 1
 * signed or 6, 32-bit float -> 2).  MC3_EIO when unreadable,
 * MC3_EUNSUPPORTED for other pixel types or pages of mixed size/type. */
int mc3_tiff_info(const char* path, int* nx, int* ny, int* nz, int* mode);
/* TiffUtil/CLoadTiffImage.cpp + CLoadTiffStack (multi-threaded): frames
 * z0..z0+nz-1 decoded (none, LZW, Deflate, PackBits; horizontal predictor)
 * into dst [nz][ny][nx] in the file's pixel type, rows bottom-up as the
 * reference stores them; threads <= 0 uses every host core. */
int mc3_tiff_read(const char* path, int z0, int nz, void* dst, int threads);

/* EerUtil/CLoadEerHeader.cpp:22-51: camera size, number of EER frames (TIFF
 * directories) and run-length bits (65001 -> 7, 65000 -> 8). */
int mc3_eer_info(const char* path, int* cam_x, int* cam_y, int* n_frames, int* bits);
/* EerUtil/CRenderMrcStack.cpp + CDecodeEerFrame.cpp: n_out rendered 8-bit
 * frames, frame i the electron counts of EER frames start[i] ..
 * start[i]+size[i]-1, at -EerSampling 1, 2 or 3 (camera size x 1, 2, 4;
 * super-resolution needs 4096-pixel rows), into dst [n_out][ny][nx]; EER
 * frames decoded on threads (<= 0: every host core). */
int mc3_eer_render(const char* path, int sampling, int n_out, const int* start, const int* size,
                   unsigned char* dst, int threads);

/* ---- host-side bookkeeping (host pointers) ---- */
/* CFmGroupParam::Setup (DataUtil/CFmGroupParam.cpp:26-78): groups of the
 * n rendered frames (start/size in raw frames) for -Group bin_z: runs holding
 * bin_z x (smallest rendered-frame size) raw frames; writes up to max_groups
 * group starts, sizes (in rendered frames) and centres (mean frame time
 * stamps) and their count in *n_groups. */
int mc3_frame_groups(const int* start, const int* size, int n, int bin_z, int max_groups,
                     int* n_groups, int* g_start, int* g_size, float* g_center);
/* CLoadRefs::PostProcess (CLoadRefs.cpp:204-229): rotation by rot x 90
 * degrees (G90Rotate2D, nearest pixel about the centre; odd factors swap the
 * size), flip (1 upside down, 2 left-right; GFlip2D), then 1/v with 0 kept
 * (GInverse2D) when inverse is set; out holds nx*ny floats and receives the
 * image at its new size *out_nx x *out_ny. */
int mc3_ref_orient(const float* in, int nx, int ny, int rot, int flip, int inverse, float* out,
                   int* out_nx, int* out_ny);
/* CLoadRefs::AugmentRefs / GAugmentRef (CLoadRefs.cpp:231-268,
 * MrcUtil/GAugmentRef.cu:10-23): a reference for frames fact times larger,
 * every pixel repeated fact x fact; out holds nx*ny*fact*fact floats. */
int mc3_ref_augment(const float* in, int nx, int ny, int fact, float* out);
/* CReadFmIntFile::DoIt (DataUtil/CReadFmIntFile.cpp:104-170): up to
 * max_entries (group size, integration size, raw-frame dose) rows of a
 * frame-integration file; two-column files take fm_dose.  MC3_EIO when the
 * file cannot be opened; *n_entries = 0 when it holds mixed doses. */
int mc3_read_fmint_file(const char* path, float fm_dose, int max_entries, int* group_size,
                        int* int_size, float* dose, int* n_entries);
/* CFmIntParam::Setup (DataUtil/CFmIntParam.cpp:29-256): rendered-frame
 * tables for n_raw raw frames from n_entries file rows (n_entries = 0: no
 * file), with -Throw / -Trunc frames dropped (raw frames without a file,
 * rendered frames with one, unless 5 or fewer would be left); fills up to
 * max_int entries of start/size/acc_dose and returns their count in *n_int,
 * *dose_weight = the file has a dose. */
int mc3_frame_integration_tables(const int* group_size, const int* int_size, const float* dose,
                                 int n_entries, int n_raw, float fm_dose, int throw_first,
                                 int throw_last, int max_int, int* n_int, int* start, int* size,
                                 float* acc_dose, int* dose_weight);
/* Align::CPeak2D::DoIt (Align/CPeak2D.cpp:39-109). */
void mc3_peak2d(const float* window, int sea_x, int sea_y, float* shift);
/* Util::CRemoveSpikes1D::DoIt(x, y, false) (Util/CRemoveSpikes1D.cpp:59-105). */
void mc3_remove_spikes(float* sx, float* sy, int n);
/* Util_LinEqs::DoIt (LibSrc/Util/Util_LinEqs.cpp:19-41); returns 1 on success. */
int mc3_lin_eqs(float* coeff, float* vals, int dim);
/* Align::CStackShift::Smooth (Align/CStackShift.cpp:180-198). */
void mc3_smooth_shifts(float* sx, float* sy, int n, float weight);
/* Align::CPatchShifts::MakeRelative (Align/CPatchShifts.cpp:263-286),
 * shifts [nz][P][2] in place. */
void mc3_patch_make_relative(float* shifts, int nz, int n_patches);
/* Align::CPatchShifts::DetectBads (Align/CPatchShifts.cpp:288-355). */
void mc3_patch_detect_bads(const float* shifts, const float* centers, int nz, int n_patches,
                           int nx, int ny, unsigned char* bad);
/* Patch starts [P][2] (alignment-image pixels) that mc3_set_patch_centers
 * derives from full-frame centres [P][2]: each centre divided by the xcf bin
 * (bin_x, bin_y) and rounded, minus half the patch (pat_x, pat_y), kept
 * inside the xcf_x x xcf_y image.  The inverse of the centres the engine
 * reports ((start + pat/2) * bin, as CPatchCenters::GetCenter scaled by
 * CFullAlign).  No counterpart in the reference (it has no given centres). */
int mc3_patch_starts_from_centers(const float* centers, int n_patches, float bin_x, float bin_y,
                                  int xcf_x, int xcf_y, int pat_x, int pat_y, int* starts);

#ifdef __cplusplus
}
#endif
#endif /* MC3_H */
