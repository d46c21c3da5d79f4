// 2D real<->complex transforms built from one-CTA shared-memory passes.
//
// Replaces Util::CCufft2D (Util/CCufft2D.cpp:23-130).  Layouts follow the
// reference: a real frame of W x H pixels lives in a padded buffer whose
// rows hold W/2+1 complex values (2*(W/2+1) floats); the half spectrum
// produced in place is [H][W/2+1] complex, DC at (0,0).
//
// A forward transform is a row pass (real FFT of every row) followed by a
// column pass (complex FFT of every kx column); the inverse runs the column
// pass first and then a real inverse per row, which only uses the real
// parts of the DC and Nyquist terms of each row (the cuFFT C2R
// convention).  Each pass reads and writes HBM once; prologue/epilogue
// operations (gain, phase shifts, scaling, Fourier cropping) ride along.
#pragma once
#include "common.cuh"

namespace mc3 {

// Device twiddle tables e^{-2 pi i k / n}, computed in FP64 on the host and
// cached per length for the lifetime of the process (per device).
const float2* twiddles(int n);
// Fills an FftDesc for an n-point complex transform whose table has
// `table_n` entries (table_n = n or 2n).
int make_desc(int n, int table_n, FftDesc* d);

// Tile sizes used by the one-CTA passes (shared-memory budget per CTA).
int col_tile(int H);      // columns per CTA for a length-H column pass
int row_tile(int M);      // rows per CTA for a row pass of M complex values

// Compile-time in-place passes (power-of-two lengths): threads per CTA,
// shared memory per CTA (two CTAs per SM) and the number of padded
// sequences of length n_padded that one CTA holds (a power of two <= 16).
constexpr int kCtThreads = 512;
constexpr int kCtBudget = 72 * 1024;
__host__ __device__ constexpr int ct_batch(int n_padded) {
  int nb = kCtBudget / (n_padded * (int)sizeof(float2));
  int p = 1;
  while (p * 2 <= nb && p < 16) p *= 2;
  return p;
}

template <typename K>
int set_smem_attr(K kernel, size_t bytes) {
  if (bytes > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)bytes);
    if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute");
  }
  return kOk;
}

// Batch addressing: item b of a launch reads in + in_off(b) and writes
// out + b * out_stride.  in_off(b) = (b % nf) * in_stride + patch_off[b / nf]
// where patch_off is an optional device array of element offsets.
struct Batch {
  int items;
  int nf;                 // items per patch group (frames)
  long in_stride;         // elements between consecutive frames
  const long* patch_off;  // device, may be null
  long out_stride;        // elements between consecutive items
};

#ifdef __CUDACC__
__device__ __forceinline__ long batch_in_off(const Batch& b, int item) {
  long off = (long)(item % b.nf) * b.in_stride;
  if (b.patch_off) off += b.patch_off[item / b.nf];
  return off;
}
#endif

// Radix-16 register passes (fft_r16.cu) for power-of-two lengths: return
// kEUnsupported for other lengths (the caller then uses another kernel).
struct ColOps;
int row_r2c_r16(const float* in, long in_pitch, float2* out, long out_pitch, int W, int H,
                const Batch& b, float scale, cudaStream_t st);
int row_c2r_r16(const float2* in, long in_pitch, float* out, long out_pitch, int W, int H,
                const Batch& b, cudaStream_t st, int keep_im = 0);
int col_fft_r16(const float2* in, float2* out, long pitch, int cmpX, int H, const Batch& b,
                const ColOps& ops, cudaStream_t st);
// MC3_FFT_R16=0 disables them (A/B runs).
bool r16_enabled();
// Whether a pipelined pass gave up waiting for its copies (*flag != 0);
// `reset` clears the record.  Synchronises with the device.
int fft_pipe_error(bool reset, int* flag);

// Row real FFT: rows of W reals (row pitch in_pitch floats) -> W/2+1
// complex (row pitch out_pitch complex), multiplied by `scale`.  In-place
// use (out aliases in with in_pitch = 2*out_pitch) is allowed.
int row_r2c(const float* in, long in_pitch, float2* out, long out_pitch, int W, int H,
            const Batch& b, float scale, cudaStream_t st);

// Whether the 2D inverse of a W x H image keeps the imaginary parts of each
// row's DC and Nyquist terms (after the column pass) in the row inverse, as
// cuFFT's single-image 2D C2R plan (the reference's cufftPlan2d,
// Util/CCufft2D.cpp:39-53) does for non-Hermitian input of that size; a
// phase-shifted spectrum is such input.
bool c2r_keep_edge_imag(int W, int H);

// Row real inverse: W/2+1 complex per row -> W reals (unnormalised).
int row_c2r(const float2* in, long in_pitch, float* out, long out_pitch, int W, int H,
            const Batch& b, cudaStream_t st);

// Column pass options.
struct ColOps {
  int dir;               // -1 forward, +1 inverse
  float scale;           // applied on output
  // prologue phase shift: v *= ex[item][kx] * ey[item][ky] when non-null
  const float2* ex;      // [items][cmpX]
  const float2* ey;      // [items][H]
  // optional second output: Fourier crop to (crop_x, crop_y)
  float2* crop;          // [items][crop_y][crop_x], null when unused
  int crop_x, crop_y;
};

// Column complex FFT of length H over columns [0, cmpX) of
// [items][H][pitch] complex data; out may alias in.
int col_fft(const float2* in, float2* out, long pitch, int cmpX, int H, const Batch& b,
            const ColOps& ops, cudaStream_t st);

}  // namespace mc3
