// Split-precision BF16 DFT-GEMMs on tensor cores (dft_gemm.cu).
#pragma once
#include "fft.cuh"

namespace mc3 {

// Whether a K-point real row transform fits the GEMM tiles (even K, at most
// 414 points: K/2+1 complex outputs in two 208-column tiles).
bool dft_rows_supported(int K);
// Row real DFT of K reals per row as a split-BF16 GEMM (hi*hi + hi*lo +
// lo*hi, FP32 accumulation): the interface of row_r2c (rows of H per item,
// items addressed by `b`), outputs times `scale`.  Not in place.
int dft_rows_r2c(const float* in, long in_pitch, float2* out, long out_pitch, int K, int H,
                 const Batch& b, float scale, cudaStream_t st);
// Error flag of the GEMM kernels (a bounded device wait gave up); reads it
// (synchronising the device) and clears it when `reset`.
int dft_gemm_error(bool reset, int* flag);

}  // namespace mc3
