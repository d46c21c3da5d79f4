// Per-element forward and backward of the shift-proposal network (strided
// convolutions + ReLU, global average pool, linear head), shared by the
// device kernels that will train it and the CPU shim that checks them
// (tests/native/proposal_core_shim.cpp).  Every output element is a gather,
// so each maps to one thread without atomics:
//   conv_fwd_at  y[co][oy][ox]      = b + sum_ci,ky,kx w x
//   conv_dx_at   dx[ci][iy][ix]     = sum over the outputs that read x[ci][iy][ix]
//   conv_dw_at   dw[co][ci][ky][kx] = sum_oy,ox dy x
// Layout: activations [C][H][W], weights [cout][cin][k][k].
#pragma once
#include <cuda_runtime.h>

#ifndef MC3_HD
#define MC3_HD __host__ __device__ __forceinline__
#endif

namespace mc3 {
namespace proposal {

struct ConvShape {
  int cin, cout, k, stride, pad;
  int H, W;    // input size
  int oh, ow;  // output size
};

MC3_HD int conv_out(int n, int k, int stride, int pad) { return (n + 2 * pad - k) / stride + 1; }

template <class T>
MC3_HD T conv_fwd_at(const T* x, const T* w, const T* b, const ConvShape& s, int co, int oy, int ox) {
  T acc = b[co];
  for (int ci = 0; ci < s.cin; ++ci)
    for (int ky = 0; ky < s.k; ++ky) {
      const int iy = oy * s.stride + ky - s.pad;
      if (iy < 0 || iy >= s.H) continue;
      for (int kx = 0; kx < s.k; ++kx) {
        const int ix = ox * s.stride + kx - s.pad;
        if (ix < 0 || ix >= s.W) continue;
        acc += w[((co * s.cin + ci) * s.k + ky) * s.k + kx] * x[(ci * s.H + iy) * s.W + ix];
      }
    }
  return acc;
}

// Input gradient at x[ci][iy][ix]: the outputs (oy, ox) with
// oy * stride + ky - pad == iy for some tap ky in [0, k).
template <class T>
MC3_HD T conv_dx_at(const T* dy, const T* w, const ConvShape& s, int ci, int iy, int ix) {
  T acc = 0;
  for (int co = 0; co < s.cout; ++co)
    for (int ky = 0; ky < s.k; ++ky) {
      const int ty = iy + s.pad - ky;
      if (ty < 0 || ty % s.stride) continue;
      const int oy = ty / s.stride;
      if (oy >= s.oh) continue;
      for (int kx = 0; kx < s.k; ++kx) {
        const int tx = ix + s.pad - kx;
        if (tx < 0 || tx % s.stride) continue;
        const int ox = tx / s.stride;
        if (ox >= s.ow) continue;
        acc += dy[(co * s.oh + oy) * s.ow + ox] * w[((co * s.cin + ci) * s.k + ky) * s.k + kx];
      }
    }
  return acc;
}

template <class T>
MC3_HD T conv_dw_at(const T* dy, const T* x, const ConvShape& s, int co, int ci, int ky, int kx) {
  T acc = 0;
  for (int oy = 0; oy < s.oh; ++oy) {
    const int iy = oy * s.stride + ky - s.pad;
    if (iy < 0 || iy >= s.H) continue;
    for (int ox = 0; ox < s.ow; ++ox) {
      const int ix = ox * s.stride + kx - s.pad;
      if (ix < 0 || ix >= s.W) continue;
      acc += dy[(co * s.oh + oy) * s.ow + ox] * x[(ci * s.H + iy) * s.W + ix];
    }
  }
  return acc;
}

template <class T>
MC3_HD T conv_db_at(const T* dy, const ConvShape& s, int co) {
  T acc = 0;
  for (int i = 0; i < s.oh * s.ow; ++i) acc += dy[co * s.oh * s.ow + i];
  return acc;
}

// ReLU'(pre) applied to the incoming gradient.
template <class T>
MC3_HD T relu_grad(T g, T pre) { return pre > T(0) ? g : T(0); }

}  // namespace proposal
}  // namespace mc3
