// Radix-16 register FFT for power-of-two lengths 128..4096.
//
// The same Stockham stage formulas as fft_core.cuh (butterfly jb of a
// radix-R stage reads x[jb + r*N/R], multiplies input r by
// w_N^(r*(jb%NS)*N/(NS*R)) and writes y[(jb/NS)*NS*R + jb%NS + r*NS]), with
// the plan N = 16 * 16 * ... * RL (RL = 16, 8, 4 or 2).  Every thread holds
// 16 values per stage (16/R butterflies of radix R), so:
//  * the first stage reads its inputs straight from global memory (or any
//    other source given by the caller) and the last stage hands its
//    outputs straight to the caller, which stores them to global memory;
//  * shared memory is touched only between stages: 4 passes at N = 4096
//    instead of the 10 of a load / radix-8 stages / store kernel;
//  * the padded layout spad16(i) = i + i/16 makes both the strided writes
//    (stride 16) and the contiguous reads of every stage bank-conflict free;
//  * one twiddle table read per butterfly, the other powers by a product
//    tree of depth <= 4.
//
// The stage functions are __host__ __device__ so that tests/native runs the
// same code sequentially (read phase of all threads, then write phase),
// which is exactly the order the __syncthreads() of the device driver
// enforces.
#pragma once
#include "fft_core.cuh"

namespace mc3 {

MC3_HD int spad16(int i) { return i + (i >> 4); }
MC3_HD constexpr int spad16_len(int n) { return n + (n >> 4) + 1; }
// Stride between the NB column sequences of a column CTA (thread t ->
// column t % NB): 64-bit shared accesses are served per half-warp, which
// holds 16/NB slots of each of NB columns, so column c must start 16/NB
// word pairs after column c-1 modulo the 16 bank pairs: stride = 16/NB
// (mod 16), at least spad16_len(n).
MC3_HD constexpr int spad16_col_stride(int n, int nb) {
  const int want = nb >= 16 ? 1 : 16 / nb;
  int ld = spad16_len(n);
  while (ld % 16 != want % 16) ++ld;
  return ld;
}

// Plan of N = 2^p: p/4 radix-16 stages, then one stage of radix 2^(p%4).
MC3_HD constexpr int r16_nstages(int n) {
  return ct_log2(n) / 4 + (ct_log2(n) % 4 ? 1 : 0);
}
MC3_HD constexpr int r16_radix(int n, int s) {
  return s < ct_log2(n) / 4 ? 16 : (1 << (ct_log2(n) % 4));
}
MC3_HD constexpr int r16_ns(int n, int s) {  // product of the earlier radices
  return s == 0 ? 1 : r16_ns(n, s - 1) * r16_radix(n, s - 1);
}

// Length-16 DFT as 4 x 4: inner 4-point DFTs over x[4 n1 + n2], twiddles
// w16^(n2 k1), outer 4-point DFTs; X[k1 + 4 k2].
template <int DIR>
struct Dft<16, DIR> {
  MC3_HD static void run(float2* v) {
    const float c1 = 0.92387953251128675613f;  // cos(pi/8)
    const float s1 = 0.38268343236508977173f;  // sin(pi/8)
    const float h = 0.70710678118654752440f;   // cos(pi/4)
    float2 a[4][4];  // a[n2][k1]
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
      float2 t[4] = {v[n2], v[4 + n2], v[8 + n2], v[12 + n2]};
      Dft<4, DIR>::run(t);
#pragma unroll
      for (int k1 = 0; k1 < 4; ++k1) a[n2][k1] = t[k1];
    }
    // w16^m for m = n2*k1 in {1, 2, 3, 4, 6, 9}; forward e^{-i pi m / 8}
    const float sg = DIR < 0 ? -1.0f : 1.0f;
    const float2 w1 = c2(c1, sg * s1), w2 = c2(h, sg * h), w3 = c2(s1, sg * c1);
    const float2 w6 = c2(-h, sg * h), w9 = c2(-c1, -sg * s1);
    a[1][1] = cmul(a[1][1], w1);
    a[1][2] = cmul(a[1][2], w2);
    a[1][3] = cmul(a[1][3], w3);
    a[2][1] = cmul(a[2][1], w2);
    a[2][2] = crot<DIR>(a[2][2]);  // w16^4 = -i (forward)
    a[2][3] = cmul(a[2][3], w6);
    a[3][1] = cmul(a[3][1], w3);
    a[3][2] = cmul(a[3][2], w6);
    a[3][3] = cmul(a[3][3], w9);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
      float2 t[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
      Dft<4, DIR>::run(t);
#pragma unroll
      for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = t[k2];
    }
  }
};

// w[1..R-1] = powers of w[1] by a product tree (depth <= 4).
template <int R>
MC3_HD void tw_powers(float2* w) {
  if constexpr (R >= 4) {
    w[2] = cmul(w[1], w[1]);
    w[3] = cmul(w[2], w[1]);
  }
  if constexpr (R >= 8) {
    w[4] = cmul(w[2], w[2]);
    w[5] = cmul(w[4], w[1]);
    w[6] = cmul(w[3], w[3]);
    w[7] = cmul(w[4], w[3]);
  }
  if constexpr (R == 16) {
    w[8] = cmul(w[4], w[4]);
    w[9] = cmul(w[8], w[1]);
    w[10] = cmul(w[5], w[5]);
    w[11] = cmul(w[8], w[3]);
    w[12] = cmul(w[6], w[6]);
    w[13] = cmul(w[8], w[5]);
    w[14] = cmul(w[7], w[7]);
    w[15] = cmul(w[8], w[7]);
  }
}

// Per-thread values of one stage: 16/R butterflies of radix R; thread slot
// j (0 <= j < N/16) owns butterflies jb = j + i*N/16.
template <int N, int S>
struct R16Stage {
  static constexpr int R = r16_radix(N, S);
  static constexpr int NB = 16 / R;  // butterflies per thread
  static constexpr int NS = r16_ns(N, S);
  static constexpr int NR = N / R;
  static constexpr bool LAST = S == r16_nstages(N) - 1;
};

// Input index of value (i, r) of slot j in stage S.
template <int N, int S>
MC3_HD int r16_in_index(int j, int i, int r) {
  using St = R16Stage<N, S>;
  return j + i * (N / 16) + r * St::NR;
}

// Twiddles, DFT and output indices of the stage: out(index, value) is
// called for the 16 outputs of slot j.
template <int DIR, int N, int S, class Out>
MC3_HD void r16_compute(float2 (&v)[16], int j, const float2* tw, int tws, Out out) {
  using St = R16Stage<N, S>;
  constexpr int R = St::R, NS = St::NS;
#pragma unroll
  for (int i = 0; i < St::NB; ++i) {
    const int jb = j + i * (N / 16);
    float2* u = v + i * R;
    const int k = jb % NS;
    if (NS > 1) {
      float2 w[R];
      w[1] = twid<DIR>(tw, tws, (N / (NS * R)) * k);
      tw_powers<R>(w);
#pragma unroll
      for (int r = 1; r < R; ++r) u[r] = cmul(u[r], w[r]);
    }
    Dft<R, DIR>::run(u);
    const int base = (jb / NS) * NS * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) out(base + r * NS, u[r]);
  }
}

#ifdef __CUDACC__
// Stages S.. of the device driver below (shared memory in, shared memory
// or store out).
template <int DIR, int N, int S, bool LAST_TO_SMEM, class StoreF>
__device__ __forceinline__ void fft_r16_rest(float2* buf, int j, const float2* __restrict__ tw,
                                             int tws, StoreF store) {
  if constexpr (S < r16_nstages(N)) {
    using St = R16Stage<N, S>;
    float2 v[16];
#pragma unroll
    for (int i = 0; i < St::NB; ++i)
#pragma unroll
      for (int r = 0; r < St::R; ++r) v[i * St::R + r] = buf[spad16(r16_in_index<N, S>(j, i, r))];
    if constexpr (St::LAST && !LAST_TO_SMEM) {
      r16_compute<DIR, N, S>(v, j, tw, tws, store);  // no shared-memory writes follow
    } else {
      __syncthreads();
      r16_compute<DIR, N, S>(v, j, tw, tws, [&](int idx, float2 x) { buf[spad16(idx)] = x; });
      __syncthreads();
      fft_r16_rest<DIR, N, S + 1, LAST_TO_SMEM>(buf, j, tw, tws, store);
    }
  }
}

// CTA driver for one sequence of length N per group of N/16 threads.  buf:
// this sequence's padded shared-memory slice (spad16 layout, spad16_len(N)
// words); j: the thread's slot.  load(idx) supplies the input x[idx] of the
// first stage; store(idx, value) receives the output y[idx] of the last
// stage (natural order).  With LAST_TO_SMEM the last stage writes buf
// instead (callers that post-process in shared memory); with
// FIRST_FROM_SMEM the first stage reads buf (load is not used).  after_first()
// runs once the first stage's inputs have all been read (after the barrier
// that follows the first stage; not called when the first stage is the
// last).  All threads of the CTA must call it.
struct NoHook {
  __device__ void operator()() const {}
};
template <int DIR, int N, bool FIRST_FROM_SMEM, bool LAST_TO_SMEM, class LoadF, class StoreF,
          class HookF = NoHook>
__device__ __forceinline__ void fft_r16(float2* buf, int j, const float2* __restrict__ tw,
                                        int tws, LoadF load, StoreF store,
                                        HookF after_first = HookF()) {
  auto to_smem = [&](int idx, float2 x) { buf[spad16(idx)] = x; };
  // stage 0
  {
    using St = R16Stage<N, 0>;
    float2 v[16];
#pragma unroll
    for (int i = 0; i < St::NB; ++i)
#pragma unroll
      for (int r = 0; r < St::R; ++r) {
        const int idx = r16_in_index<N, 0>(j, i, r);
        v[i * St::R + r] = FIRST_FROM_SMEM ? buf[spad16(idx)] : load(idx);
      }
    if (FIRST_FROM_SMEM) __syncthreads();
    if constexpr (St::LAST && !LAST_TO_SMEM) {
      r16_compute<DIR, N, 0>(v, j, tw, tws, store);
      return;
    } else {
      r16_compute<DIR, N, 0>(v, j, tw, tws, to_smem);
      __syncthreads();
      after_first();
    }
  }
  fft_r16_rest<DIR, N, 1, LAST_TO_SMEM>(buf, j, tw, tws, store);
}
#endif

}  // namespace mc3
