// Mixed-radix Stockham FFT core shared by every transform in libmc3.
//
// The reference delegates all transforms to cuFFT through Util::CCufft2D
// (Util/CCufft2D.cpp:23-120: R2C forward with optional 1/(Nx*Ny) scaling,
// unnormalised C2R inverse).  libmc3 does not link cuFFT: every 2D
// transform is split into a row pass and a column pass that each run a
// batch of 1D transforms inside one CTA's shared memory, using the
// functions below.
//
// Algorithm: out-of-place Stockham auto-sort (no bit reversal), one stage
// per factor of n.  For a stage of radix R with Ns = product of the
// earlier radices, butterfly j (0 <= j < n/R) reads x[j + r*n/R],
// multiplies input r by w_n^(r*(j%Ns)*n/(Ns*R)), applies a length-R DFT
// and writes y[(j/Ns)*Ns*R + j%Ns + r*Ns].  Radices 2, 3, 4 and 8 have
// dedicated butterflies, odd primes 5..31 a register butterfly built on
// input pairs (dft_prime); any other factor (41, 131, ...) uses a
// per-output direct DFT that reads its inputs from shared memory.
//
// Every index computation lives in __host__ __device__ functions so the
// exact same code is exercised by a sequential host driver in the CPU
// tests (fft_host_reference below) and by the CTA driver in the kernels.
#pragma once
#include <cuda_runtime.h>
#include <vector_types.h>

#ifndef MC3_HD
#define MC3_HD __host__ __device__ __forceinline__
#endif

namespace mc3 {

constexpr int kMaxStages = 24;

MC3_HD float2 c2(float x, float y) { float2 r; r.x = x; r.y = y; return r; }
MC3_HD float2 cadd(float2 a, float2 b) { return c2(a.x + b.x, a.y + b.y); }
MC3_HD float2 csub(float2 a, float2 b) { return c2(a.x - b.x, a.y - b.y); }
MC3_HD float2 cscale(float2 a, float s) { return c2(a.x * s, a.y * s); }
MC3_HD float2 cconj(float2 a) { return c2(a.x, -a.y); }
MC3_HD float2 cmul(float2 a, float2 b) {
  return c2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// Multiply by -i for the forward direction (DIR = -1, kernel e^{-i...})
// and by +i for the inverse direction (DIR = +1).
template <int DIR>
MC3_HD float2 crot(float2 a) {
  return DIR < 0 ? c2(a.y, -a.x) : c2(-a.y, a.x);
}
// Twiddle lookup: table holds e^{-2 pi i k / n}; the inverse uses the
// conjugate.
template <int DIR>
MC3_HD float2 twid(const float2* tw, int tws, int k) {
  float2 w = tw[k * tws];
  return DIR < 0 ? w : cconj(w);
}

// Description of one complex transform length.  `tw` points at a table of
// e^{-2 pi i k / n} values sampled every `tws` entries (a length-2n table
// with tws = 2 serves an n-point transform, which is how the real-data
// transforms share one table).
struct FftDesc {
  int n;
  int nstages;
  int radix[kMaxStages];
  const float2* tw;
  int tws;
};

// Factor n into stage radices: as many 8s as possible, then 4, then 2,
// then 3 (as 3), then the remaining primes in increasing order.
// Returns the number of stages, or -1 if n < 1 or too many stages.
inline int fft_factorize(int n, int* radix) {
  if (n < 1) return -1;
  int ns = 0;
  int m = n;
  int p2 = 0;
  while (m % 2 == 0) { m /= 2; ++p2; }
  // powers of two as 8s and 4s (a lone 2 only for a single factor 2)
  if (p2 >= 4 && p2 % 3 == 1) {
    radix[ns++] = 4;
    radix[ns++] = 4;
    p2 -= 4;
  }
  while (p2 >= 3) { radix[ns++] = 8; p2 -= 3; }
  if (p2 == 2) radix[ns++] = 4;
  if (p2 == 1) radix[ns++] = 2;
  for (int p = 3; m > 1; p += 2) {
    while (m % p == 0) {
      if (ns >= kMaxStages) return -1;
      radix[ns++] = p;
      m /= p;
    }
    if (p * p > m && m > 1) {
      if (ns >= kMaxStages) return -1;
      radix[ns++] = m;
      m = 1;
    }
  }
  return ns;
}

// ---- length-R DFT kernels on register arrays ---------------------------
template <int R, int DIR>
struct Dft;

template <int DIR>
struct Dft<2, DIR> {
  MC3_HD static void run(float2* v) {
    float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <int DIR>
struct Dft<4, DIR> {
  MC3_HD static void run(float2* v) {
    float2 a = cadd(v[0], v[2]);
    float2 b = csub(v[0], v[2]);
    float2 c = cadd(v[1], v[3]);
    float2 d = crot<DIR>(csub(v[1], v[3]));
    v[0] = cadd(a, c);
    v[2] = csub(a, c);
    v[1] = cadd(b, d);
    v[3] = csub(b, d);
  }
};

template <int DIR>
struct Dft<3, DIR> {
  MC3_HD static void run(float2* v) {
    // e^{-2 pi i / 3} = -1/2 - i*sqrt(3)/2 (forward)
    const float kS = 0.86602540378443864676f;
    float2 t = cadd(v[1], v[2]);
    float2 u = csub(v[1], v[2]);
    float2 m = c2(v[0].x - 0.5f * t.x, v[0].y - 0.5f * t.y);
    float2 r = crot<DIR>(cscale(u, kS));
    v[0] = cadd(v[0], t);
    v[1] = cadd(m, r);
    v[2] = csub(m, r);
  }
};

template <int DIR>
struct Dft<8, DIR> {
  MC3_HD static void run(float2* v) {
    const float kH = 0.70710678118654752440f;
    float2 e[4] = {v[0], v[2], v[4], v[6]};
    float2 o[4] = {v[1], v[3], v[5], v[7]};
    Dft<4, DIR>::run(e);
    Dft<4, DIR>::run(o);
    // o[k] *= w8^k ; w8 = e^{DIR * i pi / 4}
    float2 o1 = o[1];
    o[1] = DIR < 0 ? c2(kH * (o1.x + o1.y), kH * (o1.y - o1.x))
                   : c2(kH * (o1.x - o1.y), kH * (o1.y + o1.x));
    o[2] = crot<DIR>(o[2]);
    float2 o3 = o[3];
    o[3] = DIR < 0 ? c2(kH * (o3.y - o3.x), -kH * (o3.x + o3.y))
                   : c2(-kH * (o3.x + o3.y), kH * (o3.x - o3.y));
    for (int k = 0; k < 4; ++k) {
      v[k] = cadd(e[k], o[k]);
      v[k + 4] = csub(e[k], o[k]);
    }
  }
};

// Odd prime radices 5..31 in registers: with H = (R-1)/2 and the input
// pairs a_j = x_j + x_{R-j}, b_j = x_j - x_{R-j} (j = 1..H),
//   y_k     = x_0 + sum_j a_j cos(2 pi jk/R) + DIR i sum_j b_j sin(2 pi jk/R)
//   y_{R-k} = the same with the sine term negated,
// which needs H^2 complex-by-real products per sum instead of R^2 complex
// ones.  cos/sin of 2 pi m/R come from the stage's twiddle table
// (entry m*nR*tws holds e^{-2 pi i m / R}).
MC3_HD constexpr bool is_prime_radix(int R) {
  return R == 5 || R == 7 || R == 11 || R == 13 || R == 17 || R == 19 || R == 23 || R == 29 ||
         R == 31;
}
template <int R, int DIR>
MC3_HD void dft_prime(float2* v, const float2* tw, int tws, int nR) {
  constexpr int H = (R - 1) / 2;
  float cs[H + 1], sn[H + 1];
#pragma unroll
  for (int m = 1; m <= H; ++m) {
    const float2 w = tw[m * nR * tws];
    cs[m] = w.x;
    sn[m] = -w.y;
  }
  float2 a[H + 1], b[H + 1];
  const float2 x0 = v[0];
  float2 y0 = x0;
#pragma unroll
  for (int j = 1; j <= H; ++j) {
    a[j] = cadd(v[j], v[R - j]);
    b[j] = csub(v[j], v[R - j]);
    y0 = cadd(y0, a[j]);
  }
  v[0] = y0;  // the inputs now live in x0, a and b; outputs overwrite v
#pragma unroll
  for (int k = 1; k <= H; ++k) {
    float2 A = x0, B = c2(0.f, 0.f);
#pragma unroll
    for (int j = 1; j <= H; ++j) {
      const int m = (j * k) % R;
      const float cm = m <= H ? cs[m] : cs[R - m];
      const float sm = m <= H ? sn[m] : -sn[R - m];
      A.x += a[j].x * cm;
      A.y += a[j].y * cm;
      B.x += b[j].x * sm;
      B.y += b[j].y * sm;
    }
    // i*B = (-B.y, B.x)
    if (DIR < 0) {
      v[k] = c2(A.x + B.y, A.y - B.x);
      v[R - k] = c2(A.x - B.y, A.y + B.x);
    } else {
      v[k] = c2(A.x - B.y, A.y + B.x);
      v[R - k] = c2(A.x + B.y, A.y - B.x);
    }
  }
}

// One butterfly of a prime-radix stage (register DFT above).
template <int R, int DIR>
MC3_HD void stage_bfly_prime(const float2* A, float2* B, int n, int Ns, int j,
                             const float2* tw, int tws, int es) {
  const int nR = n / R;
  const int k = j % Ns;
  float2 v[R];
#pragma unroll
  for (int r = 0; r < R; ++r) v[r] = A[(j + r * nR) * es];
  if (Ns > 1) {
    const int step = (n / (Ns * R)) * k;
#pragma unroll
    for (int r = 1; r < R; ++r) v[r] = cmul(v[r], twid<DIR>(tw, tws, step * r));
  }
  dft_prime<R, DIR>(v, tw, tws, nR);
  const int idxD = (j / Ns) * Ns * R + k;
#pragma unroll
  for (int r = 0; r < R; ++r) B[(idxD + r * Ns) * es] = v[r];
}

// One butterfly of a dedicated-radix stage.  A/B: sequence base pointers,
// es: element stride.
template <int R, int DIR>
MC3_HD void stage_bfly(const float2* A, float2* B, int n, int Ns, int j,
                       const float2* tw, int tws, int es) {
  const int nR = n / R;
  const int k = j % Ns;
  float2 v[R];
#pragma unroll
  for (int r = 0; r < R; ++r) v[r] = A[(j + r * nR) * es];
  if (Ns > 1) {
    const int step = (n / (Ns * R)) * k;
#pragma unroll
    for (int r = 1; r < R; ++r) v[r] = cmul(v[r], twid<DIR>(tw, tws, step * r));
  }
  Dft<R, DIR>::run(v);
  const int idxD = (j / Ns) * Ns * R + k;
#pragma unroll
  for (int r = 0; r < R; ++r) B[(idxD + r * Ns) * es] = v[r];
}

// One output of a direct-DFT stage (any radix R dividing n).
// o in [0, n): j = o / R, q = o % R.
template <int DIR>
MC3_HD void stage_direct(const float2* A, float2* B, int n, int R, int Ns, int o,
                         const float2* tw, int tws, int es) {
  const int nR = n / R;
  const int j = o / R;
  const int q = o - j * R;
  const int k = j % Ns;
  const int step = (n / (Ns * R)) * k;
  float2 acc = c2(0.f, 0.f);
  for (int r = 0; r < R; ++r) {
    float2 x = A[(j + r * nR) * es];
    if (Ns > 1 && r > 0) x = cmul(x, twid<DIR>(tw, tws, step * r));
    const int m = (r * q) % R;
    if (m) x = cmul(x, twid<DIR>(tw, tws, m * nR));
    acc = cadd(acc, x);
  }
  const int idxD = (j / Ns) * Ns * R + k;
  B[(idxD + q * Ns) * es] = acc;
}

MC3_HD bool radix_is_dedicated(int R) {
  return R == 2 || R == 3 || R == 4 || R == 8 || is_prime_radix(R);
}

template <int DIR>
MC3_HD void stage_item(const float2* A, float2* B, int n, int R, int Ns, int item,
                       const float2* tw, int tws, int es) {
  switch (R) {
    case 2: stage_bfly<2, DIR>(A, B, n, Ns, item, tw, tws, es); break;
    case 3: stage_bfly<3, DIR>(A, B, n, Ns, item, tw, tws, es); break;
    case 4: stage_bfly<4, DIR>(A, B, n, Ns, item, tw, tws, es); break;
    case 8: stage_bfly<8, DIR>(A, B, n, Ns, item, tw, tws, es); break;
    case 5: stage_bfly_prime<5, DIR>(A, B, n, Ns, item, tw, tws, es); break;
    case 7: stage_bfly_prime<7, DIR>(A, B, n, Ns, item, tw, tws, es); break;
    case 11: stage_bfly_prime<11, DIR>(A, B, n, Ns, item, tw, tws, es); break;
    case 13: stage_bfly_prime<13, DIR>(A, B, n, Ns, item, tw, tws, es); break;
    case 17: stage_bfly_prime<17, DIR>(A, B, n, Ns, item, tw, tws, es); break;
    case 19: stage_bfly_prime<19, DIR>(A, B, n, Ns, item, tw, tws, es); break;
    case 23: stage_bfly_prime<23, DIR>(A, B, n, Ns, item, tw, tws, es); break;
    case 29: stage_bfly_prime<29, DIR>(A, B, n, Ns, item, tw, tws, es); break;
    case 31: stage_bfly_prime<31, DIR>(A, B, n, Ns, item, tw, tws, es); break;
    default: stage_direct<DIR>(A, B, n, R, Ns, item, tw, tws, es); break;
  }
}

MC3_HD int stage_items(int n, int R) { return radix_is_dedicated(R) ? n / R : n; }

#ifdef __CUDACC__
// CTA driver: nb sequences; sequence b, element i at A[b*bs + i*es].
// B is scratch of the same layout.  Returns the buffer holding the result.
// Must be called by all threads of the CTA; ends with __syncthreads().
template <int DIR>
__device__ float2* cta_fft(float2* A, float2* B, const FftDesc& d, int nb, int es, int bs) {
  int Ns = 1;
  for (int s = 0; s < d.nstages; ++s) {
    const int R = d.radix[s];
    const int per = stage_items(d.n, R);
    const int items = nb * per;
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
      const int b = it / per;
      const int j = it - b * per;
      stage_item<DIR>(A + b * bs, B + b * bs, d.n, R, Ns, j, d.tw, d.tws, es);
    }
    __syncthreads();
    float2* t = A; A = B; B = t;
    Ns *= R;
  }
  return A;
}
#endif

// ---- in-place variant (dedicated radices only) -----------------------
// Shared-memory index with one padding slot per 32 elements: the strided
// butterfly writes of the first stages then spread over all banks.
MC3_HD int spad(int i) { return i + (i >> 5); }
// Padded length of a sequence of n elements.
MC3_HD int spad_len(int n) { return n + (n >> 5) + 1; }

// True when every stage radix is 4 or 8 (the in-place path).
inline bool all_dedicated(const FftDesc& d) {
  for (int s = 0; s < d.nstages; ++s)
    if (d.radix[s] != 4 && d.radix[s] != 8) return false;
  return true;
}

#ifdef __CUDACC__
// One stage in place: every thread first loads the inputs of up to MAXB
// butterflies into registers, the CTA synchronises, then all outputs are
// written back to the same buffer.  Sequence b, element i lives at
// buf[b*ld + spad(i)].
template <int R, int DIR, int MAXB>
__device__ __forceinline__ void stage_inplace(float2* buf, int n, int Ns, int nb, int ld,
                                              const float2* __restrict__ tw, int tws) {
  const int per = n / R;
  const int items = nb * per;
  float2 v[MAXB][R];
  int bj[MAXB];
#pragma unroll
  for (int m = 0; m < MAXB; ++m) {
    const int it = threadIdx.x + m * blockDim.x;
    bj[m] = -1;
    if (it < items) {
      const int b = it / per;
      const int j = it - b * per;
      bj[m] = it;
      const float2* A = buf + b * ld;
#pragma unroll
      for (int r = 0; r < R; ++r) v[m][r] = A[spad(j + r * per)];
    }
  }
  __syncthreads();
#pragma unroll
  for (int m = 0; m < MAXB; ++m) {
    if (bj[m] < 0) continue;
    const int b = bj[m] / per;
    const int j = bj[m] - b * per;
    const int k = j % Ns;
    if (Ns > 1) {
      const int step = (n / (Ns * R)) * k;
#pragma unroll
      for (int r = 1; r < R; ++r) v[m][r] = cmul(v[m][r], twid<DIR>(tw, tws, step * r));
    }
    Dft<R, DIR>::run(v[m]);
    const int idxD = (j / Ns) * Ns * R + k;
    float2* A = buf + b * ld;
#pragma unroll
    for (int r = 0; r < R; ++r) A[spad(idxD + r * Ns)] = v[m][r];
  }
  __syncthreads();
}

// In-place CTA transform of nb sequences (buf[b*ld + spad(i)]); requires
// all_dedicated(d) (radices 4 and 8 only) and nb*n/R <= MAXB*blockDim.x for every stage radix R.
template <int DIR, int MAXB>
__device__ void cta_fft_inplace(float2* buf, const FftDesc& d, int nb, int ld) {
  int Ns = 1;
  for (int s = 0; s < d.nstages; ++s) {
    const int R = d.radix[s];
    if (R == 8) stage_inplace<8, DIR, MAXB>(buf, d.n, Ns, nb, ld, d.tw, d.tws);
    else stage_inplace<4, DIR, MAXB>(buf, d.n, Ns, nb, ld, d.tw, d.tws);
    Ns *= R;
  }
}
#endif

// ---- compile-time plans for power-of-two lengths -----------------------
// The same factorisation as fft_factorize, evaluated at compile time: all
// index arithmetic of a stage becomes shifts and masks and every loop
// unrolls.
MC3_HD constexpr int ct_log2(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return l;
}
MC3_HD constexpr int ct_nstages(int n) {
  int p2 = ct_log2(n), ns = 0;
  if (p2 >= 4 && p2 % 3 == 1) {
    ns += 2;
    p2 -= 4;
  }
  ns += p2 / 3;
  if (p2 % 3) ++ns;
  return ns;
}
MC3_HD constexpr int ct_radix(int n, int s) {
  int p2 = ct_log2(n), first = 0;
  if (p2 >= 4 && p2 % 3 == 1) {
    if (s < 2) return 4;
    first = 2;
    p2 -= 4;
  }
  if (s < first + p2 / 3) return 8;
  if (s == first + p2 / 3 && p2 % 3) return 1 << (p2 % 3);
  return 1;
}
// Shared-memory words of a padded sequence of n elements (spad_len).
MC3_HD constexpr int ct_spad_len(int n) { return n + (n >> 5) + 1; }

#ifdef __CUDACC__
// One in-place stage over NB sequences of N elements (sequence b at
// buf[b*LD + spad(i)]) by a CTA of T threads; the arithmetic of
// stage_inplace except for the twiddle powers (see below).
template <int R, int DIR, int N, int NS, int NB, int T, int LD>
__device__ __forceinline__ void stage_ct(float2* buf, const float2* __restrict__ tw, int tws) {
  constexpr int per = N / R;
  constexpr int items = NB * per;
  constexpr int MB = (items + T - 1) / T;
  float2 v[MB][R];
  const unsigned tid = threadIdx.x;
#pragma unroll
  for (int m = 0; m < MB; ++m) {
    const unsigned it = tid + m * T;
    if (items % T == 0 || it < (unsigned)items) {
      const unsigned b = it / per, j = it % per;
      const float2* A = buf + b * LD;
#pragma unroll
      for (int r = 0; r < R; ++r) v[m][r] = A[spad(j + r * per)];
    }
  }
  __syncthreads();
#pragma unroll
  for (int m = 0; m < MB; ++m) {
    const unsigned it = tid + m * T;
    if (items % T == 0 || it < (unsigned)items) {
      const unsigned b = it / per, j = it % per;
      const unsigned k = j % NS;
      if (NS > 1) {
        // One table read per butterfly; the other powers of the twiddle by
        // a product tree of depth <= 3 (a few FP32 ulp), which keeps the
        // shared L1/shared-memory pipe free of six more loads.
        const int step = (N / (NS * R)) * k;
        float2 w[R];
        w[1] = twid<DIR>(tw, tws, step);
        if constexpr (R >= 4) {
          w[2] = cmul(w[1], w[1]);
          w[3] = cmul(w[2], w[1]);
        }
        if constexpr (R == 8) {
          w[4] = cmul(w[2], w[2]);
          w[5] = cmul(w[4], w[1]);
          w[6] = cmul(w[3], w[3]);
          w[7] = cmul(w[4], w[3]);
        }
#pragma unroll
        for (int r = 1; r < R; ++r) v[m][r] = cmul(v[m][r], w[r]);
      }
      Dft<R, DIR>::run(v[m]);
      const unsigned idxD = (j / NS) * NS * R + k;
      float2* A = buf + b * LD;
#pragma unroll
      for (int r = 0; r < R; ++r) A[spad(idxD + r * NS)] = v[m][r];
    }
  }
  __syncthreads();
}

// In-place CTA transform of NB sequences of power-of-two length N.
template <int DIR, int N, int NB, int T, int LD, int S = 0, int NS = 1>
__device__ __forceinline__ void cta_fft_ct(float2* buf, const float2* __restrict__ tw, int tws) {
  if constexpr (S < ct_nstages(N)) {
    constexpr int R = ct_radix(N, S);
    stage_ct<R, DIR, N, NS, NB, T, LD>(buf, tw, tws);
    cta_fft_ct<DIR, N, NB, T, LD, S + 1, NS * R>(buf, tw, tws);
  }
}
#endif

// Paired real-transform helpers working in place on one row held at
// buf[i + (i >> SH)] (SH = 5: spad, SH = 4: spad16): pair p (0 <= p <= M/2)
// owns elements p and M-p.
// Forward post-processing: Z[0..M) -> X[0..M].
template <int SH = 5>
MC3_HD void r2c_post_pair(float2* buf, int M, int p, const float2* twW, float scale) {
  auto spad = [](int i) { return i + (i >> SH); };
  if (p == 0) {
    const float2 z = buf[spad(0)];
    buf[spad(0)] = c2((z.x + z.y) * scale, 0.0f);
    buf[spad(M)] = c2((z.x - z.y) * scale, 0.0f);
    return;
  }
  const int q = M - p;
  const float2 zp = buf[spad(p)];
  const float2 zq = buf[spad(q)];
  // X[k] = (Z[k] + conj Z[M-k])/2 + w_k (Z[k] - conj Z[M-k]) (-i/2)
  auto one = [&](float2 a, float2 b, int k) {
    const float2 bm = cconj(b);
    const float2 fe = c2(0.5f * (a.x + bm.x), 0.5f * (a.y + bm.y));
    const float2 dd = csub(a, bm);
    const float2 fo = c2(0.5f * dd.y, -0.5f * dd.x);
    return cscale(cadd(fe, cmul(twW[k], fo)), scale);
  };
  const float2 xp = one(zp, zq, p);
  if (q != p) {
    const float2 xq = one(zq, zp, q);
    buf[spad(q)] = xq;
  }
  buf[spad(p)] = xp;
}

// Inverse pre-processing: X[0..M] -> Z[0..M) (imaginary parts of X[0] and
// X[M] ignored unless keep_im, see c2r_pre).
template <int SH = 5>
MC3_HD void c2r_pre_pair(float2* buf, int M, int p, const float2* twW, int keep_im = 0) {
  auto spad = [](int i) { return i + (i >> SH); };
  if (p == 0) {
    const float2 x0 = buf[spad(0)], xm = buf[spad(M)];
    // Z[0] = e + i o with e = X[0] + conj(X[M]), o = X[0] - conj(X[M]); the
    // imaginary parts b0, bM of X[0] and X[M] add -(b0 + bM) to every even
    // output sample and b0 - bM to every odd one
    if (keep_im)
      buf[spad(0)] = c2(x0.x + xm.x - x0.y - xm.y, x0.x - xm.x + x0.y - xm.y);
    else
      buf[spad(0)] = c2(x0.x + xm.x, x0.x - xm.x);
    return;
  }
  const int q = M - p;
  const float2 xp = buf[spad(p)];
  const float2 xq = buf[spad(q)];
  auto one = [&](float2 a, float2 b, int k) {
    const float2 bm = cconj(b);
    const float2 e = cadd(a, bm);
    const float2 o = cmul(csub(a, bm), cconj(twW[k]));
    return c2(e.x - o.y, e.y + o.x);
  };
  const float2 zp = one(xp, xq, p);
  if (q != p) buf[spad(q)] = one(xq, xp, q);
  buf[spad(p)] = zp;
}

// Sequential host driver running the identical stage code (CPU tests).
template <int DIR>
inline float2* fft_host_reference(float2* A, float2* B, const FftDesc& d) {
  int Ns = 1;
  for (int s = 0; s < d.nstages; ++s) {
    const int R = d.radix[s];
    const int per = stage_items(d.n, R);
    for (int j = 0; j < per; ++j) stage_item<DIR>(A, B, d.n, R, Ns, j, d.tw, d.tws, 1);
    float2* t = A; A = B; B = t;
    Ns *= R;
  }
  return A;
}

// ---- real-data helpers (length W = 2M real <-> M+1 complex) -----------
// Forward: Z = FFT_M(x[2m] + i x[2m+1]); X[k] for k in [0, M].
// twW: table e^{-2 pi i k / W} (stride twWs).
MC3_HD float2 r2c_post(const float2* Z, int M, int k, const float2* twW, int twWs) {
  const float2 zk = Z[k == M ? 0 : k];
  const float2 zm = cconj(Z[k == 0 ? 0 : M - k]);
  const float2 fe = c2(0.5f * (zk.x + zm.x), 0.5f * (zk.y + zm.y));
  // fo = (zk - zm) * (-i/2)
  const float2 dd = csub(zk, zm);
  const float2 fo = c2(0.5f * dd.y, -0.5f * dd.x);
  const float2 w = twW[k * twWs];
  return cadd(fe, cmul(w, fo));
}

// Inverse pre-processing: X[0..M] (row of a half spectrum) -> Z[k], k<M.
// The imaginary parts of X[0] and X[M] are ignored, i.e. the result is the
// real part of the inverse of the Hermitian extension of the row -- unless
// keep_im, when they enter Z[0] through the same formula as every other k.
MC3_HD float2 c2r_pre(const float2* X, int M, int k, const float2* twW, int twWs,
                      int keep_im = 0) {
  float2 xa, xb;
  if (k == 0) {
    xa = keep_im ? X[0] : c2(X[0].x, 0.f);
    xb = keep_im ? cconj(X[M]) : c2(X[M].x, 0.f);
  } else {
    xa = X[k];
    xb = cconj(X[M - k]);
  }
  const float2 e = cadd(xa, xb);
  float2 o = csub(xa, xb);
  if (k) o = cmul(o, cconj(twW[k * twWs]));
  // Z = e + i*o
  return c2(e.x - o.y, e.y + o.x);
}

}  // namespace mc3
