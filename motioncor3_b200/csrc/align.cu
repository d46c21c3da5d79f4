// Alignment kernels: phase tables, aligned sums, group cross-correlation
// with pruned inverse transform, and the sub-pixel peak search.
//
// One launch of each kernel serves every still-active stack (the global
// stack, or every patch stack at once) and every frame group, replacing the
// reference's per-group, per-patch launches and host round trips
// (Align/CAlignStack.cpp:118-192, Align/GCorrelateSum2D.cu:108-140,
// Align/CPeak2D.cpp:39-109).
#include "kernels.cuh"
#include "fft_r16.cuh"

namespace mc3 {

// ---------------------------------------------------------------------
// Separable phase tables (Util/GPhaseShift2D.cu:12-38, 68-79): the
// reference multiplies by e^{i(kx*2pi*sx/Nx + ky'*2pi*sy/Ny)}; the factor
// is split into an x table and a y table computed in FP64.
// ---------------------------------------------------------------------
__global__ void k_phase_tables(const float2* sh, int cmpX, int cmpY, float2* ex, float2* ey,
                               int skip_small) {
  const int item = blockIdx.y;
  const float2 s = sh[item];
  bool unit = false;
  if (skip_small) {
    const double d = sqrtf(s.x * s.x + s.y * s.y);
    unit = d < 0.1;
  }
  const int Nx = (cmpX - 1) * 2;
  const int Ny = cmpY;
  const int n = max(cmpX, cmpY);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (i < cmpX) {
      double sn = 0.0, cs = 1.0;
      if (!unit) sincospi(2.0 * (double)i * (double)s.x / (double)Nx, &sn, &cs);
      ex[(long)item * cmpX + i] = c2((float)cs, (float)sn);
    }
    if (i < cmpY) {
      const int yy = wrap_half(i, cmpY);
      double sn = 0.0, cs = 1.0;
      if (!unit) sincospi(2.0 * (double)yy * (double)s.y / (double)Ny, &sn, &cs);
      ey[(long)item * cmpY + i] = c2((float)cs, (float)sn);
    }
  }
}

int phase_tables(const float2* sh, int items, int cmpX, int cmpY, float2* ex, float2* ey,
                 bool skip_small, cudaStream_t st) {
  const int n = cmpX > cmpY ? cmpX : cmpY;
  dim3 grid(ceil_div(n, 256), items);
  prof::Scope ps("k_phase_tables", (double)items * (cmpX + cmpY) * 8.0, st);
  k_phase_tables<<<grid, 256, 0, st>>>(sh, cmpX, cmpY, ex, ey, skip_small ? 1 : 0);
  MC3_CHECK_LAUNCH("k_phase_tables");
  return kOk;
}

// X * e^{i phi} written as in GPhaseShift2D: (c*x - s*y, c*y + s*x)
__device__ __forceinline__ float2 rot(float2 X, float2 e) {
  return c2(e.x * X.x - e.y * X.y, e.x * X.y + e.y * X.x);
}

// GPhaseShift2D::mGShiftFrame (Util/GPhaseShift2D.cu:12-38): out = X e^{i phi}
// or out += X e^{i phi}.
__global__ void k_phase_apply(const float2* in, float2* out, int cmpX, int cmpY,
                              const float2* ex, const float2* ey, int accumulate) {
  const long n = (long)cmpX * cmpY;
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int x = (int)(k % cmpX), y = (int)(k / cmpX);
  const float2 v = rot(in[k], cmul(ex[x], ey[y]));
  if (accumulate) out[k] = cadd(out[k], v);
  else out[k] = v;
}

int phase_apply(const float2* in, float2* out, int cmpX, int cmpY, const float2* ex,
                const float2* ey, bool accumulate, cudaStream_t st) {
  const long n = (long)cmpX * cmpY;
  prof::Scope ps("k_phase_apply", (double)n * (accumulate ? 24.0 : 16.0), st);
  k_phase_apply<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(in, out, cmpX, cmpY, ex, ey,
                                                            accumulate ? 1 : 0);
  MC3_CHECK_LAUNCH("k_phase_apply");
  return kOk;
}

// ---------------------------------------------------------------------
// Aligned sum (Align/CAlignedSum.cpp:69-126): frames alternate between two
// partial sums (even and odd frame index) that are added at the end.
// ---------------------------------------------------------------------
// Thread (kx, 4 consecutive rows): each frame's x phase factor is read once
// for the 4 rows.  Threads are numbered over (row group, kx) of each stack,
// so no thread idles at the end of a row when cmpX is not a multiple of the
// block size (1025 and 205 at the benchmark geometry); a warp that straddles
// two row groups reads two y factors per frame.
constexpr int kAsRows = 4;
constexpr int kAsThreads = 256;
__global__ void __launch_bounds__(kAsThreads) k_aligned_sum(const float2* __restrict__ spec,
                                                            const int* act,
                                                            const float2* __restrict__ ex,
                                                            const float2* __restrict__ ey, float2* S,
                                                            int cmpX, int cmpY, int N, long sstride) {
  const long nel = (long)cmpX * cmpY;
  const int groups = (cmpY + kAsRows - 1) / kAsRows;
  const long e = (long)blockIdx.x * kAsThreads + threadIdx.x;
  if (e >= (long)groups * cmpX) return;
  const int kx = (int)(e % cmpX);
  const int ky0 = (int)(e / cmpX) * kAsRows;
  const int a = blockIdx.y;
  const float2* X = spec + (long)act[a] * sstride;
  float2 e0[kAsRows], e1[kAsRows];
#pragma unroll
  for (int i = 0; i < kAsRows; ++i) e0[i] = e1[i] = c2(0.f, 0.f);
#pragma unroll 2
  for (int f = 0; f < N; ++f) {
    const long t = (long)a * N + f;
    const float2 exf = ex[t * cmpX + kx];
#pragma unroll
    for (int i = 0; i < kAsRows; ++i) {
      const int ky = ky0 + i;
      if (ky >= cmpY) break;
      const float2 ef = cmul(exf, ey[t * cmpY + ky]);
      const float2 v = rot(X[(long)f * nel + (long)ky * cmpX + kx], ef);
      if (f & 1) e1[i] = cadd(e1[i], v);
      else e0[i] = cadd(e0[i], v);
    }
  }
#pragma unroll
  for (int i = 0; i < kAsRows; ++i) {
    const int ky = ky0 + i;
    if (ky < cmpY) S[(long)a * nel + (long)ky * cmpX + kx] = cadd(e0[i], e1[i]);
  }
}

int aligned_sum(const float2* spec, const int* act, const float2* ex, const float2* ey, float2* S,
                const AlignDims& d, cudaStream_t st) {
  const long nel = (long)d.cmpX * d.cmpY;
  const long threads = (long)ceil_div(d.cmpY, kAsRows) * d.cmpX;
  dim3 grid((unsigned)((threads + kAsThreads - 1) / kAsThreads), d.A);
  prof::Scope ps("k_aligned_sum", (double)d.A * nel * 8.0 * (d.N + 1), st);
  k_aligned_sum<<<grid, kAsThreads, 0, st>>>(spec, act, ex, ey, S, d.cmpX, d.cmpY, d.N,
                                             d.stack_stride);
  MC3_CHECK_LAUNCH("k_aligned_sum");
  return kOk;
}

// ---------------------------------------------------------------------
// Group correlation, column pass (Align/GCorrelateSum2D.cu:13-78):
//   C = conj(G) (S - G) * exp(-B/4 (kx^2 + ky^2) / ((cmpX-1) cmpY)),
//   optional phase-only normalisation, DC = 0, times (-1)^(kx+ky),
// then the inverse FFT along ky; only the seaY rows that the 64x64 search
// window reads are written.
// ---------------------------------------------------------------------
__global__ void __launch_bounds__(256, 2) k_corr_cols(const float2* __restrict__ spec, const int* act,
                            const float2* __restrict__ ex, const float2* __restrict__ ey,
                            const float2* __restrict__ S, const int* gstart, const int* gsize,
                            float bf, int phase_only, float2* T, int cmpX, int H, int N,
                            long sstride, int G, int seaY, int TX, FftDesc dH) {
  extern __shared__ float2 sm[];
  const int ld = H + 1;
  float2* A = sm;
  float2* B = sm + TX * ld;
  const int a = blockIdx.z;
  const int g = blockIdx.y;
  const int x0 = blockIdx.x * TX;
  const long nel = (long)cmpX * H;
  const float2* X = spec + (long)act[a] * sstride;
  const float2* Sa = S + (long)a * nel;
  const int f0 = gstart[g], gs = gsize[g];
  float fFilt0 = -0.25f * bf / ((unsigned)(cmpX - 1) * (unsigned)H);
  for (int t = threadIdx.x; t < TX * H; t += blockDim.x) {
    const int y = t / TX, c = t - y * TX;
    const int x = x0 + c;
    float2 C = c2(0.f, 0.f);
    if (x < cmpX) {
      const long k = (long)y * cmpX + x;
      float2 Gs = c2(0.f, 0.f);
      for (int i = 0; i < gs; ++i) {
        const long tf = (long)a * N + f0 + i;
        const float2 e = cmul(ex[tf * cmpX + x], ey[tf * H + y]);
        const float2 v = rot(X[(long)(f0 + i) * nel + k], e);
        Gs = i ? cadd(Gs, v) : v;
      }
      float2 cs = Sa[k];
      cs.x -= Gs.x;
      cs.y -= Gs.y;
      C.x = Gs.x * cs.x + Gs.y * cs.y;
      C.y = Gs.x * cs.y - Gs.y * cs.x;
      const int yy = wrap_half(y, H);
      float fFilt = expf(fFilt0 * (float)((unsigned)(x * x) + (unsigned)(yy * yy)));
      if (phase_only) {
        float fAmp = sqrtf(C.x * C.x + C.y * C.y);
        fFilt = fFilt / (fAmp + (float)1e-20);
      }
      if (k > 0) {
        C.x *= fFilt;
        C.y *= fFilt;
      } else {
        C = c2(0.f, 0.f);
      }
      const int sgn = ((x + y) % 2 == 0) ? 1 : -1;
      C.x *= sgn;
      C.y *= sgn;
    }
    A[c * ld + y] = C;
  }
  __syncthreads();
  float2* R = cta_fft<1>(A, B, dH, TX, 1, ld);
  const int y0 = (H - seaY) / 2;
  float2* Tg = T + ((long)a * G + g) * seaY * cmpX;
  for (int t = threadIdx.x; t < TX * seaY; t += blockDim.x) {
    const int yi = t / TX, c = t - yi * TX;
    const int x = x0 + c;
    if (x < cmpX) Tg[(long)yi * cmpX + x] = R[c * ld + y0 + yi];
  }
}

// Same computation with the in-place padded FFT (power-of-two cmpY).
__device__ __forceinline__ float2 corr_value(const float2* __restrict__ X,
                                             const float2* __restrict__ ex,
                                             const float2* __restrict__ ey, const float2* Sa,
                                             int a, int N, int f0, int gs, int x, int y, int cmpX,
                                             int H, long nel, float fFilt0, int phase_only) {
  const long k = (long)y * cmpX + x;
  float2 Gs = c2(0.f, 0.f);
  for (int i = 0; i < gs; ++i) {
    const long tf = (long)a * N + f0 + i;
    const float2 e = cmul(ex[tf * cmpX + x], ey[tf * H + y]);
    const float2 v = rot(X[(long)(f0 + i) * nel + k], e);
    Gs = i ? cadd(Gs, v) : v;
  }
  float2 cs = Sa[k];
  cs.x -= Gs.x;
  cs.y -= Gs.y;
  float2 C;
  C.x = Gs.x * cs.x + Gs.y * cs.y;
  C.y = Gs.x * cs.y - Gs.y * cs.x;
  const int yy = wrap_half(y, H);
  float fFilt = expf(fFilt0 * (float)((unsigned)(x * x) + (unsigned)(yy * yy)));
  if (phase_only) {
    float fAmp = sqrtf(C.x * C.x + C.y * C.y);
    fFilt = fFilt / (fAmp + (float)1e-20);
  }
  if (k > 0) {
    C.x *= fFilt;
    C.y *= fFilt;
  } else {
    C = c2(0.f, 0.f);
  }
  const int sgn = ((x + y) % 2 == 0) ? 1 : -1;
  C.x *= sgn;
  C.y *= sgn;
  return C;
}

template <int MAXB>
__global__ void __launch_bounds__(512, 2) k_corr_cols_ip(
    const float2* __restrict__ spec, const int* act, const float2* __restrict__ ex,
    const float2* __restrict__ ey, const float2* __restrict__ S, const int* gstart,
    const int* gsize, float bf, int phase_only, float2* T, int cmpX, int H, int N, long sstride,
    int G, int seaY, int TX, FftDesc dH) {
  extern __shared__ float2 sm[];
  const int ld = spad_len(H);
  const int a = blockIdx.z;
  const int g = blockIdx.y;
  const int x0 = blockIdx.x * TX;
  const long nel = (long)cmpX * H;
  const float2* X = spec + (long)act[a] * sstride;
  const float2* Sa = S + (long)a * nel;
  const int f0 = gstart[g], gs = gsize[g];
  const float fFilt0 = -0.25f * bf / ((unsigned)(cmpX - 1) * (unsigned)H);
  for (int t = threadIdx.x; t < TX * H; t += blockDim.x) {
    const int y = t / TX, c = t - y * TX;
    const int x = x0 + c;
    float2 C = c2(0.f, 0.f);
    if (x < cmpX) C = corr_value(X, ex, ey, Sa, a, N, f0, gs, x, y, cmpX, H, nel, fFilt0, phase_only);
    sm[c * ld + spad(y)] = C;
  }
  __syncthreads();
  cta_fft_inplace<1, MAXB>(sm, dH, TX, ld);
  const int y0 = (H - seaY) / 2;
  float2* Tg = T + ((long)a * G + g) * seaY * cmpX;
  for (int t = threadIdx.x; t < TX * seaY; t += blockDim.x) {
    const int yi = t / TX, c = t - yi * TX;
    const int x = x0 + c;
    if (x < cmpX) Tg[(long)yi * cmpX + x] = sm[c * ld + spad(y0 + yi)];
  }
}

// Compile-time variant for power-of-two cmpY (H).
template <int H>
__global__ void __launch_bounds__(kCtThreads, 2) k_corr_cols_ct(
    const float2* __restrict__ spec, const int* act, const float2* __restrict__ ex,
    const float2* __restrict__ ey, const float2* __restrict__ S, const int* gstart,
    const int* gsize, float bf, int phase_only, float2* T, int cmpX, int N, long sstride, int G,
    int seaY, const float2* __restrict__ tw) {
  constexpr int LD = ct_spad_len(H);
  constexpr int TX = ct_batch(LD);
  extern __shared__ float2 sm[];
  const int a = blockIdx.z;
  const int g = blockIdx.y;
  const int x0 = blockIdx.x * TX;
  const long nel = (long)cmpX * H;
  const float2* X = spec + (long)act[a] * sstride;
  const float2* Sa = S + (long)a * nel;
  const int f0 = gstart[g], gs = gsize[g];
  const float fFilt0 = -0.25f * bf / ((unsigned)(cmpX - 1) * (unsigned)H);
#pragma unroll 4
  for (int t = threadIdx.x; t < TX * H; t += kCtThreads) {
    const int y = t / TX, c = t % TX;
    const int x = x0 + c;
    float2 C = c2(0.f, 0.f);
    if (x < cmpX) C = corr_value(X, ex, ey, Sa, a, N, f0, gs, x, y, cmpX, H, nel, fFilt0, phase_only);
    sm[c * LD + spad(y)] = C;
  }
  __syncthreads();
  cta_fft_ct<1, H, TX, kCtThreads, LD>(sm, tw, 1);
  const int y0 = (H - seaY) / 2;
  float2* Tg = T + ((long)a * G + g) * seaY * cmpX;
  for (int t = threadIdx.x; t < TX * seaY; t += kCtThreads) {
    const int yi = t / TX, c = t % TX;
    const int x = x0 + c;
    if (x < cmpX) Tg[(long)yi * cmpX + x] = sm[c * LD + spad(y0 + yi)];
  }
}

// Radix-16 register variant (fft_r16.cuh): corr_value feeds the first
// stage directly and the last stage stores only the kept window rows.
template <int H>
__global__ void __launch_bounds__(512, 2) k_corr_cols_r16(
    const float2* __restrict__ spec, const int* act, const float2* __restrict__ ex,
    const float2* __restrict__ ey, const float2* __restrict__ S, const int* gstart,
    const int* gsize, float bf, int phase_only, float2* T, int cmpX, int N, long sstride, int G,
    int seaY, const float2* __restrict__ tw) {
  constexpr int NB = 512 / (H / 16);
  constexpr int LD = spad16_col_stride(H, NB);
  extern __shared__ float2 sm[];
  const int a = blockIdx.z;
  const int g = blockIdx.y;
  const int c = threadIdx.x % NB;
  const int j = threadIdx.x / NB;
  const int x = blockIdx.x * NB + c;
  const bool live = x < cmpX;
  const long nel = (long)cmpX * H;
  const float2* X = spec + (long)act[a] * sstride;
  const float2* Sa = S + (long)a * nel;
  const int f0 = gstart[g], gs = gsize[g];
  const float fFilt0 = -0.25f * bf / ((unsigned)(cmpX - 1) * (unsigned)H);
  const int y0 = (H - seaY) / 2;
  float2* Tg = T + ((long)a * G + g) * seaY * cmpX + x;
  auto load = [&](int y) {
    return live ? corr_value(X, ex, ey, Sa, a, N, f0, gs, x, y, cmpX, H, nel, fFilt0, phase_only)
                : c2(0.f, 0.f);
  };
  auto store = [&](int y, float2 v) {
    const int yi = y - y0;
    if (live && yi >= 0 && yi < seaY) Tg[(long)yi * cmpX] = v;
  };
  fft_r16<1, H, false, false>(sm + c * LD, j, tw, 1, load, store);
}

template <int H>
int launch_corr_cols_r16(const float2* spec, const int* act, const float2* ex, const float2* ey,
                         const float2* S, const int* gstart, const int* gsize, float bfactor,
                         int phase_only, float2* T, const AlignDims& d, const float2* tw,
                         cudaStream_t st) {
  constexpr int NB = 512 / (H / 16);
  const size_t smem = (size_t)NB * spad16_col_stride(H, NB) * sizeof(float2);
  MC3_TRY(set_smem_attr(k_corr_cols_r16<H>, smem));
  dim3 grid(ceil_div(d.cmpX, NB), d.G, d.A);
  k_corr_cols_r16<H><<<grid, 512, smem, st>>>(spec, act, ex, ey, S, gstart, gsize, bfactor,
                                              phase_only, T, d.cmpX, d.N, d.stack_stride, d.G,
                                              d.seaY, tw);
  MC3_CHECK_LAUNCH("k_corr_cols_r16");
  return kOk;
}

template <int H>
int launch_corr_cols_ct(const float2* spec, const int* act, const float2* ex, const float2* ey,
                        const float2* S, const int* gstart, const int* gsize, float bfactor,
                        int phase_only, float2* T, const AlignDims& d, const float2* tw,
                        cudaStream_t st) {
  constexpr int LD = ct_spad_len(H);
  constexpr int TX = ct_batch(LD);
  const size_t smem = (size_t)TX * LD * sizeof(float2);
  MC3_TRY(set_smem_attr(k_corr_cols_ct<H>, smem));
  dim3 grid(ceil_div(d.cmpX, TX), d.G, d.A);
  k_corr_cols_ct<H><<<grid, kCtThreads, smem, st>>>(spec, act, ex, ey, S, gstart, gsize, bfactor,
                                                    phase_only, T, d.cmpX, d.N, d.stack_stride,
                                                    d.G, d.seaY, tw);
  MC3_CHECK_LAUNCH("k_corr_cols_ct");
  return kOk;
}

int corr_cols(const float2* spec, const int* act, const float2* ex, const float2* ey,
              const float2* S, const int* gstart, const int* gsize, float bfactor,
              int phase_only, float2* T, const AlignDims& d, cudaStream_t st) {
  FftDesc dH;
  MC3_TRY(make_desc(d.cmpY, d.cmpY, &dH));
  if (r16_enabled() && !getenv("MC3_FFT_PINGPONG") && !getenv("MC3_FFT_RUNTIME_PLAN")) {
    const double bytes = (double)d.A * ((double)d.cmpX * d.cmpY * 8.0 * (d.N + 1) + (double)d.G * d.seaY * d.cmpX * 8.0);
    switch (d.cmpY) {
      case 1024: {
        prof::Scope ps("k_corr_cols_r16<1024>", bytes, st);
        return launch_corr_cols_r16<1024>(spec, act, ex, ey, S, gstart, gsize, bfactor, phase_only, T, d, dH.tw, st);
      }
      case 2048: {
        prof::Scope ps("k_corr_cols_r16<2048>", bytes, st);
        return launch_corr_cols_r16<2048>(spec, act, ex, ey, S, gstart, gsize, bfactor, phase_only, T, d, dH.tw, st);
      }
      case 4096: {
        prof::Scope ps("k_corr_cols_r16<4096>", bytes, st);
        return launch_corr_cols_r16<4096>(spec, act, ex, ey, S, gstart, gsize, bfactor, phase_only, T, d, dH.tw, st);
      }
      default: break;
    }
  }
  if (all_dedicated(dH) && !getenv("MC3_FFT_PINGPONG") && !getenv("MC3_FFT_RUNTIME_PLAN")) {
    prof::Scope ps("k_corr_cols_ct", (double)d.A * ((double)d.cmpX * d.cmpY * 8.0 * (d.N + 1) + (double)d.G * d.seaY * d.cmpX * 8.0), st);
    switch (d.cmpY) {
      case 256: return launch_corr_cols_ct<256>(spec, act, ex, ey, S, gstart, gsize, bfactor, phase_only, T, d, dH.tw, st);
      case 512: return launch_corr_cols_ct<512>(spec, act, ex, ey, S, gstart, gsize, bfactor, phase_only, T, d, dH.tw, st);
      case 1024: return launch_corr_cols_ct<1024>(spec, act, ex, ey, S, gstart, gsize, bfactor, phase_only, T, d, dH.tw, st);
      case 2048: return launch_corr_cols_ct<2048>(spec, act, ex, ey, S, gstart, gsize, bfactor, phase_only, T, d, dH.tw, st);
      case 4096: return launch_corr_cols_ct<4096>(spec, act, ex, ey, S, gstart, gsize, bfactor, phase_only, T, d, dH.tw, st);
      default: break;
    }
  }
  if (all_dedicated(dH) && !getenv("MC3_FFT_PINGPONG")) {
    const int ld = spad_len(d.cmpY);
    int rmin = 8;
    for (int s = 0; s < dH.nstages; ++s) rmin = dH.radix[s] < rmin ? dH.radix[s] : rmin;
    int tx = (2 * 512) / (d.cmpY / rmin);
    const int by_smem = (72 * 1024) / (ld * (int)sizeof(float2));
    if (by_smem < tx) tx = by_smem;
    if (tx > 16) tx = 16;
    if (tx >= 1) {
      const size_t smem = (size_t)tx * ld * sizeof(float2);
      MC3_TRY(set_smem_attr(k_corr_cols_ip<2>, smem));
      dim3 grid(ceil_div(d.cmpX, tx), d.G, d.A);
      prof::Scope ps("k_corr_cols", (double)d.A * ((double)d.cmpX * d.cmpY * 8.0 * (d.N + 1) + (double)d.G * d.seaY * d.cmpX * 8.0), st);
      k_corr_cols_ip<2><<<grid, 512, smem, st>>>(spec, act, ex, ey, S, gstart, gsize, bfactor, phase_only,
                                                 T, d.cmpX, d.cmpY, d.N, d.stack_stride, d.G, d.seaY, tx, dH);
      MC3_CHECK_LAUNCH("k_corr_cols_ip");
      return kOk;
    }
  }
  const int tx = col_tile(d.cmpY);
  const size_t smem = 2 * (size_t)tx * (d.cmpY + 1) * sizeof(float2);
  if (smem > 200 * 1024) return kEUnsupported;
  MC3_TRY(set_smem_attr(k_corr_cols, smem));
  dim3 grid(ceil_div(d.cmpX, tx), d.G, d.A);
  prof::Scope ps("k_corr_cols", (double)d.A * ((double)d.cmpX * d.cmpY * 8.0 * (d.N + 1) + (double)d.G * d.seaY * d.cmpX * 8.0), st);
  k_corr_cols<<<grid, 256, smem, st>>>(spec, act, ex, ey, S, gstart, gsize, bfactor, phase_only,
                                       T, d.cmpX, d.cmpY, d.N, d.stack_stride, d.G, d.seaY, tx, dH);
  MC3_CHECK_LAUNCH("k_corr_cols");
  return kOk;
}

// ---------------------------------------------------------------------
// Row pass of the correlation: real inverse of each kept row, keeping the
// seaX central columns (the window GCorrelateSum2D.cu:130-139 copies).
// ---------------------------------------------------------------------
__global__ void __launch_bounds__(256, 2) k_corr_rows(const float2* __restrict__ T, float* win, int cmpX, int seaX, int seaY,
                            int G, int rows, FftDesc dM, int keep_im) {
  extern __shared__ float2 sm[];
  const int M = cmpX - 1;
  const int ld = M + 1;
  float2* A = sm;
  float2* B = sm + rows * ld;
  const int a = blockIdx.z, g = blockIdx.y;
  const int r0 = blockIdx.x * rows;
  const int nr = min(rows, seaY - r0);
  const float2* src = T + (((long)a * G + g) * seaY + r0) * cmpX;
  for (int t = threadIdx.x; t < nr * cmpX; t += blockDim.x) {
    const int r = t / cmpX, k = t - r * cmpX;
    B[r * ld + k] = src[(long)r * cmpX + k];
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nr * M; t += blockDim.x) {
    const int r = t / M, k = t - r * M;
    A[r * ld + k] = c2r_pre(B + r * ld, M, k, dM.tw, 1, keep_im);
  }
  __syncthreads();
  float2* R = cta_fft<1>(A, B, dM, nr, 1, ld);
  const int Nx = 2 * M;
  const int x0 = (Nx - seaX) / 2;
  float* dst = win + (((long)a * G + g) * seaY + r0) * seaX;
  for (int t = threadIdx.x; t < nr * seaX; t += blockDim.x) {
    const int r = t / seaX, xi = t - r * seaX;
    const int x = x0 + xi;
    const float2 v = R[r * ld + (x >> 1)];
    dst[(long)r * seaX + xi] = (x & 1) ? v.y : v.x;
  }
}

int corr_rows(const float2* T, float* win, const AlignDims& d, cudaStream_t st) {
  const int M = d.cmpX - 1;
  FftDesc dM;
  MC3_TRY(make_desc(M, 2 * M, &dM));
  int rows = row_tile(M);
  if (rows > d.seaY) rows = d.seaY;
  const size_t smem = 2 * (size_t)rows * (M + 1) * sizeof(float2);
  if (smem > 200 * 1024) return kEUnsupported;
  MC3_TRY(set_smem_attr(k_corr_rows, smem));
  dim3 grid(ceil_div(d.seaY, rows), d.G, d.A);
  prof::Scope ps("k_corr_rows", (double)d.A * d.G * d.seaY * (d.cmpX * 8.0 + d.seaX * 4.0), st);
  // the reference inverts the whole correlation with a cufftPlan2d C2R
  // (Align/GCorrelateSum2D.cu:127): its treatment of the rows' DC and
  // Nyquist imaginary parts at this size
  const int keep_im = c2r_keep_edge_imag(2 * M, d.cmpY) ? 1 : 0;
  k_corr_rows<<<grid, 256, smem, st>>>(T, win, d.cmpX, d.seaX, d.seaY, d.G, rows, dM, keep_im);
  MC3_CHECK_LAUNCH("k_corr_rows");
  return kOk;
}

// ---------------------------------------------------------------------
// CPeak2D::DoIt (Align/CPeak2D.cpp:39-109): first index of the maximum,
// pulled one pixel off the border, then separate 1D parabolic fits in x
// and y in FP64; offsets beyond 1 px are dropped.
// ---------------------------------------------------------------------
__global__ void k_peak(const float* win, float2* out, int seaX, int seaY, int G) {
  __shared__ float sv[256];
  __shared__ int si[256];
  const int a = blockIdx.y, g = blockIdx.x;
  const float* img = win + ((long)a * G + g) * seaX * seaY;
  const int n = seaX * seaY;
  float best = img[0];
  int bi = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float v = img[i];
    if (v > best || (v == best && i < bi)) {
      best = v;
      bi = i;
    }
  }
  sv[threadIdx.x] = best;
  si[threadIdx.x] = bi;
  __syncthreads();
  for (int off = blockDim.x / 2; off > 0; off >>= 1) {
    if (threadIdx.x < off) {
      const float v = sv[threadIdx.x + off];
      const int i = si[threadIdx.x + off];
      if (v > sv[threadIdx.x] || (v == sv[threadIdx.x] && i < si[threadIdx.x])) {
        sv[threadIdx.x] = v;
        si[threadIdx.x] = i;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  const int ip = si[0];
  int px = ip % seaX, py = ip / seaX;
  if (px == 0) px = 1;
  if (py == 0) py = 1;
  if (px == seaX - 1) px -= 1;
  if (py == seaY - 1) py -= 1;
  const int ic = py * seaX + px;
  const int xp = ic + 1, xm = ic - 1, yp = ic + seaX, ym = ic - seaX;
  double aa = (img[xp] + img[xm]) * 0.5 - img[ic];
  double bb = (img[xp] - img[xm]) * 0.5;
  double cc = (img[yp] + img[ym]) * 0.5f - img[ic];
  double dd = (img[yp] - img[ym]) * 0.5;
  double cx = -bb / (2 * aa + 1e-30);
  double cy = -dd / (2 * cc + 1e-30);
  if (fabs(cx) > 1) cx = 0;
  if (fabs(cy) > 1) cy = 0;
  const float fx = (float)(px + cx), fy = (float)(py + cy);
  out[(long)a * G + g] = c2(fx - seaX / 2, fy - seaY / 2);
}

int peak_search(const float* win, float2* out, const AlignDims& d, cudaStream_t st) {
  dim3 grid(d.G, d.A);
  prof::Scope ps("k_peak", (double)d.A * d.G * d.seaX * d.seaY * 4.0, st);
  k_peak<<<grid, 256, 0, st>>>(win, out, d.seaX, d.seaY, d.G);
  MC3_CHECK_LAUNCH("k_peak");
  return kOk;
}

}  // namespace mc3
