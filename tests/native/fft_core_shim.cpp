// Host-side shim exposing the libmc3 FFT core (fft_core.cuh) to the CPU
// tests: runs the exact Stockham stage code sequentially so the index
// arithmetic of the device kernels is checked against numpy without a GPU.
#include <cmath>
#include <cstring>
#include <vector>
#include "../../motioncor3_b200/csrc/fft_core.cuh"

using namespace mc3;

static std::vector<float2> make_table(int n) {
  std::vector<float2> t(n);
  for (int k = 0; k < n; ++k) {
    double a = -2.0 * M_PI * (double)k / (double)n;
    t[k].x = (float)std::cos(a);
    t[k].y = (float)std::sin(a);
  }
  return t;
}

extern "C" int shim_factorize(int n, int* radix) { return fft_factorize(n, radix); }

// Complex FFT of length n, dir = -1 forward, +1 inverse (unnormalised).
extern "C" int shim_cfft(const float* in, float* out, int n, int dir) {
  FftDesc d;
  d.n = n;
  d.nstages = fft_factorize(n, d.radix);
  if (d.nstages < 0) return -1;
  std::vector<float2> tw = make_table(n);
  d.tw = tw.data();
  d.tws = 1;
  std::vector<float2> A(n), B(n);
  std::memcpy(A.data(), in, sizeof(float2) * n);
  float2* r = dir < 0 ? fft_host_reference<-1>(A.data(), B.data(), d)
                      : fft_host_reference<1>(A.data(), B.data(), d);
  std::memcpy(out, r, sizeof(float2) * n);
  return 0;
}

// Real forward transform of length W (even): out has W/2+1 complex values.
extern "C" int shim_rfft(const float* in, float* out, int W) {
  const int M = W / 2;
  FftDesc d;
  d.n = M;
  d.nstages = fft_factorize(M, d.radix);
  if (d.nstages < 0) return -1;
  std::vector<float2> tw = make_table(W);
  d.tw = tw.data();
  d.tws = 2;
  std::vector<float2> A(M), B(M);
  for (int m = 0; m < M; ++m) { A[m].x = in[2 * m]; A[m].y = in[2 * m + 1]; }
  float2* Z = fft_host_reference<-1>(A.data(), B.data(), d);
  float2* o = reinterpret_cast<float2*>(out);
  for (int k = 0; k <= M; ++k) o[k] = r2c_post(Z, M, k, tw.data(), 1);
  return 0;
}

// Real inverse (unnormalised) of length W from W/2+1 complex values.
extern "C" int shim_irfft(const float* in, float* out, int W) {
  const int M = W / 2;
  FftDesc d;
  d.n = M;
  d.nstages = fft_factorize(M, d.radix);
  if (d.nstages < 0) return -1;
  std::vector<float2> tw = make_table(W);
  d.tw = tw.data();
  d.tws = 2;
  const float2* X = reinterpret_cast<const float2*>(in);
  std::vector<float2> A(M), B(M);
  for (int k = 0; k < M; ++k) A[k] = c2r_pre(X, M, k, tw.data(), 1);
  float2* z = fft_host_reference<1>(A.data(), B.data(), d);
  for (int m = 0; m < M; ++m) { out[2 * m] = z[m].x; out[2 * m + 1] = z[m].y; }
  return 0;
}

// Real transforms through the padded in-place pair helpers used by the
// in-place row kernels (same layout: element i at buf[spad(i)]).
extern "C" int shim_rfft_pairs(const float* in, float* out, int W) {
  const int M = W / 2;
  FftDesc d;
  d.n = M;
  d.nstages = fft_factorize(M, d.radix);
  std::vector<float2> tw = make_table(W);
  d.tw = tw.data();
  d.tws = 2;
  std::vector<float2> A(M), B(M);
  for (int m = 0; m < M; ++m) { A[m].x = in[2 * m]; A[m].y = in[2 * m + 1]; }
  float2* Z = fft_host_reference<-1>(A.data(), B.data(), d);
  std::vector<float2> buf(spad_len(M + 1));
  for (int m = 0; m < M; ++m) buf[spad(m)] = Z[m];
  for (int p = 0; p <= M / 2; ++p) r2c_post_pair(buf.data(), M, p, tw.data(), 1.0f);
  float2* o = reinterpret_cast<float2*>(out);
  for (int k = 0; k <= M; ++k) o[k] = buf[spad(k)];
  return 0;
}

extern "C" int shim_irfft_pairs(const float* in, float* out, int W) {
  const int M = W / 2;
  FftDesc d;
  d.n = M;
  d.nstages = fft_factorize(M, d.radix);
  std::vector<float2> tw = make_table(W);
  d.tw = tw.data();
  d.tws = 2;
  const float2* X = reinterpret_cast<const float2*>(in);
  std::vector<float2> buf(spad_len(M + 1));
  for (int k = 0; k <= M; ++k) buf[spad(k)] = X[k];
  for (int p = 0; p <= M / 2; ++p) c2r_pre_pair(buf.data(), M, p, tw.data());
  std::vector<float2> A(M), B(M);
  for (int k = 0; k < M; ++k) A[k] = buf[spad(k)];
  float2* z = fft_host_reference<1>(A.data(), B.data(), d);
  for (int m = 0; m < M; ++m) { out[2 * m] = z[m].x; out[2 * m + 1] = z[m].y; }
  return 0;
}

// ---- radix-16 register FFT (fft_r16.cuh), emulated thread by thread: each
// stage runs the read phase of every slot, then the compute/write phase of
// every slot, the order the device driver's barriers enforce.
#include "../../motioncor3_b200/csrc/fft_r16.cuh"
#include <array>

template <int DIR, int N, int S>
static void r16_host_stage(std::vector<float2>& buf, const float* in, float* out,
                           const float2* tw) {
  if constexpr (S < r16_nstages(N)) {
    using St = R16Stage<N, S>;
    const int slots = N / 16;
    std::vector<std::array<float2, 16>> v(slots);
    for (int j = 0; j < slots; ++j)
      for (int i = 0; i < St::NB; ++i)
        for (int r = 0; r < St::R; ++r) {
          const int idx = r16_in_index<N, S>(j, i, r);
          v[j][i * St::R + r] = S == 0 ? c2(in[2 * idx], in[2 * idx + 1]) : buf[spad16(idx)];
        }
    for (int j = 0; j < slots; ++j) {
      float2 u[16];
      for (int q = 0; q < 16; ++q) u[q] = v[j][q];
      if (St::LAST) {
        r16_compute<DIR, N, S>(u, j, tw, 1, [&](int idx, float2 x) {
          out[2 * idx] = x.x;
          out[2 * idx + 1] = x.y;
        });
      } else {
        r16_compute<DIR, N, S>(u, j, tw, 1, [&](int idx, float2 x) { buf[spad16(idx)] = x; });
      }
    }
    r16_host_stage<DIR, N, S + 1>(buf, in, out, tw);
  }
}

template <int N>
static int r16_host(const float* in, float* out, int dir) {
  std::vector<float2> tw = make_table(N);
  std::vector<float2> buf(spad16_len(N));
  if (dir < 0) r16_host_stage<-1, N, 0>(buf, in, out, tw.data());
  else r16_host_stage<1, N, 0>(buf, in, out, tw.data());
  return 0;
}

extern "C" int shim_cfft_r16(const float* in, float* out, int n, int dir) {
  switch (n) {
    case 128: return r16_host<128>(in, out, dir);
    case 256: return r16_host<256>(in, out, dir);
    case 512: return r16_host<512>(in, out, dir);
    case 1024: return r16_host<1024>(in, out, dir);
    case 2048: return r16_host<2048>(in, out, dir);
    case 4096: return r16_host<4096>(in, out, dir);
    default: return -1;
  }
}
