// CTF estimation on the motion-corrected sum: the role of FindCtf/
// (CFindCtfMain::DoIt, FindCtf/CFindCtfMain.cpp:49-83), which the reference
// runs on the first (unweighted) sum (Correct/CCorrectFullShift.cpp:129-144,179).
//
// Layout and kernels (per-pixel maps and the search driver in ctf_core.h):
//   * the sum is Fourier-rescaled to a pixel size >= 1.25 A (CRescaleImage)
//     with the row/column FFT passes of fft.cu, into a padded real image;
//   * all 512 x 512 tiles (50 % overlap, CGenAvgSpectrum) are normalised,
//     edge-rounded and transformed in ONE batched R2C; one kernel averages
//     their amplitude spectra in tile order;
//   * background removal (GRmBackground2D) and the full-spectrum Gaussian
//     lowpass are single launches over the 257 x 512 half spectrum;
//   * every sweep of the grid searches (CFindDefocus1D::mBrutalForceSearch,
//     the sweeps of CFindDefocus2D) is one launch that scores all of its
//     candidates at once, one warp (1D) or one CTA (2D) per candidate, over
//     the pixels of the correlation band compacted into a list; the host
//     takes the decisions in the reference's candidate order.  The reference
//     launches and synchronises once per candidate (about 6000 times).
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "ctf_core.h"
#include "engine.h"
#include "fft.cuh"

namespace mc3 {

using namespace ctf;

namespace {

// GPad2D::Pad of the rows that fit the rescaled size (bin 1).
__global__ void k_ctf_pad(const float* __restrict__ img, int nx, float* __restrict__ out, int pitch,
                          int ny) {
  const int y = blockIdx.y;
  if (y >= ny) return;
  for (int x = threadIdx.x + blockIdx.x * blockDim.x; x < pitch; x += blockDim.x * gridDim.x)
    out[(long)y * pitch + x] = x < nx ? img[(long)y * nx + x] : 0.f;
}

// Sum and sum of squares of every 512 x 512 tile (GCalcMoment2D moments 1, 2).
__global__ void __launch_bounds__(256) k_ctf_tile_stats(const float* __restrict__ img, int pitch,
                                                        const int* __restrict__ org, double* stats) {
  const int t = blockIdx.x;
  const int sx = org[2 * t], sy = org[2 * t + 1];
  double a = 0, b = 0;
  for (int i = threadIdx.x; i < kTile * kTile; i += blockDim.x) {
    const float v = img[(long)(sy + i / kTile) * pitch + sx + (i % kTile)];
    a += v;
    b += (double)v * v;
  }
  __shared__ double sa[256], sb[256];
  sa[threadIdx.x] = a;
  sb[threadIdx.x] = b;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      sa[threadIdx.x] += sa[threadIdx.x + o];
      sb[threadIdx.x] += sb[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    stats[2 * t] = sa[0];
    stats[2 * t + 1] = sb[0];
  }
}

// GNormalize2D + GRoundEdge into the padded tile stack [tiles][512][514];
// grid (512 rows, tiles).
__global__ void __launch_bounds__(256) k_ctf_tile_prep(const float* __restrict__ img, int pitch,
                                                       const int* __restrict__ org,
                                                       const double* __restrict__ stats,
                                                       float* __restrict__ tiles) {
  const int y = blockIdx.x, t = blockIdx.y;
  const int sx = org[2 * t], sy = org[2 * t + 1];
  float mean, sd;
  tile_norm(stats[2 * t], stats[2 * t + 1], &mean, &sd);
  float* row = tiles + ((long)t * kTile + y) * kTP;
  const float* src = img + (long)(sy + y) * pitch + sx;
  for (int x = threadIdx.x; x < kTP; x += blockDim.x) {
    const float w = x < kTile ? tile_edge(x, y) : 0.0f;
    row[x] = w == 0.0f ? 0.0f : ((src[x] - mean) / sd) * w;
  }
}

// Amplitude spectra of the tiles averaged in tile order (GCalcSpectrum::DoIt
// + GAddFrames), DC moved to row 256.
__global__ void k_ctf_amp_avg(const float2* __restrict__ spec, int ntiles, float fac,
                              float* __restrict__ avg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kNH) return;
  const int y = i / kCX, x = i % kCX;
  float acc = 0.f;
  for (int t = 0; t < ntiles; ++t) {
    const float2 v = spec[(long)t * kNH + i];
    acc = acc * 1.0f + sqrtf(v.x * v.x + v.y * v.y) * fac;
  }
  avg[((y + kTile / 2) % kTile) * kCX + x] = acc;
}

__global__ void k_ctf_sqrt(const float* __restrict__ in, float* __restrict__ out, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = sqrtf(in[i]);
}

__global__ void k_ctf_rmbg(const float* __restrict__ in, const float* __restrict__ sq, int box,
                           float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kNH) out[i] = remove_background_at(in, sq, box, i);
}

__global__ void k_ctf_full(const float* __restrict__ half, float* __restrict__ full) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kTP * kTile) return;
  const int s = full_source(i);
  full[i] = s < 0 ? 0.f : half[s];
}

__global__ void k_ctf_lowpass(float2* spec, float scale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kNH) return;
  const float f = lowpass_factor(i, scale);
  float2 v = spec[i];
  v.x *= f;
  v.y *= f;
  spec[i] = v;
}

__global__ void k_ctf_take_half(const float* __restrict__ full, float* __restrict__ half) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kNH) half[i] = full[take_half_source(i)];
}

// One warp per 1D candidate: out[c] = (sum cs, sum c^2, sum s^2) over the
// radial average inside [lo, hi) (GCtfCC1D, B = 0).
__global__ void __launch_bounds__(256) k_ctf_cc1d(const float2* __restrict__ cand, int ncand,
                                                  const float* __restrict__ rad, float wave, float cs,
                                                  float lo, float hi, float4* __restrict__ out) {
  const int c = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (c >= ncand) return;  // whole warps leave together
  const float2 p = cand[c];
  float a = 0.f, b = 0.f, d = 0.f;
  for (int x = lane; x < kCX; x += 32) {
    if (!(x >= lo && x < hi)) continue;
    const float v = ctf1d_term(x, p, wave, cs);
    const float s = rad[x];
    a += v * s;
    b += v * v;
    d += s * s;
  }
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
    d += __shfl_xor_sync(0xffffffffu, d, o);
  }
  if (lane == 0) out[c] = make_float4(a, b, d, 0.f);
}

// One CTA per 2D candidate over the nb band pixels (GCalcCTF2D + GCtfCC2D).
__global__ void __launch_bounds__(256) k_ctf_cc2d(const float4* __restrict__ band, int nb,
                                                  const float4* __restrict__ cand, float wave, float cs,
                                                  float4* __restrict__ out) {
  const float4 p = cand[blockIdx.x];
  float a = 0.f, b = 0.f, d = 0.f;
  for (int k = threadIdx.x; k < nb; k += blockDim.x) {
    const float4 e = band[k];
    const float v = ctf2d_term(e, p, wave, cs);
    a += v * e.w;
    b += v * v;
    d += e.w * e.w;
  }
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
    d += __shfl_xor_sync(0xffffffffu, d, o);
  }
  __shared__ float sa[8], sb[8], sd[8];
  const int w = threadIdx.x / 32;
  if ((threadIdx.x & 31) == 0) {
    sa[w] = a;
    sb[w] = b;
    sd[w] = d;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float ta = 0.f, tb = 0.f, td = 0.f;
    for (int i = 0; i < (int)(blockDim.x / 32); ++i) {
      ta += sa[i];
      tb += sb[i];
      td += sd[i];
    }
    out[blockIdx.x] = make_float4(ta, tb, td, 0.f);
  }
}

__global__ void k_ctf_model(float wave, float cs, float mean, float sigma, float azim, float add,
                            float* __restrict__ ctf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kNH) ctf[i] = ctf_model_at(i, wave, cs, mean, sigma, azim, add);
}

// GSpectralCC2D::mGCalc2D, width 10: one CTA per shell.
__global__ void __launch_bounds__(256) k_ctf_shell_cc(const float* __restrict__ ctf,
                                                      const float* __restrict__ sp, float* __restrict__ cc) {
  const int bx = blockIdx.x;
  int lo, hi;
  shell_ring(bx, &lo, &hi);
  double s[6] = {0, 0, 0, 0, 0, 0};
  for (int y = threadIdx.x; y < kTile; y += blockDim.x) {
    const float fy = fabsf(y - kTile * 0.5f);
    if (fy >= hi) continue;
    for (int x = 0; x < kCX && x < hi; ++x) {
      const float r = sqrtf((float)(x * x) + fy * fy);
      if (r < lo || r >= hi) continue;
      const float c = fabsf(ctf[y * kCX + x]) - 0.5f, v = sp[y * kCX + x];
      s[0] += c;
      s[1] += v;
      s[2] += c * v;
      s[3] += c * c;
      s[4] += v * v;
      s[5] += 1;
    }
  }
  __shared__ double sh[6][256];
  for (int k = 0; k < 6; ++k) sh[k][threadIdx.x] = s[k];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int k = 0; k < 6; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double t[6];
    for (int k = 0; k < 6; ++k) t[k] = sh[k][0];
    cc[bx] = shell_cc(t);
  }
}

// The 512 x 512 diagnostic image; grid = 512 rows.
__global__ void k_ctf_embed(const float* __restrict__ full, const float* __restrict__ ctf, float fmin,
                            float fmax, float mean, float gain, float* __restrict__ out) {
  const int y = blockIdx.x;
  for (int x = threadIdx.x; x < kTile; x += blockDim.x)
    out[y * kTile + x] = embed_at(full, ctf, x, y, fmin, fmax, mean, gain);
}

constexpr int kThreads = 256;
inline int blocks(long n) { return (int)((n + kThreads - 1) / kThreads); }

// Scores candidate sweeps on the device (the scorer of ctf::Search).
struct GpuScorer {
  CtfScratch& s;
  cudaStream_t st;
  Model m;
  float lo1 = 0, hi1 = 0;
  int nb = 0;

  int set_radial(const std::vector<float>& rad) {
    MC3_TRY(s.rad.ensure(sizeof(float) * rad.size()));
    MC3_CUDA(cudaMemcpyAsync(s.rad.p, rad.data(), sizeof(float) * rad.size(), cudaMemcpyHostToDevice, st));
    return kOk;
  }
  int set_band(const std::vector<float4>& band) {
    nb = (int)band.size();
    MC3_TRY(s.band.ensure(sizeof(float4) * (band.size() + 1)));
    if (nb)
      MC3_CUDA(cudaMemcpyAsync(s.band.p, band.data(), sizeof(float4) * nb, cudaMemcpyHostToDevice, st));
    return kOk;
  }
  int score1d(const std::vector<float2>& cand, std::vector<float>& cc) {
    const int n = (int)cand.size();
    MC3_TRY(s.cand.ensure(sizeof(float4) * n));
    MC3_TRY(s.res.ensure(sizeof(float4) * n));
    MC3_CUDA(cudaMemcpyAsync(s.cand.p, cand.data(), sizeof(float2) * n, cudaMemcpyHostToDevice, st));
    k_ctf_cc1d<<<ceil_div(n, kThreads / 32), kThreads, 0, st>>>(s.cand.as<float2>(), n, s.rad.as<float>(),
                                                                m.wave, m.cs, lo1, hi1, s.res.as<float4>());
    MC3_CHECK_LAUNCH("k_ctf_cc1d");
    std::vector<float4> r(n);
    MC3_CUDA(cudaMemcpyAsync(r.data(), s.res.p, sizeof(float4) * n, cudaMemcpyDeviceToHost, st));
    MC3_CUDA(cudaStreamSynchronize(st));
    cc.resize(n);
    for (int i = 0; i < n; ++i) {  // GCtfCC1D::DoIt (FindCtf/GCtfCC1D.cu:90-121)
      const double a = r[i].x, b = r[i].y, d = r[i].z;
      cc[i] = (b > 0 && d > 0) ? (float)(a / std::sqrt(b * d)) : 0.f;
    }
    return kOk;
  }
  int score2d(const std::vector<float4>& cand, std::vector<float>& cc) {
    const int n = (int)cand.size();
    cc.clear();
    if (!n) return kOk;
    MC3_TRY(s.cand.ensure(sizeof(float4) * n));
    MC3_TRY(s.res.ensure(sizeof(float4) * n));
    MC3_CUDA(cudaMemcpyAsync(s.cand.p, cand.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, st));
    k_ctf_cc2d<<<n, kThreads, 0, st>>>(s.band.as<float4>(), nb, s.cand.as<float4>(), m.wave, m.cs,
                                       s.res.as<float4>());
    MC3_CHECK_LAUNCH("k_ctf_cc2d");
    std::vector<float4> r(n);
    MC3_CUDA(cudaMemcpyAsync(r.data(), s.res.p, sizeof(float4) * n, cudaMemcpyDeviceToHost, st));
    MC3_CUDA(cudaStreamSynchronize(st));
    cc.resize(n);
    for (int i = 0; i < n; ++i) {  // GCtfCC2D::mGCalc1D (FindCtf/GCtfCC2D.cu:66-92)
      const float sd = sqrtf(r[i].y * r[i].z);
      cc[i] = sd == 0 ? 0.f : r[i].x / sd;
    }
    return kOk;
  }
};

}  // namespace

int estimate_ctf(const float* d_img, int nx, int ny, float pix, float kv, float cs, float ac,
                 float ext_phase, float* res6, float* image512, bool image_on_device, CtfScratch& s,
                 cudaStream_t st) {
  if (!d_img || !res6 || nx < 2 || ny < 2 || pix <= 0) return kEInval;
  if ((nx | ny) & 1) return kEUnsupported;  // the FFT passes take even sizes
  // ---- CRescaleImage::DoIt (FindCtf/CRescaleImage.cpp:28-68) ----
  int nxN, nyN;
  float pixN, bin;
  rescaled_size(nx, ny, pix, &nxN, &nyN, &pixN, &bin);
  const int pitch = (nxN / 2 + 1) * 2, cN = nxN / 2 + 1;
  // ---- tile grid (CGenAvgSpectrum::SetSizes) ----
  int nt[2], off[2], step;
  tile_grid(nxN, nyN, nt, off, &step);
  const int ntx = nt[0], nty = nt[1];
  if (ntx < 1 || nty < 1) return kEUnsupported;  // no 512 x 512 tile
  const int ntiles = ntx * nty;
  const int offx = off[0], offy = off[1];
  MC3_TRY(s.img.ensure(sizeof(float) * pitch * (size_t)nyN));
  float* img = s.img.as<float>();
  if (bin == 1) {
    k_ctf_pad<<<dim3(ceil_div(pitch, kThreads), nyN), kThreads, 0, st>>>(d_img, nx, img, pitch, nyN);
    MC3_CHECK_LAUNCH("k_ctf_pad");
  } else {
    const int cX = nx / 2 + 1;
    MC3_TRY(s.spec.ensure(sizeof(float2) * cX * (size_t)ny));
    float2* sp = s.spec.as<float2>();
    Batch b1{1, 1, 0, nullptr, 0};
    MC3_TRY(row_r2c(d_img, nx, sp, cX, nx, ny, b1, 1.0f, st));
    ColOps fwd{};
    fwd.dir = -1;
    fwd.scale = (float)(1.0 / nx / ny);
    MC3_TRY(col_fft(sp, sp, cX, cX, ny, b1, fwd, st));
    float2* cimg = reinterpret_cast<float2*>(img);
    MC3_TRY(fourier_crop(sp, cX, ny, cimg, cN, nyN, st));
    ColOps inv{};
    inv.dir = 1;
    inv.scale = 1.0f;
    MC3_TRY(col_fft(cimg, cimg, cN, cN, nyN, b1, inv, st));
    MC3_TRY(row_c2r(cimg, cN, img, pitch, nxN, nyN, b1, st));
  }
  // ---- tile spectra and their average (CGenAvgSpectrum::mAverage) ----
  std::vector<int> org(2 * ntiles);
  for (int t = 0; t < ntiles; ++t) {
    org[2 * t] = offx + (t % ntx) * step;
    org[2 * t + 1] = offy + (t / ntx) * step;
  }
  const size_t tile_f = (size_t)kTP * kTile;
  MC3_TRY(s.org.ensure(sizeof(int) * 2 * ntiles));
  MC3_TRY(s.stats.ensure(sizeof(double) * 2 * ntiles));
  MC3_TRY(s.tiles.ensure(sizeof(float) * tile_f * ntiles));
  MC3_CUDA(cudaMemcpyAsync(s.org.p, org.data(), sizeof(int) * 2 * ntiles, cudaMemcpyHostToDevice, st));
  k_ctf_tile_stats<<<ntiles, kThreads, 0, st>>>(img, pitch, s.org.as<int>(), s.stats.as<double>());
  MC3_CHECK_LAUNCH("k_ctf_tile_stats");
  k_ctf_tile_prep<<<dim3(kTile, ntiles), kThreads, 0, st>>>(img, pitch, s.org.as<int>(), s.stats.as<double>(),
                                                           s.tiles.as<float>());
  MC3_CHECK_LAUNCH("k_ctf_tile_prep");
  float2* tsp = s.tiles.as<float2>();
  {
    Batch br{ntiles, ntiles, (long)tile_f, nullptr, (long)kNH};
    MC3_TRY(row_r2c(s.tiles.as<float>(), kTP, tsp, kCX, kTile, kTile, br, 1.0f, st));
    Batch bc{ntiles, ntiles, (long)kNH, nullptr, (long)kNH};
    ColOps fwd{};
    fwd.dir = -1;
    fwd.scale = 1.0f;
    MC3_TRY(col_fft(tsp, tsp, kCX, kCX, kTile, bc, fwd, st));
  }
  MC3_TRY(s.half.ensure(sizeof(float) * 3 * kNH));
  float* raw = s.half.as<float>();
  float* sq = raw + kNH;
  float* half = raw + 2 * kNH;
  k_ctf_amp_avg<<<blocks(kNH), kThreads, 0, st>>>(tsp, ntiles, 1.0f / ntiles, raw);
  MC3_CHECK_LAUNCH("k_ctf_amp_avg");
  // ---- background (CGenAvgSpectrum::mRmBackground) ----
  k_ctf_sqrt<<<blocks(kNH), kThreads, 0, st>>>(raw, sq, kNH);
  k_ctf_rmbg<<<blocks(kNH), kThreads, 0, st>>>(raw, sq, background_box(), half);
  MC3_CHECK_LAUNCH("k_ctf_rmbg");
  // ---- lowpass (CGenAvgSpectrum::mLowpass) ----
  MC3_TRY(s.full.ensure(sizeof(float) * tile_f));
  float* full = s.full.as<float>();
  float2* fsp = s.full.as<float2>();
  k_ctf_full<<<blocks((long)tile_f), kThreads, 0, st>>>(half, full);
  MC3_CHECK_LAUNCH("k_ctf_full");
  {
    Batch b1{1, 1, 0, nullptr, 0};
    MC3_TRY(row_r2c(full, kTP, fsp, kCX, kTile, kTile, b1, 1.0f, st));
    ColOps fwd{};
    fwd.dir = -1;
    fwd.scale = (float)(1.0 / kTile / kTile);
    MC3_TRY(col_fft(fsp, fsp, kCX, kCX, kTile, b1, fwd, st));
    const double tmp = (double)kTile * kTile + (double)kTile * kTile;
    k_ctf_lowpass<<<blocks(kNH), kThreads, 0, st>>>(fsp, (float)(-5.0f / tmp));
    MC3_CHECK_LAUNCH("k_ctf_lowpass");
    ColOps inv{};
    inv.dir = 1;
    inv.scale = 1.0f;
    MC3_TRY(col_fft(fsp, fsp, kCX, kCX, kTile, b1, inv, st));
    MC3_TRY(row_c2r(fsp, kCX, full, kTP, kTile, kTile, b1, st));
  }
  k_ctf_take_half<<<blocks(kNH), kThreads, 0, st>>>(full, half);
  MC3_CHECK_LAUNCH("k_ctf_take_half");
  std::vector<float> hs(kNH);
  MC3_CUDA(cudaMemcpyAsync(hs.data(), half, sizeof(float) * kNH, cudaMemcpyDeviceToHost, st));
  MC3_CUDA(cudaStreamSynchronize(st));
  // ---- fit (CFindCtfMain::mFindCTF, FindCtf/CFindCtfMain.cpp:96-116) ----
  GpuScorer sc{s, st, make_model(kv, cs, ac, pixN)};
  float rr[2];
  res_range(pixN, rr);
  const float res1 = ((kCX - 1) * 2) * pixN;  // CFindDefocus1D::mCorrelate
  sc.lo1 = res1 / rr[0];
  sc.hi1 = res1 / rr[1];
  Search<GpuScorer> search{sc, sc.m};
  Fit fit;
  MC3_TRY(search.run(hs.data(), ext_phase, &fit));
  // ---- resolution (CFindDefocus2D::mCalcCtfRes) ----
  MC3_TRY(s.ctf.ensure(sizeof(float) * (kNH + kCX)));
  float* ctfm = s.ctf.as<float>();
  float* shell_ccs = ctfm + kNH;
  k_ctf_model<<<blocks(kNH), kThreads, 0, st>>>(sc.m.wave, sc.m.cs, 0.5f * (fit.dfmin + fit.dfmax),
                                                0.5f * (fit.dfmax - fit.dfmin), fit.azim, sc.m.amp + fit.ext,
                                                ctfm);
  MC3_CHECK_LAUNCH("k_ctf_model");
  k_ctf_shell_cc<<<kCX, kThreads, 0, st>>>(ctfm, half, shell_ccs);
  MC3_CHECK_LAUNCH("k_ctf_shell_cc");
  std::vector<float> scc(kCX);
  MC3_CUDA(cudaMemcpyAsync(scc.data(), shell_ccs, sizeof(float) * kCX, cudaMemcpyDeviceToHost, st));
  MC3_CUDA(cudaStreamSynchronize(st));
  fit_result(fit, pixN, fit_shell(scc.data()), res6);
  if (!image512) return kOk;
  // ---- diagnostic image (CFindCtfMain::mEmbedCTF + mAddSpectrumToPackage) ----
  double m1 = 0, m2 = 0;
  for (float v : hs) {
    m1 += v;
    m2 += (double)v * v;
  }
  const float mean = (float)(m1 / kNH);
  float sd = (float)(m2 / kNH) - mean * mean;
  sd = sd < 0 ? 0.0f : std::sqrt(sd);
  MC3_TRY(s.out.ensure(sizeof(float) * kTile * kTile));
  k_ctf_embed<<<kTile, kThreads, 0, st>>>(full, ctfm, pixN / rr[0], pixN / rr[1], mean, sd * 1.5f,
                                          s.out.as<float>());
  MC3_CHECK_LAUNCH("k_ctf_embed");
  MC3_CUDA(cudaMemcpyAsync(image512, s.out.p, sizeof(float) * kTile * kTile,
                           image_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
  MC3_CUDA(cudaStreamSynchronize(st));
  return kOk;
}

}  // namespace mc3
