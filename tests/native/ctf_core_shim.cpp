// Host-side shim over libmc3's CTF core (motioncor3_b200/csrc/ctf_core.h):
// the per-pixel maps of the CTF kernels and the search driver, run on the CPU
// with a scorer that evaluates each candidate sweep sequentially, so the CPU
// tests check the device path's index arithmetic and decision logic against
// the oracle and the reference's own drivers without a GPU.
#include <cmath>
#include <thread>
#include <vector>
#include "../../motioncor3_b200/csrc/ctf_core.h"

using namespace mc3::ctf;

namespace {

struct CpuScorer {
  Model m;
  float lo1 = 0, hi1 = 0;
  std::vector<float> rad;
  std::vector<float4> band;
  int set_radial(const std::vector<float>& r) {
    rad = r;
    return 0;
  }
  int set_band(const std::vector<float4>& b) {
    band = b;
    return 0;
  }
  int score1d(const std::vector<float2>& cand, std::vector<float>& cc) {
    cc.resize(cand.size());
    for (size_t c = 0; c < cand.size(); ++c) {
      double a = 0, b = 0, d = 0;
      for (int x = 0; x < kCX; ++x) {
        if (!(x >= lo1 && x < hi1)) continue;
        const float v = ctf1d_term(x, cand[c], m.wave, m.cs), s = rad[x];
        a += v * s;
        b += v * v;
        d += s * s;
      }
      cc[c] = (b > 0 && d > 0) ? (float)(a / std::sqrt(b * d)) : 0.f;
    }
    return 0;
  }
  int score2d(const std::vector<float4>& cand, std::vector<float>& cc) {
    cc.assign(cand.size(), 0.f);
    const int nt = 8;
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t)
      th.emplace_back([&, t] {
        for (size_t c = t; c < cand.size(); c += nt) {
          double a = 0, b = 0, d = 0;
          for (const float4& e : band) {
            const float v = ctf2d_term(e, cand[c], m.wave, m.cs);
            a += v * e.w;
            b += v * v;
            d += e.w * e.w;
          }
          const float sd = sqrtf((float)b * (float)d);
          cc[c] = sd == 0 ? 0.f : (float)a / sd;
        }
      });
    for (auto& x : th) x.join();
    return 0;
  }
};

void shell_ccs(const float* ctf, const float* sp, float* cc) {
  for (int bx = 0; bx < kCX; ++bx) {
    int lo, hi;
    shell_ring(bx, &lo, &hi);
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int y = 0; y < kTile; ++y) {
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
    cc[bx] = shell_cc(s);
  }
}

}  // namespace

extern "C" {

// The device path's fit of a half spectrum: res6 as the _Ctf.txt line, fit4 =
// (defocus min px, defocus max px, azimuth rad, extra phase rad).
int shim_ctf_search(const float* half, float pix, float kv, float cs, float ac, float ext_phase, float* res6,
                    float* fit4) {
  CpuScorer sc;
  sc.m = make_model(kv, cs, ac, pix);
  float rr[2];
  res_range(pix, rr);
  const float res1 = ((kCX - 1) * 2) * pix;
  sc.lo1 = res1 / rr[0];
  sc.hi1 = res1 / rr[1];
  Search<CpuScorer> s{sc, sc.m};
  Fit fit;
  if (s.run(half, ext_phase, &fit)) return 1;
  std::vector<float> ctf(kNH), cc(kCX);
  for (int i = 0; i < kNH; ++i)
    ctf[i] = ctf_model_at(i, sc.m.wave, sc.m.cs, 0.5f * (fit.dfmin + fit.dfmax), 0.5f * (fit.dfmax - fit.dfmin),
                          fit.azim, sc.m.amp + fit.ext);
  shell_ccs(ctf.data(), half, cc.data());
  fit_result(fit, pix, fit_shell(cc.data()), res6);
  fit4[0] = fit.dfmin;
  fit4[1] = fit.dfmax;
  fit4[2] = fit.azim;
  fit4[3] = fit.ext;
  return 0;
}

// Rescaled size and tile grid: out7 = (nxN, nyN, ntx, nty, offx, offy, step);
// pixN.
void shim_ctf_geometry(int nx, int ny, float pix, int* out7, float* pix_n) {
  float bin;
  rescaled_size(nx, ny, pix, &out7[0], &out7[1], pix_n, &bin);
  tile_grid(out7[0], out7[1], &out7[2], &out7[4], &out7[6]);
}

// k_ctf_tile_stats + k_ctf_tile_prep for one tile at (sx, sy) of a padded
// image: the normalised, edge-rounded tile [512][514].
void shim_ctf_tile(const float* img, int pitch, int sx, int sy, float* tile) {
  double a = 0, b = 0;
  for (int i = 0; i < kTile * kTile; ++i) {
    const float v = img[(long)(sy + i / kTile) * pitch + sx + (i % kTile)];
    a += v;
    b += (double)v * v;
  }
  float mean, sd;
  tile_norm(a, b, &mean, &sd);
  for (int y = 0; y < kTile; ++y)
    for (int x = 0; x < kTP; ++x) {
      const float w = x < kTile ? tile_edge(x, y) : 0.0f;
      const float* src = img + (long)(sy + y) * pitch + sx;
      tile[y * kTP + x] = w == 0.0f ? 0.0f : ((src[x] - mean) / sd) * w;
    }
}

void shim_ctf_remove_background(const float* raw, float* out) {
  std::vector<float> sq(kNH);
  for (int i = 0; i < kNH; ++i) sq[i] = sqrtf(raw[i]);
  for (int i = 0; i < kNH; ++i) out[i] = remove_background_at(raw, sq.data(), background_box(), i);
}

void shim_ctf_full(const float* half, float* full) {
  for (int i = 0; i < kTP * kTile; ++i) {
    const int s = full_source(i);
    full[i] = s < 0 ? 0.f : half[s];
  }
}

void shim_ctf_lowpass_factors(float* out) {
  const double tmp = (double)kTile * kTile + (double)kTile * kTile;
  for (int i = 0; i < kNH; ++i) out[i] = lowpass_factor(i, (float)(-5.0f / tmp));
}

void shim_ctf_take_half(const float* full, float* half) {
  for (int i = 0; i < kNH; ++i) half[i] = full[take_half_source(i)];
}

void shim_ctf_radial(const float* half, float* rad) {
  for (int r = 0; r < kCX; ++r) rad[r] = radial_at(half, r);
}

// The diagnostic image from the lowpassed full spectrum ([512][514]), the half
// spectrum and the fit (fit4 as shim_ctf_search returns it).
void shim_ctf_image(const float* full, const float* half, float pix, float kv, float cs, float ac,
                    const float* fit4, float* out) {
  const Model m = make_model(kv, cs, ac, pix);
  std::vector<float> ctf(kNH);
  for (int i = 0; i < kNH; ++i)
    ctf[i] = ctf_model_at(i, m.wave, m.cs, 0.5f * (fit4[0] + fit4[1]), 0.5f * (fit4[1] - fit4[0]), fit4[2],
                          m.amp + fit4[3]);
  double m1 = 0, m2 = 0;
  for (int i = 0; i < kNH; ++i) {
    m1 += half[i];
    m2 += (double)half[i] * half[i];
  }
  const float mean = (float)(m1 / kNH);
  float sd = (float)(m2 / kNH) - mean * mean;
  sd = sd < 0 ? 0.0f : std::sqrt(sd);
  float rr[2];
  res_range(pix, rr);
  for (int y = 0; y < kTile; ++y)
    for (int x = 0; x < kTile; ++x)
      out[y * kTile + x] = embed_at(full, ctf.data(), x, y, pix / rr[0], pix / rr[1], mean, sd * 1.5f);
}

}  // extern "C"
