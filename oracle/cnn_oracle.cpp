// FP64 CPU oracle of the learned shift proposal (the warm-start network of
// the accelerated form (4)): a stack of strided convolutions with ReLU, a
// global average pool and a linear head that maps a binned frame pair
// [2][H][W] to shift outputs (global x, y, then per-patch x, y).  Forward and
// backward are written out directly so the device kernels that will train
// the network have a checker for their activations and gradients.
// TEST INFRASTRUCTURE ONLY: nothing in the product links it.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

namespace {

struct Conv {
  int cin, cout, k, stride, pad;
  std::vector<double> w, b;  // w[cout][cin][k][k]
};

struct Net {
  std::vector<Conv> conv;
  int nout = 0, nfeat = 0;
  std::vector<double> lw, lb;  // lw[nout][nfeat]
};

int out_size(int n, const Conv& c) { return (n + 2 * c.pad - c.k) / c.stride + 1; }

// y[co][oy][ox] = b[co] + sum w[co][ci][ky][kx] x[ci][oy*s+ky-p][ox*s+kx-p]
void conv_fwd(const Conv& c, const std::vector<double>& x, int H, int W, std::vector<double>& y, int* Ho,
              int* Wo) {
  const int oh = out_size(H, c), ow = out_size(W, c);
  *Ho = oh;
  *Wo = ow;
  y.assign((size_t)c.cout * oh * ow, 0.0);
  for (int co = 0; co < c.cout; ++co)
    for (int oy = 0; oy < oh; ++oy)
      for (int ox = 0; ox < ow; ++ox) {
        double acc = c.b[co];
        for (int ci = 0; ci < c.cin; ++ci)
          for (int ky = 0; ky < c.k; ++ky) {
            const int iy = oy * c.stride + ky - c.pad;
            if (iy < 0 || iy >= H) continue;
            for (int kx = 0; kx < c.k; ++kx) {
              const int ix = ox * c.stride + kx - c.pad;
              if (ix < 0 || ix >= W) continue;
              acc += c.w[(((size_t)co * c.cin + ci) * c.k + ky) * c.k + kx] * x[((size_t)ci * H + iy) * W + ix];
            }
          }
        y[((size_t)co * oh + oy) * ow + ox] = acc;
      }
}

// Gradients of conv_fwd: dw, db accumulated; dx written (may be skipped).
void conv_bwd(const Conv& c, const std::vector<double>& x, int H, int W, const std::vector<double>& dy, int oh,
              int ow, std::vector<double>& dw, std::vector<double>& db, std::vector<double>* dx) {
  if (dx) dx->assign((size_t)c.cin * H * W, 0.0);
  for (int co = 0; co < c.cout; ++co)
    for (int oy = 0; oy < oh; ++oy)
      for (int ox = 0; ox < ow; ++ox) {
        const double g = dy[((size_t)co * oh + oy) * ow + ox];
        if (g == 0.0) continue;
        db[co] += g;
        for (int ci = 0; ci < c.cin; ++ci)
          for (int ky = 0; ky < c.k; ++ky) {
            const int iy = oy * c.stride + ky - c.pad;
            if (iy < 0 || iy >= H) continue;
            for (int kx = 0; kx < c.k; ++kx) {
              const int ix = ox * c.stride + kx - c.pad;
              if (ix < 0 || ix >= W) continue;
              const size_t wi = (((size_t)co * c.cin + ci) * c.k + ky) * c.k + kx;
              const size_t xi = ((size_t)ci * H + iy) * W + ix;
              dw[wi] += g * x[xi];
              if (dx) (*dx)[xi] += g * c.w[wi];
            }
          }
      }
}

size_t num_params(const Net& n) {
  size_t s = n.lw.size() + n.lb.size();
  for (const Conv& c : n.conv) s += c.w.size() + c.b.size();
  return s;
}

// Parameter order: per conv w then b, then the head's w then b.
template <class F>
void for_params(Net& n, F f) {
  for (Conv& c : n.conv) {
    f(c.w);
    f(c.b);
  }
  f(n.lw);
  f(n.lb);
}

}  // namespace

extern "C" {

// spec: n_conv groups of (cin, cout, k, stride, pad); weights He-initialised
// from `seed`, biases 0.
void* cnn_create(int n_conv, const int* spec, int nout, unsigned seed) {
  Net* n = new Net;
  std::mt19937_64 rng(seed);
  std::normal_distribution<double> N01(0.0, 1.0);
  for (int i = 0; i < n_conv; ++i) {
    Conv c{spec[5 * i], spec[5 * i + 1], spec[5 * i + 2], spec[5 * i + 3], spec[5 * i + 4], {}, {}};
    c.w.resize((size_t)c.cout * c.cin * c.k * c.k);
    const double sd = std::sqrt(2.0 / (c.cin * c.k * c.k));
    for (double& v : c.w) v = sd * N01(rng);
    c.b.assign(c.cout, 0.0);
    n->conv.push_back(c);
  }
  n->nfeat = n_conv ? n->conv.back().cout : 0;
  n->nout = nout;
  n->lw.resize((size_t)nout * n->nfeat);
  const double sd = std::sqrt(1.0 / (n->nfeat > 0 ? n->nfeat : 1));
  for (double& v : n->lw) v = sd * N01(rng);
  n->lb.assign(nout, 0.0);
  return n;
}

void cnn_destroy(void* h) { delete static_cast<Net*>(h); }

long cnn_num_params(void* h) { return (long)num_params(*static_cast<Net*>(h)); }

void cnn_get_params(void* h, double* out) {
  size_t o = 0;
  for_params(*static_cast<Net*>(h), [&](std::vector<double>& v) {
    std::memcpy(out + o, v.data(), sizeof(double) * v.size());
    o += v.size();
  });
}

void cnn_set_params(void* h, const double* in) {
  size_t o = 0;
  for_params(*static_cast<Net*>(h), [&](std::vector<double>& v) {
    std::memcpy(v.data(), in + o, sizeof(double) * v.size());
    o += v.size();
  });
}

// One sample x[C][H][W]: out[nout] (may be NULL); with a target, returns the
// loss 0.5 * |out - target|^2 and, when grad is not NULL, ADDS its gradient
// (parameter order of cnn_get_params) to grad.
double cnn_loss_grad(void* h, const double* x, int C, int H, int W, const double* target, double* grad,
                     double* out) {
  Net& n = *static_cast<Net*>(h);
  const int L = (int)n.conv.size();
  if (L == 0 || n.conv[0].cin != C) return -1.0;
  std::vector<std::vector<double>> act(L + 1), pre(L);
  std::vector<int> hs(L + 1), ws(L + 1);
  act[0].assign(x, x + (size_t)C * H * W);
  hs[0] = H;
  ws[0] = W;
  for (int l = 0; l < L; ++l) {
    conv_fwd(n.conv[l], act[l], hs[l], ws[l], pre[l], &hs[l + 1], &ws[l + 1]);
    act[l + 1] = pre[l];
    for (double& v : act[l + 1]) v = v > 0 ? v : 0.0;  // ReLU
  }
  const int F = n.nfeat, P = hs[L] * ws[L];
  std::vector<double> feat(F, 0.0);
  for (int f = 0; f < F; ++f) {
    double s = 0;
    for (int i = 0; i < P; ++i) s += act[L][(size_t)f * P + i];
    feat[f] = s / P;  // global average pool
  }
  std::vector<double> y(n.nout);
  for (int o = 0; o < n.nout; ++o) {
    double s = n.lb[o];
    for (int f = 0; f < F; ++f) s += n.lw[(size_t)o * F + f] * feat[f];
    y[o] = s;
  }
  if (out) std::memcpy(out, y.data(), sizeof(double) * n.nout);
  if (!target) return 0.0;
  double loss = 0;
  std::vector<double> dy(n.nout);
  for (int o = 0; o < n.nout; ++o) {
    dy[o] = y[o] - target[o];
    loss += 0.5 * dy[o] * dy[o];
  }
  if (!grad) return loss;
  // gradient layout: conv params first, head last
  std::vector<size_t> off(L + 1);
  size_t o0 = 0;
  for (int l = 0; l < L; ++l) {
    off[l] = o0;
    o0 += n.conv[l].w.size() + n.conv[l].b.size();
  }
  off[L] = o0;
  double* glw = grad + off[L];
  double* glb = glw + n.lw.size();
  std::vector<double> dfeat(F, 0.0);
  for (int o = 0; o < n.nout; ++o) {
    glb[o] += dy[o];
    for (int f = 0; f < F; ++f) {
      glw[(size_t)o * F + f] += dy[o] * feat[f];
      dfeat[f] += dy[o] * n.lw[(size_t)o * F + f];
    }
  }
  std::vector<double> d((size_t)F * P);
  for (int f = 0; f < F; ++f)
    for (int i = 0; i < P; ++i) d[(size_t)f * P + i] = dfeat[f] / P;
  for (int l = L - 1; l >= 0; --l) {
    for (size_t i = 0; i < d.size(); ++i)
      if (pre[l][i] <= 0) d[i] = 0.0;  // ReLU'
    const Conv& c = n.conv[l];
    std::vector<double> dw(c.w.size(), 0.0), db(c.b.size(), 0.0), dx;
    conv_bwd(c, act[l], hs[l], ws[l], d, hs[l + 1], ws[l + 1], dw, db, l > 0 ? &dx : nullptr);
    double* g = grad + off[l];
    for (size_t i = 0; i < dw.size(); ++i) g[i] += dw[i];
    for (size_t i = 0; i < db.size(); ++i) g[dw.size() + i] += db[i];
    if (l > 0) d.swap(dx);
  }
  return loss;
}

}  // extern "C"
