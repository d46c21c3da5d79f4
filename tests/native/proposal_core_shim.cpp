// Host-side shim over libmc3's proposal-network core
// (motioncor3_b200/csrc/proposal_core.h): a whole forward and backward pass
// built from the per-element gather functions the device kernels use, in
// double, with the parameter layout of the FP64 oracle (oracle/cnn_oracle.cpp:
// per convolution its weights then biases, then the head's weights and
// biases), so the CPU tests compare them value for value.
#include <cstring>
#include <vector>
#include "../../motioncor3_b200/csrc/proposal_core.h"

using namespace mc3::proposal;

extern "C" double shim_proposal_loss_grad(int n_conv, const int* spec, int nout, const double* params,
                                          const double* x, int C, int H, int W, const double* target,
                                          double* grad, double* out) {
  std::vector<ConvShape> sh(n_conv);
  std::vector<const double*> wp(n_conv), bp(n_conv);
  size_t off = 0;
  int h = H, w = W;
  for (int l = 0; l < n_conv; ++l) {
    ConvShape& s = sh[l];
    s.cin = spec[5 * l];
    s.cout = spec[5 * l + 1];
    s.k = spec[5 * l + 2];
    s.stride = spec[5 * l + 3];
    s.pad = spec[5 * l + 4];
    s.H = h;
    s.W = w;
    s.oh = conv_out(h, s.k, s.stride, s.pad);
    s.ow = conv_out(w, s.k, s.stride, s.pad);
    h = s.oh;
    w = s.ow;
    wp[l] = params + off;
    off += (size_t)s.cout * s.cin * s.k * s.k;
    bp[l] = params + off;
    off += s.cout;
  }
  if (n_conv == 0 || sh[0].cin != C) return -1.0;
  const int F = sh[n_conv - 1].cout, P = h * w;
  const double* lw = params + off;
  const double* lb = lw + (size_t)nout * F;
  std::vector<std::vector<double>> act(n_conv + 1), pre(n_conv);
  act[0].assign(x, x + (size_t)C * H * W);
  for (int l = 0; l < n_conv; ++l) {
    const ConvShape& s = sh[l];
    pre[l].resize((size_t)s.cout * s.oh * s.ow);
    for (int co = 0; co < s.cout; ++co)
      for (int oy = 0; oy < s.oh; ++oy)
        for (int ox = 0; ox < s.ow; ++ox)
          pre[l][((size_t)co * s.oh + oy) * s.ow + ox] = conv_fwd_at(act[l].data(), wp[l], bp[l], s, co, oy, ox);
    act[l + 1] = pre[l];
    for (double& v : act[l + 1]) v = v > 0 ? v : 0.0;
  }
  std::vector<double> feat(F, 0.0), y(nout);
  for (int f = 0; f < F; ++f) {
    double s = 0;
    for (int i = 0; i < P; ++i) s += act[n_conv][(size_t)f * P + i];
    feat[f] = s / P;
  }
  for (int o = 0; o < nout; ++o) {
    double s = lb[o];
    for (int f = 0; f < F; ++f) s += lw[(size_t)o * F + f] * feat[f];
    y[o] = s;
  }
  if (out) std::memcpy(out, y.data(), sizeof(double) * nout);
  if (!target) return 0.0;
  double loss = 0;
  std::vector<double> dy(nout);
  for (int o = 0; o < nout; ++o) {
    dy[o] = y[o] - target[o];
    loss += 0.5 * dy[o] * dy[o];
  }
  if (!grad) return loss;
  double* glw = grad + off;
  double* glb = glw + (size_t)nout * F;
  std::vector<double> dfeat(F, 0.0);
  for (int o = 0; o < nout; ++o) {
    glb[o] += dy[o];
    for (int f = 0; f < F; ++f) {
      glw[(size_t)o * F + f] += dy[o] * feat[f];
      dfeat[f] += dy[o] * lw[(size_t)o * F + f];
    }
  }
  std::vector<double> d((size_t)F * P);
  for (int f = 0; f < F; ++f)
    for (int i = 0; i < P; ++i) d[(size_t)f * P + i] = dfeat[f] / P;
  size_t goff = off;
  for (int l = n_conv - 1; l >= 0; --l) {
    const ConvShape& s = sh[l];
    for (size_t i = 0; i < d.size(); ++i) d[i] = relu_grad(d[i], pre[l][i]);
    const size_t nw = (size_t)s.cout * s.cin * s.k * s.k;
    goff -= nw + s.cout;
    double* gw = grad + goff;
    double* gb = gw + nw;
    for (int co = 0; co < s.cout; ++co) {
      gb[co] += conv_db_at(d.data(), s, co);
      for (int ci = 0; ci < s.cin; ++ci)
        for (int ky = 0; ky < s.k; ++ky)
          for (int kx = 0; kx < s.k; ++kx)
            gw[((size_t)(co * s.cin + ci) * s.k + ky) * s.k + kx] += conv_dw_at(d.data(), act[l].data(), s, co, ci, ky, kx);
    }
    if (l == 0) break;
    std::vector<double> dx((size_t)s.cin * s.H * s.W);
    for (int ci = 0; ci < s.cin; ++ci)
      for (int iy = 0; iy < s.H; ++iy)
        for (int ix = 0; ix < s.W; ++ix)
          dx[((size_t)ci * s.H + iy) * s.W + ix] = conv_dx_at(d.data(), wp[l], s, ci, iy, ix);
    d.swap(dx);
  }
  return loss;
}
