// Learned shift proposal on the device: forward, backward and Adam training
// of the proposal network (strided convolutions + ReLU, global average
// pool, linear head; the same network as the FP64 oracle), whose output
// warm-starts the full-frame alignment (mc3_set_first_iterate).
//
// Every activation, gradient and weight element is computed by one thread
// from the gathers of proposal_core.h (no atomics, FP32 accumulation in a
// fixed order, so a batch's gradient is deterministic); weight gradients
// are block reductions over the batch and the output pixels.  Layout:
// activations [batch][C][H][W], weights [cout][cin][k][k], head [nout][F].
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "kernels.cuh"
#include "proposal.h"
#include "proposal_core.h"

namespace mc3 {
namespace proposal {

namespace {

constexpr int kThreads = 256;

// pre[n][co][oy][ox] = conv(x)[n]; act = max(pre, 0)
__global__ void k_conv_fwd(const float* __restrict__ x, const float* __restrict__ w,
                           const float* __restrict__ b, ConvShape s, int batch, float* pre,
                           float* act) {
  const long per = (long)s.cout * s.oh * s.ow;
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= per * batch) return;
  const int n = (int)(i / per);
  const long r = i - n * per;
  const int co = (int)(r / ((long)s.oh * s.ow));
  const int oy = (int)((r / s.ow) % s.oh), ox = (int)(r % s.ow);
  const float v = conv_fwd_at(x + (long)n * s.cin * s.H * s.W, w, b, s, co, oy, ox);
  pre[i] = v;
  act[i] = v > 0.0f ? v : 0.0f;
}

// dx[n][ci][iy][ix] of the layer input, times ReLU'(pre_in) of the layer
// below (pre_in null for the network input: no gradient needed there).
__global__ void k_conv_dx(const float* __restrict__ dy, const float* __restrict__ w, ConvShape s,
                          int batch, const float* __restrict__ pre_in, float* dx) {
  const long per = (long)s.cin * s.H * s.W;
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= per * batch) return;
  const int n = (int)(i / per);
  const long r = i - n * per;
  const int ci = (int)(r / ((long)s.H * s.W));
  const int iy = (int)((r / s.W) % s.H), ix = (int)(r % s.W);
  const float g = conv_dx_at(dy + (long)n * s.cout * s.oh * s.ow, w, s, ci, iy, ix);
  dx[i] = relu_grad(g, pre_in[i]);
}

// dw[co][ci][ky][kx] (blockIdx.x = weight index; blockIdx.x == nw: the
// biases, one per thread group) summed over the batch.
__global__ void k_conv_dw(const float* __restrict__ dy, const float* __restrict__ x, ConvShape s,
                          int batch, float* dw, float* db) {
  __shared__ float red[kThreads];
  const int nw = s.cout * s.cin * s.k * s.k;
  const int wi = blockIdx.x;
  float acc = 0.0f;
  const long npix = (long)s.oh * s.ow;
  if (wi < nw) {
    const int kx = wi % s.k, ky = (wi / s.k) % s.k, ci = (wi / (s.k * s.k)) % s.cin,
              co = wi / (s.k * s.k * s.cin);
    for (long t = threadIdx.x; t < npix * batch; t += blockDim.x) {
      const int n = (int)(t / npix);
      const long p = t - n * npix;
      const int oy = (int)(p / s.ow), ox = (int)(p % s.ow);
      const int iy = oy * s.stride + ky - s.pad, ix = ox * s.stride + kx - s.pad;
      if (iy < 0 || iy >= s.H || ix < 0 || ix >= s.W) continue;
      acc += dy[((long)n * s.cout + co) * npix + p] *
             x[(((long)n * s.cin + ci) * s.H + iy) * s.W + ix];
    }
  } else {
    const int co = wi - nw;
    for (long t = threadIdx.x; t < npix * batch; t += blockDim.x) {
      const int n = (int)(t / npix);
      acc += dy[((long)n * s.cout + co) * npix + (t - n * npix)];
    }
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (wi < nw) dw[wi] = red[0];
    else db[wi - nw] = red[0];
  }
}

// Pool + head + loss for sample n (one CTA): feat = mean over pixels of
// act[F][P]; out = lb + lw feat; with targets, loss_n = 0.5 |out - t|^2,
// dout = out - t, the head's gradient contributions per sample (summed by
// k_head_grad) and the gradient of the pooled features spread back over
// the pixels (dact, times ReLU' of the last layer).
__global__ void k_head(const float* __restrict__ act, const float* __restrict__ pre, int F, int P,
                       const float* __restrict__ lw, const float* __restrict__ lb, int nout,
                       const float* __restrict__ target, float* out, float* feat_out,
                       float* dout, float* loss, float* dact) {
  extern __shared__ float sh[];
  float* feat = sh;          // [F]
  float* dfeat = sh + F;     // [F]
  float* dy = sh + 2 * F;    // [nout]
  const int n = blockIdx.x;
  const float* a = act + (long)n * F * P;
  for (int f = threadIdx.x; f < F; f += blockDim.x) {
    float s = 0.0f;
    for (int i = 0; i < P; ++i) s += a[(long)f * P + i];
    feat[f] = s / P;
    feat_out[(long)n * F + f] = feat[f];
  }
  __syncthreads();
  for (int o = threadIdx.x; o < nout; o += blockDim.x) {
    float s = lb[o];
    for (int f = 0; f < F; ++f) s += lw[(long)o * F + f] * feat[f];
    out[(long)n * nout + o] = s;
    dy[o] = target ? s - target[(long)n * nout + o] : 0.0f;
    if (target) dout[(long)n * nout + o] = dy[o];
  }
  __syncthreads();
  if (!target) return;
  if (threadIdx.x == 0) {
    float l = 0.0f;
    for (int o = 0; o < nout; ++o) l += 0.5f * dy[o] * dy[o];
    loss[n] = l;
  }
  for (int f = threadIdx.x; f < F; f += blockDim.x) {
    float s = 0.0f;
    for (int o = 0; o < nout; ++o) s += dy[o] * lw[(long)o * F + f];
    dfeat[f] = s / P;
  }
  __syncthreads();
  const float* pr = pre + (long)n * F * P;
  float* d = dact + (long)n * F * P;
  for (long i = threadIdx.x; i < (long)F * P; i += blockDim.x)
    d[i] = relu_grad(dfeat[i / P], pr[i]);
}

// Head gradients summed over the batch: glw[o][f] = sum_n dout[n][o] feat[n][f],
// glb[o] = sum_n dout[n][o].
__global__ void k_head_grad(const float* __restrict__ dout, const float* __restrict__ feat, int F,
                            int nout, int batch, float* glw, float* glb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nout * F) {
    const int o = i / F, f = i % F;
    float s = 0.0f;
    for (int n = 0; n < batch; ++n) s += dout[(long)n * nout + o] * feat[(long)n * F + f];
    glw[i] = s;
  } else if (i < nout * F + nout) {
    const int o = i - nout * F;
    float s = 0.0f;
    for (int n = 0; n < batch; ++n) s += dout[(long)n * nout + o];
    glb[o] = s;
  }
}

// Adam (Kingma & Ba 2015) on all parameters: the batch-summed gradient
// scaled by 1/batch.
__global__ void k_adam(float* p, const float* g, float* m, float* v, long n, float lr, float b1,
                       float b2, float eps, float scale, float c1, float c2) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i] * scale;
  m[i] = b1 * m[i] + (1.0f - b1) * gi;
  v[i] = b2 * v[i] + (1.0f - b2) * gi * gi;
  p[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
}

// Network input of a frame pair: both frames binned by `bin` (block sums),
// then normalised together by the pair's mean and standard deviation
// (one CTA per sample; x [n][2][bh][bw], frames [nz][H][W]).
__global__ void k_pair_input(const float* __restrict__ frames, int W, int H, long fstride,
                             const int* __restrict__ pairs, int bin, float* x) {
  __shared__ double red[2][kThreads];
  const int n = blockIdx.x;
  const int bw = W / bin, bh = H / bin;
  const long np = (long)bw * bh;
  float* xo = x + (long)n * 2 * np;
  double s = 0.0, s2 = 0.0;
  for (int c = 0; c < 2; ++c) {
    const float* f = frames + (long)pairs[2 * n + c] * fstride;
    for (long i = threadIdx.x; i < np; i += blockDim.x) {
      const int by = (int)(i / bw), bx = (int)(i % bw);
      float acc = 0.0f;
      for (int yy = 0; yy < bin; ++yy)
        for (int xx = 0; xx < bin; ++xx) acc += f[(long)(by * bin + yy) * W + bx * bin + xx];
      xo[c * np + i] = acc;
      s += acc;
      s2 += (double)acc * acc;
    }
  }
  red[0][threadIdx.x] = s;
  red[1][threadIdx.x] = s2;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) {
      red[0][threadIdx.x] += red[0][threadIdx.x + h];
      red[1][threadIdx.x] += red[1][threadIdx.x + h];
    }
    __syncthreads();
  }
  const double mean = red[0][0] / (2.0 * np);
  const double var = red[1][0] / (2.0 * np) - mean * mean;
  const float inv = (float)(1.0 / sqrt(var > 1e-12 ? var : 1e-12));
  for (long i = threadIdx.x; i < 2 * np; i += blockDim.x) xo[i] = (xo[i] - (float)mean) * inv;
}

unsigned blocks(long n) { return (unsigned)((n + kThreads - 1) / kThreads); }

}  // namespace

// ---------------------------------------------------------------------------
Net::~Net() { release(); }

void Net::release() {
  for (float** p : {&d_params, &d_grad, &d_m, &d_v, &d_act, &d_pre, &d_dact, &d_dbuf, &d_out,
                    &d_feat, &d_dout, &d_loss, &d_target, &d_x})
    if (*p) {
      cudaFree(*p);
      *p = nullptr;
    }
  cap_batch = 0;
}

int Net::create(const std::vector<int>& spec, int nout_, unsigned seed) {
  if (spec.size() % 5 || spec.empty() || nout_ < 1) return kEInval;
  release();
  layers.clear();
  for (size_t i = 0; i < spec.size(); i += 5) {
    Layer L;
    L.cin = spec[i], L.cout = spec[i + 1], L.k = spec[i + 2], L.stride = spec[i + 3],
    L.pad = spec[i + 4];
    if (L.cin < 1 || L.cout < 1 || L.k < 1 || L.stride < 1 || L.pad < 0) return kEInval;
    if (!layers.empty() && layers.back().cout != L.cin) return kEInval;
    layers.push_back(L);
  }
  nout = nout_;
  nfeat = layers.back().cout;
  // parameter offsets: per layer w then b, then the head's w then b (the
  // oracle's order)
  long o = 0;
  for (Layer& L : layers) {
    L.w_off = o;
    o += (long)L.cout * L.cin * L.k * L.k;
    L.b_off = o;
    o += L.cout;
  }
  lw_off = o;
  o += (long)nout * nfeat;
  lb_off = o;
  o += nout;
  nparams = o;
  // He initialisation from `seed` (weights), zero biases
  std::vector<float> h(nparams, 0.0f);
  std::mt19937_64 rng(seed);
  std::normal_distribution<double> N01(0.0, 1.0);
  for (const Layer& L : layers) {
    const double sd = std::sqrt(2.0 / (L.cin * L.k * L.k));
    for (long i = 0; i < (long)L.cout * L.cin * L.k * L.k; ++i) h[L.w_off + i] = (float)(sd * N01(rng));
  }
  const double sd = std::sqrt(1.0 / nfeat);
  for (long i = 0; i < (long)nout * nfeat; ++i) h[lw_off + i] = (float)(sd * N01(rng));
  MC3_CUDA(cudaMalloc(&d_params, sizeof(float) * nparams));
  MC3_CUDA(cudaMalloc(&d_grad, sizeof(float) * nparams));
  MC3_CUDA(cudaMalloc(&d_m, sizeof(float) * nparams));
  MC3_CUDA(cudaMalloc(&d_v, sizeof(float) * nparams));
  MC3_CUDA(cudaMemcpy(d_params, h.data(), sizeof(float) * nparams, cudaMemcpyHostToDevice));
  MC3_CUDA(cudaMemset(d_m, 0, sizeof(float) * nparams));
  MC3_CUDA(cudaMemset(d_v, 0, sizeof(float) * nparams));
  adam_t = 0;
  return kOk;
}

// Shapes of every layer for inputs of H x W; activation element counts.
int Net::shapes(int H, int W, std::vector<ConvShape>& s, long* act_elems) const {
  s.clear();
  long tot = 0;
  int h = H, w = W;
  for (const Layer& L : layers) {
    ConvShape c;
    c.cin = L.cin, c.cout = L.cout, c.k = L.k, c.stride = L.stride, c.pad = L.pad;
    c.H = h, c.W = w;
    c.oh = conv_out(h, L.k, L.stride, L.pad);
    c.ow = conv_out(w, L.k, L.stride, L.pad);
    if (c.oh < 1 || c.ow < 1) return kEInval;
    s.push_back(c);
    tot += (long)c.cout * c.oh * c.ow;
    h = c.oh;
    w = c.ow;
  }
  *act_elems = tot;
  return kOk;
}

int Net::ensure(int batch, int H, int W, cudaStream_t st) {
  (void)st;
  long act = 0;
  std::vector<ConvShape> s;
  MC3_TRY(shapes(H, W, s, &act));
  long maxin = (long)layers[0].cin * H * W;
  for (const ConvShape& c : s) maxin = std::max(maxin, (long)c.cin * c.H * c.W);
  if (batch <= cap_batch && H == cap_h && W == cap_w) return kOk;
  for (float** p : {&d_act, &d_pre, &d_dact, &d_dbuf, &d_out, &d_feat, &d_dout, &d_loss,
                    &d_target, &d_x})
    if (*p) {
      cudaFree(*p);
      *p = nullptr;
    }
  MC3_CUDA(cudaMalloc(&d_act, sizeof(float) * act * batch));
  MC3_CUDA(cudaMalloc(&d_pre, sizeof(float) * act * batch));
  MC3_CUDA(cudaMalloc(&d_dact, sizeof(float) * std::max(act, maxin) * batch));
  MC3_CUDA(cudaMalloc(&d_dbuf, sizeof(float) * std::max(act, maxin) * batch));
  MC3_CUDA(cudaMalloc(&d_out, sizeof(float) * nout * batch));
  MC3_CUDA(cudaMalloc(&d_feat, sizeof(float) * nfeat * batch));
  MC3_CUDA(cudaMalloc(&d_dout, sizeof(float) * nout * batch));
  MC3_CUDA(cudaMalloc(&d_loss, sizeof(float) * batch));
  MC3_CUDA(cudaMalloc(&d_target, sizeof(float) * nout * batch));
  MC3_CUDA(cudaMalloc(&d_x, sizeof(float) * (long)layers[0].cin * H * W * batch));
  cap_batch = batch;
  cap_h = H;
  cap_w = W;
  return kOk;
}

// Forward of a batch x [batch][cin][H][W] (device) -> d_out; with targets
// (device [batch][nout]) also the loss per sample and the batch-summed
// gradient in d_grad.
int Net::run(const float* x, int batch, int H, int W, const float* target, cudaStream_t st) {
  std::vector<ConvShape> s;
  long act = 0;
  MC3_TRY(shapes(H, W, s, &act));
  MC3_TRY(ensure(batch, H, W, st));
  const int L = (int)layers.size();
  std::vector<long> aoff(L + 1, 0);  // activation offsets (per batch, all samples)
  for (int l = 0; l < L; ++l) aoff[l + 1] = aoff[l] + (long)s[l].cout * s[l].oh * s[l].ow * batch;
  const float* in = x;
  for (int l = 0; l < L; ++l) {
    const long n = (long)s[l].cout * s[l].oh * s[l].ow * batch;
    prof::Scope ps("k_proposal_conv_fwd", (double)n * 4.0 * 2.0, st);
    k_conv_fwd<<<blocks(n), kThreads, 0, st>>>(in, d_params + layers[l].w_off,
                                               d_params + layers[l].b_off, s[l], batch,
                                               d_pre + aoff[l], d_act + aoff[l]);
    MC3_CHECK_LAUNCH("k_proposal_conv_fwd");
    in = d_act + aoff[l];
  }
  const int P = s[L - 1].oh * s[L - 1].ow;
  const size_t shm = sizeof(float) * (2 * nfeat + nout);
  {
    prof::Scope ps("k_proposal_head", (double)batch * nfeat * P * 4.0, st);
    k_head<<<batch, kThreads, shm, st>>>(d_act + aoff[L - 1], d_pre + aoff[L - 1], nfeat, P,
                                         d_params + lw_off, d_params + lb_off, nout, target, d_out,
                                         d_feat, d_dout, d_loss, d_dact);
    MC3_CHECK_LAUNCH("k_proposal_head");
  }
  if (!target) return kOk;
  {
    const int n = nout * nfeat + nout;
    k_head_grad<<<blocks(n), kThreads, 0, st>>>(d_dout, d_feat, nfeat, nout, batch,
                                                d_grad + lw_off, d_grad + lb_off);
    MC3_CHECK_LAUNCH("k_proposal_head_grad");
  }
  // backward through the convolutions: d_dact holds dL/dpre of layer l
  float* dcur = d_dact;
  float* dnext = d_dbuf;
  for (int l = L - 1; l >= 0; --l) {
    const float* xin = l > 0 ? d_act + aoff[l - 1] : x;
    const int nw = s[l].cout * s[l].cin * s[l].k * s[l].k;
    {
      prof::Scope ps("k_proposal_conv_dw", (double)nw * batch * s[l].oh * s[l].ow * 8.0, st);
      k_conv_dw<<<nw + s[l].cout, kThreads, 0, st>>>(dcur, xin, s[l], batch,
                                                      d_grad + layers[l].w_off,
                                                      d_grad + layers[l].b_off);
      MC3_CHECK_LAUNCH("k_proposal_conv_dw");
    }
    if (l > 0) {
      const long n = (long)s[l].cin * s[l].H * s[l].W * batch;
      prof::Scope ps("k_proposal_conv_dx", (double)n * 8.0, st);
      k_conv_dx<<<blocks(n), kThreads, 0, st>>>(dcur, d_params + layers[l].w_off, s[l], batch,
                                                d_pre + aoff[l - 1], dnext);
      MC3_CHECK_LAUNCH("k_proposal_conv_dx");
      std::swap(dcur, dnext);
    }
  }
  return kOk;
}

int Net::adam_step(int batch, float lr, cudaStream_t st) {
  ++adam_t;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - std::pow(b1, (float)adam_t), c2 = 1.0f - std::pow(b2, (float)adam_t);
  k_adam<<<blocks(nparams), kThreads, 0, st>>>(d_params, d_grad, d_m, d_v, nparams, lr, b1, b2,
                                               1e-8f, 1.0f / batch, c1, c2);
  MC3_CHECK_LAUNCH("k_proposal_adam");
  return kOk;
}

int pair_inputs(const float* frames, int W, int H, long fstride, const int* d_pairs, int n,
                int bin, float* x, cudaStream_t st) {
  if (bin < 1 || W / bin < 1 || H / bin < 1 || n < 1) return kEInval;
  prof::Scope ps("k_proposal_pair_input", (double)n * 2.0 * W * H * 4.0, st);
  k_pair_input<<<n, kThreads, 0, st>>>(frames, W, H, fstride, d_pairs, bin, x);
  MC3_CHECK_LAUNCH("k_proposal_pair_input");
  return kOk;
}

}  // namespace proposal
}  // namespace mc3
