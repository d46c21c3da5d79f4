// Device state of the learned shift proposal (proposal.cu).
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "proposal_core.h"

namespace mc3 {
namespace proposal {

struct Layer {
  int cin, cout, k, stride, pad;
  long w_off = 0, b_off = 0;  // offsets in the parameter vector
};

class Net {
 public:
  ~Net();
  // spec: groups of (cin, cout, k, stride, pad); He-initialised from seed.
  int create(const std::vector<int>& spec, int nout, unsigned seed);
  // Forward (and, with targets, the batch-summed gradient in d_grad) of a
  // device batch x [batch][cin][H][W]; outputs in d_out, losses in d_loss.
  int run(const float* x, int batch, int H, int W, const float* target, cudaStream_t st);
  // One Adam step with the gradient of the last run() divided by batch.
  int adam_step(int batch, float lr, cudaStream_t st);
  int shapes(int H, int W, std::vector<ConvShape>& s, long* act_elems) const;
  int ensure(int batch, int H, int W, cudaStream_t st);
  void release();

  std::vector<Layer> layers;
  int nout = 0, nfeat = 0;
  long nparams = 0, lw_off = 0, lb_off = 0;
  int adam_t = 0;
  int cap_batch = 0, cap_h = 0, cap_w = 0;
  float *d_params = nullptr, *d_grad = nullptr, *d_m = nullptr, *d_v = nullptr;
  float *d_act = nullptr, *d_pre = nullptr, *d_dact = nullptr, *d_dbuf = nullptr;
  float *d_out = nullptr, *d_feat = nullptr, *d_dout = nullptr, *d_loss = nullptr;
  float *d_target = nullptr, *d_x = nullptr;
};

// Network inputs of n frame pairs (d_pairs [n][2] frame indices into
// frames [nz][H][W] with frame stride fstride floats): each pair binned by
// `bin` and normalised by its mean and standard deviation, x [n][2][H/bin][W/bin].
int pair_inputs(const float* frames, int W, int H, long fstride, const int* d_pairs, int n,
                int bin, float* x, cudaStream_t st);

}  // namespace proposal
}  // namespace mc3
