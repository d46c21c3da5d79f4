"""The learned shift proposal on the GPU (mc3_proposal_*, csrc/proposal.cu)
and its use as the warm start of the full-frame alignment
(mc3_set_first_iterate).

* The device forward and backward (FP32) against the FP64 oracle
  (oracle/cnn_oracle.cpp) with the same parameters: outputs, loss and every
  gradient entry.
* Training on the GPU with the library's kernels on frame pairs of 512
  synthetic movies whose labels are the plain aligner's own shifts (each
  batch flipped or transposed at random, the shift label with it); on
  held-out movies the proposal's error against the plain aligner is stated
  and must beat predicting no motion by a wide margin.
* The warm start: with the proposal's first iterate the aligner runs at most
  three iterations and keeps the plain aligner's shifts within 0.05 px (up
  to a translation of the whole movie, which global mode does not fix); when
  it has not converged the plain aligner runs from zero (every iteration
  counted).  The iterations used are stated beside the cold start's, and the
  movies whose warm start converged used no more iterations than cold.
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SPEC = [(2, 8, 5, 2, 2), (8, 16, 3, 2, 1), (16, 16, 3, 2, 1), (16, 16, 3, 2, 1)]
# the trained network: 128^2 pairs -> 4^2 x 64 features -> pooled -> (dx, dy)
TRAIN_SPEC = [(2, 16, 5, 2, 2), (16, 32, 3, 2, 1), (32, 64, 3, 2, 1), (64, 64, 3, 2, 1),
              (64, 64, 3, 2, 1)]


@pytest.mark.parametrize("layers,size,batch", [
    ([(2, 4, 3, 2, 1), (4, 6, 3, 2, 1)], 12, 3),
    ([(2, 3, 4, 3, 0), (3, 5, 3, 1, 1)], 17, 2),
    (SPEC, 64, 4)])
def test_device_gradients_match_fp64_oracle(mc3lib, oracle, torch_cuda, layers, size, batch):
    from motioncor3_b200 import api
    dev = api.ShiftProposal(layers, 5, seed=3)
    ref = oracle.ShiftNet(layers, 5, seed=3)
    ref.set_params(dev.params().astype(np.float64))  # the device's FP32 parameters exactly
    rng = np.random.default_rng(size)
    x = rng.standard_normal((batch, 2, size, size)).astype(np.float32)
    t = rng.standard_normal((batch, 5)).astype(np.float32)
    g_ref = np.zeros(ref.n_params)
    loss_ref = sum(ref.loss_grad(x[i].astype(np.float64), t[i].astype(np.float64), g_ref)
                   for i in range(batch))
    out_ref = np.array([ref.forward(x[i].astype(np.float64)) for i in range(batch)])
    loss, g, out = dev.loss_grad(x, t)
    err_g = np.abs(g - g_ref).max() / np.abs(g_ref).max()
    print(f"{len(layers)} layers, {size}^2 x {batch}: loss {loss:.6g} vs {loss_ref:.6g}, "
          f"max gradient error {err_g:.2e} of the largest entry")
    assert abs(loss - loss_ref) <= 1e-5 * max(1.0, abs(loss_ref))
    assert np.abs(out - out_ref).max() <= 1e-5 * max(1.0, np.abs(out_ref).max())
    assert err_g <= 1e-4


def _movies(n, seed0, nz=16, size=256):
    """Movies with larger, jumpier drifts than the default generator's,
    generated on the GPU (frames as CUDA tensors)."""
    from motioncor3_b200 import synthetic as S
    return [S.make_movie(size, size, nz, dose=4.0, seed=seed0 + i, drift_step=1.5, jump=6.0,
                         backend="torch", device="cuda")
            for i in range(n)]


def _pairs_and_labels(torch, api, movies, shifts, bin_, per_movie=None, seed=0):
    """Inputs (frame f, frame g) and targets s_f - s_g (px / 4): per_movie
    random ordered pairs of distinct frames (training), or g = the central
    frame (per_movie None)."""
    rng = np.random.default_rng(seed)
    xs, ts = [], []
    for m, s in zip(movies, shifts):
        nz, ny, nx = m.frames.shape
        ref = nz // 2
        if per_movie:
            every = np.array([[f, g] for f in range(nz) for g in range(nz) if f != g], np.int32)
            pairs = every[rng.choice(len(every), per_movie, replace=False)]
        else:
            pairs = np.array([[f, ref] for f in range(nz)], np.int32)
        fr = m.frames.contiguous()
        x = torch.empty((len(pairs), 2, ny // bin_, nx // bin_), dtype=torch.float32, device="cuda")
        api.ShiftProposal.pair_inputs(fr, pairs, bin_, x)
        xs.append(x)
        ts.append(torch.from_numpy(((s[pairs[:, 0]] - s[pairs[:, 1]]) / 4.0).astype(np.float32)).cuda())
    return torch.cat(xs), torch.cat(ts)


def test_trained_proposal_warm_starts_the_aligner(mc3lib, torch_cuda):
    torch = torch_cuda
    from motioncor3_b200 import api
    p = api.Params(iter=15, tol=0.05, bft=(150, 100), pix_size=1.0)
    train, test = _movies(512, 500), _movies(8, 900)
    with api.MotionCor3(p) as mc:
        lab_tr = [mc.process(m.frames).global_shifts for m in train]
        cold = [mc.process(m.frames) for m in test]
    bin_ = 2
    xtr, ttr = _pairs_and_labels(torch, api, train, lab_tr, bin_, per_movie=64)
    xte, tte = _pairs_and_labels(torch, api, test, [c.global_shifts for c in cold], bin_)
    frames_test = [m.frames.cpu().numpy() for m in test]
    del train
    net = api.ShiftProposal(TRAIN_SPEC, 2, seed=11)
    gen = torch.Generator(device="cuda").manual_seed(0)
    aug = np.random.default_rng(1)
    losses = []
    steps = 7000                      # 64-pair batches drawn from 32k pairs
    t0 = time.perf_counter()
    for st in range(steps):
        i = torch.randint(0, xtr.shape[0], (64,), device="cuda", generator=gen)
        xb, tb = xtr[i], ttr[i].clone()
        # the same flip / transpose of both frames moves the shift with them
        k = int(aug.integers(0, 8))
        if k & 1:
            xb, tb[:, 0] = xb.flip(-1), -tb[:, 0]
        if k & 2:
            xb, tb[:, 1] = xb.flip(-2), -tb[:, 1]
        if k & 4:
            xb, tb = xb.transpose(-1, -2), tb[:, [1, 0]]
        lr = 2e-3 if st < 5000 else 4e-4
        losses.append(net.train_step(xb.contiguous(), tb.contiguous(), lr=lr))
    train_s = time.perf_counter() - t0
    pred = net.predict(xte.contiguous()) * 4.0
    truth = tte.cpu().numpy() * 4.0
    err = float(np.sqrt(np.mean((pred - truth) ** 2)))
    base = float(np.sqrt(np.mean(truth ** 2)))
    print(f"proposal on held-out movies: {err:.3f} px RMS against the plain aligner's shifts "
          f"(no-motion guess {base:.3f} px); training loss {np.mean(losses[:24]):.3f} -> "
          f"{np.mean(losses[-24:]):.3f} over {len(losses)} GPU steps ({train_s:.0f} s)")
    assert np.mean(losses[-24:]) < 0.5 * np.mean(losses[:24])
    assert err < 0.5 * base
    warm_iters, cold_iters, kept, worst, offs = [], [], [], 0.0, []
    with api.MotionCor3(p) as mc:
        for k, (fr, c) in enumerate(zip(frames_test, cold)):
            nz = fr.shape[0]
            d = pred[k * nz:(k + 1) * nz].astype(np.float64)
            # first iterate: the plain aligner's convention (its shifts of
            # these movies have about zero mean), in full-frame pixels
            mc.set_first_iterate((d - d.mean(0)).astype(np.float32), max_iter=3)
            w = mc.process(fr)
            assert w.first_iterate in (1, 2)
            # global-mode shifts are not made relative to a frame (neither
            # here nor in the reference), so a warm start can end at the same
            # alignment translated as a whole: compared up to that offset,
            # which is reported
            dd = w.global_shifts.astype(np.float64) - c.global_shifts
            offs.append(np.round(dd.mean(0), 3).tolist())
            worst = max(worst, float(np.abs(dd - dd.mean(0)).max()))
            warm_iters.append(int(w.iterations[0]))
            cold_iters.append(int(c.iterations[0]))
            kept.append(w.first_iterate == 1)
    print(f"iterations: cold {cold_iters}, warm {warm_iters} (warm start kept: {kept}); "
          f"max |warm - cold| after each movie's mean offset {worst:.4f} px; "
          f"mean warm - cold per movie {offs}")
    assert worst <= 0.05
    assert all(wi <= ci for wi, ci, k in zip(warm_iters, cold_iters, kept) if k)
