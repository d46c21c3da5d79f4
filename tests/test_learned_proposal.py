"""Oracle of the learned shift proposal (the warm-start network of the
accelerated form (4); oracle/cnn_oracle.cpp): FP64 forward and backward of
strided convolutions + ReLU, global average pool and a linear head.  Its
gradients are checked by central differences (the checker the device
training kernels will be held to), and a short training run on frame pairs
with known shifts shows that it learns a usable first iterate."""
import numpy as np
import pytest


def _pairs(n, size=32, seed=0, max_shift=2.0):
    """Smooth random images and their Fourier-shifted copies, normalised;
    targets are the shifts divided by max_shift."""
    rng = np.random.default_rng(seed)
    ky = np.fft.fftfreq(size)[:, None]
    kx = np.fft.fftfreq(size)[None, :]
    filt = np.exp(-(kx ** 2 + ky ** 2) / (2 * 0.08 ** 2))
    xs, ts = [], []
    for _ in range(n):
        F = np.fft.fft2(rng.standard_normal((size, size))) * filt
        s = rng.uniform(-max_shift, max_shift, 2)
        a = np.real(np.fft.ifft2(F))
        b = np.real(np.fft.ifft2(F * np.exp(-2j * np.pi * (kx * s[0] + ky * s[1]))))
        m, sd = a.mean(), a.std()
        xs.append(np.stack([(a - m) / sd, (b - m) / sd]))
        ts.append(s / max_shift)
    return np.array(xs), np.array(ts)


def test_gradients_match_finite_differences(oracle):
    net = oracle.ShiftNet([(2, 4, 3, 2, 1), (4, 6, 3, 2, 1)], 4, seed=1)
    rng = np.random.default_rng(2)
    x, t = rng.standard_normal((2, 12, 12)), rng.standard_normal(4)
    g = np.zeros(net.n_params)
    net.loss_grad(x, t, g)
    p0 = net.params()
    num = np.zeros_like(p0)
    eps = 1e-6
    for i in range(len(p0)):
        p = p0.copy()
        p[i] += eps
        net.set_params(p)
        lp = net.loss_grad(x, t, np.zeros(len(p0)))
        p[i] -= 2 * eps
        net.set_params(p)
        lm = net.loss_grad(x, t, np.zeros(len(p0)))
        num[i] = (lp - lm) / (2 * eps)
    net.set_params(p0)
    rel = np.abs(g - num) / np.maximum(1e-8, np.abs(g) + np.abs(num))
    assert rel.max() < 1e-5, rel.max()


def test_network_learns_frame_pair_shifts(oracle):
    """Ten epochs of Adam on 256 pairs: the held-out shift error falls well
    below that of predicting no motion."""
    xtr, ttr = _pairs(256, seed=1)
    xte, tte = _pairs(64, seed=2)
    net = oracle.ShiftNet([(2, 8, 5, 2, 2), (8, 16, 3, 2, 1), (16, 16, 3, 2, 1)], 2, seed=3)
    p = net.params()
    m, v = np.zeros_like(p), np.zeros_like(p)
    lr, b1, b2, step = 3e-3, 0.9, 0.999, 0
    for ep in range(10):
        idx = np.random.default_rng(ep).permutation(len(xtr))
        for bs in range(0, len(idx), 16):
            g = np.zeros_like(p)
            for i in idx[bs:bs + 16]:
                net.loss_grad(xtr[i], ttr[i], g)
            g /= 16
            step += 1
            m = b1 * m + (1 - b1) * g
            v = b2 * v + (1 - b2) * g * g
            p -= lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + 1e-8)
            net.set_params(p)
    pred = np.array([net.forward(x) for x in xte])
    err = np.sqrt(np.mean((pred - tte) ** 2))
    base = np.sqrt(np.mean(tte ** 2))
    assert err < 0.45 * base, (err, base)


@pytest.mark.parametrize("seed", [21, 24])
def test_warm_start_keeps_the_cold_result(oracle, seed):
    """The aligner started from a first iterate (the proposal's role) ends
    at the cold-start shifts within 0.05 px and never needs more iterations
    (at least two always run).  On these small-drift movies the cold start
    itself needs only three, so the gain a proposal can bring here is at most
    one iteration."""
    from motioncor3_b200 import synthetic as S
    m = S.make_movie(256, 256, 14, dose=5.0, seed=seed)
    spec = np.stack([oracle.rfft2(f.astype(np.float64)) for f in m.frames])
    cold, it0 = oracle.iterative_align(spec, 1, 15, 0.05, 150.0)
    warm, it1 = oracle.iterative_align(spec, 1, 15, 0.05, 150.0, init=cold)
    assert it1 <= it0 and it1 >= 2
    assert np.abs(warm - cold).max() <= 0.05


@pytest.mark.parametrize("layers,size", [([(2, 4, 3, 2, 1), (4, 6, 3, 2, 1)], 12),
                                         ([(2, 8, 5, 2, 2), (8, 16, 3, 2, 1), (16, 16, 3, 2, 1)], 32),
                                         ([(2, 3, 4, 3, 0), (3, 5, 3, 1, 1)], 17)])
def test_device_core_matches_oracle(oracle, proposal_shim, layers, size):
    """The per-element gathers the device kernels are built from
    (csrc/proposal_core.h: conv_fwd_at, conv_dx_at, conv_dw_at, conv_db_at,
    relu_grad), assembled into a whole pass in double, give the oracle's
    output, loss and gradient (strides 1-3, padding 0-2, odd sizes)."""
    import ctypes
    net = oracle.ShiftNet(layers, 5, seed=4)
    rng = np.random.default_rng(5)
    x = rng.standard_normal((2, size, size))
    t = rng.standard_normal(5)
    p = net.params()
    g_ref = np.zeros(net.n_params)
    loss_ref = net.loss_grad(x, t, g_ref)
    out_ref = net.forward(x)
    spec = np.array(layers, np.int32).ravel()
    g = np.zeros(net.n_params)
    out = np.zeros(5)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    loss = proposal_shim.shim_proposal_loss_grad(len(layers), P(spec), 5, P(p), P(x), 2, size, size, P(t),
                                                 P(g), P(out))
    assert abs(loss - loss_ref) <= 1e-12 * max(1.0, abs(loss_ref))
    assert np.allclose(out, out_ref, rtol=1e-12, atol=1e-12)
    assert np.abs(g - g_ref).max() <= 1e-10 * np.abs(g_ref).max()
