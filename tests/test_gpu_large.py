"""GPU parity at the benchmark's frame sizes, against the FP64 oracle.

The benchmark movie (60 x 4096^2, 5x5 patches) runs with an alignment image
binned by 2 (xcf 2048^2: the crop epilogue of the forward column pass and the
scaling of every shift by the bin), 408^2 patch transforms (odd radix 17) and
the 25-patch gather.  These cases run the same geometry on fewer frames, so
that the FP64 oracle finishes in about a minute:

* 12 x 4096^2, -Patch 5 5 -Iter 10 -Bft 500 150, dose weighting, gain;
* 10 x 5760x4092 at 3 e/px/frame, -Patch 7 5 (35 patches): xcf bin 1.998
  (2882 x 2048, a non-power-of-two transform) and 410 x 408 patches.

Shifts within 0.05 px of the oracle's, patch centres identical, and the sums
of the oracle corrected with the GPU's own shifts within 1e-4 relative RMS.
The movies are generated on the GPU (seeded) and copied to the host for the
oracle.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b ** 2)))


def _host_movie(nx, ny, nz, dose, seed, gain, local):
    from motioncor3_b200 import synthetic as S
    m = S.make_movie(nx, ny, nz, dose=dose, seed=seed, gain=gain, local=local, backend="torch")
    frames = m.frames.cpu().numpy()
    g = m.gain.cpu().numpy() if m.gain is not None else None
    return frames, g, m


def _run_and_compare(frames, gain, params, oracle_kw):
    from motioncor3_b200 import api
    from oracle import oracle as O
    with api.MotionCor3(params) as mc:
        if gain is not None:
            mc.set_gain(gain)
        info = mc.plan(frames.shape[2], frames.shape[1], frames.shape[0])
        res = mc.process(frames)
    orc = O.process_movie(frames, gain=gain, **oracle_kw)
    dg = float(np.abs(res.global_shifts - orc["global_shifts"]).max())
    dp = float(np.abs(res.patch_shifts - orc["patch_shifts"]).max())
    print(f"xcf {info['xcf_size']} bin {info['xcf_bin']} patch {info['patch_size']}: "
          f"global max |d| {dg:.4f} px, patch max |d| {dp:.4f} px, "
          f"iterations {res.iterations.tolist()} / oracle {orc['iterations'].tolist()}")
    assert dg <= 0.05, dg
    assert np.array_equal(res.patch_centers, orc["patch_centers"])
    assert dp <= 0.05, dp
    force = dict(global_shifts=res.global_shifts, patch_shifts=res.patch_shifts,
                 patch_centers=res.patch_centers, patch_bad=res.patch_bad)
    same = O.process_movie(frames, gain=gain, force=force, **oracle_kw)
    assert res.n_sums == same["n_sums"]
    for s in range(res.n_sums):
        e = _rel_rms(res.sums[s], same["sums"][s])
        print(f"  sum {s}: rel RMS {e:.2e} against the oracle with the same shifts")
        assert e <= 1e-4, (s, e)
    return res, info


def test_benchmark_geometry_4096_bin2_25_patches(mc3lib, oracle, torch_cuda):
    from motioncor3_b200 import api
    frames, gain, _ = _host_movie(4096, 4096, 12, 0.8, 1201, True, True)
    p = api.Params(patch=(5, 5), iter=10, tol=0.1, bft=(500, 150), fm_dose=1.161, pix_size=0.83,
                   kv=300)
    kw = dict(patch=(5, 5), iter=10, tol=0.1, bft=(500, 150), fm_dose=1.161, pix_size=0.83, kv=300)
    res, info = _run_and_compare(frames, gain, p, kw)
    assert info["xcf_size"] == (2048, 2048) and info["patch_size"] == (408, 408)
    assert abs(info["xcf_bin"][0] - 2.0) < 1e-6 and res.n_patches == 25 and res.n_sums == 3


def test_5760x4092_bin_1998_35_patches(mc3lib, oracle, torch_cuda):
    from motioncor3_b200 import api
    # 3 e/px/frame: enough signal per 410 x 408 patch for the patch
    # alignment to converge, so that the geometry, not the noise, is compared
    frames, gain, _ = _host_movie(5760, 4092, 10, 3.0, 1202, False, True)
    p = api.Params(patch=(7, 5), iter=10, tol=0.1, bft=(500, 150), fm_dose=1.2, pix_size=1.0,
                   kv=300)
    kw = dict(patch=(7, 5), iter=10, tol=0.1, bft=(500, 150), fm_dose=1.2, pix_size=1.0, kv=300)
    res, info = _run_and_compare(frames, gain, p, kw)
    assert info["xcf_size"] == (2882, 2048) and info["patch_size"] == (410, 408) and res.n_patches == 35
