"""The FP64 oracle pinned before it is trusted: its FFT against numpy, its
solver against the reference's own known-answer test, its host bookkeeping
against golden vectors produced by the reference's own host code, and its
whole path on small synthetic movies."""
import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("shape", [(64, 64), (96, 128), (408, 408), (410, 408), (256, 512)])
def test_oracle_fft2_matches_numpy(oracle, shape):
    ny, nx = shape
    rng = np.random.default_rng(nx * ny)
    img = rng.standard_normal((ny, nx))
    spec = oracle.rfft2(img, normalise=True)
    ref = np.fft.rfft2(img) / (nx * ny)
    assert np.abs(spec - ref).max() < 1e-12 * np.abs(ref).max() * nx
    half = rng.standard_normal((ny, nx // 2 + 1)) + 1j * rng.standard_normal((ny, nx // 2 + 1))
    back = oracle.irfft2(half, nx)
    refb = np.fft.irfft2(half, s=(ny, nx)) * nx * ny
    assert np.abs(back - refb).max() < 1e-10 * np.abs(refb).max()


def test_oracle_cfft_prime_lengths(oracle):
    for n in (17, 31, 41, 131, 2882):
        x = np.random.default_rng(n).standard_normal(n) + 0j
        assert np.allclose(oracle.cfft(x, -1), np.fft.fft(x), atol=1e-9 * n)


def test_lin_eqs_reference_kat(oracle):
    kat = json.load(open(os.path.join(GOLD, "lin_eqs_kat.json")))
    ok, sol = oracle.lin_eqs(np.array(kat["coeff"]), np.array(kat["vals"]))
    assert ok
    assert np.allclose(sol, kat["solution"], atol=0.5 * 10 ** -kat["solution_decimals"] + 1e-4)


def test_oracle_host_bookkeeping_golden(oracle):
    g = json.load(open(os.path.join(GOLD, "host_bookkeeping.json")))
    for c in g["peak2d"]:
        w = np.array(c["window"], np.float32).reshape(64, 64)
        assert np.array_equal(oracle.peak2d(w), np.array(c["shift"], np.float32))
    for c in g["remove_spikes"]:
        x, y = oracle.remove_spikes(np.array(c["x"]), np.array(c["y"]))
        assert np.array_equal(x, np.array(c["x_out"], np.float32))
        assert np.array_equal(y, np.array(c["y_out"], np.float32))
    for c in g["patch_shifts"]:
        N, P = c["N"], c["P"]
        raw = np.array(c["raw"], np.float32).reshape(P, N, 2)
        cen = np.array(c["centers"], np.float32).reshape(P, 2)
        tab = np.ascontiguousarray(raw.transpose(1, 0, 2))
        rel = oracle.patch_make_relative(tab)
        assert np.array_equal(rel, np.array(c["shifts"], np.float32).reshape(N, P, 2))
        bad = oracle.patch_detect_bads(rel, cen, 4096, 4096)
        assert np.array_equal(bad, np.array(c["bad"], np.uint8).reshape(N, P))


def test_oracle_recovers_drift(oracle):
    from motioncor3_b200 import synthetic as S
    m = S.make_movie(256, 256, 20, dose=6.0, seed=11)
    r = oracle.process_movie(m.frames, iter=10, tol=0.05, bft=(150, 100), pix_size=1.0)
    est = r["global_shifts"] - r["global_shifts"][10]
    true = -(m.drift - m.drift[10])
    # the reference smooths the trajectory twice, so a jittery random walk is
    # followed only to about a pixel
    assert np.abs(est - true).max() < 1.5
    assert np.corrcoef(est[:, 0], true[:, 0])[0, 1] > 0.9
    assert r["n_sums"] == 1 and r["sums"][0].min() >= 0


def test_oracle_patch_and_dose_paths_run(oracle):
    from motioncor3_b200 import synthetic as S
    m = S.make_movie(256, 256, 12, dose=4.0, seed=5, gain=True, local=True)
    r = oracle.process_movie(m.frames, gain=m.gain, patch=(3, 3), iter=4, tol=0.2,
                             bft=(150, 100), fm_dose=1.0, pix_size=1.0, kv=300)
    assert r["n_sums"] == 3
    assert r["patch_shifts"].shape == (12, 9, 2)
    assert np.isfinite(r["sums"]).all()
    # with forced shifts the oracle reproduces its own sums
    f = oracle.process_movie(m.frames, gain=m.gain, patch=(3, 3), iter=4, tol=0.2,
                             bft=(150, 100), fm_dose=1.0, pix_size=1.0, kv=300,
                             force=dict(global_shifts=r["global_shifts"],
                                        patch_shifts=r["patch_shifts"],
                                        patch_centers=r["patch_centers"],
                                        patch_bad=r["patch_bad"]))
    assert np.array_equal(f["sums"], r["sums"])


def test_patch_sum_sensitivity_to_shift_rounding(oracle):
    """Patch-mode sums are pinned by nearest-pixel gathers of untruncated
    patch shifts (Correct/GCorrectPatchShift.cu:17-66): moving every nonzero
    patch shift by ~1e-6 px -- FP32 rounding of the peak fit -- changes the
    sums by ~1e-4 relative RMS, while shifts of 1e-7 leave them unchanged.
    This is why patch-mode sums are compared to the reference program with
    a 1e-3 bound (global mode keeps 1e-4)."""
    from motioncor3_b200 import synthetic as S
    m = S.make_movie(256, 256, 8, dose=4.0, seed=33, gain=False, local=True)
    kw = dict(patch=(3, 3), iter=4, tol=0.2, bft=(500, 150), pix_size=1.0)
    r0 = oracle.process_movie(m.frames, **kw)
    ps0 = r0["patch_shifts"]
    rng = np.random.default_rng(0)
    rels = {}
    for eps in (1e-7, 1e-5):
        ps = ps0 + np.where(ps0 != 0, rng.normal(0, eps, ps0.shape), 0).astype(np.float32)
        r1 = oracle.process_movie(m.frames, force=dict(global_shifts=r0["global_shifts"], patch_shifts=ps,
                                                       patch_centers=r0["patch_centers"],
                                                       patch_bad=r0["patch_bad"]), **kw)
        a, b = r0["sums"][0].astype(np.float64), r1["sums"][0].astype(np.float64)
        rels[eps] = np.sqrt(np.mean((a - b) ** 2) / np.mean(a ** 2))
    assert rels[1e-7] < 1e-5
    assert rels[1e-5] > 1e-4


def test_oracle_split_sums_partition_the_weighted_sum(oracle):
    """-SplitSum: the _ODD (even frame indices) and _EVN sums of the dose-
    weighted frames add up to the _DW sum (before positivity clamping, which
    a positive movie does not reach), as CCorrectFullShift::mGenSums builds
    them (Correct/CCorrectFullShift.cpp:271-300)."""
    from motioncor3_b200 import synthetic as S
    m = S.make_movie(128, 96, 7, dose=20.0, seed=8)
    kw = dict(iter=4, tol=0.2, bft=(300, 100), fm_dose=1.2, pix_size=0.9, kv=300)
    r = oracle.process_movie(m.frames, split_sum=1, **kw)
    assert r["n_sums"] == 5
    plain = oracle.process_movie(m.frames, **kw)
    assert plain["n_sums"] == 3
    for i in range(3):
        assert np.array_equal(r["sums"][i], plain["sums"][i])
    dw, odd, evn = (r["sums"][i].astype(np.float64) for i in (1, 3, 4))
    assert np.abs(odd + evn - dw).max() <= 1e-4 * np.abs(dw).max()
    assert np.abs(odd - evn).max() > 1e-3 * np.abs(dw).max()


def test_oracle_fourier_binned_sums(oracle):
    """-FtBin 2: the output sum is the Fourier crop of the full-size sum to
    the binned size (CInput::GetBinnedSize rounding), inverted unnormalised,
    i.e. the band-limited half-size image with the same mean."""
    from motioncor3_b200 import synthetic as S
    m = S.make_movie(200, 150, 6, dose=20.0, seed=9)
    kw = dict(iter=4, tol=0.2, bft=(300, 100), pix_size=1.0)
    full = oracle.process_movie(m.frames, **kw)["sums"][0].astype(np.float64)
    binned = oracle.process_movie(m.frames, ft_bin=2.0, **kw)["sums"][0].astype(np.float64)
    oh, ow = 74, 100                   # (int)(150/2 + 0.5) = 75, made even
    assert binned.shape == (oh, ow)
    F = np.fft.rfft2(full) / full.size
    rows = [yo if yo <= oh // 2 else yo - oh + 150 for yo in range(oh)]
    crop = F[rows, : ow // 2 + 1]
    ref = np.fft.irfft2(crop, s=(oh, ow)) * (oh * ow)
    assert np.abs(binned - np.maximum(ref, 0)).max() <= 1e-3 * np.abs(ref).max()
    assert abs(binned.mean() - full.mean()) <= 1e-3 * full.mean()


def test_oracle_aligned_stack_and_zbin(oracle):
    """-OutStack: the aligned frames add up to the plain sum (before its
    positivity clamp, which a positive movie does not reach), and -OutStack
    1 3 holds the FP32 group sums of three consecutive frames, the last
    group shorter (CZbinStack::DoIt, Align/CZbinStack.cpp:27-71)."""
    from motioncor3_b200 import synthetic as S
    m = S.make_movie(128, 96, 7, dose=20.0, seed=10)
    kw = dict(iter=4, tol=0.2, bft=(300, 100), fm_dose=1.2, pix_size=0.9, kv=300, ft_bin=1.5)
    one = oracle.process_movie(m.frames, out_stack=(1, 1), **kw)
    st = one["stack"]
    assert st.shape == (7,) + one["sums"][0].shape
    tot = st.astype(np.float64).sum(axis=0)
    plain = one["sums"][0].astype(np.float64)
    assert np.abs(tot - plain).max() <= 1e-5 * np.abs(plain).max()
    three = oracle.process_movie(m.frames, out_stack=(1, 3), **kw)
    assert three["stack"].shape[0] == 3
    for g, (a, b) in enumerate([(0, 3), (3, 6), (6, 7)]):
        ref = st[a].copy()
        for k in range(a + 1, b):
            ref = (ref + st[k]).astype(np.float32)
        assert np.array_equal(three["stack"][g], ref), g
    for i in range(one["n_sums"]):  # the stack leaves the sums alone
        assert np.array_equal(three["sums"][i], one["sums"][i])


def test_oracle_loaded_patch_alignment_is_made_relative(oracle):
    """-InAln in patch mode: CPatchAlign::mCorrectFullShift makes the loaded
    full-frame shifts relative to the reference frame (Align/CPatchAlign.cpp:47-52),
    so an offset added to every loaded shift changes nothing."""
    from motioncor3_b200 import synthetic as S
    m = S.make_movie(192, 192, 6, dose=20.0, seed=11)
    kw = dict(patch=(2, 2), iter=3, tol=0.2, bft=(300, 100), pix_size=1.0, group=(1, 2))
    r = oracle.process_movie(m.frames, **kw)
    force = dict(global_shifts=r["global_shifts"], patch_shifts=r["patch_shifts"],
                 patch_centers=r["patch_centers"], patch_bad=np.zeros_like(r["patch_bad"]))
    a = oracle.process_movie(m.frames, force=force, **kw)
    force["global_shifts"] = r["global_shifts"] + np.float32(1.25)
    b = oracle.process_movie(m.frames, force=force, **kw)
    assert np.array_equal(a["global_shifts"], r["global_shifts"])
    # (s + c) - (s_ref + c) rounds differently from s - s_ref by ~1e-7 px
    assert np.abs(b["global_shifts"] - a["global_shifts"]).max() <= 1e-6
    for i in range(a["n_sums"]):
        d = a["sums"][i].astype(np.float64) - b["sums"][i]
        assert np.sqrt(np.mean(d ** 2) / np.mean(a["sums"][i].astype(np.float64) ** 2)) <= 1e-3


def test_mrc_four_bit_round_trip(tmp_path):
    """Mode 101 files: packed rows of (nx+1)//2 bytes, even pixel in the low
    nibble (LibSrc/Mrcfile/Image/C4BitImage.cpp), odd widths included."""
    from motioncor3_b200 import mrcio
    rng = np.random.default_rng(5)
    for nx in (6, 7):
        a = rng.integers(0, 16, size=(3, 5, nx)).astype(np.uint8)
        pk = mrcio.pack4(a)
        assert pk.shape == (3, 5, (nx + 1) // 2)
        assert pk[0, 0, 0] == (a[0, 0, 0] | (a[0, 0, 1] << 4))
        f = str(tmp_path / f"m{nx}.mrc")
        mrcio.write(f, a, four_bit=True)
        h = mrcio.read_header(f)
        assert (h["nx"], h["mode"]) == (nx, 101)
        assert np.array_equal(mrcio.read(f), a)


def test_oracle_mag_stretch_of_the_sums(oracle):
    """-Mag major minor angle: each sum is resampled bilinearly at
    m ((x, y) - c) + c with m the inverse stretch (Correct/GStretch.cu); at
    angle 0 that reads the plain sum at ((x - c)/s + c, y), s = major/minor.
    Equal major and minor leave the sums untouched."""
    from motioncor3_b200 import synthetic as S
    m = S.make_movie(160, 128, 6, dose=20.0, seed=13)
    kw = dict(iter=4, tol=0.2, bft=(300, 100), pix_size=1.0)
    plain = oracle.process_movie(m.frames, **kw)["sums"][0].astype(np.float64)
    same = oracle.process_movie(m.frames, mag=(1.02, 1.02, 10.0), **kw)["sums"][0]
    assert np.array_equal(same, plain.astype(np.float32))
    s = 1.04
    st = oracle.process_movie(m.frames, mag=(s, 1.0, 0.0), **kw)["sums"][0].astype(np.float64)
    H, W = plain.shape
    xs = (np.arange(W) - W / 2) / np.float32(s) + W / 2
    ix = np.floor(xs).astype(int)
    wx = xs - ix
    ref = (1 - wx) * plain[:, ix] + wx * plain[:, np.minimum(ix + 1, W - 1)]
    inner = (slice(4, H - 4), slice(8, W - 8))
    rel = np.abs(st[inner] - ref[inner]).max() / np.abs(ref[inner]).max()
    assert rel < 2e-3, rel


def test_oracle_in_frame_motion_weighting(oracle):
    """-InFmMotion: each aligned frame is damped by the directional sinc of
    its motion (MotionDecon/GMotionWeight.cu); the DC term (the mean) is
    untouched and high frequencies lose power."""
    from motioncor3_b200 import synthetic as S
    m = S.make_movie(192, 160, 8, dose=20.0, seed=14)
    kw = dict(iter=4, tol=0.2, bft=(300, 100), pix_size=1.0)
    a = oracle.process_movie(m.frames, **kw)
    b = oracle.process_movie(m.frames, in_fm_motion=1, **kw)
    assert np.array_equal(a["global_shifts"], b["global_shifts"])
    sa, sb = a["sums"][0].astype(np.float64), b["sums"][0].astype(np.float64)
    assert abs(sa.mean() - sb.mean()) <= 1e-5 * sa.mean()
    Fa, Fb = np.abs(np.fft.rfft2(sa)), np.abs(np.fft.rfft2(sb))
    hi = np.zeros_like(Fa, bool)
    hi[40:-40, 40:] = True
    assert Fb[hi].sum() < 0.99 * Fa[hi].sum()


@pytest.mark.parametrize("nx,ny,keeps", [(1024, 1024, False), (2048, 2048, True), (1024, 2048, True),
                                         (2048, 1024, False), (2882, 2048, False)])
def test_inverse_keeps_edge_imaginary_parts_where_cufft_does(oracle, nx, ny, keeps):
    """The oracle's C2R of a non-Hermitian half spectrum restates cufftPlan2d
    (the reference's inverse, probed on the B200): the real part after the
    column transform, plus -(b0 + bM) on even and b0 - bM on odd samples of
    each row at the sizes where cuFFT keeps the rows' DC / Nyquist imaginary
    parts (both sides powers of two, ny >= 2048)."""
    rng = np.random.default_rng(nx + 3 * ny)
    cx = nx // 2 + 1
    half = rng.standard_normal((ny, cx)) + 1j * rng.standard_normal((ny, cx))
    got = oracle.irfft2(half, nx)
    want = np.fft.irfft2(half, s=(ny, nx)) * nx * ny
    if keeps:
        col = np.fft.ifft(half, axis=0) * ny
        b0, bm = col[:, 0].imag, col[:, nx // 2].imag
        want[:, 0::2] += (-(b0 + bm))[:, None]
        want[:, 1::2] += (b0 - bm)[:, None]
    assert np.abs(got - want).max() <= 1e-9 * np.abs(want).max()
