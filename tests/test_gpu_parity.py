"""GPU parity: every libmc3 kernel and the whole path against the FP64
oracle (and numpy / cuFFT for the transforms).  Tolerances: FFTs 2e-6
relative to the spectrum maximum; correlation windows 1e-4 relative; shifts
within 0.05 px; sums within 1e-4 relative RMS; integer / gather work exact."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b ** 2)))


def _keeps_edge_imag(nx, ny):
    """cufftPlan2d C2R keeps the rows' DC / Nyquist imaginary parts for these
    sizes (both powers of two, ny >= 2048; probed on the B200)."""
    p2 = lambda n: n > 0 and (n & (n - 1)) == 0
    return p2(nx) and p2(ny) and ny >= 2048


def _c2r_reference(half, nx, ny):
    """Unnormalised 2D C2R of half spectra [nz][ny][nx/2+1] as cufftPlan2d
    computes it: numpy's inverse (real part after the column transform), plus,
    at the sizes where cuFFT keeps them, -(b0 + bM) on even and b0 - bM on odd
    samples of each row (b0, bM: imaginary parts of the row's DC and Nyquist
    terms after the column inverse)."""
    out = np.fft.irfft2(half.astype(np.complex128), s=(ny, nx), axes=(-2, -1)) * nx * ny
    if _keeps_edge_imag(nx, ny):
        col = np.fft.ifft(half.astype(np.complex128), axis=-2) * ny
        b0, bm = col[..., 0].imag, col[..., nx // 2].imag
        out[..., 0::2] += (-(b0 + bm))[..., None]
        out[..., 1::2] += (b0 - bm)[..., None]
    return out


def _cufft_plan2d_c2r(torch, half):
    """The reference's inverse (cufftPlan2d C2R, in place) as a comparator;
    None when libcufft cannot be loaded."""
    import ctypes
    try:
        cf = ctypes.CDLL("/usr/local/cuda/lib64/libcufft.so")
    except OSError:
        return None
    ny, cx = half.shape
    nx = (cx - 1) * 2
    buf = torch.view_as_real(torch.from_numpy(half.astype(np.complex64)).cuda()).reshape(ny, 2 * cx).contiguous()
    plan = ctypes.c_int()
    assert cf.cufftPlan2d(ctypes.byref(plan), ny, nx, 0x2C) == 0
    assert cf.cufftExecC2R(plan, ctypes.c_void_p(buf.data_ptr()), ctypes.c_void_p(buf.data_ptr())) == 0
    torch.cuda.synchronize()
    cf.cufftDestroy(plan)
    return buf[:, :nx].cpu().numpy()


@pytest.fixture(scope="module")
def api(mc3lib, torch_cuda):
    from motioncor3_b200 import api as A
    return A


@pytest.mark.parametrize("ny,nx", [(64, 64), (256, 256), (408, 408), (408, 410), (1024, 1024),
                                   (2048, 2048), (4096, 4096), (4092, 5760)])
def test_fft_forward_inverse(api, torch_cuda, ny, nx):
    torch = torch_cuda
    rng = np.random.default_rng(nx + ny)
    nz = 2
    img = rng.standard_normal((nz, ny, nx)).astype(np.float32)
    cx = nx // 2 + 1
    buf = torch.zeros((nz, ny, 2 * cx), dtype=torch.float32, device="cuda")
    buf[:, :, :nx] = torch.from_numpy(img).cuda()
    api.fft_forward(buf, nx, ny, normalise=True)
    torch.cuda.synchronize()
    spec = torch.view_as_complex(buf.view(nz, ny, cx, 2)).cpu().numpy()
    ref = np.fft.rfft2(img.astype(np.float64)) / (nx * ny)
    assert np.abs(spec - ref).max() / np.abs(ref).max() < 2e-6
    # Non-Hermitian input to the inverse (a phase-shifted spectrum has a
    # non-Hermitian Nyquist column): the reference's plan type
    # (Util/CCufft2D.cpp:49, cufftPlan2d) takes the real part after the
    # column transform, except that at some sizes the imaginary parts of the
    # rows' DC and Nyquist terms also reach the output (_c2r_reference).
    half = (rng.standard_normal((nz, ny, cx)) + 1j * rng.standard_normal((nz, ny, cx))).astype(np.complex64)
    hb = torch.view_as_real(torch.from_numpy(half).cuda()).reshape(nz, ny, 2 * cx).contiguous()
    api.fft_inverse(hb, nx, ny)
    torch.cuda.synchronize()
    out = hb[:, :, :nx].cpu().numpy()
    refb = _c2r_reference(half, nx, ny)
    assert np.abs(out - refb).max() / np.abs(refb).max() < 2e-6
    cu = _cufft_plan2d_c2r(torch, half[0])
    if cu is not None:
        assert np.abs(out[0] - cu).max() / np.abs(cu).max() < 2e-6


@pytest.mark.parametrize("nx,ny", [(64, 64), (384, 320), (192, 160), (408, 408), (410, 408),
                                   (1024, 1024), (1536, 1536), (2048, 1024), (1024, 2048),
                                   (2048, 2048), (2882, 2048), (4096, 2048), (2048, 4096),
                                   (4096, 4096), (5760, 4092)])
def test_inverse_of_shifted_spectra_matches_cufft_plan2d(api, torch_cuda, nx, ny):
    """The inverse of a phase-shifted spectrum (non-Hermitian in the DC and
    Nyquist columns) against the reference's own inverse, cufftPlan2d C2R, at
    every frame, alignment and output size the configurations use."""
    torch = torch_cuda
    rng = np.random.default_rng(nx * 7 + ny)
    img = rng.poisson(1.0, (ny, nx)).astype(np.float64)
    cx = nx // 2 + 1
    kx = np.arange(cx)[None, :]
    ky = np.arange(ny)[:, None]
    ky = np.where(ky > ny // 2, ky - ny, ky)
    half = np.fft.rfft2(img) / (nx * ny) * np.exp(2j * np.pi * (kx * 0.37 / nx - ky * 1.21 / ny))
    cu = _cufft_plan2d_c2r(torch, half)
    if cu is None:
        pytest.skip("libcufft not available as a comparator")
    hb = torch.view_as_real(torch.from_numpy(half.astype(np.complex64)).cuda()).reshape(1, ny, 2 * cx).contiguous()
    api.fft_inverse(hb, nx, ny)
    torch.cuda.synchronize()
    out = hb[0, :, :nx].cpu().numpy()
    rel = np.sqrt(np.mean((out - cu) ** 2) / np.mean(cu ** 2))
    print(f"{nx}x{ny}: rel RMS {rel:.2e} against cufftPlan2d "
          f"({'keeps' if _keeps_edge_imag(nx, ny) else 'drops'} the edge imaginary parts)")
    assert rel < 1e-6


def test_phase_shift(api, torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(2)
    cy, cx = 128, 65
    X = (rng.standard_normal((cy, cx)) + 1j * rng.standard_normal((cy, cx))).astype(np.complex64)
    src = torch.from_numpy(X).cuda()
    dst = torch.zeros_like(src)
    sx, sy = 3.37, -7.81
    api.phase_shift(src, dst, sx, sy)
    torch.cuda.synchronize()
    kx = np.arange(cx)[None, :]
    ky = np.fft.fftfreq(cy, 1.0 / cy)[:, None]
    ky = np.where(np.arange(cy)[:, None] > cy // 2, np.arange(cy)[:, None] - cy, np.arange(cy)[:, None])
    ref = X * np.exp(2j * np.pi * (kx * sx / ((cx - 1) * 2) + ky * sy / cy))
    assert np.abs(dst.cpu().numpy() - ref).max() < 1e-5 * np.abs(ref).max()
    api.phase_shift(src, dst, sx, sy, accumulate=True)
    torch.cuda.synchronize()
    assert np.abs(dst.cpu().numpy() - 2 * ref).max() < 2e-5 * np.abs(ref).max()


@pytest.mark.parametrize("cy,cx,phase_only", [(256, 129, 0), (408, 205, 0), (512, 257, 1)])
def test_correlate_window_and_peak(api, oracle, torch_cuda, cy, cx, phase_only):
    torch = torch_cuda
    from motioncor3_b200 import synthetic as S
    rng = np.random.default_rng(cy)
    nx = (cx - 1) * 2
    truth = S.truth_image(nx, cy, rng, n_blobs=60)
    a = rng.poisson(4 * truth).astype(np.float64)
    b = rng.poisson(4 * np.roll(truth, (3, -5), (0, 1))).astype(np.float64)
    G = oracle.rfft2(a) * 1.0
    Sm = oracle.rfft2(a) + oracle.rfft2(b)
    win_o = oracle.correlate_window(G, Sm, 150.0, phase_only)
    sh_o = oracle.peak2d(win_o)
    g = torch.from_numpy(G.astype(np.complex64)).cuda()
    s = torch.from_numpy(Sm.astype(np.complex64)).cuda()
    win = torch.zeros((64, 64), dtype=torch.float32, device="cuda")
    sh = api.correlate(g, s, 150.0, phase_only, (64, 64), win)
    w = win.cpu().numpy()
    assert np.abs(w - win_o).max() < 1e-4 * np.abs(win_o).max()
    assert np.abs(sh - sh_o).max() < 0.01
    assert np.allclose(np.abs(sh_o), [5, 3], atol=0.6)


def test_bad_pixel_detection_and_fill(api, oracle, torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(9)
    ny, nx, nz = 200, 256, 3
    frames = rng.poisson(20.0, (nz, ny, nx)).astype(np.float32)
    frames[:, 50, 60] = 400.0            # hot pixel
    frames[:, 120:126, 30:36] = 2.0      # dark defect block
    frames[:, 128:130, 31:33] = 90.0
    total = frames.astype(np.float64).sum(0)
    bad_o = oracle.detect_bad(total)
    cx = nx // 2 + 1
    pad = torch.zeros((nz, ny, 2 * cx), dtype=torch.float32, device="cuda")
    pad[:, :, :nx] = torch.from_numpy(frames).cuda()
    ssum = torch.zeros((ny, 2 * cx), dtype=torch.float32, device="cuda")
    ssum[:, :nx] = torch.from_numpy(frames.sum(0)).cuda()
    bad = torch.zeros((ny, nx), dtype=torch.uint8, device="cuda")
    api.detect_bad_pixels(ssum, nx, ny, bad)
    bad_g = bad.cpu().numpy()
    assert bad_o[50, 60] == 1 and bad_o.sum() > 1
    assert np.array_equal(bad_g, bad_o)
    api.correct_bad_pixels(pad, nx, ny, bad)
    torch.cuda.synchronize()
    got = pad[:, :, :nx].cpu().numpy()
    for f in range(nz):
        ref = oracle.correct_bad(frames[f], bad_o)
        assert np.array_equal(got[f], ref.astype(np.float32))


def _local_shift_f64(nx, ny, cen, sh, bad):
    """The per-pixel weighted patch shift of mGCorrect3D in FP64."""
    yy, xx = np.mgrid[0:ny, 0:nx].astype(np.float64)
    sx = np.zeros((ny, nx))
    sy = np.zeros((ny, nx))
    sw = np.zeros((ny, nx))
    for p in range(len(cen)):
        if bad[p]:
            continue
        r = np.sqrt(((xx - cen[p, 0]) / nx) ** 2 + ((yy - cen[p, 1]) / ny) ** 2)
        w = np.where(r <= 0.6, np.exp(-100.0 * r), 0.0)
        sw += w
        sx += w * sh[p, 0]
        sy += w * sh[p, 1]
    ok = sw > 0
    sx[ok] /= sw[ok]
    sy[ok] /= sw[ok]
    return xx - sx, yy - sy


def _check_gather(got, ref, nx, ny, cen, sh, bad, limit=1e-4):
    """Every pixel equal, except where the source coordinate lies within
    `limit` px of a pixel boundary (the host's expf and unfused FP32 adds in
    the oracle against the device's expf and FMAs can truncate such a
    coordinate to the neighbouring pixel).  Returns the mismatch fraction."""
    mism = got != ref.astype(np.float32)
    if mism.any():
        u, v = _local_shift_f64(nx, ny, cen, sh, bad)
        du = np.abs(u - np.round(u))
        dv = np.abs(v - np.round(v))
        near = np.minimum(du, dv)[mism]
        assert near.max() < limit, (int(mism.sum()), float(near.max()))
    return float(mism.mean())


@pytest.mark.parametrize("P,grid", [(9, 3), (100, 10)])
def test_local_gather_exact(api, oracle, torch_cuda, P, grid):
    """mGCorrect3D gathers against the oracle: identical pixels, except at
    sources on a pixel boundary (checked pixel by pixel).  P = 100 runs the
    kernel for more than 64 patches (chunked patch loop)."""
    torch = torch_cuda
    rng = np.random.default_rng(4 + P)
    ny, nx = 384, 512
    img = rng.standard_normal((ny, nx)).astype(np.float32)
    cen = np.array([[(i % grid + 0.5) * nx / grid + rng.normal(0, 9),
                     (i // grid + 0.5) * ny / grid + rng.normal(0, 9)] for i in range(P)], np.float32)
    sh = rng.normal(0, 2.5, (P, 2)).astype(np.float32)
    bad = np.zeros(P, np.uint8)
    bad[4] = 1
    bad[P - 3] = 1
    ref = oracle.local_gather(img, cen, sh, bad)
    cx = nx // 2 + 1
    src = torch.zeros((ny, 2 * cx), dtype=torch.float32, device="cuda")
    src[:, :nx] = torch.from_numpy(img).cuda()
    dst = torch.zeros_like(src)
    api.local_gather(src, dst, nx, ny, torch.from_numpy(cen).cuda(), torch.from_numpy(sh).cuda(),
                     torch.from_numpy(bad).cuda())
    torch.cuda.synchronize()
    got = dst[:, :nx].cpu().numpy()
    frac = _check_gather(got, ref, nx, ny, cen.astype(np.float64), sh.astype(np.float64), bad)
    assert frac < 1e-4, frac


def test_iterative_align_component(api, oracle, torch_cuda):
    torch = torch_cuda
    from motioncor3_b200 import synthetic as S
    m = S.make_movie(256, 256, 14, dose=5.0, seed=21)
    spec = np.stack([oracle.rfft2(f.astype(np.float64)) for f in m.frames])
    ref, it_o = oracle.iterative_align(spec, 1, 8, 0.05, 150.0)
    with api.MotionCor3(api.Params()) as mc:
        t = torch.from_numpy(spec.astype(np.complex64)).cuda()
        got, it_g = mc.iterative_align(t, 1, 8, 0.05, 150.0)
    assert it_g == it_o
    assert np.abs(got - ref).max() <= 0.05


def _compare_movie(api, oracle, movie, params, forced_sum_tol=1e-4):
    """Runs the GPU path and the oracle on the same raw frames: shifts within
    0.05 px and sums (oracle corrected with the GPU's shifts) within 1e-4."""
    kw = dict(patch=params.patch[:2], iter=params.iter, tol=params.tol, bft=params.bft,
              fm_dose=params.fm_dose, pix_size=params.pix_size, kv=params.kv, group=params.group,
              split_sum=params.split_sum, ft_bin=params.ft_bin)
    with api.MotionCor3(params) as mc:
        if movie.gain is not None:
            mc.set_gain(np.asarray(movie.gain))
        res = mc.process(np.asarray(movie.frames))
    orc = oracle.process_movie(np.asarray(movie.frames),
                               gain=None if movie.gain is None else np.asarray(movie.gain), **kw)
    assert res.n_sums == orc["n_sums"]
    dg = np.abs(res.global_shifts - orc["global_shifts"]).max()
    assert dg <= 0.05, dg
    force = dict(global_shifts=res.global_shifts)
    if res.n_patches:
        assert np.abs(res.patch_shifts - orc["patch_shifts"]).max() <= 0.05
        assert np.array_equal(res.patch_centers, orc["patch_centers"])
        force.update(patch_shifts=res.patch_shifts, patch_centers=res.patch_centers,
                     patch_bad=res.patch_bad)
    same = oracle.process_movie(np.asarray(movie.frames),
                                gain=None if movie.gain is None else np.asarray(movie.gain),
                                force=force, **kw)
    for s in range(res.n_sums):
        e = _rel_rms(res.sums[s], same["sums"][s])
        assert e <= forced_sum_tol, (s, e)
    return res, orc


def test_pipeline_global_small(api, oracle, torch_cuda):
    from motioncor3_b200 import synthetic as S
    m = S.make_movie(256, 256, 16, dose=4.0, seed=31)
    p = api.Params(iter=7, tol=0.5, bft=(150, 100), pix_size=1.0)
    _compare_movie(api, oracle, m, p)


def test_pipeline_global_dose_weighted_gain(api, oracle, torch_cuda):
    from motioncor3_b200 import synthetic as S
    m = S.make_movie(384, 320, 12, dose=3.0, seed=32, gain=True)
    p = api.Params(iter=6, tol=0.2, bft=(300, 100), fm_dose=1.2, pix_size=0.9, kv=300)
    res, _ = _compare_movie(api, oracle, m, p)
    assert res.n_sums == 3


@pytest.mark.parametrize("dose", [0.0, 1.2])
def test_pipeline_split_sums(api, oracle, torch_cuda, dose):
    """-SplitSum 1: odd/even frame sums after the plain (and DW, DWS) sums."""
    from motioncor3_b200 import synthetic as S
    m = S.make_movie(320, 256, 11, dose=3.0, seed=36, gain=False)
    p = api.Params(iter=6, tol=0.2, bft=(300, 100), fm_dose=dose, pix_size=0.9, kv=300,
                   split_sum=1)
    res, _ = _compare_movie(api, oracle, m, p)
    assert res.n_sums == (5 if dose > 0 else 3)


@pytest.mark.parametrize("ft_bin", [2.0, 1.5])
def test_pipeline_fourier_binned_sums(api, oracle, torch_cuda, ft_bin):
    """-FtBin: sums Fourier-cropped to the binned size before the inverse."""
    from motioncor3_b200 import synthetic as S
    m = S.make_movie(384, 320, 10, dose=3.0, seed=37, gain=False)
    p = api.Params(iter=6, tol=0.2, bft=(300, 100), fm_dose=1.2, pix_size=0.9, kv=300,
                   ft_bin=ft_bin)
    res, _ = _compare_movie(api, oracle, m, p)
    ob = int(np.float32(384) / np.float32(ft_bin) + np.float32(0.5)) // 2 * 2
    oh = int(np.float32(320) / np.float32(ft_bin) + np.float32(0.5)) // 2 * 2
    assert res.sums.shape == (3, oh, ob)


def test_pipeline_patch_small(api, oracle, torch_cuda):
    from motioncor3_b200 import synthetic as S
    m = S.make_movie(512, 512, 12, dose=4.0, seed=33, gain=True, local=True)
    p = api.Params(patch=(3, 3), iter=5, tol=0.2, bft=(500, 150), fm_dose=1.0, pix_size=1.0, kv=300)
    res, _ = _compare_movie(api, oracle, m, p)
    assert res.n_patches == 9


def _oracle_kw(params):
    return dict(patch=params.patch[:2], iter=params.iter, tol=params.tol, bft=params.bft,
                fm_dose=params.fm_dose, pix_size=params.pix_size, kv=params.kv,
                group=params.group, split_sum=params.split_sum, ft_bin=params.ft_bin,
                out_stack=params.out_stack)


@pytest.mark.parametrize("ft_bin,zbin", [(1.0, 1), (1.5, 3)])
def test_pipeline_aligned_stack(api, oracle, torch_cuda, ft_bin, zbin):
    """-OutStack 1 zbin: the aligned frames (phase-shifted spectra, Fourier
    crop, C2R, no clamp) and their group sums against the oracle corrected
    with the GPU's shifts; the sums are unchanged by the stack."""
    from motioncor3_b200 import synthetic as S
    m = S.make_movie(384, 320, 10, dose=3.0, seed=38, gain=False)
    p = api.Params(iter=6, tol=0.2, bft=(300, 100), fm_dose=1.2, pix_size=0.9, kv=300,
                   ft_bin=ft_bin, out_stack=(1, zbin))
    with api.MotionCor3(p) as mc:
        res = mc.process(np.asarray(m.frames))
    with api.MotionCor3(api.Params(iter=6, tol=0.2, bft=(300, 100), fm_dose=1.2, pix_size=0.9,
                                   kv=300, ft_bin=ft_bin)) as mc:
        plain = mc.process(np.asarray(m.frames))
    for i in range(res.n_sums):
        assert np.array_equal(res.sums[i], plain.sums[i])
    same = oracle.process_movie(np.asarray(m.frames), force=dict(global_shifts=res.global_shifts),
                                **_oracle_kw(p))
    assert res.stack.shape == same["stack"].shape == ((10 + zbin - 1) // zbin,) + res.sums[0].shape
    for f in range(res.stack.shape[0]):
        e = _rel_rms(res.stack[f], same["stack"][f])
        assert e <= 1e-5, (f, e)


def test_pipeline_aligned_stack_patch(api, oracle, torch_cuda):
    """-OutStack in patch mode: the locally corrected frames."""
    from motioncor3_b200 import synthetic as S
    m = S.make_movie(512, 512, 12, dose=4.0, seed=33, gain=True, local=True)
    p = api.Params(patch=(3, 3), iter=5, tol=0.2, bft=(500, 150), fm_dose=1.0, pix_size=1.0,
                   kv=300, out_stack=(1, 1))
    with api.MotionCor3(p) as mc:
        mc.set_gain(np.asarray(m.gain))
        res = mc.process(np.asarray(m.frames))
    force = dict(global_shifts=res.global_shifts, patch_shifts=res.patch_shifts,
                 patch_centers=res.patch_centers, patch_bad=res.patch_bad)
    same = oracle.process_movie(np.asarray(m.frames), gain=np.asarray(m.gain), force=force,
                                **_oracle_kw(p))
    assert res.stack.shape == same["stack"].shape == (12, 512, 512)
    for f in range(12):
        e = _rel_rms(res.stack[f], same["stack"][f])
        assert e <= 1e-4, (f, e)


@pytest.mark.parametrize("patch", [False, True])
def test_pipeline_loaded_alignment(api, oracle, torch_cuda, patch):
    """mc3_set_alignment (-InAln): the movie is corrected with the given
    shifts, nothing is measured (0 iterations), and the sums match the
    oracle corrected with the same tables (all patches good)."""
    from motioncor3_b200 import synthetic as S
    if patch:
        m = S.make_movie(512, 512, 12, dose=4.0, seed=33, gain=False, local=True)
        p = api.Params(patch=(3, 3), iter=5, tol=0.2, bft=(500, 150), fm_dose=1.0, pix_size=1.0)
    else:
        m = S.make_movie(384, 320, 12, dose=3.0, seed=32, gain=False)
        p = api.Params(iter=6, tol=0.2, bft=(300, 100), fm_dose=1.2, pix_size=0.9)
    with api.MotionCor3(p) as mc:
        first = mc.process(np.asarray(m.frames))
        g = first.global_shifts + np.float32(0.5)  # patch mode makes them relative again
        mc.set_alignment(g if patch else first.global_shifts,
                         first.patch_shifts if patch else None,
                         first.patch_centers if patch else None)
        res = mc.process(np.asarray(m.frames))
        mc.set_alignment(None)
        again = mc.process(np.asarray(m.frames))
    assert res.iterations.max() == 0 and first.iterations[0] > 0
    assert np.array_equal(again.global_shifts, first.global_shifts)
    if not patch:
        assert np.array_equal(res.global_shifts, first.global_shifts)
        for i in range(res.n_sums):  # same shifts, same kernels: same bits
            assert np.array_equal(res.sums[i], first.sums[i])
        return
    assert np.abs(res.global_shifts - first.global_shifts).max() <= 1e-6
    assert np.array_equal(res.patch_shifts, first.patch_shifts)
    assert not res.patch_bad.any()
    force = dict(global_shifts=res.global_shifts, patch_shifts=res.patch_shifts,
                 patch_centers=res.patch_centers, patch_bad=res.patch_bad)
    same = oracle.process_movie(np.asarray(m.frames), force=force, **_oracle_kw(p))
    for i in range(res.n_sums):
        e = _rel_rms(res.sums[i], same["sums"][i])
        assert e <= 1e-4, (i, e)


@pytest.mark.parametrize("nx", [320, 330])
def test_pipeline_four_bit_frames(api, torch_cuda, nx):
    """MRC mode 101 (two 4-bit pixels per byte, GApplyRefsToFrame mGDoPkd):
    the packed movie gives the same sums, bit for bit, as its uint8
    unpacking (the engine takes even widths; odd packed rows are covered by
    the CPU packing test)."""
    from motioncor3_b200 import mrcio, synthetic as S
    m = S.make_movie(nx, 256, 8, dose=2.0, seed=41, gain=True)
    u8 = np.minimum(np.asarray(m.frames), 15).astype(np.uint8)
    pk = mrcio.pack4(u8)
    assert np.array_equal(mrcio.unpack4(pk, nx), u8)
    p = api.Params(iter=5, tol=0.2, bft=(300, 100), fm_dose=1.0, pix_size=1.0)
    with api.MotionCor3(p) as mc:
        mc.set_gain(np.asarray(m.gain))
        a = mc.process(u8)
        b = mc.process(pk, nx4=nx)
    assert np.array_equal(a.global_shifts, b.global_shifts)
    for i in range(a.n_sums):
        assert np.array_equal(a.sums[i], b.sums[i])


def _render(raw, size):
    """Rendered frames of the reference's 8-bit integration (sums mod 256)."""
    out, r = [], 0
    for n in size:
        out.append(raw[r:r + n].astype(np.uint32).sum(axis=0) % 256)
        r += n
    return np.stack(out).astype(np.float32)


@pytest.mark.parametrize("packed,high", [(False, False), (False, True), (True, False)])
def test_pipeline_frame_integration(api, oracle, torch_cuda, packed, high):
    """-FmIntFile: 26 raw frames rendered as 3+3+...(+leftovers) frames
    (CFmIntParam::mCalcIntFms), summed modulo 256 as the reference's 8-bit
    rendered stack (high: counts that wrap), then aligned with groups by
    raw-frame count and dose-weighted by the file's dose; against the
    oracle run on the rendered frames with the same tables."""
    from motioncor3_b200 import mrcio, synthetic as S
    m = S.make_movie(384, 320, 26, dose=1.0, seed=43, gain=False)
    raw = np.minimum(np.asarray(m.frames), 15).astype(np.uint8)
    if high:
        raw = (raw.astype(np.uint16) * 17 + 40).astype(np.uint8)  # rendered sums wrap
    tabs = api.frame_integration_tables(([26], [3], [0.4]), 26)
    assert tabs["size"].tolist() == [3] * 6 + [4, 4]
    p = api.Params(iter=6, tol=0.2, bft=(300, 100), pix_size=0.9, kv=300, group=(2, 4))
    with api.MotionCor3(p) as mc:
        mc.set_frame_integration(tabs, n_raw=26)
        res = mc.process(mrcio.pack4(raw) if packed else raw, nx4=384 if packed else None)
    assert res.n_sums == 3 and res.global_shifts.shape == (8, 2)
    rend = _render(raw, tabs["size"])
    kw = dict(iter=6, tol=0.2, bft=(300, 100), pix_size=0.9, kv=300, group=(2, 4),
              dose_weight=1)
    orc = oracle.process_movie(rend, int_size=tabs["size"], acc_dose=tabs["acc_dose"], **kw)
    assert np.abs(res.global_shifts - orc["global_shifts"]).max() <= 0.05
    same = oracle.process_movie(rend, int_size=tabs["size"], acc_dose=tabs["acc_dose"],
                                force=dict(global_shifts=res.global_shifts), **kw)
    for i in range(res.n_sums):
        e = _rel_rms(res.sums[i], same["sums"][i])
        assert e <= 1e-4, (i, e)


def test_pipeline_dark_and_gain(api, oracle, torch_cuda):
    """(raw - dark) * gain (GApplyRefsToFrame, MrcUtil/GApplyRefsToFrame.cu:56-72)."""
    from motioncor3_b200 import synthetic as S
    m = S.make_movie(384, 320, 10, dose=4.0, seed=45, gain=True)
    dark = np.random.default_rng(45).uniform(0.0, 0.6, (320, 384)).astype(np.float32)
    p = api.Params(iter=6, tol=0.2, bft=(300, 100), fm_dose=1.2, pix_size=0.9)
    with api.MotionCor3(p) as mc:
        mc.set_gain(np.asarray(m.gain))
        mc.set_dark(dark)
        res = mc.process(np.asarray(m.frames))
    kw = dict(iter=6, tol=0.2, bft=(300, 100), fm_dose=1.2, pix_size=0.9)
    orc = oracle.process_movie(np.asarray(m.frames), gain=np.asarray(m.gain), dark=dark, **kw)
    assert np.abs(res.global_shifts - orc["global_shifts"]).max() <= 0.05
    same = oracle.process_movie(np.asarray(m.frames), gain=np.asarray(m.gain), dark=dark,
                                force=dict(global_shifts=res.global_shifts), **kw)
    for i in range(res.n_sums):
        e = _rel_rms(res.sums[i], same["sums"][i])
        assert e <= 1e-4, (i, e)


@pytest.mark.parametrize("patch", [False, True])
def test_pipeline_mag_correction(api, oracle, torch_cuda, patch):
    """-Mag 1.05 1.0 25: every sum stretched in real space
    (CCorrectFullShift::mCorrectMag + GStretch) before the output crop."""
    from motioncor3_b200 import synthetic as S
    if patch:
        m = S.make_movie(512, 512, 12, dose=4.0, seed=33, gain=False, local=True)
        p = api.Params(patch=(3, 3), iter=5, tol=0.2, bft=(500, 150), fm_dose=1.0, pix_size=1.0,
                       mag=(1.05, 1.0, 25.0))
    else:
        m = S.make_movie(384, 320, 10, dose=3.0, seed=48, gain=False)
        p = api.Params(iter=6, tol=0.2, bft=(300, 100), fm_dose=1.2, pix_size=0.9,
                       mag=(1.05, 1.0, 25.0), ft_bin=1.5)
    with api.MotionCor3(p) as mc:
        res = mc.process(np.asarray(m.frames))
    force = dict(global_shifts=res.global_shifts)
    if patch:
        force.update(patch_shifts=res.patch_shifts, patch_centers=res.patch_centers,
                     patch_bad=res.patch_bad)
    kw = _oracle_kw(p)
    kw["mag"] = p.mag
    same = oracle.process_movie(np.asarray(m.frames), force=force, **kw)
    for i in range(res.n_sums):
        e = _rel_rms(res.sums[i], same["sums"][i])
        assert e <= 1e-4, (i, e)


@pytest.mark.parametrize("patch", [False, True])
def test_pipeline_in_frame_motion(api, oracle, torch_cuda, patch):
    """-InFmMotion 1: the directional sinc weight of each frame's motion
    (CCorrectFullShift::mMotionDecon in global mode, CGenRealStack on the
    globally corrected frames in patch mode), against the oracle."""
    from motioncor3_b200 import synthetic as S
    if patch:
        m = S.make_movie(512, 512, 12, dose=4.0, seed=33, gain=False, local=True)
        p = api.Params(patch=(3, 3), iter=5, tol=0.2, bft=(500, 150), fm_dose=1.0, pix_size=1.0,
                       in_fm_motion=1, out_stack=(1, 1), corr_interp=1)
    else:
        m = S.make_movie(384, 320, 10, dose=3.0, seed=50, gain=False)
        p = api.Params(iter=6, tol=0.2, bft=(300, 100), fm_dose=1.2, pix_size=0.9,
                       in_fm_motion=1, out_stack=(1, 1))
    with api.MotionCor3(p) as mc:
        res = mc.process(np.asarray(m.frames))
    force = dict(global_shifts=res.global_shifts)
    if patch:
        force.update(patch_shifts=res.patch_shifts, patch_centers=res.patch_centers,
                     patch_bad=res.patch_bad)
    kw = _oracle_kw(p)
    kw["in_fm_motion"] = 1
    kw["corr_interp"] = p.corr_interp
    same = oracle.process_movie(np.asarray(m.frames), force=force, **kw)
    for i in range(res.n_sums):
        e = _rel_rms(res.sums[i], same["sums"][i])
        assert e <= 1e-4, (i, e)
    for f in range(res.stack.shape[0]):
        e = _rel_rms(res.stack[f], same["stack"][f])
        assert e <= 1e-4, (f, e)


def test_pipeline_known_defects(api, oracle, torch_cuda):
    """-DefectFile / -DefectMap: known defects join the detected bad pixels
    before the fill (BadPixel/CDetectMain.cpp:146-260); the fill itself is
    the reference's pseudo-random one, so frames and sums agree exactly."""
    from motioncor3_b200 import synthetic as S
    m = S.make_movie(384, 320, 10, dose=3.0, seed=55, gain=False)
    defects = np.zeros((320, 384), np.uint8)
    defects[100:104, 50:300] = 1   # a few dead rows
    defects[:, 200] = 1            # a dead column
    p = api.Params(iter=6, tol=0.2, bft=(300, 100), fm_dose=1.2, pix_size=0.9)
    with api.MotionCor3(p) as mc:
        mc.set_defects(defects)
        res = mc.process(np.asarray(m.frames))
        mc.set_defects(None)
        plain = mc.process(np.asarray(m.frames))
    assert not np.array_equal(res.sums[0], plain.sums[0])
    kw = dict(iter=6, tol=0.2, bft=(300, 100), fm_dose=1.2, pix_size=0.9)
    same = oracle.process_movie(np.asarray(m.frames), defects=defects,
                                force=dict(global_shifts=res.global_shifts), **kw)
    assert same["bad_map"][defects == 1].all()
    for i in range(res.n_sums):
        e = _rel_rms(res.sums[i], same["sums"][i])
        assert e <= 1e-4, (i, e)


def test_pipeline_config1_full_size(api, oracle, torch_cuda):
    """40 frames of 1024x1024, global alignment only (-Patch 0 0 -Iter 7
    -Tol 0.5 -Bft 150 -PixSize 1.0), dose 1 e/px/frame, unit gain."""
    from motioncor3_b200 import synthetic as S
    m = S.make_movie(1024, 1024, 40, dose=1.0, seed=101)
    p = api.Params(iter=7, tol=0.5, bft=(150, 100), pix_size=1.0)
    _compare_movie(api, oracle, m, p)


def test_pipeline_patch_10x10(api, oracle, torch_cuda):
    """-Patch 10 10 (100 patches: more than a 64-bit patch mask holds), the
    whole path against the oracle."""
    from motioncor3_b200 import synthetic as S
    m = S.make_movie(1024, 1024, 10, dose=3.0, seed=57, gain=False, local=True)
    p = api.Params(patch=(10, 10), iter=5, tol=0.2, bft=(500, 150), fm_dose=1.0, pix_size=1.0,
                   kv=300)
    res, _ = _compare_movie(api, oracle, m, p)
    assert res.n_patches == 100
