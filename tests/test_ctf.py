"""CTF estimation on the corrected sum (FindCtf/, run by
CCorrectFullShift::mEstimateCtf on the first sum): the oracle restatement
pinned against the reference's own fitting drivers (CFindCtf2D,
CFindDefocus1D/2D, CCtfParam compiled unmodified from the reference tree into
oracle/_ref/libmc3ref_ctf.so, with host stand-ins for the kernels they call),
and against CTFs planted in synthetic micrographs."""
import ctypes

import numpy as np
import pytest


@pytest.fixture(scope="module")
def ref_ctf():
    from oracle import oracle as O
    L = O.ref_ctf()
    if L is None:
        pytest.skip("reference CTF checker not available")
    return L


def _f(v):
    return ctypes.c_float(v)


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@pytest.mark.parametrize("kv,cs,ac,pix", [(300, 2.7, 0.07, 1.25), (200, 2.0, 0.1, 1.6),
                                          (300, 0.01, 0.0, 2.5)])
def test_ctf_parameters_match_reference(oracle, ref_ctf, kv, cs, ac, pix):
    """CCtfParam::Setup: wavelength and Cs in pixels, amplitude-contrast phase."""
    ref = np.zeros(3, np.float32)
    ref_ctf.ref_ctf_param(_f(kv), _f(cs), _f(ac), _f(pix), _ptr(ref))
    assert np.array_equal(oracle.ctf_param(kv, cs, ac, pix), ref)


_REF_FITS = {}


def _ref_fit(oracle, ref_ctf, ctf_image, phase, ext):
    """(half spectrum, pixel size, the reference drivers' res6), computed once."""
    if (phase, ext) not in _REF_FITS:
        img = ctf_image(n=1024, df=12000.0, ast=0.03, ang=-40.0, phase=phase, seed=5)
        avg, _, pn = oracle.ctf_spectrum(img, 1.0)
        ref = np.zeros(6, np.float32)
        ref_ctf.ref_ctf_search(_ptr(np.ascontiguousarray(avg)), _f(pn), _f(300), _f(2.7), _f(0.07),
                               _f(ext), _ptr(ref))
        _REF_FITS[(phase, ext)] = (avg, pn, ref)
    return _REF_FITS[(phase, ext)]


@pytest.mark.parametrize("phase,ext", [(0.0, 0.0), (30.0, 30.0)])
def test_search_matches_reference_drivers(oracle, ref_ctf, ctf_image, phase, ext):
    """The 1D brute-force search, the 2D astigmatism / angle / defocus / phase
    sweeps with their acceptance rules and the fit resolution give the
    reference's numbers exactly on the same half spectrum (-ExtPhase 30
    searches the extra phase in [0, 60] degrees)."""
    avg, pn, ref = _ref_fit(oracle, ref_ctf, ctf_image, phase, ext)
    got = oracle.ctf_search(avg, pn, 300, 2.7, 0.07, ext)
    assert np.array_equal(got, ref), (got, ref)
    assert abs(0.5 * (ref[0] + ref[1]) - 12000.0) < 250.0
    if ext:
        assert abs(ref[3] - phase) < 6.0


@pytest.mark.parametrize("phase,ext", [(0.0, 0.0), (30.0, 30.0)])
def test_device_search_logic_matches_reference_drivers(oracle, ref_ctf, ctf_shim, ctf_image, phase, ext):
    """The device path's search driver and per-candidate expressions
    (csrc/ctf_core.h: ctf::Search, ctf1d_term, ctf2d_term, make_band,
    fit_shell), run on the host with a sequential scorer, give the
    reference's numbers exactly."""
    avg, pn, ref = _ref_fit(oracle, ref_ctf, ctf_image, phase, ext)
    res, fit = np.zeros(6, np.float32), np.zeros(4, np.float32)
    assert ctf_shim.shim_ctf_search(_ptr(np.ascontiguousarray(avg)), _f(pn), _f(300), _f(2.7), _f(0.07),
                                    _f(ext), _ptr(res), _ptr(fit)) == 0
    assert np.array_equal(res, ref), (res, ref)


def test_device_spectrum_maps_match_oracle(oracle, ctf_shim, ctf_image):
    """The index maps of the device kernels (csrc/ctf_core.h) on the oracle's
    intermediate spectra: background removal (exact), the full spectrum,
    lowpass factors and copy-back (with numpy's FFT between them), the radial
    average and the diagnostic image."""
    img = ctf_image(n=2048, pix=1.0, df=15000.0, ast=0.02, ang=30.0, seed=1)
    st = oracle.ctf_stages(img, 1.0)
    bg = np.zeros((512, 257), np.float32)
    ctf_shim.shim_ctf_remove_background(_ptr(st["raw"]), _ptr(bg))
    assert np.array_equal(bg, st["bg"])
    full = np.zeros((512, 514), np.float32)
    ctf_shim.shim_ctf_full(_ptr(bg), _ptr(full))
    assert not full[:, 512:].any()
    lp = np.zeros((512, 257), np.float32)
    ctf_shim.shim_ctf_lowpass_factors(_ptr(lp))
    spec = np.fft.rfft2(full[:, :512].astype(np.float64)) / (512 * 512) * lp
    low = np.zeros((512, 514), np.float32)
    low[:, :512] = np.fft.irfft2(spec, s=(512, 512)) * (512 * 512)
    assert np.abs(low[:, :512] - st["full"]).max() <= 1e-5 * np.abs(st["full"]).max()
    half = np.zeros((512, 257), np.float32)
    ctf_shim.shim_ctf_take_half(_ptr(low), _ptr(half))
    assert np.abs(half - st["half"]).max() <= 1e-5 * np.abs(st["half"]).max()
    rad = np.zeros(257, np.float32)
    ctf_shim.shim_ctf_radial(_ptr(st["half"]), _ptr(rad))
    ref_rad = np.zeros(257)
    f32 = np.float32
    for r in range(257):  # GRadialAvg restated in numpy with its FP32 expressions
        n = min(max(int(f32(3.1415926) * f32(r) + f32(0.5)), 1), 180)
        a = (f32(-90.0) + np.arange(n, dtype=f32) * f32(f32(180.0) / f32(n))) * f32(0.017453)
        x = np.minimum((f32(r) * np.cos(a) + f32(0.5)).astype(int), 256)
        y = np.minimum((f32(r) * np.sin(a) + f32(256.5)).astype(int), 511)
        ref_rad[r] = st["half"][y, x].mean()
    # an index can flip where float32 cos/sin differ by an ulp at a .5 boundary
    same = np.abs(rad - ref_rad) <= 1e-5 * np.abs(ref_rad).max()
    assert same.mean() >= 0.97, np.flatnonzero(~same)
    res, fit = np.zeros(6, np.float32), np.zeros(4, np.float32)
    ctf_shim.shim_ctf_search(_ptr(st["half"]), _f(st["pix_n"]), _f(300), _f(2.7), _f(0.07), _f(0),
                             _ptr(res), _ptr(fit))
    ores, oimg = oracle.find_ctf(img, 1.0)
    assert np.array_equal(res, ores)
    out = np.zeros((512, 512), np.float32)
    fl = np.zeros((512, 514), np.float32)
    fl[:, :512] = st["full"]
    ctf_shim.shim_ctf_image(_ptr(fl), _ptr(st["half"]), _f(st["pix_n"]), _f(300), _f(2.7), _f(0.07),
                            _ptr(fit), _ptr(out))
    assert np.abs(out - oimg).max() <= 1e-5 * np.abs(oimg).max()


@pytest.mark.parametrize("pix,nx,ny", [(1.6, 1300, 1100), (1.0, 1280, 1600)])
def test_device_tile_stage_matches_oracle(oracle, ctf_shim, ctf_image, pix, nx, ny):
    """The device path's rescaled size, tile grid and tile preparation
    (csrc/ctf_core.h) with numpy standing in for the FFTs reproduce the
    oracle's averaged amplitude spectrum (CGenAvgSpectrum::mAverage)."""
    img = ctf_image(n=nx, ny=ny, pix=pix, seed=9)
    g = np.zeros(7, np.int32)
    pn = ctypes.c_float(0)
    ctf_shim.shim_ctf_geometry(nx, ny, _f(pix), _ptr(g), ctypes.byref(pn))
    nxN, nyN, ntx, nty, offx, offy, step = (int(v) for v in g)
    st = oracle.ctf_stages(img, pix)
    assert abs(pn.value - st["pix_n"]) == 0.0
    pitch = (nxN // 2 + 1) * 2
    if nxN == nx and nyN == ny:
        scaled = img.astype(np.float64)
    else:  # Fourier crop (GFourierResize2D) between a normalised R2C and a C2R
        F = np.fft.rfft2(img.astype(np.float64)) / (nx * ny)
        keep = np.r_[0:nyN // 2 + 1, ny - nyN // 2 + 1:ny]
        C = F[keep][:, :nxN // 2 + 1]
        scaled = np.fft.irfft2(C, s=(nyN, nxN)) * (nxN * nyN)
    pad = np.zeros((nyN, pitch), np.float32)
    pad[:, :nxN] = scaled
    acc = np.zeros((512, 257), np.float32)
    fac = np.float32(1.0 / (ntx * nty))
    tile = np.zeros((512, 514), np.float32)
    for t in range(ntx * nty):
        sx, sy = offx + (t % ntx) * step, offy + (t // ntx) * step
        ctf_shim.shim_ctf_tile(_ptr(pad), pitch, sx, sy, _ptr(tile))
        assert not tile[:, 512:].any()
        amp = np.abs(np.fft.rfft2(tile[:, :512].astype(np.float64))).astype(np.float32)
        acc = acc + np.roll(amp, 256, axis=0) * fac
    assert np.abs(acc - st["raw"]).max() <= 1e-4 * np.abs(st["raw"]).max()


@pytest.mark.parametrize("pix,n", [(1.0, 2048), (1.6, 2048)])
def test_oracle_recovers_planted_ctf(oracle, ctf_image, pix, n):
    """Pixel size 1.0 A is Fourier-rescaled to 1.25 A before tiling
    (CRescaleImage); 1.6 A is tiled as it is."""
    img = ctf_image(n=n, pix=pix, df=15000.0, ast=0.02, ang=30.0, seed=1)
    res, spec = oracle.find_ctf(img, pix)
    dfmax, dfmin, ang, ph, score, resol = res
    assert abs(dfmax - 15300.0) < 150.0 and abs(dfmin - 14700.0) < 150.0, res
    assert abs(ang - 30.0) < 3.0, res
    assert ph == 0.0 and score > 0.5 and resol < 10.0, res
    assert spec.shape == (512, 512) and np.isfinite(spec).all()


def test_spectrum_needs_a_tile(oracle, ctf_image):
    img = ctf_image(n=400, pix=1.0)  # 320 px after rescaling: no 512 x 512 tile
    assert oracle.ctf_spectrum(img, 1.0) is None
    assert oracle.find_ctf(img, 1.0) is None


def test_estimate_ctf_argument_checks(mc3lib):
    from motioncor3_b200 import api
    img = np.zeros((600, 600), np.float32)
    res = np.zeros(6, np.float32)
    rc = mc3lib.mc3_estimate_ctf(None, _ptr(img), 600, 600, 0, 1.0, 300.0, 2.7, 0.07, 0.0,
                                 _ptr(res), None)
    assert rc == api.MC3_EINVAL
    d = api.Params()
    assert d.cs == 0.0 and d.amp_cont == 0.07  # the library does not estimate unless asked


def test_searches_match_golden_reference_fits(oracle, ctf_shim):
    """tests/golden/ctf_fits.json holds the reference drivers' fits (made by
    tests/golden/make_golden.py) of the oracle's spectra of seeded
    micrographs: the oracle's search and the device path's search driver
    reproduce every value without the reference tree (three cases: no extra
    phase, an extra-phase search, 200 kV / 1.6 A)."""
    import json
    import os
    from conftest import make_ctf_image
    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ctf_fits.json")))
    assert len(gold["cases"]) == 3
    import hashlib
    for c in gold["cases"]:
        avg, _, pn = oracle.ctf_spectrum(make_ctf_image(**c["image"]), c["pix"])
        sha = hashlib.sha256(np.ascontiguousarray(avg, np.float32).tobytes()).hexdigest()
        # the input first: the micrograph is made with numpy's FFT, and a
        # changed spectrum is a changed input, not a changed search
        assert sha == c["spectrum_sha256"], (
            "averaged spectrum differs from the one the golden fits were made from "
            "(numpy's FFT changed?); rerun tests/golden/make_golden.py", c["image"])
        assert np.float32(pn) == np.float32(c["pix_n"])
        ref = np.array(c["res6"], np.float32)
        got = oracle.ctf_search(avg, pn, c["kv"], c["cs"], c["ac"], c["ext_phase"])
        assert np.array_equal(got, ref), (c["image"], got, ref)
        res, fit = np.zeros(6, np.float32), np.zeros(4, np.float32)
        ctf_shim.shim_ctf_search(_ptr(np.ascontiguousarray(avg)), _f(pn), _f(c["kv"]), _f(c["cs"]),
                                 _f(c["ac"]), _f(c["ext_phase"]), _ptr(res), _ptr(fit))
        assert np.array_equal(res, ref), (c["image"], res, ref)
