"""CTF estimation on the GPU (mc3_estimate_ctf, and the estimate
mc3_process_movie makes on the first sum when cs > 0.001): against the
oracle on micrographs with a planted CTF, and the command line against the
reference program's <stem>_Ctf.txt / _Ctf.mrc (FindCtf/,
CSaveSerialCryoEM::mSaveCtfStack / mSaveCtfFit).

Tolerances: the searches are discrete (defocus steps of 20 A in the 2D
refinement, 1 degree in azimuth), so results are compared within a few
steps; FP32 device transforms against the FP64 oracle move the spectrum by
~1e-5 relative."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _close(got, ref, df_tol=60.0, ang_tol=2.0, score_tol=0.01, res_tol=0.15):
    assert abs(got[0] - ref[0]) <= df_tol and abs(got[1] - ref[1]) <= df_tol, (got, ref)
    assert abs(got[2] - ref[2]) <= ang_tol, (got, ref)
    assert abs(got[3] - ref[3]) <= 2.0, (got, ref)
    assert abs(got[4] - ref[4]) <= score_tol, (got, ref)
    assert abs(got[5] / ref[5] - 1.0) <= res_tol, (got, ref)


@pytest.mark.parametrize("pix", [1.0, 1.6])
def test_estimate_matches_oracle(mc3lib, oracle, ctf_image, pix):
    """Pixel size 1.0 A: Fourier rescale to 1.25 A (1638 px, 25 tiles);
    1.6 A: tiled as it is (49 tiles)."""
    from motioncor3_b200 import api
    img = ctf_image(n=2048, pix=pix, df=15000.0, ast=0.02, ang=30.0, seed=1)
    with api.MotionCor3() as mc:
        got, spec = mc.estimate_ctf(img, pix)
    ref, rspec = oracle.find_ctf(img, pix)
    _close(got, ref)
    # right half of the diagnostic image: the lowpassed average spectrum
    a = spec[8:504, 264:504].astype(np.float64)
    b = rspec[8:504, 264:504].astype(np.float64)
    assert np.sqrt(np.mean((a - b) ** 2)) <= 1e-3 * np.sqrt(np.mean(b ** 2))


def test_estimate_rejects_images_without_a_tile(mc3lib, ctf_image):
    from motioncor3_b200 import api
    img = ctf_image(n=400, pix=1.0)
    with api.MotionCor3() as mc:
        with pytest.raises(api.MC3Error) as e:
            mc.estimate_ctf(img, 1.0)
    assert e.value.code == api.MC3_EUNSUPPORTED


def _ctf_movie(ctf_image, n=1280, frames=8, dose=20.0, seed=3):
    """Frames of Poisson counts around a CTF-carrying image; n = 1280 and 1600
    rescale (1 A -> 1.25 A) to 1024 and 1280 pixels."""
    truth = ctf_image(n=n, pix=1.0, df=14000.0, ast=0.03, ang=-25.0, seed=seed)
    truth = truth / truth.mean()
    rng = np.random.default_rng(seed + 1)
    return rng.poisson(dose * np.clip(truth, 0, None)[None].repeat(frames, 0)).astype(np.float32)


def test_movie_estimate_is_the_estimate_of_its_first_sum(mc3lib, oracle, ctf_image):
    """mc3_process_movie with cs = 2.7 estimates the CTF of the first sum at the
    final pixel size, outside the timed region."""
    from motioncor3_b200 import api
    frames = _ctf_movie(ctf_image)
    p = api.Params(patch=(0, 0), iter=3, tol=0.5, bft=(150.0, 100.0), pix_size=1.0, kv=300, cs=2.7)
    with api.MotionCor3(p) as mc:
        r = mc.process(frames)
        assert r.ctf is not None and r.ctf_spectrum.shape == (512, 512)
        again, spec = mc.estimate_ctf(r.sums[0], 1.0)
    assert np.array_equal(r.ctf, again)
    assert np.array_equal(r.ctf_spectrum, spec)
    ref, _ = oracle.find_ctf(r.sums[0], 1.0)
    _close(r.ctf, ref, df_tol=100.0, ang_tol=5.0, score_tol=0.02)
    assert abs(0.5 * (r.ctf[0] + r.ctf[1]) - 14000.0) < 400.0
    with api.MotionCor3(api.Params(patch=(0, 0), iter=3, pix_size=1.0)) as mc:
        assert mc.process(frames).ctf is None  # cs 0: no estimate


def _ctf_txt(path):
    rows = [l.split() for l in open(path) if l.strip() and not l.startswith("#")]
    assert len(rows) == 1 and len(rows[0]) == 6
    return np.array([float(v) for v in rows[0]])


def test_cli_ctf_matches_reference_program(tmp_path, mc3lib, ctf_image):
    """-Cs 2.7 -PixSize 1 -kV 300 on a movie whose frames carry a CTF: the fit
    line of <stem>_Ctf.txt and the spectrum of <stem>_Ctf.mrc.  The
    reference's spectrum has two undefined reads (row 0 of the full spectrum,
    the x-Nyquist column), so row 0..7 and the outer columns are left out of
    the image comparison."""
    from test_gpu_reference import OUR_BIN, REF_BIN, run_program
    from motioncor3_b200 import build, mrcio
    if not os.path.exists(REF_BIN):
        pytest.skip("reference program not built (oracle/ref_full)")
    build.build()
    frames = _ctf_movie(ctf_image, n=1600, frames=6, seed=7)
    tags = "-Patch 0 0 -Iter 5 -Tol 0.5 -Bft 150 -PixSize 1 -kV 300".split()
    ref = run_program(REF_BIN, str(tmp_path / "ref"), frames, None, tags, cs="2.7")
    ours = run_program(OUR_BIN, str(tmp_path / "ours"), frames, None, tags, cs="2.7")
    assert "CTF estimate" in ref["stdout"] and "CTF estimate" in ours["stdout"]
    a = _ctf_txt(str(tmp_path / "ref" / "sum_Ctf.txt"))
    b = _ctf_txt(str(tmp_path / "ours" / "sum_Ctf.txt"))
    # the outermost shells of the reference's resolution search see its
    # undefined x-Nyquist column, so the resolution is compared loosely
    _close(b, a, df_tol=150.0, ang_tol=5.0, score_tol=0.03, res_tol=0.3)
    ia = mrcio.read(str(tmp_path / "ref" / "sum_Ctf.mrc"))[0].astype(np.float64)
    ib = mrcio.read(str(tmp_path / "ours" / "sum_Ctf.mrc"))[0].astype(np.float64)
    assert ia.shape == ib.shape == (512, 512)
    ra, rb = ia[8:504, 264:504], ib[8:504, 264:504]
    assert np.sqrt(np.mean((ra - rb) ** 2)) <= 1e-2 * np.sqrt(np.mean(ra ** 2))
