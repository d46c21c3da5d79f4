"""The C ABI: the library loads, exports every entry point include/mc3.h
declares, reports the reference's defaults, and refuses to run without a
GPU (no CPU fallback)."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"\b(mc3_[a-z0-9_]+)\s*\(", txt))
    return sorted(names)


def test_exports_every_declared_symbol(mc3lib):
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(mc3lib, s), s


def test_defaults_match_reference_cinput(mc3lib):
    from motioncor3_b200 import api
    p = api._Params()
    mc3lib.mc3_params_default(ctypes.byref(p))
    # CInput::CInput (CInput.cpp:82-127)
    assert p.iter == 15 and abs(p.tol - 0.1) < 1e-7
    assert (p.bft[0], p.bft[1]) == (500.0, 100.0)
    assert (p.group[0], p.group[1]) == (1, 4)
    assert p.kv == 300 and p.fm_ref == -1
    assert (p.sum_range[0], p.sum_range[1]) == (3.0, 25.0)
    assert (p.out_stack[0], p.out_stack[1]) == (0, 1)  # m_aiOutStack (CInput.cpp:107-108)


def test_strerror_and_version(mc3lib):
    from motioncor3_b200 import api
    assert b"sm_100a" in mc3lib.mc3_version()
    assert mc3lib.mc3_strerror(api.MC3_EINVAL) == b"invalid argument or size"


def test_no_cpu_fallback(mc3lib):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from motioncor3_b200 import api
    with pytest.raises(api.MC3Error) as e:
        api.MotionCor3(api.Params())
    assert e.value.code == api.MC3_ECUDA


def test_bad_arguments_rejected(mc3lib):
    from motioncor3_b200 import api
    p = api.Params(iter=0).to_c()
    h = ctypes.c_void_p()
    assert mc3lib.mc3_create(ctypes.byref(p), ctypes.byref(h)) == api.MC3_EINVAL
    assert mc3lib.mc3_destroy(None) == api.MC3_EINVAL
    assert mc3lib.mc3_fft_forward(None, 64, 64, 1, 1, None) == api.MC3_EINVAL


def _write(tmp_path, name, text):
    f = tmp_path / name
    f.write_text(text)
    return str(f)


def test_read_fmint_file_parsing(mc3lib, tmp_path):
    """CReadFmIntFile::DoIt (DataUtil/CReadFmIntFile.cpp:104-170)."""
    from motioncor3_b200 import api
    g, n, d = api.read_fmint_file(_write(tmp_path, "a.txt", "40 4 0.5\n20 2 0.5\n"), 9.0)
    assert g.tolist() == [40, 20] and n.tolist() == [4, 2] and np.allclose(d, 0.5)
    # two columns: the raw-frame dose is -FmDose
    g, n, d = api.read_fmint_file(_write(tmp_path, "b.txt", "40 4\n10 1\n"), 0.7)
    assert g.tolist() == [40, 10] and n.tolist() == [4, 1] and np.allclose(d, 0.7)
    # three columns: a line that does not scan repeats the previous entry
    # (the reference compares the scan count instead of assigning it)
    g, n, d = api.read_fmint_file(_write(tmp_path, "c.txt", "40 4 0.5\n\n20 2 0.5\n"), 0.0)
    assert g.tolist() == [40, 40, 20]
    # different raw-frame doses: the file is dropped
    g, n, d = api.read_fmint_file(_write(tmp_path, "d.txt", "40 4 0.5\n20 2 0.6\n"), 0.0)
    assert len(g) == 0
    with pytest.raises(api.MC3Error):
        api.read_fmint_file(str(tmp_path / "missing.txt"), 0.0)


def _tables(entries, n_raw, fm_dose=0.0):
    """Independent restatement of CFmIntParam::mCalcIntFms (DataUtil/CFmIntParam.cpp:138-229)."""
    gs = [e[0] for e in entries]
    isz = [e[1] for e in entries]
    extra = sum(gs) - n_raw
    if extra > 0:
        for i in range(len(gs) - 1, -1, -1):
            g0 = gs[i]
            gs[i] -= extra
            if gs[i] <= 0:
                gs[i] = 0
            else:
                extra -= g0
            if extra <= 0:
                break
    elif extra < 0:
        gs[-1] -= extra
    nint = []
    for i in range(len(gs) - 1):
        nint.append(gs[i] // isz[i])
        gs[i + 1] += gs[i] % isz[i]
    left = gs[-1] % isz[-1]
    nint.append(gs[-1] // isz[-1])
    size = [isz[i] for i in range(len(gs)) for _ in range(nint[i])]
    for i in range(left):
        size[len(size) - 1 - i] += 1
    start = [0]
    for s in size[:-1]:
        start.append(start[-1] + s)
    acc = np.cumsum(np.float32(entries[0][2]) * np.array(size, np.float32), dtype=np.float32)
    return start, size, acc


@pytest.mark.parametrize("entries,n_raw", [([(40, 4, 0.5)], 40), ([(40, 4, 0.5)], 42),
                                           ([(40, 4, 0.5)], 37),
                                           ([(20, 2, 0.25), (30, 3, 0.25)], 50),
                                           ([(21, 2, 0.25), (30, 3, 0.25)], 51),
                                           ([(21, 2, 0.25), (30, 3, 0.25)], 44)])
def test_frame_integration_tables(mc3lib, entries, n_raw):
    """CFmIntParam::Setup with a frame-integration file: rendered frames,
    leftovers moved to the next entry and spread over the last frames."""
    from motioncor3_b200 import api
    e = ([x[0] for x in entries], [x[1] for x in entries], [x[2] for x in entries])
    t = api.frame_integration_tables(e, n_raw)
    start, size, acc = _tables(entries, n_raw)
    if len(size) - 3 > 5:  # -Throw 2 -Trunc 1 drop rendered frames, doses kept
        tt = api.frame_integration_tables(e, n_raw, throw=(2, 1))
        assert tt["start"].tolist() == start[2:-1] and tt["size"].tolist() == size[2:-1]
        assert np.allclose(tt["acc_dose"], acc[2:-1], rtol=1e-6)
    assert t["size"].tolist() == size and t["start"].tolist() == start
    assert sum(size) == n_raw
    assert np.allclose(t["acc_dose"], acc, rtol=1e-6)
    assert t["dose_weight"] == 1


def test_frame_integration_tables_without_integration(mc3lib):
    """All integration sizes 1 (or no file): one raw frame per frame with
    -FmDose (CFmIntParam::mSetup); the file's dose still turns dose
    weighting on (CFmIntParam::bDoseWeight)."""
    from motioncor3_b200 import api
    t = api.frame_integration_tables(([30], [1], [0.8]), 30, fm_dose=1.5)
    assert t["size"].tolist() == [1] * 30 and t["start"].tolist() == list(range(30))
    assert np.allclose(t["acc_dose"], 1.5 * np.arange(1, 31, dtype=np.float32))
    assert t["dose_weight"] == 1
    t = api.frame_integration_tables(None, 12, fm_dose=0.0)
    assert t["dose_weight"] == 0 and len(t["size"]) == 12


@pytest.mark.parametrize("rot", [0, 1, 2, 3])
@pytest.mark.parametrize("flip", [0, 1, 2])
def test_ref_orient(mc3lib, rot, flip):
    """CLoadRefs::PostProcess: G90Rotate2D's nearest-pixel rotation about the
    centre (restated here from its index formula), GFlip2D, GInverse2D."""
    from motioncor3_b200 import api
    rng = np.random.default_rng(rot * 3 + flip)
    ny, nx = 6, 10
    a = rng.uniform(0.5, 1.5, (ny, nx)).astype(np.float32)
    a[2, 3] = 0.0
    out = api.ref_orient(a, rot, flip, 1)
    c, s = [(1, 0), (0, 1), (-1, 0), (0, -1)][rot]
    rx, ry = (ny, nx) if rot % 2 else (nx, ny)
    ref = np.zeros((ry, rx), np.float32)
    for y in range(ry):
        for x in range(rx):
            fx = (x - (rx - 1) / 2) * c + (y - (ry - 1) / 2) * s
            fy = -(x - (rx - 1) / 2) * s + (y - (ry - 1) / 2) * c
            ref[y, x] = a[int(fy + (ny - 1) / 2 + 0.5), int(fx + (nx - 1) / 2 + 0.5)]
    if flip == 1:
        ref = ref[::-1]
    elif flip == 2:
        ref = ref[:, ::-1]
    with np.errstate(divide="ignore"):
        ref = np.where(ref == 0, 0, 1.0 / ref).astype(np.float32)
    assert out.shape == ref.shape
    assert np.array_equal(out, ref)
    if rot == 2 and flip == 0:  # half turn = both flips
        assert np.array_equal(api.ref_orient(a, 2), a[::-1, ::-1])


def test_ref_augment(mc3lib):
    from motioncor3_b200 import api
    a = np.arange(12, dtype=np.float32).reshape(3, 4)
    assert np.array_equal(api.ref_augment(a, 2), np.repeat(np.repeat(a, 2, 0), 2, 1))


def test_frame_tables_with_throws(mc3lib):
    """CFmIntParam::mSetup with -Throw 2 -Trunc 3: the kept raw frames,
    doses counted again from the first kept frame; with a file, throwing
    that would leave 5 or fewer rendered frames is ignored
    (CFmIntParam::mThrowIntFrames)."""
    from motioncor3_b200 import api
    t = api.frame_integration_tables(None, 20, fm_dose=0.5, throw=(2, 3))
    assert t["start"].tolist() == list(range(2, 17)) and t["size"].tolist() == [1] * 15
    assert np.allclose(t["acc_dose"], 0.5 * np.arange(1, 16, dtype=np.float32))
    t = api.frame_integration_tables(([24], [4], [0.5]), 24, throw=(1, 1))
    assert t["size"].tolist() == [4] * 6  # 6 - 2 = 4 <= 5: throws ignored


def test_argument_checks_without_gpu(mc3lib):
    """Entry points reject bad arguments with a status code (never abort),
    before touching a device."""
    from motioncor3_b200 import api
    L = api._lib()
    EINVAL = api.MC3_EINVAL
    assert L.mc3_set_alignment(None, None) == EINVAL
    assert L.mc3_set_frame_integration(None, None) == EINVAL
    assert L.mc3_set_dark(None, None, 0, 0, 0) == EINVAL
    assert L.mc3_set_defects(None, None, 0, 0) == EINVAL
    img = np.ones((4, 6), np.float32)
    out = np.zeros(24, np.float32)
    nx, ny = ctypes.c_int(0), ctypes.c_int(0)
    assert L.mc3_ref_orient(img.ctypes.data, 6, 4, 0, 3, 0, out.ctypes.data, ctypes.byref(nx),
                            ctypes.byref(ny)) == EINVAL  # flip must be 0, 1 or 2
    assert L.mc3_ref_augment(img.ctypes.data, 6, 4, 0, out.ctypes.data) == EINVAL
    n = ctypes.c_int(0)
    assert L.mc3_frame_integration_tables(None, None, None, 0, 10, ctypes.c_float(1.0), -1, 0, 10,
                                          ctypes.byref(n), None, None, None, None) == EINVAL
    assert L.mc3_frame_integration_tables(None, None, None, 0, 10, ctypes.c_float(1.0), 6, 5, 10,
                                          ctypes.byref(n), None, None, None, None) == EINVAL
    assert L.mc3_frame_groups(None, None, 0, 1, 0, ctypes.byref(n), None, None, None) == EINVAL
    assert L.mc3_eer_render(None, 1, 1, None, None, None, 0) == EINVAL
    assert L.mc3_tiff_read(b"x.tif", -1, 1, out.ctypes.data, 1) == EINVAL


def test_create_without_a_gpu_fails_cleanly(mc3lib):
    """Without a CUDA device mc3_create returns an error status instead of
    aborting the process (CSimpleFuncs.cpp:203-212 resets the device and
    asserts instead)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from motioncor3_b200 import api
    p = api.Params().to_c()
    h = ctypes.c_void_p()
    rc = api._lib().mc3_create(ctypes.byref(p), ctypes.byref(h))
    assert rc != api.MC3_OK and not h.value


def test_cli_ctf_gate(mc3lib, tmp_path):
    """-Cs defaults to the reference's 2.7 on the command line; with -Cs 0 (or
    no -PixSize) the reference's 'Skip CTF estimation' notice is printed
    (CFindCtfMain::bEstimate).  Runs before any GPU work: the movie does not
    exist."""
    import subprocess
    from motioncor3_b200 import build
    exe = build.CLI
    base = [exe, "-InMrc", str(tmp_path / "none.mrc"), "-OutMrc", str(tmp_path / "o.mrc")]
    off = subprocess.run(base + ["-PixSize", "1", "-Cs", "0"], capture_output=True, text=True, timeout=60)
    assert "Skip CTF estimation" in off.stdout and "Cs value:     0.000000" in off.stdout
    on = subprocess.run(base + ["-PixSize", "1", "-AmpCont", "0.1", "-ExtPhase", "20"],
                        capture_output=True, text=True, timeout=60)
    assert "Skip CTF estimation" not in on.stdout
    assert "outside the implemented path" not in on.stderr  # the CTF tags are parsed
    nopix = subprocess.run(base, capture_output=True, text=True, timeout=60)
    assert "Pixel size:   0.000000" in nopix.stdout


def test_queue_entry_points_check_their_arguments(mc3lib):
    import ctypes
    from motioncor3_b200 import api
    L = mc3lib
    t = ctypes.c_int()
    assert L.mc3_submit(None, None, None, ctypes.byref(t)) == api.MC3_EINVAL
    assert L.mc3_wait(None, 1, None) == api.MC3_EINVAL
    assert L.mc3_rfft_rows(None, 8, None, 5, 8, 1, 1, None) == api.MC3_EINVAL


def test_proposal_and_warm_start_entry_points_check_their_arguments(mc3lib):
    import ctypes
    from motioncor3_b200 import api
    L = mc3lib
    h = ctypes.c_void_p()
    spec = (ctypes.c_int * 5)(3, 4, 3, 2, 1)   # the first layer must take the two frames
    assert L.mc3_proposal_create(spec, 1, 2, 0, 0, ctypes.byref(h)) == api.MC3_EINVAL
    assert L.mc3_proposal_create(None, 1, 2, 0, 0, ctypes.byref(h)) == api.MC3_EINVAL
    assert L.mc3_proposal_destroy(None) == api.MC3_EINVAL
    assert L.mc3_proposal_predict(None, None, 1, 8, 8, 0, None) == api.MC3_EINVAL
    assert L.mc3_proposal_pair_inputs(None, 8, 8, 2, None, 1, 2, None, None) == api.MC3_EINVAL
    assert L.mc3_set_first_iterate(None, None, 0, 0) == api.MC3_EINVAL
    assert L.mc3_autotune(None, 64, 64, 4, None, None) == api.MC3_EINVAL
    assert L.mc3_load_tuning(None, b"x.json") == api.MC3_EINVAL
    c = (ctypes.c_float * 4)(10.0, 20.0, 30.0, 40.0)
    assert L.mc3_set_patch_centers(None, c, 2) == api.MC3_EINVAL


class _DeviceTensorStandIn:
    """Enough of a CUDA tensor for the Python wrappers' argument checks,
    which run before anything is handed to the library."""

    def __init__(self, shape, dtype="float32"):
        self.shape, self.dtype, self.is_cuda = tuple(shape), f"torch.{dtype}", True

    def data_ptr(self):
        return 0

    def is_contiguous(self):
        return True


def test_device_wrappers_check_output_sizes(mc3lib):
    """The C entry points take raw device pointers and cannot see a buffer's
    size, so the wrappers compare each tensor's shape with what the call
    writes: an output sized for fewer frame pairs, a wrong target or a frame
    of the wrong row length is refused with ValueError."""
    from motioncor3_b200 import api
    T = _DeviceTensorStandIn
    pairs = np.array([[f, g] for f in range(16) for g in range(16) if f != g], np.int32)
    with pytest.raises(ValueError, match="pair_inputs out"):
        api.ShiftProposal.pair_inputs(T((16, 256, 256)), pairs, 2, T((16, 2, 128, 128)))
    with pytest.raises(ValueError, match="pair_inputs out"):
        api.ShiftProposal.pair_inputs(T((16, 256, 256)), pairs, 2, T((240, 2, 64, 64)))
    with pytest.raises(ValueError, match="fft_forward"):
        api.fft_forward(T((2, 64, 64)), 64, 64)
    with pytest.raises(ValueError, match="fft_inverse"):
        api.fft_inverse(T((2, 64, 66), "complex64"), 64, 64)
    net = api.ShiftProposal.__new__(api.ShiftProposal)  # no device state needed for the check
    net.nout, net._h = 2, None
    with pytest.raises(ValueError, match="train_step target"):
        net.train_step(T((8, 2, 32, 32)), T((4, 2)))
