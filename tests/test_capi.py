"""The C ABI: the library loads, exports every entry point include/mc3.h
declares, reports the reference's defaults, and refuses to run without a
GPU (no CPU fallback)."""
import ctypes
import os
import re

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
