"""The autotuner's table file (csrc/tuning.cpp, compiled for the host):
entries written as JSON read back exactly; foreign or damaged text is
rejected; every combination of the three variant switches is a candidate."""
import ctypes
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def tshim():
    out_dir = os.path.join(ROOT, "tests", "_build")
    os.makedirs(out_dir, exist_ok=True)
    so = os.path.join(out_dir, "tuning_shim.so")
    src = os.path.join(ROOT, "tests", "native", "tuning_shim.cpp")
    deps = [src, os.path.join(ROOT, "motioncor3_b200", "csrc", "tuning.cpp"),
            os.path.join(ROOT, "motioncor3_b200", "csrc", "tuning.h")]
    if not os.path.exists(so) or os.path.getmtime(so) < max(map(os.path.getmtime, deps)):
        cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
        subprocess.run([cxx, "-O1", "-std=c++17", "-shared", "-fPIC", src, "-o", so], check=True)
    L = ctypes.CDLL(so)
    L.shim_tuning_parse.argtypes = [ctypes.c_char_p]
    return L


def test_tuning_file_round_trip(tshim):
    buf = ctypes.create_string_buffer(1 << 16)
    assert tshim.shim_tuning_roundtrip(buf, len(buf)) == 0
    doc = json.loads(buf.value.decode())          # valid JSON for other tools too
    assert doc["mc3_tuning"] == 1 and len(doc["entries"]) == 2
    e0 = doc["entries"][0]
    assert (e0["nx"], e0["patch"], e0["col_wide"], e0["gather_px"]) == (4096, [5, 5], 1, 1)
    assert len(e0["candidates"]) == 8 and e0["candidates"][3]["ms"] == pytest.approx(43.0)


def test_tuning_file_rejects_other_text(tshim):
    assert tshim.shim_tuning_parse(b'{"entries": []}') == -1
    assert tshim.shim_tuning_parse(b'{"mc3_tuning": 1, "entries": [\n{"nx": 64, "ny": 64}\n]}') == -1
    assert tshim.shim_tuning_parse(b'{"mc3_tuning": 1, "device": "", "entries": [\n]}') == 0


def test_every_variant_is_a_candidate(tshim):
    assert tshim.shim_tuning_candidates() == 8
    assert tshim.shim_tuning_candidate_faults() == 0
