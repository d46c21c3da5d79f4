"""Regenerates tests/golden/*.json from the reference tree.

lin_eqs_kat.json: the known-answer test that the reference ships with its
Gauss-Jordan solver (Util_LinEqs::Test, LibSrc/Util/Util_LinEqs.cpp:160-180):
coefficient matrix, right-hand side and expected solution, parsed from the
source text.

host_bookkeeping.json: inputs and outputs of the reference's own host-side
shift bookkeeping (CPeak2D, CRemoveSpikes1D, CStackShift::Smooth,
CInterpolateShift, CPatchShifts) compiled unmodified from the reference
sources by oracle/ref_host (seeded random inputs).

ctf_fits.json: the fits of the reference's own CTF drivers (CFindCtf2D,
CFindDefocus1D/2D, compiled unmodified by oracle/ref_host with host
stand-ins for their kernels) on the half spectra the oracle makes from
seeded micrographs with a planted CTF (tests/conftest.py make_ctf_image);
the inputs are stored as the image parameters.

Run from the repository root: python tests/golden/make_golden.py
"""
import ctypes
import hashlib
import json
import os
import re
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
# The reference source tree: $MC3_REFERENCE, else "reference" beside the repository.
REF = os.environ.get("MC3_REFERENCE") or os.path.normpath(os.path.join(ROOT, "..", "reference"))
OUT = os.path.dirname(os.path.abspath(__file__))


def _floats(block: str):
    return [float(v.rstrip("f")) for v in re.findall(r"-?\d+\.\d+f?", block)]


def lin_eqs_kat():
    src = open(os.path.join(REF, "LibSrc/Util/Util_LinEqs.cpp")).read()
    body = src[src.index("void Util_LinEqs::Test"):]
    coeff = _floats(body[body.index("afCoeff[]"):body.index("afVals[]")])
    vals = _floats(body[body.index("afVals[]"):body.index("afSol[]")])
    sol = _floats(body[body.index("afSol[]"):body.index("iDim")])
    return {"source": "LibSrc/Util/Util_LinEqs.cpp Util_LinEqs::Test", "dim": 4,
            "coeff": coeff, "vals": vals, "solution": sol, "solution_decimals": 4}


def host_bookkeeping():
    from oracle import oracle as O
    L = O.ref_host()
    P = ctypes.c_void_p
    f = lambda a: a.ctypes.data_as(P)
    rng = np.random.default_rng(20261203)
    cases = {"peak2d": [], "remove_spikes": [], "smooth": [], "interpolate": [], "patch_shifts": []}
    for t in range(6):
        w = rng.standard_normal((64, 64)).astype(np.float32)
        y0, x0 = rng.integers(0, 64, 2)
        w[y0, x0] += 8.0
        out = np.zeros(2, np.float32)
        L.ref_peak2d(f(w), 64, 64, f(out))
        cases["peak2d"].append({"window": w.ravel().tolist(), "shift": out.tolist()})
    for n in (12, 30, 40, 60, 80):
        x = np.cumsum(rng.normal(0, 0.8, n)).astype(np.float32)
        y = np.cumsum(rng.normal(0, 0.8, n)).astype(np.float32)
        x[n // 3] += 15
        y[n // 2] -= 9
        xo, yo = x.copy(), y.copy()
        L.ref_remove_spikes(f(xo), f(yo), n)
        cases["remove_spikes"].append({"x": x.tolist(), "y": y.tolist(), "x_out": xo.tolist(),
                                       "y_out": yo.tolist()})
        xs, ys = x.copy(), y.copy()
        L.ref_smooth(f(xs), f(ys), n, ctypes.c_float(0.5))
        cases["smooth"].append({"x": x.tolist(), "y": y.tolist(), "w": 0.5, "x_out": xs.tolist(),
                                "y_out": ys.tolist()})
        for binz in (1, 4):
            ng = (n + binz - 1) // binz
            g = rng.normal(0, 2, (ng, 2)).astype(np.float32)
            for nearest in (0, 1):
                o = np.zeros((n, 2), np.float32)
                L.ref_interpolate(f(g), n, binz, nearest, f(o))
                cases["interpolate"].append({"n": n, "binz": binz, "nearest": nearest,
                                             "groups": g.ravel().tolist(), "out": o.ravel().tolist()})
    for (N, Px, Py) in ((20, 3, 3), (40, 5, 5)):
        Pn = Px * Py
        raw = rng.normal(0, 1.5, (Pn, N, 2)).astype(np.float32)
        cen = np.array([[(i % Px + 0.5) * 4096 / Px, (i // Px + 0.5) * 4096 / Py] for i in range(Pn)],
                       np.float32)
        sh = np.zeros((N, Pn, 2), np.float32)
        bad = np.zeros((N, Pn), np.uint8)
        L.ref_patch_shifts(f(raw), f(cen), N, Pn, 4096, 4096, f(sh), f(bad))
        cases["patch_shifts"].append({"N": N, "P": Pn, "raw": raw.ravel().tolist(),
                                      "centers": cen.ravel().tolist(), "shifts": sh.ravel().tolist(),
                                      "bad": bad.ravel().tolist()})
    return cases


CTF_CASES = [
    {"image": {"n": 1024, "df": 12000.0, "ast": 0.03, "ang": -40.0, "phase": 0.0, "seed": 5},
     "pix": 1.0, "kv": 300.0, "cs": 2.7, "ac": 0.07, "ext_phase": 0.0},
    {"image": {"n": 1024, "df": 12000.0, "ast": 0.03, "ang": -40.0, "phase": 30.0, "seed": 5},
     "pix": 1.0, "kv": 300.0, "cs": 2.7, "ac": 0.07, "ext_phase": 30.0},
    {"image": {"n": 1280, "pix": 1.6, "df": 22000.0, "ast": 0.01, "ang": 70.0, "phase": 0.0, "seed": 6,
               "kv": 200.0, "cs": 2.0, "ac": 0.1},
     "pix": 1.6, "kv": 200.0, "cs": 2.0, "ac": 0.1, "ext_phase": 0.0},
]


def ctf_fits():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import make_ctf_image
    from oracle import oracle as O
    L = O.ref_ctf()
    f = ctypes.c_float
    out = []
    for c in CTF_CASES:
        avg, _, pn = O.ctf_spectrum(make_ctf_image(**c["image"]), c["pix"])
        res = np.zeros(6, np.float32)
        L.ref_ctf_search(np.ascontiguousarray(avg).ctypes.data_as(ctypes.c_void_p), f(pn), f(c["kv"]),
                         f(c["cs"]), f(c["ac"]), f(c["ext_phase"]), res.ctypes.data_as(ctypes.c_void_p))
        # the spectrum's hash, so that a change of the input (the image is
        # made with numpy's FFT) is told apart from a change of the search
        sha = hashlib.sha256(np.ascontiguousarray(avg, np.float32).tobytes()).hexdigest()
        out.append(dict(c, pix_n=float(pn), spectrum_sha256=sha, res6=[float(v) for v in res]))
    return {"source": "FindCtf/CFindCtf2D.cpp, CFindDefocus1D.cpp, CFindDefocus2D.cpp", "cases": out}


if __name__ == "__main__":
    with open(os.path.join(OUT, "lin_eqs_kat.json"), "w") as fh:
        json.dump(lin_eqs_kat(), fh, indent=1)
    with open(os.path.join(OUT, "host_bookkeeping.json"), "w") as fh:
        json.dump(host_bookkeeping(), fh)
    with open(os.path.join(OUT, "ctf_fits.json"), "w") as fh:
        json.dump(ctf_fits(), fh, indent=1)
    print("written")
