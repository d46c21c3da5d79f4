"""libmc3's host-side shift bookkeeping (C ABI, no GPU needed) against the
reference's own host classes compiled from its sources: bit-exact."""
import ctypes
import json
import os

import numpy as np
import pytest

from conftest import fp

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_peak2d_bit_exact(mc3lib, ref_host):
    from motioncor3_b200 import api
    rng = np.random.default_rng(7)
    for t in range(500):
        w = rng.standard_normal((64, 64)).astype(np.float32)
        if t % 2:
            w[rng.integers(0, 64), rng.integers(0, 64)] += 6
        if t % 7 == 0:
            w[0, 0] = 50  # border peak gets pulled inside
        ref = np.zeros(2, np.float32)
        ref_host.ref_peak2d(fp(w), 64, 64, fp(ref))
        assert np.array_equal(api.peak2d(w), ref)


@pytest.mark.parametrize("n", [3, 8, 29, 30, 31, 45, 60, 61, 90, 120])
def test_remove_spikes_bit_exact(mc3lib, ref_host, n):
    from motioncor3_b200 import api
    rng = np.random.default_rng(n)
    for t in range(20):
        x = np.cumsum(rng.normal(0, 1.0, n)).astype(np.float32)
        y = np.cumsum(rng.normal(0, 1.0, n)).astype(np.float32)
        if t % 2:
            x[rng.integers(0, n)] += 25
            y[rng.integers(0, n)] -= 14
        xr, yr = x.copy(), y.copy()
        ref_host.ref_remove_spikes(fp(xr), fp(yr), n)
        xm, ym = api.remove_spikes(x, y)
        assert np.array_equal(xm, xr) and np.array_equal(ym, yr)


def test_smooth_and_lin_eqs(mc3lib, ref_host):
    from motioncor3_b200 import api
    rng = np.random.default_rng(3)
    for w in (0.4, 0.5, 0.7, 0.9):
        x = rng.normal(0, 3, 50).astype(np.float32)
        y = rng.normal(0, 3, 50).astype(np.float32)
        xr, yr = x.copy(), y.copy()
        ref_host.ref_smooth(fp(xr), fp(yr), 50, ctypes.c_float(w))
        xm, ym = api.smooth_shifts(x, y, w)
        assert np.array_equal(xm, xr) and np.array_equal(ym, yr)
    for dim in (3, 4, 6, 9):
        A = rng.normal(0, 1, (dim, dim)).astype(np.float32) + np.eye(dim, dtype=np.float32) * 3
        b = rng.normal(0, 1, dim).astype(np.float32)
        Ar, br = A.copy(), b.copy()
        ref_host.ref_lin_eqs(fp(Ar), fp(br), dim)
        ok, bm = api.lin_eqs(A, b)
        assert ok and np.array_equal(bm, br)


def test_lin_eqs_reference_kat(mc3lib):
    from motioncor3_b200 import api
    kat = json.load(open(os.path.join(GOLD, "lin_eqs_kat.json")))
    ok, sol = api.lin_eqs(np.array(kat["coeff"]), np.array(kat["vals"]))
    assert ok and np.allclose(sol, kat["solution"], atol=1e-4)


def test_patch_bookkeeping_bit_exact(mc3lib, ref_host):
    from motioncor3_b200 import api
    rng = np.random.default_rng(11)
    for (N, Px, Py) in ((10, 2, 2), (30, 5, 5), (41, 7, 5), (60, 5, 5)):
        P = Px * Py
        raw = rng.normal(0, 2.0, (P, N, 2)).astype(np.float32)
        raw[rng.integers(0, P), rng.integers(0, N)] += 15
        cen = np.array([[(i % Px + 0.5) * 4096 / Px + rng.normal(0, 40),
                         (i // Px + 0.5) * 4096 / Py + rng.normal(0, 40)] for i in range(P)], np.float32)
        sh = np.zeros((N, P, 2), np.float32)
        bad = np.zeros((N, P), np.uint8)
        ref_host.ref_patch_shifts(fp(raw), fp(cen), N, P, 4096, 4096, fp(sh), fp(bad))
        tab = np.ascontiguousarray(raw.transpose(1, 0, 2))
        rel = api.patch_make_relative(tab)
        assert np.array_equal(rel, sh)
        assert np.array_equal(api.patch_detect_bads(rel, cen, 4096, 4096), bad)


def test_golden_vectors(mc3lib):
    """Same checks from the committed fixtures (no reference tree needed)."""
    from motioncor3_b200 import api
    g = json.load(open(os.path.join(GOLD, "host_bookkeeping.json")))
    for c in g["peak2d"]:
        w = np.array(c["window"], np.float32).reshape(64, 64)
        assert np.array_equal(api.peak2d(w), np.array(c["shift"], np.float32))
    for c in g["remove_spikes"]:
        x, y = api.remove_spikes(np.array(c["x"]), np.array(c["y"]))
        assert np.array_equal(x, np.array(c["x_out"], np.float32))
        assert np.array_equal(y, np.array(c["y_out"], np.float32))
    for c in g["smooth"]:
        x, y = api.smooth_shifts(np.array(c["x"]), np.array(c["y"]), c["w"])
        assert np.array_equal(x, np.array(c["x_out"], np.float32))
        assert np.array_equal(y, np.array(c["y_out"], np.float32))


def _ref_fmint(ref_host, path, fm_dose, throws, n_raw, bin_z):
    n = n_raw
    I = lambda: np.zeros(n, np.int32)
    F = lambda: np.zeros(n, np.float32)
    st, sz, acc, cen, gs, gz, gc = I(), I(), F(), F(), I(), I(), F()
    ni, ng, hd = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
    ref_host.ref_fmint(path.encode() if path else None, ctypes.c_float(fm_dose), throws[0],
                       throws[1], n_raw, bin_z, n, ctypes.byref(ni), fp(st), fp(sz), fp(acc),
                       fp(cen), ctypes.byref(ng), fp(gs), fp(gz), fp(gc), ctypes.byref(hd))
    k, g = ni.value, ng.value
    return dict(start=st[:k], size=sz[:k], acc=acc[:k], center=cen[:k], g_start=gs[:g],
                g_size=gz[:g], g_center=gc[:g], has_dose=hd.value)


@pytest.mark.parametrize("text,fm_dose,n_raw,throws,bin_z", [
    ("40 4 0.5\n", 0.0, 40, (0, 0), 1),
    ("40 4 0.5\n", 0.0, 43, (0, 0), 2),
    ("40 4 0.5\n", 0.0, 37, (1, 2), 3),
    ("20 2 0.25\n30 3 0.25\n", 0.0, 50, (0, 0), 2),
    ("21 2 0.25\n30 3 0.25\n", 0.0, 51, (2, 0), 4),
    ("21 2 0.25\n\n30 3 0.25\n", 0.0, 60, (0, 1), 2),   # blank line: repeated entry
    ("40 4\n10 1\n", 0.7, 50, (0, 0), 2),                # two columns: -FmDose
    ("40 4 0.5\n20 2 0.6\n", 1.5, 30, (0, 0), 3),        # mixed doses: file dropped
    ("30 1 0.8\n", 1.2, 30, (2, 1), 4),                  # no integration: -FmDose doses
    (None, 0.9, 25, (3, 2), 3),                          # no file at all
])
def test_frame_tables_and_groups_match_reference(mc3lib, ref_host, tmp_path, text, fm_dose,
                                                 n_raw, throws, bin_z):
    """CReadFmIntFile::DoIt + CFmIntParam::Setup + CFmGroupParam::Setup of the
    reference, compiled from its sources, against mc3_read_fmint_file +
    mc3_frame_integration_tables + mc3_frame_groups: same rendered frames,
    doses, time stamps and groups (bit for bit)."""
    from motioncor3_b200 import api
    path = None
    if text is not None:
        f = tmp_path / "fmint.txt"
        f.write_text(text)
        path = str(f)
    ref = _ref_fmint(ref_host, path, fm_dose, throws, n_raw, bin_z)
    entries = api.read_fmint_file(path, fm_dose) if path else None
    t = api.frame_integration_tables(entries, n_raw, fm_dose=fm_dose, throw=throws)
    assert t["start"].tolist() == ref["start"].tolist()
    assert t["size"].tolist() == ref["size"].tolist()
    assert np.array_equal(t["acc_dose"], ref["acc"])
    assert t["dose_weight"] == ref["has_dose"]
    g = api.frame_groups(t["start"], t["size"], bin_z)
    assert g["start"].tolist() == ref["g_start"].tolist()
    assert g["size"].tolist() == ref["g_size"].tolist()
    assert np.array_equal(g["center"], ref["g_center"])


def _eer_module():
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "eer_t", os.path.join(os.path.dirname(__file__), "test_eer.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


@pytest.mark.parametrize("bits,sampling,cx,cy", [(7, 1, 96, 64), (8, 1, 96, 64), (7, 2, 4096, 8),
                                                 (7, 3, 4096, 8), (8, 2, 4096, 8)])
def test_eer_decoding_matches_reference(mc3lib, ref_host, tmp_path, bits, sampling, cx, cy):
    """mc3_eer_render against the reference's CDecodeEerFrame compiled from
    its sources (EerUtil/CDecodeEerFrame.cpp), on the same EER streams: the
    same electron counts at the same pixels, the 8-bit super-resolution
    branch included."""
    from motioncor3_b200 import api
    E = _eer_module()
    rng = np.random.default_rng(bits * 10 + sampling)
    cam = cx * cy
    fact = {1: 1, 2: 2, 3: 4}[sampling]
    raws = []
    for f in range(3):
        pix = np.sort(rng.choice(cam, size=400 + 50 * f, replace=False))
        sub = rng.integers(0, 16, size=pix.size)
        raws.append(E._encode7(pix, sub, cam) if bits == 7 else E._encode8(pix, cam))
    path = str(tmp_path / "r.eer")
    E._write_eer(path, cx, cy, raws, 65001 if bits == 7 else 65000)
    ours = api.eer_render(path, [0, 1], [1, 2], sampling=sampling)
    for i, frames in enumerate([[0], [1, 2]]):
        ref = np.zeros((cy * fact, cx * fact), np.uint8)
        for f in frames:
            b = np.frombuffer(raws[f], np.uint8).copy()
            ref_host.ref_eer_decode(fp(b), b.size, cx, cy, sampling, bits, fp(ref))
        assert np.array_equal(ours[i], ref), i
