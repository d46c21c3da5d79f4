"""EER movies (mc3_eer_info / mc3_eer_render; EerUtil/CLoadEerFrames.cpp,
CDecodeEerFrame.cpp, CRenderMrcStack.cpp).  The reference program here is
built without libtiff, so the decoder is pinned by an encoder written here
from the same stream layout: run lengths of 7 bits (compression 65001) or
8 bits (65000) with 127 / 255 meaning "run continues, no electron", each
electron followed by a 4-bit sub-pixel code (stored XOR 0xA in the 7-bit
form), codes packed least-significant bit first (7-bit) or as 12-bit pairs
in three bytes (8-bit)."""
import struct

import numpy as np
import pytest


def _encode7(pix, sub, cam):
    bits = []

    def put(v, n):
        bits.extend((v >> k) & 1 for k in range(n))

    cur = 0
    for n, s in zip(pix, sub):
        gap = n - cur
        while gap >= 127:
            put(127, 7)
            gap -= 127
        put(gap, 7)
        put(s ^ 0x0A, 4)
        cur = n + 1
    rest = cam - cur
    while rest > 0:  # runs past the end stop the decoder
        put(127 if rest >= 127 else rest, 7)
        rest -= 127
    while len(bits) % 8:
        bits.append(0)
    b = np.packbits(np.array(bits, np.uint8).reshape(-1, 8)[:, ::-1], axis=1).ravel()
    return bytes(b)


def _encode8(pix, cam):
    codes = []
    cur = 0
    for n in pix:
        gap = n - cur
        while gap >= 255:
            codes.append(255)
            gap -= 255
        codes.append(gap)
        cur = n + 1
    rest = cam - cur
    while rest > 0:
        codes.append(255 if rest >= 255 else rest)
        rest -= 255
    if len(codes) % 2:
        codes.append(255)
    out = bytearray()
    for a, c in zip(codes[0::2], codes[1::2]):  # sub-pixel codes 0 (not used when counting)
        out += bytes([a & 0xFF, (c & 0x0F) << 4, (c >> 4) & 0x0F])
    return bytes(out)


def _write_eer(path, cam_x, cam_y, frames, compression):
    """Classic little-endian TIFF, one directory and one strip per frame."""
    data = bytearray(b"II" + struct.pack("<HI", 42, 0))
    ptr = 4
    for raw in frames:
        off = len(data)
        data += raw
        if len(data) % 2:
            data += b"\0"
        tags = [(256, 4, cam_x), (257, 4, cam_y), (258, 3, 8), (259, 3, compression),
                (273, 4, off), (277, 3, 1), (278, 4, cam_y), (279, 4, len(raw))]
        ifd = len(data)
        struct.pack_into("<I", data, ptr, ifd)
        data += struct.pack("<H", len(tags))
        for tag, typ, val in tags:
            v = struct.pack("<H", val) + b"\0\0" if typ == 3 else struct.pack("<I", val)
            data += struct.pack("<HHI", tag, typ, 1) + v
        ptr = len(data)
        data += b"\0\0\0\0"
    with open(path, "wb") as fh:
        fh.write(bytes(data))


def _electrons(rng, cam, n):
    pix = np.sort(rng.choice(cam, size=n, replace=False))
    sub = rng.integers(0, 16, size=n)
    return pix, sub


@pytest.mark.parametrize("bits", [7, 8])
def test_counted_rendering_and_integration(mc3lib, tmp_path, bits):
    from motioncor3_b200 import api
    rng = np.random.default_rng(bits)
    cx, cy, nfr = 96, 64, 7
    cam = cx * cy
    ev, raws = [], []
    for f in range(nfr):
        pix, sub = _electrons(rng, cam, 300 + 40 * f)
        ev.append(pix)
        raws.append(_encode7(pix, sub, cam) if bits == 7 else _encode8(pix, cam))
    path = str(tmp_path / "m.eer")
    _write_eer(path, cx, cy, raws, 65001 if bits == 7 else 65000)
    assert api.eer_info(path) == dict(cam_x=cx, cam_y=cy, n_frames=nfr, bits=bits)
    out = api.eer_render(path, [0, 2, 5], [2, 3, 2])
    for i, (a, b) in enumerate([(0, 2), (2, 5), (5, 7)]):
        ref = np.zeros(cam, np.uint16)
        for f in range(a, b):
            ref[ev[f]] += 1
        assert np.array_equal(out[i].ravel(), (ref % 256).astype(np.uint8)), i


@pytest.mark.parametrize("sampling", [2, 3])
def test_super_resolution_positions(mc3lib, tmp_path, sampling):
    """7-bit streams at -EerSampling 2 / 3: the electron lands at
    ((n mod 4096) << k | sub-pixel x bits, (n / 4096) << k | sub-pixel y bits)
    of the 2x / 4x grid (CDecodeEerFrame::mFindElectron)."""
    from motioncor3_b200 import api
    rng = np.random.default_rng(20 + sampling)
    cx, cy = 4096, 8
    cam = cx * cy
    pix, sub = _electrons(rng, cam, 500)
    path = str(tmp_path / "s.eer")
    _write_eer(path, cx, cy, [_encode7(pix, sub, cam)], 65001)
    out = api.eer_render(path, [0], [1], sampling=sampling)
    k, fact = (1, 2) if sampling == 2 else (2, 4)
    assert out.shape == (1, cy * fact, cx * fact)
    ref = np.zeros((cy * fact, cx * fact), np.uint8)
    for n, s in zip(pix, sub):
        if sampling == 2:
            x = ((n & 4095) << 1) | ((s & 2) >> 1)
            y = ((n >> 12) << 1) | ((s & 8) >> 3)
        else:
            x = ((n & 4095) << 2) | (s & 3)
            y = ((n >> 12) << 2) | ((s & 12) >> 2)
        ref[y, x] += 1
    assert np.array_equal(out[0], ref)


def test_unsupported_inputs(mc3lib, tmp_path):
    from motioncor3_b200 import api
    path = str(tmp_path / "odd.eer")
    _write_eer(path, 100, 4, [_encode7(np.array([5]), np.array([0]), 400)], 65001)
    with pytest.raises(api.MC3Error):  # super-resolution needs 4096-pixel rows
        api.eer_render(path, [0], [1], sampling=2)
    _write_eer(path, 100, 4, [b"\0" * 16], 65002)
    with pytest.raises(api.MC3Error):
        api.eer_info(path)
