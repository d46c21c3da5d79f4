"""Minimal MRC read/write helpers (numpy) for movies, gains and sums.

Header fields follow the MRC2014 layout the reference writes
(LibSrc/Mrcfile/Header/CSaveMainHeader.cpp); reading supports modes 0, 1, 2
and 6 in either byte order.
"""
from __future__ import annotations

import numpy as np

_DT = {0: np.uint8, 1: np.int16, 2: np.float32, 6: np.uint16}
_MODE = {np.dtype(np.uint8): 0, np.dtype(np.int16): 1, np.dtype(np.float32): 2, np.dtype(np.uint16): 6}


def read_header(path: str) -> dict:
    raw = np.fromfile(path, dtype=np.uint8, count=1024)
    for order in ("<", ">"):
        ints = raw[:96].view(order + "i4")
        if int(ints[3]) in _DT or int(ints[3]) == 101:
            floats = raw[:96].view(order + "f4")
            return dict(nx=int(ints[0]), ny=int(ints[1]), nz=int(ints[2]), mode=int(ints[3]),
                        nsymbt=int(ints[23]), amin=float(floats[19]), amax=float(floats[20]),
                        amean=float(floats[21]), xlen=float(floats[10]), mx=int(ints[7]),
                        order=order, raw=raw)
    raise ValueError(f"{path}: not an MRC file with a supported mode")


def pack4(frames: np.ndarray) -> np.ndarray:
    """[nz][ny][nx] values 0..15 -> mode-101 bytes [nz][ny][(nx+1)//2], the
    even pixel in the low nibble (LibSrc/Mrcfile/Image/C4BitImage.cpp)."""
    a = np.asarray(frames, np.uint8) & 0xF
    nz, ny, nx = a.shape
    if nx % 2:
        a = np.concatenate([a, np.zeros((nz, ny, 1), np.uint8)], axis=2)
    return (a[:, :, 0::2] | (a[:, :, 1::2] << 4)).astype(np.uint8)


def unpack4(packed: np.ndarray, nx: int) -> np.ndarray:
    p = np.asarray(packed, np.uint8)
    out = np.empty(p.shape[:2] + (2 * p.shape[2],), np.uint8)
    out[:, :, 0::2] = p & 0xF
    out[:, :, 1::2] = p >> 4
    return out[:, :, :nx]


def read(path: str) -> np.ndarray:
    h = read_header(path)
    if h["mode"] == 101:
        pk = (h["nx"] + 1) // 2
        a = np.fromfile(path, dtype=np.uint8, count=pk * h["ny"] * h["nz"],
                        offset=1024 + h["nsymbt"])
        return unpack4(a.reshape(h["nz"], h["ny"], pk), h["nx"])
    dt = np.dtype(_DT[h["mode"]]).newbyteorder(h["order"])
    n = h["nx"] * h["ny"] * h["nz"]
    a = np.fromfile(path, dtype=dt, count=n, offset=1024 + h["nsymbt"])
    return a.reshape(h["nz"], h["ny"], h["nx"]).astype(dt.newbyteorder("="))


def write(path: str, data: np.ndarray, pix: float = 1.0, four_bit: bool = False) -> None:
    """four_bit: store uint8 values 0..15 as packed mode 101."""
    a = np.ascontiguousarray(data)
    if a.ndim == 2:
        a = a[None]
    mode = 101 if four_bit else _MODE[a.dtype]
    nz, ny, nx = a.shape
    h = np.zeros(256, np.int32)
    f = h.view(np.float32)
    h[0:4] = (nx, ny, nz, mode)
    h[7:10] = (nx, ny, nz)
    f[10:13] = (nx * pix, ny * pix, nz * pix)
    f[13:16] = 90.0
    h[16:19] = (1, 2, 3)
    af = a.astype(np.float64)
    f[19], f[20], f[21] = af.min(), af.max(), af.mean()
    b = h.view(np.uint8).copy()
    b[208:212] = np.frombuffer(b"MAP ", np.uint8)
    b[212:216] = (0x44, 0x44, 0, 0)
    with open(path, "wb") as fh:
        fh.write(b.tobytes())
        fh.write(pack4(a).tobytes() if four_bit else a.tobytes())
