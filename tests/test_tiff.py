"""TIFF movie reader (mc3_tiff_info / mc3_tiff_read, the role of
TiffUtil/CLoadTiffHeader.cpp + CLoadTiffImage.cpp).  Files written by Pillow
(its bundled libtiff: uncompressed, LZW, Deflate, PackBits strips) pin the
decoders against an independent encoder; a small writer here covers what
Pillow does not write (big-endian byte order, tiles, the horizontal
predictor, signed 16-bit samples, BigTIFF).  Frames come back bottom-up, as
CLoadTiffImage::mReadByStrip stores them."""
import struct
import zlib

import numpy as np
import pytest

PIL = pytest.importorskip("PIL.Image")


def _pillow_write(path, frames, compression):
    ims = [PIL.fromarray(f) for f in frames]
    ims[0].save(path, save_all=True, append_images=ims[1:], compression=compression)


@pytest.mark.parametrize("dtype,mode", [(np.uint8, 0), (np.uint16, 6), (np.float32, 2)])
@pytest.mark.parametrize("compression", ["raw", "tiff_lzw", "tiff_deflate", "packbits"])
def test_pillow_written_movies(mc3lib, tmp_path, dtype, mode, compression):
    from motioncor3_b200 import api
    if dtype == np.float32 and compression == "packbits":
        pytest.skip("Pillow does not write PackBits floats")
    rng = np.random.default_rng(7)
    hi = 256 if dtype == np.uint8 else 3000
    frames = rng.integers(0, hi, (4, 161, 203)).astype(dtype)
    frames[:, :20] = 5  # long runs as well as noise
    path = str(tmp_path / "m.tif")
    _pillow_write(path, frames, compression)
    info = api.tiff_info(path)
    assert info == dict(nx=203, ny=161, nz=4, mode=mode)
    out = api.tiff_read(path)
    assert np.array_equal(out, frames[:, ::-1])
    part = api.tiff_read(path, z0=1, nz=2, threads=1)
    assert np.array_equal(part, frames[1:3, ::-1])


def _write_tiff(path, frames, *, big_endian=False, tile=None, predictor=1, deflate=False,
                signed=False, bigtiff=False):
    """Minimal multi-page TIFF writer (TIFF 6.0 / BigTIFF layout)."""
    e = ">" if big_endian else "<"
    nz, ny, nx = frames.shape
    dt = frames.dtype
    bps = dt.itemsize * 8
    fmt = 3 if dt == np.float32 else (2 if signed else 1)
    data = bytearray()
    head = (b"MM" if big_endian else b"II") + (struct.pack(e + "HHHQ", 43, 8, 0, 0) if bigtiff
                                                else struct.pack(e + "HI", 42, 0))
    data += head
    ifd_ptr_pos = 8 if bigtiff else 4
    for z in range(nz):
        img = frames[z]
        blocks = []
        if tile:
            tw, th = tile
            for ty in range(0, ny, th):
                for tx in range(0, nx, tw):
                    t = np.zeros((th, tw), dt)
                    part = img[ty:ty + th, tx:tx + tw]
                    t[:part.shape[0], :part.shape[1]] = part
                    blocks.append(t)
        else:
            rps = 16
            blocks = [img[r:r + rps] for r in range(0, ny, rps)]
        raw = []
        for b in blocks:
            b = np.ascontiguousarray(b)
            if predictor == 2:
                d = b.copy()
                d[:, 1:] = b[:, 1:] - b[:, :-1]
                b = d
            by = b.astype(dt.newbyteorder(e)).tobytes()
            raw.append(zlib.compress(by) if deflate else by)
        offsets = []
        for r in raw:
            offsets.append(len(data))
            data += r
        if len(data) % 2:
            data += b"\0"
        tags = [(256, 4, [nx]), (257, 4, [ny]), (258, 3, [bps]), (259, 3, [8 if deflate else 1]),
                (277, 3, [1]), (339, 3, [fmt])]
        if predictor == 2:
            tags.append((317, 3, [2]))
        if tile:
            tags += [(322, 4, [tile[0]]), (323, 4, [tile[1]]), (324, 4, offsets),
                     (325, 4, [len(r) for r in raw])]
        else:
            tags += [(273, 4, offsets), (278, 4, [16]), (279, 4, [len(r) for r in raw])]
        tags.sort()
        ifd_off = len(data)
        struct.pack_into(e + ("Q" if bigtiff else "I"), data, ifd_ptr_pos, ifd_off)
        # out-of-line values first
        ents = []
        extra = bytearray()
        esz, cnt_fmt, inl = (20, "Q", 8) if bigtiff else (12, "I", 4)
        n_ifd_bytes = (8 if bigtiff else 2) + len(tags) * esz + (8 if bigtiff else 4)
        base = ifd_off + n_ifd_bytes
        for tag, typ, vals in tags:
            f = "H" if typ == 3 else "I"
            payload = struct.pack(e + f * len(vals), *vals)
            if len(payload) <= inl:
                ents.append(struct.pack(e + "HH" + cnt_fmt, tag, typ, len(vals)) +
                            payload.ljust(inl, b"\0"))
            else:
                off = base + len(extra)
                extra += payload
                ents.append(struct.pack(e + "HH" + cnt_fmt, tag, typ, len(vals)) +
                            struct.pack(e + ("Q" if bigtiff else "I"), off))
        data += struct.pack(e + ("Q" if bigtiff else "H"), len(tags)) + b"".join(ents)
        ifd_ptr_pos = len(data)
        data += b"\0" * (8 if bigtiff else 4)
        data += extra
    with open(path, "wb") as fh:
        fh.write(bytes(data))


@pytest.mark.parametrize("opts", [dict(big_endian=True), dict(tile=(32, 16)),
                                  dict(tile=(48, 32), deflate=True, big_endian=True),
                                  dict(predictor=2, deflate=True), dict(signed=True),
                                  dict(bigtiff=True, deflate=True)])
def test_written_layouts(mc3lib, tmp_path, opts):
    from motioncor3_b200 import api
    rng = np.random.default_rng(11)
    dt = np.int16 if opts.get("signed") else np.uint16
    frames = rng.integers(0 if dt == np.uint16 else -500, 3000, (3, 70, 90)).astype(dt)
    path = str(tmp_path / "w.tif")
    _write_tiff(path, frames, **opts)
    info = api.tiff_info(path)
    assert info["nx"] == 90 and info["ny"] == 70 and info["nz"] == 3
    assert info["mode"] == (1 if opts.get("signed") else 6)
    assert np.array_equal(api.tiff_read(path), frames[:, ::-1])


def test_eight_bit_predictor_and_tiles(mc3lib, tmp_path):
    from motioncor3_b200 import api
    rng = np.random.default_rng(12)
    frames = rng.integers(0, 256, (2, 45, 77)).astype(np.uint8)
    path = str(tmp_path / "p.tif")
    _write_tiff(path, frames, tile=(16, 16), predictor=2, deflate=True)
    assert api.tiff_info(path)["mode"] == 0
    assert np.array_equal(api.tiff_read(path), frames[:, ::-1])


def test_unreadable_and_unsupported(mc3lib, tmp_path):
    from motioncor3_b200 import api
    with pytest.raises(api.MC3Error) as e:
        api.tiff_info(str(tmp_path / "none.tif"))
    assert e.value.code == api.MC3_EIO
    rgb = np.zeros((20, 30, 3), np.uint8)
    path = str(tmp_path / "rgb.tif")
    PIL.fromarray(rgb).save(path)
    with pytest.raises(api.MC3Error) as e:
        api.tiff_info(path)
    assert e.value.code == api.MC3_EUNSUPPORTED
