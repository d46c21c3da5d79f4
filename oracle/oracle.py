"""ctypes binding of the FP64 CPU oracle (TEST INFRASTRUCTURE ONLY).

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline / reference arm.  Builds oracle/_build/libmc3_oracle.so with the
Makefile beside this file when it is missing or stale, and the reference
host-code checker oracle/_ref/libmc3ref_host.so when the reference tree is
present (the prebuilt .so is used otherwise).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libmc3_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libmc3ref_host.so")
REF_CTF_LIB = os.path.join(HERE, "_ref", "libmc3ref_ctf.so")
# The reference source tree: $MC3_REFERENCE, else a directory named
# "reference" beside the repository.  Absent on machines that only run the
# prebuilt checkers.
REF_TREE = os.environ.get("MC3_REFERENCE") or os.path.normpath(
    os.path.join(HERE, "..", "..", "reference"))
_VP = ctypes.c_void_p


def _cxx_env():
    env = dict(os.environ)
    if os.path.exists("/usr/bin/g++"):
        env["CXX"] = "/usr/bin/g++"
    return env


def build() -> str:
    srcs = [os.path.join(HERE, f) for f in ("mc3_oracle.cpp", "mc3_oracle.h", "ctf_oracle.cpp",
                                            "cnn_oracle.cpp", "Makefile")]
    if not os.path.exists(LIB) or any(os.path.getmtime(s) > os.path.getmtime(LIB) for s in srcs):
        subprocess.run(["make", "-C", HERE], check=True, env=_cxx_env(), capture_output=True)
    return LIB


def build_ref_host() -> str | None:
    """Compiles the reference's own host classes when the reference tree exists."""
    if os.path.isdir(REF_TREE):
        d = os.path.join(HERE, "ref_host")
        subprocess.run(["make", "-C", d, f"REF={REF_TREE}"], check=True, capture_output=True)
    return REF_LIB if os.path.exists(REF_LIB) else None


def build_ref_program() -> str | None:
    """Compiles the reference program itself (checker for the command line)
    from the reference tree when it exists; make keeps it incremental."""
    exe = os.path.join(HERE, "_ref", "MotionCor3")
    if os.path.isdir(REF_TREE):
        d = os.path.join(HERE, "ref_full")
        subprocess.run(["make", "-C", d, f"REF={REF_TREE}", "-j8"], check=True, capture_output=True)
    return exe if os.path.exists(exe) else None


class OracleParams(ctypes.Structure):
    _fields_ = [
        ("patch", ctypes.c_int * 2),
        ("iter", ctypes.c_int),
        ("tol", ctypes.c_float),
        ("bft", ctypes.c_float * 2),
        ("phase_only", ctypes.c_int),
        ("fm_dose", ctypes.c_float),
        ("pix_size", ctypes.c_float),
        ("kv", ctypes.c_int),
        ("group", ctypes.c_int * 2),
        ("fm_ref", ctypes.c_int),
        ("sum_range", ctypes.c_float * 2),
        ("correct_bad", ctypes.c_int),
        ("split_sum", ctypes.c_int),
        ("ft_bin", ctypes.c_float),
        ("out_stack", ctypes.c_int * 2),
        ("int_size", _VP),
        ("acc_dose", _VP),
        ("dose_weight", ctypes.c_int),
        ("dark", _VP),
        ("mag", ctypes.c_float * 3),
        ("in_fm_motion", ctypes.c_int),
        ("corr_interp", ctypes.c_int),
        ("defects", _VP),
    ]


class OracleResult(ctypes.Structure):
    _fields_ = [
        ("n_sums", ctypes.c_int),
        ("sums", _VP),
        ("global_shifts", _VP),
        ("n_patches", ctypes.c_int),
        ("patch_shifts", _VP),
        ("patch_centers", _VP),
        ("patch_bad", _VP),
        ("iterations", _VP),
        ("bad_map", _VP),
        ("use_global_shifts", _VP),
        ("use_patch_shifts", _VP),
        ("use_patch_centers", _VP),
        ("use_patch_bad", _VP),
        ("stack", _VP),
        ("stack_frames", ctypes.c_int),
    ]


_L = None


def lib() -> ctypes.CDLL:
    global _L
    if _L is None:
        _L = ctypes.CDLL(build())
    return _L


def _p(a):
    return None if a is None else a.ctypes.data_as(_VP)


def params(**kw) -> OracleParams:
    p = OracleParams()
    lib().oracle_default_params(ctypes.byref(p))
    for k, v in kw.items():
        if k in ("patch", "bft", "group", "sum_range", "out_stack", "mag"):
            arr = getattr(p, k)
            for i, x in enumerate(v[:len(arr)]):
                arr[i] = x
        else:
            setattr(p, k, v)
    return p


def process_movie(frames: np.ndarray, gain=None, force=None, int_size=None, acc_dose=None,
                  dark=None, defects=None, **kw) -> dict:
    """Runs the whole oracle path.  `force` may hold global_shifts (and
    patch_shifts / patch_centers / patch_bad) to correct with given shifts;
    int_size / acc_dose describe rendered frames of a frame-integration file."""
    p = params(**kw)
    tabs = []
    if int_size is not None:
        isz = np.ascontiguousarray(int_size, np.int32)
        tabs.append(isz)
        p.int_size = isz.ctypes.data
    if acc_dose is not None:
        acc = np.ascontiguousarray(acc_dose, np.float32)
        tabs.append(acc)
        p.acc_dose = acc.ctypes.data
    if dark is not None:
        dk = np.ascontiguousarray(dark, np.float32)
        tabs.append(dk)
        p.dark = dk.ctypes.data
    if defects is not None:
        df = np.ascontiguousarray(defects, np.uint8)
        tabs.append(df)
        p.defects = df.ctypes.data
    nz, ny, nx = frames.shape
    fr = np.ascontiguousarray(frames, np.float32)
    g = None if gain is None else np.ascontiguousarray(gain, np.float32)
    P = (p.patch[0] * p.patch[1]) if (p.patch[0] > 1 and p.patch[1] > 1) else 0
    ob, oh = nx, ny
    if p.ft_bin > 0:  # CInput::GetBinnedSize (CInput.cpp:678-688)
        ob = int(np.float32(nx) / np.float32(p.ft_bin) + np.float32(0.5)) // 2 * 2
        oh = int(np.float32(ny) / np.float32(p.ft_bin) + np.float32(0.5)) // 2 * 2
    sums = np.zeros((5, oh, ob), np.float32)
    gsh = np.zeros((nz, 2), np.float32)
    psh = np.zeros((nz, max(P, 1), 2), np.float32)
    pc = np.zeros((max(P, 1), 2), np.float32)
    pb = np.zeros((nz, max(P, 1)), np.uint8)
    its = np.zeros(1 + P, np.int32)
    bad = np.zeros((ny, nx), np.uint8)
    r = OracleResult()
    r.sums = sums.ctypes.data
    r.global_shifts = gsh.ctypes.data
    r.patch_shifts = psh.ctypes.data
    r.patch_centers = pc.ctypes.data
    r.patch_bad = pb.ctypes.data
    r.iterations = its.ctypes.data
    r.bad_map = bad.ctypes.data
    stack = None
    if p.out_stack[0]:
        stack = np.zeros((nz, oh, ob), np.float32)
        r.stack = stack.ctypes.data
    keep = []
    if force:
        for key in ("global_shifts", "patch_shifts", "patch_centers", "patch_bad"):
            if force.get(key) is not None:
                dt = np.uint8 if key == "patch_bad" else np.float32
                a = np.ascontiguousarray(force[key], dt)
                keep.append(a)
                setattr(r, "use_" + key, a.ctypes.data)
    rc = lib().oracle_process_movie(ctypes.byref(p), _p(fr), nx, ny, nz, _p(g), ctypes.byref(r))
    if rc != 0:
        raise RuntimeError(f"oracle_process_movie failed ({rc})")
    return dict(sums=sums[: r.n_sums], global_shifts=gsh, patch_shifts=psh if P else None,
                patch_centers=pc if P else None, patch_bad=pb if P else None, iterations=its,
                bad_map=bad, n_sums=r.n_sums,
                stack=None if stack is None else stack[: r.stack_frames])


def rfft2(img: np.ndarray, normalise: bool = True) -> np.ndarray:
    ny, nx = img.shape
    a = np.ascontiguousarray(img, np.float64)
    out = np.zeros((ny, nx // 2 + 1), np.complex128)
    lib().oracle_rfft2(_p(a), _p(out), nx, ny, int(normalise))
    return out


def irfft2(spec: np.ndarray, nx: int) -> np.ndarray:
    ny = spec.shape[0]
    a = np.ascontiguousarray(spec, np.complex128)
    out = np.zeros((ny, nx), np.float64)
    lib().oracle_irfft2(_p(a), _p(out), nx, ny)
    return out


def cfft(x: np.ndarray, direction: int) -> np.ndarray:
    a = np.ascontiguousarray(x, np.complex128)
    out = np.zeros_like(a)
    lib().oracle_cfft(_p(a), _p(out), len(a), direction)
    return out


def detect_bad(sum_img: np.ndarray) -> np.ndarray:
    ny, nx = sum_img.shape
    a = np.ascontiguousarray(sum_img, np.float64)
    bad = np.zeros((ny, nx), np.uint8)
    lib().oracle_detect_bad(_p(a), nx, ny, _p(bad))
    return bad


def correct_bad(frame: np.ndarray, bad: np.ndarray) -> np.ndarray:
    ny, nx = frame.shape
    a = np.ascontiguousarray(frame, np.float64).copy()
    b = np.ascontiguousarray(bad, np.uint8)
    lib().oracle_correct_bad(_p(a), _p(b), nx, ny)
    return a


def correlate_window(grp: np.ndarray, sum_: np.ndarray, bfactor: float, phase_only=0, sea=(64, 64)):
    cy, cx = grp.shape
    g = np.ascontiguousarray(grp, np.complex128)
    s = np.ascontiguousarray(sum_, np.complex128)
    win = np.zeros((sea[1], sea[0]), np.float32)
    lib().oracle_correlate_window(_p(g), _p(s), cx, cy, ctypes.c_float(bfactor), phase_only, sea[0],
                                  sea[1], _p(win))
    return win


def peak2d(win: np.ndarray) -> np.ndarray:
    w = np.ascontiguousarray(win, np.float32)
    out = np.zeros(2, np.float32)
    lib().oracle_peak2d(_p(w), w.shape[1], w.shape[0], _p(out))
    return out


def iterative_align(spec: np.ndarray, group: int, max_iter: int, tol: float, bfactor: float,
                    phase_only: int = 0, init=None):
    """init: optional first iterate [n][2] of the per-frame shifts (warm start)."""
    n, cy, cx = spec.shape
    s = np.ascontiguousarray(spec, np.complex128)
    out = np.zeros((n, 2), np.float32)
    ini = None if init is None else np.ascontiguousarray(init, np.float32)
    it = lib().oracle_iterative_align_warm(_p(s), cx, cy, n, group, max_iter, ctypes.c_float(tol),
                                           ctypes.c_float(bfactor), phase_only, _p(ini), _p(out))
    return out, it


def local_gather(img: np.ndarray, centers, shifts, bad=None) -> np.ndarray:
    ny, nx = img.shape
    a = np.ascontiguousarray(img, np.float64)
    out = np.zeros_like(a)
    c = np.ascontiguousarray(centers, np.float32)
    s = np.ascontiguousarray(shifts, np.float32)
    b = None if bad is None else np.ascontiguousarray(bad, np.uint8)
    lib().oracle_local_gather(_p(a), _p(out), nx, ny, _p(c), _p(s), _p(b), len(c))
    return out


def dose_weights(acc_dose, frame: int, cmpx: int, cmpy: int, pix: float, kv: int) -> np.ndarray:
    acc = np.ascontiguousarray(acc_dose, np.float32)
    out = np.zeros((cmpy, cmpx), np.float64)
    lib().oracle_dose_weights(_p(acc), len(acc), frame, cmpx, cmpy, ctypes.c_float(pix), kv, _p(out))
    return out


def remove_spikes(sx, sy):
    x = np.ascontiguousarray(sx, np.float32).copy()
    y = np.ascontiguousarray(sy, np.float32).copy()
    lib().oracle_remove_spikes(_p(x), _p(y), len(x))
    return x, y


def lin_eqs(a, b):
    A = np.ascontiguousarray(a, np.float32).copy()
    B = np.ascontiguousarray(b, np.float32).copy()
    ok = lib().oracle_lin_eqs(_p(A), _p(B), len(B))
    return bool(ok), B


def patch_make_relative(shifts):
    s = np.ascontiguousarray(shifts, np.float32).copy()
    lib().oracle_patch_make_relative(_p(s), s.shape[0], s.shape[1])
    return s


def patch_detect_bads(shifts, centers, nx, ny):
    s = np.ascontiguousarray(shifts, np.float32)
    c = np.ascontiguousarray(centers, np.float32)
    bad = np.zeros(s.shape[:2], np.uint8)
    lib().oracle_patch_detect_bads(_p(s), _p(c), s.shape[0], s.shape[1], nx, ny, _p(bad))
    return bad


def ctf_spectrum(img: np.ndarray, pix: float):
    """(half spectrum [512][257], lowpassed full spectrum [512][512], pixel
    size) the CTF is fitted to, or None when no 512 x 512 tile fits."""
    im = np.ascontiguousarray(img, np.float32)
    avg = np.zeros((512, 257), np.float32)
    full = np.zeros((512, 512), np.float32)
    pn = ctypes.c_float(0)
    if lib().oracle_ctf_spectrum(_p(im), im.shape[1], im.shape[0], ctypes.c_float(pix), _p(avg),
                                 _p(full), ctypes.byref(pn)):
        return None
    return avg, full, pn.value


def ctf_stages(img: np.ndarray, pix: float):
    """dict(raw, bg, half, full, pix_n) of the spectrum stages, or None."""
    im = np.ascontiguousarray(img, np.float32)
    raw = np.zeros((512, 257), np.float32)
    bg = np.zeros((512, 257), np.float32)
    half = np.zeros((512, 257), np.float32)
    full = np.zeros((512, 512), np.float32)
    pn = ctypes.c_float(0)
    if lib().oracle_ctf_stages(_p(im), im.shape[1], im.shape[0], ctypes.c_float(pix), _p(raw), _p(bg),
                               _p(half), _p(full), ctypes.byref(pn)):
        return None
    return dict(raw=raw, bg=bg, half=half, full=full, pix_n=pn.value)


def ctf_search(avg: np.ndarray, pix_n: float, kv=300.0, cs=2.7, ac=0.07, ext_phase=0.0) -> np.ndarray:
    a = np.ascontiguousarray(avg, np.float32)
    res = np.zeros(6, np.float32)
    f = ctypes.c_float
    lib().oracle_ctf_search(_p(a), f(pix_n), f(kv), f(cs), f(ac), f(ext_phase), _p(res))
    return res


def find_ctf(img: np.ndarray, pix: float, kv=300.0, cs=2.7, ac=0.07, ext_phase=0.0):
    """(res6, 512 x 512 diagnostic image) or None when no tile fits."""
    im = np.ascontiguousarray(img, np.float32)
    res = np.zeros(6, np.float32)
    out = np.zeros((512, 512), np.float32)
    f = ctypes.c_float
    if lib().oracle_find_ctf(_p(im), im.shape[1], im.shape[0], f(pix), f(kv), f(cs), f(ac),
                             f(ext_phase), _p(res), _p(out)):
        return None
    return res, out


def ctf_param(kv: float, cs: float, ac: float, pix: float) -> np.ndarray:
    out = np.zeros(3, np.float32)
    f = ctypes.c_float
    lib().oracle_ctf_param(f(kv), f(cs), f(ac), f(pix), _p(out))
    return out


def ctf_model(kv, cs, ac, pix, dfmin_px, dfmax_px, azim_rad, ext_rad) -> np.ndarray:
    out = np.zeros((512, 257), np.float32)
    f = ctypes.c_float
    lib().oracle_ctf_model(f(kv), f(cs), f(ac), f(pix), f(dfmin_px), f(dfmax_px), f(azim_rad),
                           f(ext_rad), _p(out))
    return out


class ShiftNet:
    """FP64 oracle of the shift-proposal network (cnn_oracle.cpp): strided
    convolutions + ReLU, global average pool, linear head."""

    def __init__(self, layers, nout: int, seed: int = 0):
        L = lib()
        L.cnn_create.restype = _VP
        L.cnn_num_params.restype = ctypes.c_long
        L.cnn_loss_grad.restype = ctypes.c_double
        spec = np.ascontiguousarray(np.array(layers, np.int32).ravel())
        self._L = L
        self._h = _VP(L.cnn_create(len(layers), _p(spec), nout, ctypes.c_uint(seed)))
        self.nout = nout
        self.cin = int(layers[0][0])

    def __del__(self):
        if getattr(self, "_h", None):
            self._L.cnn_destroy(self._h)
            self._h = None

    @property
    def n_params(self) -> int:
        return int(self._L.cnn_num_params(self._h))

    def params(self) -> np.ndarray:
        out = np.zeros(self.n_params)
        self._L.cnn_get_params(self._h, _p(out))
        return out

    def set_params(self, p: np.ndarray) -> None:
        self._L.cnn_set_params(self._h, _p(np.ascontiguousarray(p, np.float64)))

    def forward(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float64)
        out = np.zeros(self.nout)
        self._L.cnn_loss_grad(self._h, _p(x), *x.shape, None, None, _p(out))
        return out

    def loss_grad(self, x: np.ndarray, target: np.ndarray, grad: np.ndarray) -> float:
        """Loss 0.5 |f(x) - target|^2; its gradient is ADDED to grad."""
        x = np.ascontiguousarray(x, np.float64)
        t = np.ascontiguousarray(target, np.float64)
        return float(self._L.cnn_loss_grad(self._h, _p(x), *x.shape, _p(t), _p(grad), None))


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even), kept as float32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32)


def split_bf16_matmul(a: np.ndarray, b: np.ndarray, products: int = 3) -> np.ndarray:
    """a @ b as the tensor-core form computes it: each FP32 operand split into
    BF16 hi + lo, products hi*hi + hi*lo + lo*hi (products=3) or hi*hi alone
    (products=1), each exact in FP32 and accumulated in FP32."""
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    ah, bh = bf16(a), bf16(b)
    out = (ah @ bh).astype(np.float32)
    if products == 3:
        al, bl = bf16(a - ah), bf16(b - bh)
        out = out + (ah @ bl).astype(np.float32) + (al @ bh).astype(np.float32)
    return out


def split_bf16_dft(x: np.ndarray, products: int = 3) -> np.ndarray:
    """Complex DFT along axis 0 of x [n][m] as four real split-BF16 GEMMs with
    the FP32 DFT matrix (the form (1) transform of the patch stacks)."""
    n = x.shape[0]
    k = np.arange(n)
    w = np.exp(-2j * np.pi * np.outer(k, k) / n)
    wr, wi = w.real.astype(np.float32), w.imag.astype(np.float32)
    xr, xi = x.real.astype(np.float32), x.imag.astype(np.float32)
    mm = lambda a, b: split_bf16_matmul(a, b, products)
    return (mm(wr, xr) - mm(wi, xi)) + 1j * (mm(wr, xi) + mm(wi, xr))


def ref_ctf():
    """The reference's CTF fitting drivers with host stand-ins for their
    kernels (None when neither the tree nor the prebuilt checker exists)."""
    build_ref_host()
    if not os.path.exists(REF_CTF_LIB):
        return None
    L = ctypes.CDLL(REF_CTF_LIB)
    L.ref_ctf_param.restype = None
    L.ref_ctf_search.restype = None
    return L


def ref_host():
    """The reference's own host classes (None when neither the tree nor the
    prebuilt checker is available)."""
    path = build_ref_host()
    return ctypes.CDLL(path) if path else None
