"""ctypes binding of libmc3 (include/mc3.h).

`MotionCor3` mirrors the reference program's single-movie flow
(CMain::mDoSingleCryoEM, CMain.cpp:93): options as in CInput (CInput.cpp:82-127),
one call from raw frames to the unweighted / dose-weighted sums and the
global and patch shift tables.  Component functions expose the individual
replaced interfaces (FFT, phase shift, correlation + peak, bad pixels, local
gather, dose-weighted sums, host bookkeeping) for integrators and tests.

Device arrays are passed as torch CUDA tensors (their data_ptr); host arrays
as numpy arrays.  Errors raise MC3Error carrying the library status code.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
lib_path = os.path.join(_HERE, "libmc3.so")

MC3_OK, MC3_EINVAL, MC3_ENOMEM, MC3_ECUDA, MC3_ETIMEOUT, MC3_EIO, MC3_EUNSUPPORTED = range(7)


class MC3Error(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        msg = _lib().mc3_strerror(code).decode() if _LIB is not None else f"status {code}"
        super().__init__(f"{what}: {msg} (status {code})" if what else f"{msg} (status {code})")


class _Params(ctypes.Structure):
    _fields_ = [
        ("patch", ctypes.c_int * 3),
        ("iter", ctypes.c_int),
        ("tol", ctypes.c_float),
        ("bft", ctypes.c_float * 2),
        ("phase_only", ctypes.c_int),
        ("ft_bin", ctypes.c_float),
        ("init_dose", ctypes.c_float),
        ("fm_dose", ctypes.c_float),
        ("pix_size", ctypes.c_float),
        ("kv", ctypes.c_int),
        ("group", ctypes.c_int * 2),
        ("fm_ref", ctypes.c_int),
        ("sum_range", ctypes.c_float * 2),
        ("align", ctypes.c_int),
        ("correct_bad", ctypes.c_int),
        ("gpu", ctypes.c_int),
        ("split_sum", ctypes.c_int),
        ("out_stack", ctypes.c_int * 2),
        ("mag", ctypes.c_float * 3),
        ("in_fm_motion", ctypes.c_int),
        ("corr_interp", ctypes.c_int),
        ("cs", ctypes.c_float),
        ("amp_cont", ctypes.c_float),
        ("ext_phase", ctypes.c_float),
        ("dft_gemm", ctypes.c_int),
    ]


class _PlanInfo(ctypes.Structure):
    _fields_ = [
        ("n_sums", ctypes.c_int),
        ("n_patches", ctypes.c_int),
        ("xcf_size", ctypes.c_int * 2),
        ("patch_size", ctypes.c_int * 2),
        ("xcf_bin", ctypes.c_float * 2),
        ("device_bytes", ctypes.c_size_t),
        ("out_size", ctypes.c_int * 2),
        ("n_frames", ctypes.c_int),
    ]


class _Movie(ctypes.Structure):
    _fields_ = [
        ("frames", ctypes.c_void_p),
        ("mode", ctypes.c_int),
        ("nx", ctypes.c_int),
        ("ny", ctypes.c_int),
        ("nz", ctypes.c_int),
        ("on_device", ctypes.c_int),
    ]


class _Result(ctypes.Structure):
    _fields_ = [
        ("sums", ctypes.c_void_p),
        ("sums_on_device", ctypes.c_int),
        ("global_shifts", ctypes.c_void_p),
        ("patch_shifts", ctypes.c_void_p),
        ("patch_centers", ctypes.c_void_p),
        ("patch_bad", ctypes.c_void_p),
        ("iterations", ctypes.c_void_p),
        ("errors", ctypes.c_void_p),
        ("n_sums", ctypes.c_int),
        ("n_patches", ctypes.c_int),
        ("time_ms", ctypes.c_double),
        ("stack", ctypes.c_void_p),
        ("stack_on_device", ctypes.c_int),
        ("stack_frames", ctypes.c_int),
        ("hot_map", ctypes.c_void_p),
        ("ctf", ctypes.c_float * 6),
        ("ctf_done", ctypes.c_int),
        ("ctf_spectrum", ctypes.c_void_p),
        ("ctf_spectrum_on_device", ctypes.c_int),
        ("first_iterate", ctypes.c_int),
    ]


class _FrameIntegration(ctypes.Structure):
    _fields_ = [
        ("n_raw", ctypes.c_int),
        ("n_int", ctypes.c_int),
        ("start", ctypes.c_void_p),
        ("size", ctypes.c_void_p),
        ("acc_dose", ctypes.c_void_p),
        ("dose_weight", ctypes.c_int),
        ("rendered", ctypes.c_int),
    ]


class _Alignment(ctypes.Structure):
    _fields_ = [
        ("nz", ctypes.c_int),
        ("global_shifts", ctypes.c_void_p),
        ("n_patches", ctypes.c_int),
        ("patch_shifts", ctypes.c_void_p),
        ("patch_centers", ctypes.c_void_p),
    ]


_LIB: Optional[ctypes.CDLL] = None
_VP = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float

_SIGS = {
    "mc3_version": ([], ctypes.c_char_p),
    "mc3_strerror": ([_I], ctypes.c_char_p),
    "mc3_params_default": ([ctypes.POINTER(_Params)], None),
    "mc3_create": ([ctypes.POINTER(_Params), ctypes.POINTER(_VP)], _I),
    "mc3_destroy": ([_VP], _I),
    "mc3_set_stream": ([_VP, _VP], _I),
    "mc3_plan": ([_VP, _I, _I, _I, ctypes.POINTER(_PlanInfo)], _I),
    "mc3_host_alloc": ([ctypes.c_size_t, ctypes.POINTER(_VP)], _I),
    "mc3_host_free": ([_VP], _I),
    "mc3_set_gain": ([_VP, _VP, _I, _I, _I], _I),
    "mc3_set_dark": ([_VP, _VP, _I, _I, _I], _I),
    "mc3_set_defects": ([_VP, _VP, _I, _I], _I),
    "mc3_ref_orient": ([_VP, _I, _I, _I, _I, _I, _VP, _VP, _VP], _I),
    "mc3_ref_augment": ([_VP, _I, _I, _I, _VP], _I),
    "mc3_tiff_info": ([ctypes.c_char_p, _VP, _VP, _VP, _VP], _I),
    "mc3_tiff_read": ([ctypes.c_char_p, _I, _I, _VP, _I], _I),
    "mc3_eer_info": ([ctypes.c_char_p, _VP, _VP, _VP, _VP], _I),
    "mc3_eer_render": ([ctypes.c_char_p, _I, _I, _VP, _VP, _VP, _I], _I),
    "mc3_process_movie": ([_VP, ctypes.POINTER(_Movie), ctypes.POINTER(_Result)], _I),
    "mc3_estimate_ctf": ([_VP, _VP, _I, _I, _I, _F, _F, _F, _F, _F, _VP, _VP], _I),
    "mc3_prefetch_movie": ([_VP, ctypes.POINTER(_Movie)], _I),
    "mc3_set_alignment": ([_VP, ctypes.POINTER(_Alignment)], _I),
    "mc3_set_frame_integration": ([_VP, ctypes.POINTER(_FrameIntegration)], _I),
    "mc3_read_fmint_file": ([ctypes.c_char_p, _F, _I, _VP, _VP, _VP, _VP], _I),
    "mc3_frame_groups": ([_VP, _VP, _I, _I, _I, _VP, _VP, _VP, _VP], _I),
    "mc3_frame_integration_tables": ([_VP, _VP, _VP, _I, _I, _F, _I, _I, _I, _VP, _VP, _VP, _VP,
                                      _VP], _I),
    "mc3_fft_forward": ([_VP, _I, _I, _I, _I, _VP], _I),
    "mc3_fft_inverse": ([_VP, _I, _I, _I, _VP], _I),
    "mc3_rfft_rows": ([_VP, _I, _VP, _I, _I, _I, _I, _VP], _I),
    "mc3_submit": ([_VP, _VP, _VP, _VP], _I),
    "mc3_set_first_iterate": ([_VP, _VP, _I, _I], _I),
    "mc3_set_patch_centers": ([_VP, _VP, _I], _I),
    "mc3_proposal_create": ([_VP, _I, _I, ctypes.c_uint, _I, _VP], _I),
    "mc3_proposal_destroy": ([_VP], _I),
    "mc3_proposal_num_params": ([_VP, _VP], _I),
    "mc3_proposal_get_params": ([_VP, _VP], _I),
    "mc3_proposal_set_params": ([_VP, _VP], _I),
    "mc3_proposal_loss_grad": ([_VP, _VP, _I, _I, _I, _VP, _VP, _VP, _VP], _I),
    "mc3_proposal_train_step": ([_VP, _VP, _VP, _I, _I, _I, _I, ctypes.c_float, _VP], _I),
    "mc3_proposal_predict": ([_VP, _VP, _I, _I, _I, _I, _VP], _I),
    "mc3_proposal_pair_inputs": ([_VP, _I, _I, _I, _VP, _I, _I, _VP, _VP], _I),
    "mc3_autotune": ([_VP, _I, _I, _I, ctypes.c_char_p, _VP], _I),
    "mc3_load_tuning": ([_VP, ctypes.c_char_p], _I),
    "mc3_wait": ([_VP, _I, _VP], _I),
    "mc3_phase_shift": ([_VP, _VP, _I, _I, _F, _F, _I, _VP], _I),
    "mc3_fourier_crop": ([_VP, _I, _I, _VP, _I, _I, _VP], _I),
    "mc3_correlate": ([_VP, _VP, _I, _I, _F, _I, _I, _I, _VP, _VP, _VP], _I),
    "mc3_iterative_align": ([_VP, _VP, _I, _I, _I, _I, _I, _F, _F, _I, _VP, _VP], _I),
    "mc3_detect_bad_pixels": ([_VP, _I, _I, _VP, _VP], _I),
    "mc3_correct_bad_pixels": ([_VP, _I, _I, _I, _VP, _VP], _I),
    "mc3_local_gather": ([_VP, _VP, _I, _I, _VP, _VP, _VP, _I, _VP], _I),
    "mc3_dose_weighted_sums": ([_VP, _VP, _I, _I, _I, _VP, _VP, _VP], _I),
    "mc3_profile_enable": ([_I], None),
    "mc3_profile_read": ([ctypes.c_char_p, ctypes.c_size_t, _I], _I),
    "mc3_kernel_launches": ([], ctypes.c_ulonglong),
    "mc3_peak2d": ([_VP, _I, _I, _VP], None),
    "mc3_remove_spikes": ([_VP, _VP, _I], None),
    "mc3_lin_eqs": ([_VP, _VP, _I], _I),
    "mc3_smooth_shifts": ([_VP, _VP, _I, _F], None),
    "mc3_patch_make_relative": ([_VP, _I, _I], None),
    "mc3_patch_detect_bads": ([_VP, _VP, _I, _I, _I, _I, _VP], None),
    "mc3_patch_starts_from_centers": ([_VP, _I, ctypes.c_float, ctypes.c_float, _I, _I, _I, _I,
                                       _VP], _I),
}


def _lib() -> ctypes.CDLL:
    """Loads libmc3.so (built in place by motioncor3_b200.build); raises if absent."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(lib_path):
            raise RuntimeError(
                f"libmc3.so not found at {lib_path}; build it with "
                "`python -m motioncor3_b200.build` (there is no fallback path)")
        L = ctypes.CDLL(lib_path)
        for name, (args, res) in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _LIB = L
    return _LIB


lib = _lib


def _check(code: int, what: str) -> None:
    if code != MC3_OK:
        raise MC3Error(code, what)


def _hp(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(_VP)


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dp(t) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def _need(t, what: str, shape=None, dtype=None) -> None:
    """Checks a device tensor handed to the library as a raw pointer (the C
    entry points cannot see its size): a contiguous CUDA tensor, of the given
    dtype, whose shape equals `shape` (None entries are free)."""
    if not (hasattr(t, "data_ptr") and getattr(t, "is_cuda", False)):
        raise ValueError(f"{what}: a CUDA tensor is required")
    if not t.is_contiguous():
        raise ValueError(f"{what}: a contiguous tensor is required")
    if dtype is not None and str(t.dtype) != f"torch.{dtype}":
        raise ValueError(f"{what}: dtype {t.dtype}, {dtype} required")
    if shape is not None:
        if len(t.shape) != len(shape) or any(w is not None and int(g) != int(w)
                                             for g, w in zip(t.shape, shape)):
            raise ValueError(f"{what}: shape {tuple(t.shape)}, {tuple(shape)} required")


@dataclasses.dataclass
class Params:
    """In-scope MotionCor3 options; defaults of CInput::CInput (CInput.cpp:82-127)."""
    patch: tuple = (0, 0)
    iter: int = 15
    tol: float = 0.1
    bft: tuple = (500.0, 100.0)
    phase_only: int = 0
    ft_bin: float = 1.0
    init_dose: float = 0.0
    fm_dose: float = 0.0
    pix_size: float = 0.0
    kv: int = 300
    group: tuple = (1, 4)
    fm_ref: int = -1
    sum_range: tuple = (3.0, 25.0)
    align: int = 1
    correct_bad: int = 1
    gpu: int = 0
    split_sum: int = 0
    out_stack: tuple = (0, 1)
    mag: tuple = (1.0, 1.0, 0.0)
    in_fm_motion: int = 0
    corr_interp: int = 0
    cs: float = 0.0          # > 0.001 (with pix_size, kv) turns the CTF estimate on
    amp_cont: float = 0.07
    ext_phase: float = 0.0
    dft_gemm: int = 0        # 1: patch row transforms as split-BF16 DFT GEMMs (tensor cores)

    def to_c(self) -> _Params:
        p = _Params()
        _lib().mc3_params_default(ctypes.byref(p))
        px = list(self.patch) + [0] * (3 - len(self.patch))
        for i in range(3):
            p.patch[i] = int(px[i])
        p.iter = int(self.iter)
        p.tol = float(self.tol)
        p.bft[0], p.bft[1] = float(self.bft[0]), float(self.bft[1])
        p.phase_only = int(self.phase_only)
        p.ft_bin = float(self.ft_bin)
        p.init_dose = float(self.init_dose)
        p.fm_dose = float(self.fm_dose)
        p.pix_size = float(self.pix_size)
        p.kv = int(self.kv)
        p.group[0], p.group[1] = int(self.group[0]), int(self.group[1])
        p.fm_ref = int(self.fm_ref)
        p.sum_range[0], p.sum_range[1] = float(self.sum_range[0]), float(self.sum_range[1])
        p.align = int(self.align)
        p.correct_bad = int(self.correct_bad)
        p.gpu = int(self.gpu)
        p.split_sum = int(self.split_sum)
        p.out_stack[0], p.out_stack[1] = int(self.out_stack[0]), int(self.out_stack[1])
        for i in range(3):
            p.mag[i] = float(self.mag[i])
        p.in_fm_motion = int(self.in_fm_motion)
        p.corr_interp = int(self.corr_interp)
        p.cs = float(self.cs)
        p.amp_cont = float(self.amp_cont)
        p.ext_phase = float(self.ext_phase)
        p.dft_gemm = int(self.dft_gemm)
        return p


@dataclasses.dataclass
class Result:
    sums: object                 # [n_sums][ny][nx] numpy (host) or torch tensor (device)
    global_shifts: np.ndarray    # [nz][2]
    patch_shifts: Optional[np.ndarray]
    patch_centers: Optional[np.ndarray]
    patch_bad: Optional[np.ndarray]
    iterations: np.ndarray       # [1 + n_patches]
    errors: np.ndarray           # [1 + n_patches][iter]
    n_sums: int
    n_patches: int
    time_ms: float
    first_iterate: int = 0       # 0 cold start, 1 warm start kept, 2 fell back to cold
    stack: Optional[np.ndarray] = None  # [stack_frames][ny][nx] aligned frames (-OutStack)
    ctf: Optional[np.ndarray] = None    # dfmax, dfmin (A), azimuth, phase (deg), score, res (A)
    ctf_spectrum: Optional[np.ndarray] = None  # [512][512] diagnostic spectrum


_MODES = {np.dtype(np.uint8): 0, np.dtype(np.int16): 1, np.dtype(np.float32): 2, np.dtype(np.uint16): 6}


class MotionCor3:
    """One processing context on one GPU (mc3_create / mc3_process_movie)."""

    def __init__(self, params: Optional[Params] = None):
        self.params = params or Params()
        self._p = self.params.to_c()
        h = _VP()
        _check(_lib().mc3_create(ctypes.byref(self._p), ctypes.byref(h)), "mc3_create")
        self._h = h
        self._prefetched = []  # host arrays whose copies are in flight
        self._queued = {}      # ticket -> buffers of a submitted movie

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib().mc3_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_stream(self, stream) -> None:
        _check(_lib().mc3_set_stream(self._h, stream), "mc3_set_stream")

    def plan(self, nx: int, ny: int, nz: int) -> dict:
        info = _PlanInfo()
        _check(_lib().mc3_plan(self._h, nx, ny, nz, ctypes.byref(info)), "mc3_plan")
        return dict(n_sums=info.n_sums, n_patches=info.n_patches, xcf_size=tuple(info.xcf_size),
                    patch_size=tuple(info.patch_size), xcf_bin=tuple(info.xcf_bin),
                    device_bytes=info.device_bytes, out_size=tuple(info.out_size),
                    n_frames=info.n_frames)

    def set_gain(self, gain) -> None:
        if gain is None:
            _check(_lib().mc3_set_gain(self._h, None, 0, 0, 0), "mc3_set_gain")
            return
        if hasattr(gain, "data_ptr"):
            _check(_lib().mc3_set_gain(self._h, _dp(gain), gain.shape[1], gain.shape[0], 1),
                   "mc3_set_gain")
        else:
            g = np.ascontiguousarray(gain, dtype=np.float32)
            _check(_lib().mc3_set_gain(self._h, _hp(g), g.shape[1], g.shape[0], 0), "mc3_set_gain")

    def set_dark(self, dark) -> None:
        """Dark reference [ny][nx] (mc3_set_dark); None clears it."""
        if dark is None:
            _check(_lib().mc3_set_dark(self._h, None, 0, 0, 0), "mc3_set_dark")
            return
        d = np.ascontiguousarray(dark, dtype=np.float32)
        _check(_lib().mc3_set_dark(self._h, _hp(d), d.shape[1], d.shape[0], 0), "mc3_set_dark")

    def set_defects(self, mask) -> None:
        """Known camera defects [ny][nx] (nonzero = bad; mc3_set_defects); None clears."""
        if mask is None:
            _check(_lib().mc3_set_defects(self._h, None, 0, 0), "mc3_set_defects")
            return
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        _check(_lib().mc3_set_defects(self._h, _hp(m), m.shape[1], m.shape[0]), "mc3_set_defects")

    @staticmethod
    def _movie(frames, nx4=None):
        if nx4 is not None:  # packed 4-bit frames [nz][ny][(nx4+1)//2] (MRC mode 101)
            on_dev = hasattr(frames, "data_ptr")
            keep = frames if on_dev else np.ascontiguousarray(frames, np.uint8)
            nz, ny, pk = keep.shape
            if pk != (nx4 + 1) // 2:
                raise MC3Error(MC3_EINVAL, "packed row length")
            fptr = _dp(keep) if on_dev else keep.ctypes.data_as(_VP)
            return _Movie(fptr, 101, nx4, ny, nz, 1 if on_dev else 0), keep
        on_dev = hasattr(frames, "data_ptr")
        if on_dev:
            import torch
            dt = {torch.uint8: 0, torch.int16: 1, torch.float32: 2}.get(frames.dtype)
            if dt is None:
                raise MC3Error(MC3_EUNSUPPORTED, "frame dtype")
            nz, ny, nx = frames.shape
            fptr = _dp(frames)
            keep = frames
        else:
            keep = np.ascontiguousarray(frames)
            dt = _MODES.get(keep.dtype)
            if dt is None:
                raise MC3Error(MC3_EUNSUPPORTED, "frame dtype")
            nz, ny, nx = keep.shape
            fptr = keep.ctypes.data_as(_VP)
        return _Movie(fptr, dt, nx, ny, nz, 1 if on_dev else 0), keep

    def prefetch(self, frames, nx4=None) -> None:
        """Starts copying a later movie's host frames to the device
        (mc3_prefetch_movie); pass the same array to a later process()."""
        mv, keep = self._movie(frames, nx4)
        _check(_lib().mc3_prefetch_movie(self._h, ctypes.byref(mv)), "mc3_prefetch_movie")
        if not mv.on_device:
            self._prefetched.append(keep)

    def set_alignment(self, global_shifts=None, patch_shifts=None, patch_centers=None) -> None:
        """Known alignment for the following movies (mc3_set_alignment, the
        -InAln path); global_shifts None clears it.  global_shifts [nz][2],
        patch_shifts [nz][P][2], patch_centers [P][2]."""
        if global_shifts is None:
            _check(_lib().mc3_set_alignment(self._h, None), "mc3_set_alignment")
            return
        g = np.ascontiguousarray(global_shifts, np.float32)
        a = _Alignment()
        a.nz = g.shape[0]
        a.global_shifts = g.ctypes.data
        keep = [g]
        if patch_shifts is not None:
            ps = np.ascontiguousarray(patch_shifts, np.float32)
            pc = np.ascontiguousarray(patch_centers, np.float32)
            a.n_patches = ps.shape[1]
            a.patch_shifts = ps.ctypes.data
            a.patch_centers = pc.ctypes.data
            keep += [ps, pc]
        _check(_lib().mc3_set_alignment(self._h, ctypes.byref(a)), "mc3_set_alignment")
        del keep  # the library copies the tables

    def set_frame_integration(self, tables: Optional[dict], n_raw: int = 0,
                              rendered: bool = False) -> None:
        """Rendered frames for the following movies of n_raw raw frames
        (mc3_set_frame_integration); tables as frame_integration_tables()
        returns them; None clears."""
        if tables is None:
            _check(_lib().mc3_set_frame_integration(self._h, None), "mc3_set_frame_integration")
            return
        st = np.ascontiguousarray(tables["start"], np.int32)
        sz = np.ascontiguousarray(tables["size"], np.int32)
        acc = np.ascontiguousarray(tables["acc_dose"], np.float32)
        fi = _FrameIntegration(n_raw, len(st), st.ctypes.data, sz.ctypes.data, acc.ctypes.data,
                               int(tables.get("dose_weight", 0)), int(rendered))
        _check(_lib().mc3_set_frame_integration(self._h, ctypes.byref(fi)),
               "mc3_set_frame_integration")

    def _prepare(self, frames, sums_out, nx4):
        """The mc3_movie, an mc3_result pointing at freshly allocated host
        tables, and everything that must stay alive until the call is done."""
        mv, keep = self._movie(frames, nx4)
        nx, ny, nz = mv.nx, mv.ny, mv.nz
        info = self.plan(nx, ny, nz)
        ns, P = info["n_sums"], info["n_patches"]
        nz = info["n_frames"]  # rendered frames: the tables below are per rendered frame
        it = int(self.params.iter)
        h = dict(keep=keep, mv=mv, P=P,
                 gsh=np.zeros((nz, 2), np.float32),
                 psh=np.zeros((nz, max(P, 1), 2), np.float32),
                 pc=np.zeros((max(P, 1), 2), np.float32),
                 pb=np.zeros((nz, max(P, 1)), np.uint8),
                 iters=np.zeros(1 + P, np.int32),
                 errs=np.zeros((1 + P, it), np.float32), stack=None, ctf_img=None)
        r = _Result()
        if sums_out is not None and hasattr(sums_out, "data_ptr"):
            r.sums = sums_out.data_ptr()
            r.sums_on_device = 1
            sums = sums_out
        elif sums_out is not None:
            sums = sums_out
            r.sums = sums.ctypes.data
            r.sums_on_device = 0
        else:
            ox, oy = info["out_size"]
            sums = np.zeros((ns, oy, ox), np.float32)
            r.sums = sums.ctypes.data
            r.sums_on_device = 0
        h["sums"] = sums
        r.global_shifts = h["gsh"].ctypes.data
        r.patch_shifts = h["psh"].ctypes.data if P else None
        r.patch_centers = h["pc"].ctypes.data if P else None
        r.patch_bad = h["pb"].ctypes.data if P else None
        r.iterations = h["iters"].ctypes.data
        r.errors = h["errs"].ctypes.data
        if int(self.params.out_stack[0]):
            ox, oy = info["out_size"]
            h["stack"] = np.zeros((nz, oy, ox), np.float32)
            r.stack = h["stack"].ctypes.data
        if float(self.params.cs) > 0.001 and self.params.kv and self.params.pix_size:
            h["ctf_img"] = np.zeros((512, 512), np.float32)  # CFindCtfMain::bEstimate
            r.ctf_spectrum = h["ctf_img"].ctypes.data
        h["r"] = r
        return h

    @staticmethod
    def _finish(h) -> Result:
        r, P, stack = h["r"], h["P"], h["stack"]
        if stack is not None:
            stack = stack[:r.stack_frames]
        return Result(sums=h["sums"], global_shifts=h["gsh"], patch_shifts=h["psh"] if P else None,
                      patch_centers=h["pc"] if P else None, patch_bad=h["pb"] if P else None,
                      iterations=h["iters"], errors=h["errs"], n_sums=r.n_sums,
                      n_patches=r.n_patches, time_ms=r.time_ms, stack=stack,
                      first_iterate=r.first_iterate,
                      ctf=np.array(r.ctf[:], np.float32) if r.ctf_done else None,
                      ctf_spectrum=h["ctf_img"] if r.ctf_done else None)

    def process(self, frames, sums_out=None, nx4=None) -> Result:
        """frames: [nz][ny][nx] numpy array (host) or torch CUDA tensor; with
        nx4, packed 4-bit frames [nz][ny][(nx4+1)//2] of width nx4."""
        h = self._prepare(frames, sums_out, nx4)
        _check(_lib().mc3_process_movie(self._h, ctypes.byref(h["mv"]), ctypes.byref(h["r"])),
               "mc3_process_movie")
        if not h["mv"].on_device and self._prefetched:
            self._prefetched.pop(0)
        return self._finish(h)

    def submit(self, frames, sums_out=None, nx4=None) -> int:
        """Queues a movie on the context's worker thread (mc3_submit) and
        returns its ticket; the frames must not change until wait(ticket)."""
        h = self._prepare(frames, sums_out, nx4)
        t = ctypes.c_int()
        _check(_lib().mc3_submit(self._h, ctypes.byref(h["mv"]), ctypes.byref(h["r"]),
                                 ctypes.byref(t)), "mc3_submit")
        self._queued[t.value] = h
        return t.value

    def autotune(self, nx: int, ny: int, nz: int, json_path: Optional[str] = None) -> float:
        """Picks the fastest kernel variants for movies of this size
        (mc3_autotune); returns the winner's device time per movie in ms."""
        ms = ctypes.c_double()
        _check(_lib().mc3_autotune(self._h, nx, ny, nz,
                                   json_path.encode() if json_path else None, ctypes.byref(ms)),
               "mc3_autotune")
        return ms.value

    def set_first_iterate(self, global_shifts=None, max_iter: int = 3) -> None:
        """Warm start of the next movie's full-frame alignment
        (mc3_set_first_iterate): global_shifts [nz][2] in full-frame pixels;
        None clears it."""
        if global_shifts is None:
            _check(_lib().mc3_set_first_iterate(self._h, None, 0, 0), "mc3_set_first_iterate")
            return
        g = np.ascontiguousarray(global_shifts, np.float32)
        _check(_lib().mc3_set_first_iterate(self._h, g.ctypes.data, g.shape[0], max_iter),
               "mc3_set_first_iterate")

    def set_patch_centers(self, centers=None) -> None:
        """Patch centres [P][2] (full-frame pixels) for the following movies
        instead of the feature-based placement (mc3_set_patch_centers); None
        clears them."""
        if centers is None:
            _check(_lib().mc3_set_patch_centers(self._h, None, 0), "mc3_set_patch_centers")
            return
        c = np.ascontiguousarray(centers, np.float32).reshape(-1, 2)
        _check(_lib().mc3_set_patch_centers(self._h, c.ctypes.data, c.shape[0]),
               "mc3_set_patch_centers")

    def load_tuning(self, json_path: str) -> None:
        _check(_lib().mc3_load_tuning(self._h, json_path.encode()), "mc3_load_tuning")

    def wait(self, ticket: int):
        """(Result, latency in ms from submit to done) of a queued movie (mc3_wait)."""
        lat = ctypes.c_double()
        code = _lib().mc3_wait(self._h, ticket, ctypes.byref(lat))
        h = self._queued.pop(ticket)
        _check(code, "mc3_wait")
        return self._finish(h), lat.value

    def estimate_ctf(self, image, pix_size: float, kv: float = 300.0, cs: float = 2.7,
                     amp_cont: float = 0.07, ext_phase: float = 0.0):
        """CTF of one image [ny][nx] (numpy float32, or a CUDA tensor):
        (res6, spectrum512) with res6 = dfmax, dfmin (A), azimuth, phase (deg),
        score, resolution (A) (mc3_estimate_ctf)."""
        res = np.zeros(6, np.float32)
        if hasattr(image, "data_ptr"):
            import torch
            ny, nx = image.shape
            spec = torch.empty((512, 512), dtype=torch.float32, device=image.device)
            _check(_lib().mc3_estimate_ctf(self._h, _dp(image), nx, ny, 1, pix_size, kv, cs, amp_cont,
                                           ext_phase, _hp(res), _dp(spec)), "mc3_estimate_ctf")
            torch.cuda.synchronize()
            return res, spec.cpu().numpy()
        img = np.ascontiguousarray(image, np.float32)
        ny, nx = img.shape
        spec = np.zeros((512, 512), np.float32)
        _check(_lib().mc3_estimate_ctf(self._h, _hp(img), nx, ny, 0, pix_size, kv, cs, amp_cont,
                                       ext_phase, _hp(res), _hp(spec)), "mc3_estimate_ctf")
        return res, spec

    # ---- component entry points needing the context ----
    def iterative_align(self, stack, group: int, max_iter: int, tol: float, bfactor: float,
                        phase_only: int = 0):
        """stack: torch complex64 CUDA tensor [n][cmp_y][cmp_x]."""
        n, cy, cx = stack.shape
        sh = np.zeros((n, 2), np.float32)
        its = ctypes.c_int(0)
        _check(_lib().mc3_iterative_align(self._h, _dp(stack), cx, cy, n, group, max_iter, tol,
                                          bfactor, phase_only, _hp(sh), ctypes.byref(its)),
               "mc3_iterative_align")
        return sh, its.value

    def dose_weighted_sums(self, spectra, nx: int, ny: int, shifts: np.ndarray, sums):
        nz = spectra.shape[0]
        s = np.ascontiguousarray(shifts, np.float32)
        ns = ctypes.c_int(0)
        _check(_lib().mc3_dose_weighted_sums(self._h, _dp(spectra), nx, ny, nz, _hp(s), _dp(sums),
                                             ctypes.byref(ns)), "mc3_dose_weighted_sums")
        return ns.value


# ---- stateless components (device tensors) ----
class ShiftProposal:
    """The learned shift proposal on the GPU (mc3_proposal_*): strided
    convolutions + ReLU, global average pool and a linear head, trained by
    the library's own kernels.  spec: [(cin, cout, k, stride, pad), ...]."""

    def __init__(self, spec, nout: int = 2, seed: int = 0, gpu: int = 0):
        flat = (ctypes.c_int * (5 * len(spec)))(*[int(v) for layer in spec for v in layer])
        h = _VP()
        _check(_lib().mc3_proposal_create(flat, len(spec), nout, seed, gpu, ctypes.byref(h)),
               "mc3_proposal_create")
        self._h, self.nout = h, nout
        n = ctypes.c_long()
        _check(_lib().mc3_proposal_num_params(self._h, ctypes.byref(n)), "mc3_proposal_num_params")
        self.n_params = n.value

    def close(self):
        if getattr(self, "_h", None):
            _lib().mc3_proposal_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        p = np.zeros(self.n_params, np.float32)
        _check(_lib().mc3_proposal_get_params(self._h, p.ctypes.data), "mc3_proposal_get_params")
        return p

    def set_params(self, p) -> None:
        a = np.ascontiguousarray(p, np.float32)
        _check(_lib().mc3_proposal_set_params(self._h, a.ctypes.data), "mc3_proposal_set_params")

    def loss_grad(self, x, target):
        """(summed loss, summed gradient, outputs) of a host batch x [n][2][h][w]."""
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(target, np.float32)
        n, _, h, w = x.shape
        g = np.zeros(self.n_params, np.float32)
        out = np.zeros((n, self.nout), np.float32)
        loss = ctypes.c_double()
        _check(_lib().mc3_proposal_loss_grad(self._h, x.ctypes.data, n, h, w, t.ctypes.data,
                                             ctypes.byref(loss), g.ctypes.data, out.ctypes.data),
               "mc3_proposal_loss_grad")
        return loss.value, g, out

    def train_step(self, x, target, lr: float = 1e-3) -> float:
        """One Adam step on a batch (torch CUDA tensors or host arrays); mean loss."""
        loss = ctypes.c_double()
        if hasattr(x, "data_ptr"):
            _need(x, "train_step x", (None, 2, None, None), "float32")
            n, _, h, w = x.shape
            _need(target, "train_step target", (n, self.nout), "float32")
            _check(_lib().mc3_proposal_train_step(self._h, _dp(x), _dp(target), n, h, w, 1, lr,
                                                  ctypes.byref(loss)), "mc3_proposal_train_step")
        else:
            xa = np.ascontiguousarray(x, np.float32)
            ta = np.ascontiguousarray(target, np.float32)
            n, _, h, w = xa.shape
            _check(_lib().mc3_proposal_train_step(self._h, xa.ctypes.data, ta.ctypes.data, n, h, w,
                                                  0, lr, ctypes.byref(loss)),
                   "mc3_proposal_train_step")
        return loss.value

    def predict(self, x) -> np.ndarray:
        n, _, h, w = x.shape
        out = np.zeros((n, self.nout), np.float32)
        if hasattr(x, "data_ptr"):
            _need(x, "predict x", (None, 2, None, None), "float32")
            _check(_lib().mc3_proposal_predict(self._h, _dp(x), n, h, w, 1, out.ctypes.data),
                   "mc3_proposal_predict")
        else:
            xa = np.ascontiguousarray(x, np.float32)
            _check(_lib().mc3_proposal_predict(self._h, xa.ctypes.data, n, h, w, 0, out.ctypes.data),
                   "mc3_proposal_predict")
        return out

    @staticmethod
    def pair_inputs(frames, pairs, bin: int, out):
        """Inputs of frame pairs from a device movie (torch float32 [nz][ny][nx])
        into out (torch float32 [n][2][ny/bin][nx/bin])."""
        _need(frames, "pair_inputs frames", (None, None, None), "float32")
        nz, ny, nx = frames.shape
        pr = np.ascontiguousarray(pairs, np.int32).reshape(-1, 2)
        _need(out, "pair_inputs out", (pr.shape[0], 2, ny // bin, nx // bin), "float32")
        _check(_lib().mc3_proposal_pair_inputs(_dp(frames), nx, ny, nz, pr.ctypes.data, pr.shape[0],
                                               bin, _dp(out), _stream()), "mc3_proposal_pair_inputs")


def fft_forward(frames, nx: int, ny: int, normalise: bool = True) -> None:
    """In place on a float32 CUDA tensor [nz][ny][2*(nx//2+1)]."""
    _need(frames, "fft_forward frames", (None, ny, 2 * (nx // 2 + 1)), "float32")
    nz = frames.shape[0]
    _check(_lib().mc3_fft_forward(_dp(frames), nx, ny, nz, int(normalise), _stream()), "mc3_fft_forward")


def rfft_rows(src, dst, nx: int, method: int = 0) -> None:
    """Real DFT of every row of src [rows][>= nx] (float32, device) into dst
    [rows][>= nx/2+1] (complex64, device): method 0 the FP32 FFT, 1 the
    split-precision BF16 DFT GEMM on the tensor cores."""
    rows = src.shape[0]
    ok = (getattr(src, "is_cuda", False) and getattr(dst, "is_cuda", False) and
          str(src.dtype) == "torch.float32" and str(dst.dtype) == "torch.complex64" and
          src.dim() == 2 and dst.dim() == 2 and src.stride(1) == 1 and dst.stride(1) == 1 and
          src.shape[1] >= nx and dst.shape[0] >= rows and dst.shape[1] >= nx // 2 + 1)
    if not ok:
        raise ValueError("rfft_rows: src float32 CUDA [rows][>= nx] and dst complex64 CUDA "
                         "[>= rows][>= nx/2+1], both with unit inner stride")
    _check(_lib().mc3_rfft_rows(_dp(src), src.stride(0), _dp(dst), dst.stride(0), nx, rows, method,
                                _stream()), "mc3_rfft_rows")


def fft_inverse(frames, nx: int, ny: int) -> None:
    _need(frames, "fft_inverse frames", (None, ny, 2 * (nx // 2 + 1)), "float32")
    nz = frames.shape[0]
    _check(_lib().mc3_fft_inverse(_dp(frames), nx, ny, nz, _stream()), "mc3_fft_inverse")


def phase_shift(src, dst, sx: float, sy: float, accumulate: bool = False) -> None:
    cy, cx = src.shape[-2], src.shape[-1]
    _check(_lib().mc3_phase_shift(_dp(src), _dp(dst), cx, cy, sx, sy, int(accumulate), _stream()),
           "mc3_phase_shift")


def fourier_crop(src, dst) -> None:
    _check(_lib().mc3_fourier_crop(_dp(src), src.shape[-1], src.shape[-2], _dp(dst), dst.shape[-1],
                                   dst.shape[-2], _stream()), "mc3_fourier_crop")


def correlate(group, sum_, bfactor: float, phase_only: int = 0, sea=(64, 64), window=None):
    cy, cx = group.shape[-2], group.shape[-1]
    sh = np.zeros(2, np.float32)
    _check(_lib().mc3_correlate(_dp(group), _dp(sum_), cx, cy, bfactor, phase_only, sea[0], sea[1],
                                _dp(window) if window is not None else None, _hp(sh), _stream()),
           "mc3_correlate")
    return sh


def detect_bad_pixels(sum_padded, nx: int, ny: int, bad) -> None:
    _check(_lib().mc3_detect_bad_pixels(_dp(sum_padded), nx, ny, _dp(bad), _stream()),
           "mc3_detect_bad_pixels")


def correct_bad_pixels(frames, nx: int, ny: int, bad) -> None:
    _check(_lib().mc3_correct_bad_pixels(_dp(frames), nx, ny, frames.shape[0], _dp(bad), _stream()),
           "mc3_correct_bad_pixels")


def local_gather(src, dst, nx: int, ny: int, centers, shifts, bad=None) -> None:
    P = centers.shape[0]
    _check(_lib().mc3_local_gather(_dp(src), _dp(dst), nx, ny, _dp(centers), _dp(shifts),
                                   _dp(bad) if bad is not None else None, P, _stream()),
           "mc3_local_gather")


# ---- reference images (host) ----
def ref_orient(img: np.ndarray, rot: int = 0, flip: int = 0, inverse: int = 0) -> np.ndarray:
    """CLoadRefs::PostProcess: rotate by rot x 90 degrees, flip (1 upside
    down, 2 left-right), invert (mc3_ref_orient)."""
    a = np.ascontiguousarray(img, np.float32)
    out = np.zeros(a.size, np.float32)
    nx, ny = ctypes.c_int(0), ctypes.c_int(0)
    _check(_lib().mc3_ref_orient(_hp(a), a.shape[1], a.shape[0], rot, flip, inverse, _hp(out),
                                 ctypes.byref(nx), ctypes.byref(ny)), "mc3_ref_orient")
    return out.reshape(ny.value, nx.value)


def ref_augment(img: np.ndarray, fact: int) -> np.ndarray:
    """CLoadRefs::AugmentRefs: every pixel repeated fact x fact (mc3_ref_augment)."""
    a = np.ascontiguousarray(img, np.float32)
    out = np.zeros((a.shape[0] * fact, a.shape[1] * fact), np.float32)
    _check(_lib().mc3_ref_augment(_hp(a), a.shape[1], a.shape[0], fact, _hp(out)),
           "mc3_ref_augment")
    return out


# ---- movie files (host) ----
_TIFF_DT = {0: np.uint8, 1: np.int16, 2: np.float32, 6: np.uint16}


def tiff_info(path: str) -> dict:
    """mc3_tiff_info: size, frame count and MRC-equivalent mode of a TIFF movie."""
    v = [ctypes.c_int(0) for _ in range(4)]
    _check(_lib().mc3_tiff_info(path.encode(), *[ctypes.byref(x) for x in v]), "mc3_tiff_info")
    return dict(nx=v[0].value, ny=v[1].value, nz=v[2].value, mode=v[3].value)


def tiff_read(path: str, z0: int = 0, nz: Optional[int] = None, threads: int = 0) -> np.ndarray:
    """mc3_tiff_read: frames [nz][ny][nx] in the file's pixel type, rows
    bottom-up as the reference stores them."""
    info = tiff_info(path)
    nz = info["nz"] - z0 if nz is None else nz
    out = np.zeros((nz, info["ny"], info["nx"]), _TIFF_DT[info["mode"]])
    _check(_lib().mc3_tiff_read(path.encode(), z0, nz, out.ctypes.data, threads), "mc3_tiff_read")
    return out


def eer_info(path: str) -> dict:
    """mc3_eer_info: camera size, EER frame count and run-length bits."""
    v = [ctypes.c_int(0) for _ in range(4)]
    _check(_lib().mc3_eer_info(path.encode(), *[ctypes.byref(x) for x in v]), "mc3_eer_info")
    return dict(cam_x=v[0].value, cam_y=v[1].value, n_frames=v[2].value, bits=v[3].value)


def eer_render(path: str, start, size, sampling: int = 1, threads: int = 0) -> np.ndarray:
    """mc3_eer_render: rendered 8-bit frames, frame i the electrons of EER
    frames start[i] .. start[i]+size[i]-1."""
    info = eer_info(path)
    f = {1: 1, 2: 2, 3: 4}[sampling]
    st = np.ascontiguousarray(start, np.int32)
    sz = np.ascontiguousarray(size, np.int32)
    out = np.zeros((len(st), info["cam_y"] * f, info["cam_x"] * f), np.uint8)
    _check(_lib().mc3_eer_render(path.encode(), sampling, len(st), st.ctypes.data, sz.ctypes.data,
                                 out.ctypes.data, threads), "mc3_eer_render")
    return out


# ---- frame integration (host) ----
def read_fmint_file(path: str, fm_dose: float = 0.0, max_entries: int = 4096):
    """CReadFmIntFile::DoIt: (group_size, int_size, dose) arrays of a
    frame-integration file (empty when it mixes doses)."""
    g = np.zeros(max_entries, np.int32)
    n = np.zeros(max_entries, np.int32)
    d = np.zeros(max_entries, np.float32)
    ne = ctypes.c_int(0)
    _check(_lib().mc3_read_fmint_file(path.encode(), fm_dose, max_entries, _hp(g), _hp(n), _hp(d),
                                      ctypes.byref(ne)), "mc3_read_fmint_file")
    k = min(ne.value, max_entries)
    return g[:k], n[:k], d[:k]


def frame_integration_tables(entries, n_raw: int, fm_dose: float = 0.0, throw=(0, 0)) -> dict:
    """CFmIntParam::Setup: rendered-frame tables for n_raw raw frames from
    (group_size, int_size, dose) entries (None or empty: no file)."""
    if entries is None or len(entries[0]) == 0:
        g = n = d = None
        ne = 0
    else:
        g = np.ascontiguousarray(entries[0], np.int32)
        n = np.ascontiguousarray(entries[1], np.int32)
        d = np.ascontiguousarray(entries[2], np.float32)
        ne = len(g)
    start = np.zeros(n_raw, np.int32)
    size = np.zeros(n_raw, np.int32)
    acc = np.zeros(n_raw, np.float32)
    nint = ctypes.c_int(0)
    dwt = ctypes.c_int(0)
    _check(_lib().mc3_frame_integration_tables(_hp(g), _hp(n), _hp(d), ne, n_raw, fm_dose,
                                               int(throw[0]), int(throw[1]), n_raw,
                                               ctypes.byref(nint), _hp(start), _hp(size), _hp(acc),
                                               ctypes.byref(dwt)), "mc3_frame_integration_tables")
    k = nint.value
    return dict(start=start[:k], size=size[:k], acc_dose=acc[:k], dose_weight=dwt.value)


def frame_groups(start, size, bin_z: int) -> dict:
    """CFmGroupParam::Setup over rendered frames (mc3_frame_groups)."""
    st = np.ascontiguousarray(start, np.int32)
    sz = np.ascontiguousarray(size, np.int32)
    n = len(st)
    gs = np.zeros(n, np.int32)
    gz = np.zeros(n, np.int32)
    gc = np.zeros(n, np.float32)
    ng = ctypes.c_int(0)
    _check(_lib().mc3_frame_groups(_hp(st), _hp(sz), n, bin_z, n, ctypes.byref(ng), _hp(gs),
                                   _hp(gz), _hp(gc)), "mc3_frame_groups")
    k = ng.value
    return dict(start=gs[:k], size=gz[:k], center=gc[:k])


# ---- diagnostics ----
def profile_enable(on: bool) -> None:
    _lib().mc3_profile_enable(int(on))


def profile_read(reset: bool = False) -> dict:
    import json
    buf = ctypes.create_string_buffer(1 << 16)
    _check(_lib().mc3_profile_read(buf, len(buf), int(reset)), "mc3_profile_read")
    return json.loads(buf.value.decode())


def kernel_launches() -> int:
    return int(_lib().mc3_kernel_launches())


# ---- host bookkeeping ----
def peak2d(window: np.ndarray) -> np.ndarray:
    w = np.ascontiguousarray(window, np.float32)
    out = np.zeros(2, np.float32)
    _lib().mc3_peak2d(_hp(w), w.shape[1], w.shape[0], _hp(out))
    return out


def remove_spikes(sx: np.ndarray, sy: np.ndarray):
    x = np.ascontiguousarray(sx, np.float32).copy()
    y = np.ascontiguousarray(sy, np.float32).copy()
    _lib().mc3_remove_spikes(_hp(x), _hp(y), len(x))
    return x, y


def lin_eqs(coeff: np.ndarray, vals: np.ndarray):
    a = np.ascontiguousarray(coeff, np.float32).copy()
    b = np.ascontiguousarray(vals, np.float32).copy()
    ok = _lib().mc3_lin_eqs(_hp(a), _hp(b), len(b))
    return bool(ok), b


def smooth_shifts(sx: np.ndarray, sy: np.ndarray, weight: float):
    x = np.ascontiguousarray(sx, np.float32).copy()
    y = np.ascontiguousarray(sy, np.float32).copy()
    _lib().mc3_smooth_shifts(_hp(x), _hp(y), len(x), weight)
    return x, y


def patch_make_relative(shifts: np.ndarray) -> np.ndarray:
    s = np.ascontiguousarray(shifts, np.float32).copy()
    _lib().mc3_patch_make_relative(_hp(s), s.shape[0], s.shape[1])
    return s


def patch_detect_bads(shifts: np.ndarray, centers: np.ndarray, nx: int, ny: int) -> np.ndarray:
    s = np.ascontiguousarray(shifts, np.float32)
    c = np.ascontiguousarray(centers, np.float32)
    bad = np.zeros(s.shape[:2], np.uint8)
    _lib().mc3_patch_detect_bads(_hp(s), _hp(c), s.shape[0], s.shape[1], nx, ny, _hp(bad))
    return bad


def patch_starts_from_centers(centers, bin_xy, xcf_size, patch_size) -> np.ndarray:
    """Patch starts [P][2] in the alignment image for full-frame centres
    [P][2] (mc3_patch_starts_from_centers): what mc3_set_patch_centers uses."""
    c = np.ascontiguousarray(centers, np.float32).reshape(-1, 2)
    out = np.zeros((c.shape[0], 2), np.int32)
    _check(_lib().mc3_patch_starts_from_centers(_hp(c), c.shape[0], float(bin_xy[0]),
                                                float(bin_xy[1]), int(xcf_size[0]),
                                                int(xcf_size[1]), int(patch_size[0]),
                                                int(patch_size[1]), _hp(out)),
           "mc3_patch_starts_from_centers")
    return out
