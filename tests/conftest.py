"""Shared fixtures.  `gpu` marks tests that need a CUDA device; everything
else runs on the CPU (oracle, reference-host checker, host bookkeeping,
symbol checks)."""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on the B200 box)")


@pytest.fixture(scope="session")
def mc3lib():
    from motioncor3_b200 import build
    build.build()
    from motioncor3_b200 import api
    return api._lib()


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def ref_host():
    from oracle import oracle as O
    L = O.ref_host()
    if L is None:
        pytest.skip("reference host checker not available")
    P = ctypes.c_void_p
    L.ref_interpolate.restype = ctypes.c_int
    L.ref_lin_eqs.restype = ctypes.c_int
    if hasattr(L, "ref_fmint"):
        L.ref_fmint.restype = ctypes.c_int
    return L


@pytest.fixture(scope="session")
def shim():
    out_dir = os.path.join(ROOT, "tests", "_build")
    os.makedirs(out_dir, exist_ok=True)
    so = os.path.join(out_dir, "fft_core_shim.so")
    src = os.path.join(ROOT, "tests", "native", "fft_core_shim.cpp")
    hdr = os.path.join(ROOT, "motioncor3_b200", "csrc", "fft_core.cuh")
    hdr16 = os.path.join(ROOT, "motioncor3_b200", "csrc", "fft_r16.cuh")
    if not os.path.exists(so) or os.path.getmtime(so) < max(os.path.getmtime(src), os.path.getmtime(hdr), os.path.getmtime(hdr16)):
        cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
        subprocess.run([cxx, "-O2", "-shared", "-fPIC", "-I/usr/local/cuda/include", src, "-o", so],
                       check=True)
    return ctypes.CDLL(so)


@pytest.fixture(scope="session")
def ctf_shim():
    """libmc3's CTF core (csrc/ctf_core.h) compiled for the host."""
    out_dir = os.path.join(ROOT, "tests", "_build")
    os.makedirs(out_dir, exist_ok=True)
    so = os.path.join(out_dir, "ctf_core_shim.so")
    src = os.path.join(ROOT, "tests", "native", "ctf_core_shim.cpp")
    hdr = os.path.join(ROOT, "motioncor3_b200", "csrc", "ctf_core.h")
    if not os.path.exists(so) or os.path.getmtime(so) < max(os.path.getmtime(src), os.path.getmtime(hdr)):
        cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
        subprocess.run([cxx, "-O2", "-std=c++17", "-pthread", "-shared", "-fPIC", "-I/usr/local/cuda/include",
                        src, "-o", so], check=True)
    L = ctypes.CDLL(so)
    L.shim_ctf_search.restype = ctypes.c_int
    return L


@pytest.fixture(scope="session")
def proposal_shim():
    """libmc3's proposal-network core (csrc/proposal_core.h) compiled for the host."""
    out_dir = os.path.join(ROOT, "tests", "_build")
    os.makedirs(out_dir, exist_ok=True)
    so = os.path.join(out_dir, "proposal_core_shim.so")
    src = os.path.join(ROOT, "tests", "native", "proposal_core_shim.cpp")
    hdr = os.path.join(ROOT, "motioncor3_b200", "csrc", "proposal_core.h")
    if not os.path.exists(so) or os.path.getmtime(so) < max(os.path.getmtime(src), os.path.getmtime(hdr)):
        cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
        subprocess.run([cxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-I/usr/local/cuda/include",
                        src, "-o", so], check=True)
    L = ctypes.CDLL(so)
    L.shim_proposal_loss_grad.restype = ctypes.c_double
    return L


@pytest.fixture(scope="session")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def fp(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@pytest.fixture
def rng():
    return np.random.default_rng(1234)


def make_ctf_image(n=2048, pix=1.0, df=15000.0, ast=0.02, ang=30.0, kv=300.0, cs=2.7, ac=0.07,
                   phase=0.0, seed=0, ny=None):
    """A seeded micrograph whose power spectrum carries a known CTF: white
    noise filtered by |CTF| (CCtfTheory convention: defocus
    df_mean (1 + ast cos 2(theta - angle)), angle in degrees) under a
    Gaussian envelope, plus an offset."""
    ny = ny or n
    rng = np.random.default_rng(seed)
    ky = np.fft.fftfreq(ny)[:, None]
    kx = np.fft.fftfreq(n)[None, :]
    s2 = (kx ** 2 + ky ** 2) / pix ** 2
    th = np.arctan2(ky, kx + 1e-30)
    lam = 12.26 / np.sqrt(kv * 1000 + 0.9784 * kv * kv)
    dfa = df + df * ast * np.cos(2 * (th - np.deg2rad(ang)))
    chi = (np.pi * lam * s2 * (dfa - 0.5 * lam ** 2 * s2 * cs * 1e7)
           + np.arctan(ac / np.sqrt(1 - ac * ac)) + np.deg2rad(phase))
    F = np.fft.fft2(rng.standard_normal((ny, n))) * (np.abs(np.sin(chi)) * np.exp(-40 * s2) + 0.3)
    return (np.real(np.fft.ifft2(F)) + 10.0).astype(np.float32)


@pytest.fixture(scope="session")
def ctf_image():
    """Factory of micrographs with a planted CTF (make_ctf_image)."""
    return make_ctf_image
