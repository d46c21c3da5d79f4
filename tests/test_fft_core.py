"""The Stockham FFT core shared by every libmc3 transform, run through its
sequential host driver (same index arithmetic as the device kernels),
against numpy at every length the configurations use."""
import ctypes

import numpy as np
import pytest

from conftest import fp

LENGTHS = [1, 2, 3, 4, 5, 6, 8, 12, 16, 17, 34, 41, 51, 64, 102, 128, 131, 204, 205, 256, 408,
           410, 512, 1023, 1024, 1441, 2046, 2048, 2882, 4092, 4096]


@pytest.mark.parametrize("n", LENGTHS)
def test_complex_fft(shim, n):
    rng = np.random.default_rng(n)
    x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    f = np.empty_like(x)
    b = np.empty_like(x)
    assert shim.shim_cfft(fp(x), fp(f), n, -1) == 0
    assert shim.shim_cfft(fp(x), fp(b), n, 1) == 0
    ref = np.fft.fft(x.astype(np.complex128))
    refb = np.fft.ifft(x.astype(np.complex128)) * n
    assert np.abs(f - ref).max() / np.abs(ref).max() < 2e-6
    assert np.abs(b - refb).max() / np.abs(refb).max() < 2e-6


@pytest.mark.parametrize("w", [2, 4, 6, 16, 128, 408, 410, 1024, 2048, 2882, 4092, 4096, 5760])
def test_real_fft_pair(shim, w):
    rng = np.random.default_rng(w)
    x = rng.standard_normal(w).astype(np.float32)
    X = np.empty(w // 2 + 1, np.complex64)
    assert shim.shim_rfft(fp(x), fp(X), w) == 0
    ref = np.fft.rfft(x.astype(np.float64))
    assert np.abs(X - ref).max() / np.abs(ref).max() < 2e-6
    # inverse of a non-Hermitian half spectrum: imaginary parts of DC and
    # Nyquist are ignored, as numpy's irfft (and cuFFT's C2R) do
    Y = (rng.standard_normal(w // 2 + 1) + 1j * rng.standard_normal(w // 2 + 1)).astype(np.complex64)
    y = np.empty(w, np.float32)
    assert shim.shim_irfft(fp(Y), fp(y), w) == 0
    refy = np.fft.irfft(Y.astype(np.complex128), w) * w
    assert np.abs(y - refy).max() / np.abs(refy).max() < 2e-6


def test_factorisation_covers_lengths(shim):
    radix = (ctypes.c_int * 24)()
    for n in LENGTHS:
        k = shim.shim_factorize(n, radix)
        assert k >= 0
        assert int(np.prod([radix[i] for i in range(k)])) == n


@pytest.mark.parametrize("w", [2, 4, 6, 16, 128, 408, 1024, 4096])
def test_real_fft_pair_helpers(shim, w):
    """The in-place paired pre/post-processing of the row kernels."""
    rng = np.random.default_rng(w + 1)
    x = rng.standard_normal(w).astype(np.float32)
    X = np.empty(w // 2 + 1, np.complex64)
    assert shim.shim_rfft_pairs(fp(x), fp(X), w) == 0
    ref = np.fft.rfft(x.astype(np.float64))
    assert np.abs(X - ref).max() / np.abs(ref).max() < 2e-6
    Y = (rng.standard_normal(w // 2 + 1) + 1j * rng.standard_normal(w // 2 + 1)).astype(np.complex64)
    y = np.empty(w, np.float32)
    assert shim.shim_irfft_pairs(fp(Y), fp(y), w) == 0
    refy = np.fft.irfft(Y.astype(np.complex128), w) * w
    assert np.abs(y - refy).max() / np.abs(refy).max() < 2e-6


@pytest.mark.parametrize("n", [128, 256, 512, 1024, 2048, 4096])
@pytest.mark.parametrize("direction", [-1, 1])
def test_radix16_register_fft(shim, n, direction):
    """The radix-16 register FFT (fft_r16.cuh: 16,16,..,RL plan, spad16
    layout, product-tree twiddles), run thread by thread in barrier order,
    against numpy."""
    rng = np.random.default_rng(n)
    x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    out = np.zeros(n, np.complex64)
    assert shim.shim_cfft_r16(fp(x), fp(out), n, direction) == 0
    ref = np.fft.fft(x.astype(np.complex128)) if direction < 0 else np.fft.ifft(x.astype(np.complex128)) * n
    assert np.abs(out - ref).max() < 2e-6 * np.abs(ref).max()
