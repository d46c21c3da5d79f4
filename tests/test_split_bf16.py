"""Numerics of the accelerated form (1), split-precision BF16 DFT-GEMMs,
before any tensor-core kernel exists: oracle.split_bf16_dft restates the
arithmetic (FP32 operands split into BF16 hi + lo, hi*hi + hi*lo + lo*hi,
FP32 accumulation) so the error budget of the 408-point patch transforms can
be checked against FP64 and the 0.05 px shift tolerance."""
import numpy as np


def test_split_bf16_dft_error(oracle):
    rng = np.random.default_rng(0)
    n = 408
    x = rng.standard_normal((n, 64)) + 1j * rng.standard_normal((n, 64))
    ref = np.fft.fft(x, axis=0)
    scale = np.sqrt(np.mean(np.abs(ref) ** 2))
    e3 = np.sqrt(np.mean(np.abs(oracle.split_bf16_dft(x, 3) - ref) ** 2)) / scale
    e1 = np.sqrt(np.mean(np.abs(oracle.split_bf16_dft(x, 1) - ref) ** 2)) / scale
    assert e3 < 1e-5, e3      # measured 3.9e-6: FP32-FFT class
    assert e1 > 1e-3, e1      # one BF16 product alone: 2.1e-3


def test_split_bf16_patch_shift(oracle):
    """A 408 x 408 patch pair transformed by split-BF16 GEMMs (columns, then
    rows) gives the same correlation peak as FP64 to 1e-4 px."""
    rng = np.random.default_rng(1)
    n = 408
    ky = np.fft.fftfreq(n)[:, None]
    kx = np.fft.fftfreq(n)[None, :]
    a = np.real(np.fft.ifft2(np.fft.fft2(rng.standard_normal((n, n))) * np.exp(-(kx ** 2 + ky ** 2) / 0.005)))
    s = (1.37, -2.61)
    b = np.real(np.fft.ifft2(np.fft.fft2(a) * np.exp(-2j * np.pi * (kx * s[0] + ky * s[1]))))

    def fft2(img):
        t = oracle.split_bf16_dft(img.astype(np.complex128))
        return oracle.split_bf16_dft(t.T.copy()).T

    def peak(f1, f2):
        c = np.fft.fftshift(np.real(np.fft.ifft2(np.conj(f1) * f2)))
        iy, ix = np.unravel_index(np.argmax(c), c.shape)
        fit = lambda m, z, p: 0.5 * (m - p) / (m + p - 2 * z)
        return np.array([ix + fit(c[iy, ix - 1], c[iy, ix], c[iy, ix + 1]) - n // 2,
                         iy + fit(c[iy - 1, ix], c[iy, ix], c[iy + 1, ix]) - n // 2])

    p64 = peak(np.fft.fft2(a), np.fft.fft2(b))
    p3 = peak(fft2(a), fft2(b))
    assert np.abs(p64 - np.array(s)).max() < 0.05
    assert np.abs(p3 - p64).max() < 1e-4, (p3, p64)
