"""Seeded synthetic cryo-EM movies with known drift (no dataset is needed).

Truth image: 1/f^2-power random-phase noise plus Gaussian blobs (sigma 2-8
px), normalised to mean 1.  Global drift: a random walk with N(0, step) px
steps plus an early jump over the first frames.  Optional local motion: a
second-order polynomial field in (x, y) times a linear-in-frame factor.
Each frame is a Poisson sample of dose * shifted truth / gain, so applying
the gain restores the dose-scaled image.

`backend="numpy"` is used by the tests (small sizes, bit-reproducible);
`backend="torch"` generates large movies directly on the GPU for the
benchmark.
"""
from __future__ import annotations

import dataclasses
from typing import Optional

import numpy as np


@dataclasses.dataclass
class Movie:
    frames: object           # [nz][ny][nx] float32 (numpy or torch)
    gain: Optional[object]   # [ny][nx] float32 or None
    drift: np.ndarray        # [nz][2] true global displacement (px) of frame content
    local_coef: Optional[np.ndarray]  # [2][6] polynomial coefficients of the local field
    seed: int


def truth_image(nx: int, ny: int, rng: np.random.Generator, n_blobs: int = 200,
                sigma=(2.0, 8.0)) -> np.ndarray:
    kx = np.fft.rfftfreq(nx)[None, :]
    ky = np.fft.fftfreq(ny)[:, None]
    k2 = kx * kx + ky * ky
    k2[0, 0] = 1.0
    amp = 1.0 / np.sqrt(k2)          # power ~ 1/f^2
    amp[0, 0] = 0.0
    ph = rng.uniform(0, 2 * np.pi, size=amp.shape)
    noise = np.fft.irfft2(amp * np.exp(1j * ph), s=(ny, nx))
    noise /= noise.std() + 1e-30
    img = 0.25 * noise
    yy, xx = np.mgrid[0:ny, 0:nx]
    for _ in range(n_blobs):
        cx, cy = rng.uniform(0, nx), rng.uniform(0, ny)
        s = rng.uniform(*sigma)
        a = rng.uniform(0.5, 1.5)
        dx = (xx - cx + nx / 2) % nx - nx / 2
        dy = (yy - cy + ny / 2) % ny - ny / 2
        img += a * np.exp(-(dx * dx + dy * dy) / (2 * s * s))
    img -= img.min()
    img += 0.05 * img.mean()
    img /= img.mean()
    return img


def drift_trajectory(nz: int, rng: np.random.Generator, step: float = 0.7,
                     jump: float = 3.0, jump_frames: int = 4) -> np.ndarray:
    d = np.cumsum(rng.normal(0.0, step, size=(nz, 2)), axis=0)
    ang = rng.uniform(0, 2 * np.pi)
    u = np.array([np.cos(ang), np.sin(ang)])
    for f in range(min(jump_frames, nz)):
        d[f] += jump * u * (1.0 - f / max(jump_frames - 1, 1))
    d -= d[nz // 2]
    return d


def local_coefficients(rng: np.random.Generator, amp: float = 2.0) -> np.ndarray:
    c = rng.normal(0.0, 1.0, size=(2, 6))
    # |field| <= sum |c| for x, y in [-1, 1]; scale so the end frames reach <= amp
    c *= amp / np.abs(c).sum(axis=1, keepdims=True)
    return c


def _poly(c: np.ndarray, xh, yh):
    return c[0] + c[1] * xh + c[2] * yh + c[3] * xh * xh + c[4] * xh * yh + c[5] * yh * yh


def _shift_fourier(img: np.ndarray, dx: float, dy: float) -> np.ndarray:
    ny, nx = img.shape
    F = np.fft.rfft2(img)
    kx = np.fft.rfftfreq(nx)[None, :]
    ky = np.fft.fftfreq(ny)[:, None]
    return np.fft.irfft2(F * np.exp(-2j * np.pi * (kx * dx + ky * dy)), s=(ny, nx))


def make_movie(nx: int, ny: int, nz: int, dose: float = 1.0, seed: int = 0, gain: bool = False,
               local: bool = False, local_amp: float = 2.0, n_blobs: int = 200,
               backend: str = "numpy", device: str = "cuda", drift_step: float = 0.7,
               jump: float = 3.0) -> Movie:
    """drift_step: standard deviation of the random walk's steps (px); jump:
    size of the early jump over the first four frames (px)."""
    rng = np.random.default_rng(seed)
    truth = truth_image(nx, ny, rng, n_blobs=n_blobs)
    drift = drift_trajectory(nz, rng, step=drift_step, jump=jump)
    coef = local_coefficients(rng, local_amp) if local else None
    g = rng.uniform(0.9, 1.1, size=(ny, nx)).astype(np.float32) if gain else None
    if backend == "torch":
        return _make_torch(truth, drift, coef, g, dose, seed, device)
    frames = np.empty((nz, ny, nx), np.float32)
    yy, xx = np.mgrid[0:ny, 0:nx].astype(np.float64)
    xh, yh = 2 * xx / nx - 1, 2 * yy / ny - 1
    for f in range(nz):
        img = _shift_fourier(truth, drift[f, 0], drift[f, 1])
        if coef is not None:
            from scipy import ndimage
            t = (f - nz // 2) / max(nz // 2, 1)
            ux, uy = t * _poly(coef[0], xh, yh), t * _poly(coef[1], xh, yh)
            img = ndimage.map_coordinates(img, [yy - uy, xx - ux], order=3, mode="wrap")
        lam = np.clip(dose * img, 0, None)
        if g is not None:
            lam = lam / g
        frames[f] = rng.poisson(lam).astype(np.float32)
    return Movie(frames=frames, gain=g, drift=drift, local_coef=coef, seed=seed)


def _make_torch(truth, drift, coef, g, dose, seed, device) -> Movie:
    import torch
    ny, nx = truth.shape
    nz = drift.shape[0]
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    T = torch.fft.rfft2(torch.as_tensor(truth, dtype=torch.float64, device=device))
    kx = torch.fft.rfftfreq(nx, device=device, dtype=torch.float64)[None, :]
    ky = torch.fft.fftfreq(ny, device=device, dtype=torch.float64)[:, None]
    frames = torch.empty((nz, ny, nx), dtype=torch.float32, device=device)
    gd = torch.as_tensor(g, device=device) if g is not None else None
    if coef is not None:
        yy, xx = torch.meshgrid(torch.arange(ny, device=device, dtype=torch.float64),
                                torch.arange(nx, device=device, dtype=torch.float64), indexing="ij")
        xh, yh = 2 * xx / nx - 1, 2 * yy / ny - 1
        cx = torch.as_tensor(coef[0], device=device)
        cy = torch.as_tensor(coef[1], device=device)
        px = cx[0] + cx[1] * xh + cx[2] * yh + cx[3] * xh * xh + cx[4] * xh * yh + cx[5] * yh * yh
        py = cy[0] + cy[1] * xh + cy[2] * yh + cy[3] * xh * xh + cy[4] * xh * yh + cy[5] * yh * yh
    for f in range(nz):
        ph = torch.exp(-2j * torch.pi * (kx * float(drift[f, 0]) + ky * float(drift[f, 1])))
        img = torch.fft.irfft2(T * ph, s=(ny, nx))
        if coef is not None:
            t = (f - nz // 2) / max(nz // 2, 1)
            sx = (xx - t * px) / (nx - 1) * 2 - 1
            sy = (yy - t * py) / (ny - 1) * 2 - 1
            grid = torch.stack([sx, sy], dim=-1)[None].float()
            img = torch.nn.functional.grid_sample(img[None, None].float(), grid, mode="bicubic",
                                                  padding_mode="reflection",
                                                  align_corners=True)[0, 0].double()
        lam = torch.clamp(dose * img, min=0)
        if gd is not None:
            lam = lam / gd
        frames[f] = torch.poisson(lam.float(), generator=gen)
    return Movie(frames=frames, gain=gd, drift=drift, local_coef=coef, seed=seed)
