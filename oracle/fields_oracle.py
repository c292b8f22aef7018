"""CPU oracle of the orientation and deformation fields (test infrastructure only).

Restates src/fields.c of the reference in numpy (complex 2-D FFTs, FP64):
write_phi (fields.c:103-216) and write_chi (fields.c:218-343). Only the tests
import this module, as the checker of the GPU path (pfcg_fields); it is itself
pinned to the reference tool compiled over the FFT shim (oracle/_ref/fields).
"""
from __future__ import annotations

import math

import numpy as np


def _k(W, H, dx, dy):
    """Wave numbers of the complex transform: index i < W/2 -> i, else i - W (fields.c:143-152)."""
    i = np.arange(W)
    j = np.arange(H)
    kx = np.where(i < W // 2, i, i - W) * (2 * math.pi / (dx * W))
    ky = np.where(j < H // 2, j, j - H) * (2 * math.pi / (dy * H))
    return np.meshgrid(kx, ky)


def orientation(p: np.ndarray, dx: float, dy: float, fold: int, sk: float, sb: float):
    """(psi, Z): the complex orientation field normalised to max |psi| = 1 and
    the smoothed spectrum it came from (fields.c:121-200)."""
    H, W = p.shape
    KX, KY = _k(W, H, dx, dy)
    n = W * H
    s = p - p.min()
    z = np.fft.fft2(s.astype(complex))
    q = np.sqrt(KX ** 2 + KY ** 2) - 1.0
    z *= np.exp(-0.5 / sk ** 2 * q * q) * np.exp(1j * fold * np.arctan2(KY, KX)) / n
    z = np.fft.ifft2(z) * n
    z *= s
    Z = np.fft.fft2(z) * np.exp(-0.5 / sb ** 2 * (KX ** 2 + KY ** 2)) / n
    z = np.fft.ifft2(Z) * n
    return z / np.abs(z).max(), Z


def deformation(Z: np.ndarray, dx: float, dy: float, power: float) -> np.ndarray:
    """The deformation field from the smoothed spectrum Z (fields.c:247-320):
    sum over Gaussian scales 1/n, n = 2, 4, ... while n * 4 pi / sqrt(3) < L/2,
    of the convolution of |grad psi|^power normalised to its maximum."""
    H, W = Z.shape
    KX, KY = _k(W, H, dx, dy)
    n = W * H
    zx = np.fft.ifft2(1j * KX * Z) * n
    zy = np.fft.ifft2(1j * KY * Z) * n
    g = (np.abs(zx) ** 2 + np.abs(zy) ** 2) ** (0.5 * power)
    G = np.fft.fft2(g.astype(complex))
    l0 = 4.0 * math.pi / math.sqrt(3.0)
    L = min(W * dx, H * dy)
    out = np.zeros((H, W))
    m = 2
    while l0 * m < 0.5 * L:
        r = (np.fft.ifft2(np.exp(-0.5 * m * m * (KX ** 2 + KY ** 2)) / n * G) * n).real
        out += r / r.max()
        m *= 2
    return out
