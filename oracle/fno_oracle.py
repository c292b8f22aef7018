"""CPU oracle of the warm-start network (test infrastructure only).

Only the tests import this module, as the checker of the CUDA kernels in
pfc_b200/csrc/fno.cu; the product path never calls it.
The network has no counterpart in the reference. Its definition is the
Fourier neural operator of Li et al., "Fourier Neural Operator for Parametric
Partial Differential Equations" (ICLR 2021), in the fixed shape of
include/pfc_b200.h: lift, four spectral + pointwise layers with GELU (none
after the last), projection added to the input. The spectral convolution
keeps modes kx = 0..MODES_X-1 and ky = -MODES_Y/2..MODES_Y/2-1 of
torch.fft.rfft2 and maps back with torch.fft.irfft2, evaluated in float64
with the BF16-rounded weights the kernels read; gradients come from torch
autograd, an implementation independent of the hand-written adjoints.
A finite-difference test pins this oracle's gradients, and a test of explicit
Fourier sums pins its spectral convolution.
"""
from __future__ import annotations

import numpy as np
import torch

C, L, MX, MY = 32, 4, 8, 16


def _blocks(flat: torch.Tensor) -> dict:
    out, off = {}, 0

    def take(name, shape):
        nonlocal off
        n = int(np.prod(shape))
        out[name] = flat[off:off + n].reshape(shape)
        off += n

    take("P", (C, 2))
    take("p", (C,))
    for l in range(L):
        take("W%d" % l, (C, C))
        take("b%d" % l, (C,))
        take("Rr%d" % l, (C, C, MY, MX))
        take("Ri%d" % l, (C, C, MY, MX))
    take("Q", (2, C))
    take("q", (2,))
    assert off == flat.numel()
    return out


def spectral(v: torch.Tensor, Rr: torch.Tensor, Ri: torch.Tensor) -> torch.Tensor:
    """irfft2 of sum_i R[i, o] * rfft2(v)[i] on the retained modes. v: [B, C, T, T]."""
    T = v.shape[-1]
    V = torch.fft.rfft2(v)                                  # [B, C, T, T/2+1]
    rows = list(range(MY // 2)) + list(range(T - MY // 2, T))
    Vk = V[:, :, rows, :MX]                                 # [B, C, MY, MX]
    R = torch.complex(Rr, Ri)                               # [in, out, MY, MX]
    Yk = torch.einsum("bikm,iokm->bokm", Vk, R)
    H = torch.zeros(v.shape[0], C, T, T // 2 + 1, dtype=V.dtype)
    H[:, :, rows, :MX] = Yk
    return torch.fft.irfft2(H, s=(T, T))


def forward(flat: torch.Tensor, x: torch.Tensor) -> torch.Tensor:
    """y = network(x), x: [B, 2, T, T] float64."""
    w = _blocks(flat)
    v = torch.einsum("ci,bixy->bcxy", w["P"], x) + w["p"][None, :, None, None]
    for l in range(L):
        z = torch.einsum("oi,bixy->boxy", w["W%d" % l], v) + w["b%d" % l][None, :, None, None] \
            + spectral(v, w["Rr%d" % l], w["Ri%d" % l])
        v = torch.nn.functional.gelu(z) if l < L - 1 else z
    return x + torch.einsum("jc,bcxy->bjxy", w["Q"], v) + w["q"][None, :, None, None]


def loss_and_grad(flat_bf16: np.ndarray, x: np.ndarray, target: np.ndarray):
    """Mean-square error over all points of both fields and its gradient with
    respect to the (BF16-rounded) weights, in float64."""
    p = torch.tensor(np.asarray(flat_bf16, dtype=np.float64), requires_grad=True)
    xt = torch.tensor(np.asarray(x, dtype=np.float64))
    tt = torch.tensor(np.asarray(target, dtype=np.float64))
    y = forward(p, xt)
    loss = ((y - tt) ** 2).mean()
    loss.backward()
    return float(loss.detach()), p.grad.numpy().copy(), y.detach().numpy()


def apply_tiled(flat_bf16: np.ndarray, fields: np.ndarray, T: int) -> np.ndarray:
    """Tiled application on a periodic grid (2, Ny, Nx): T x T tiles whose central
    T/2 block is kept, T/4 points of periodic halo; each field's mean restored."""
    halo, core = T // 4, T // 2
    _, Ny, Nx = fields.shape
    p = torch.tensor(np.asarray(flat_bf16, dtype=np.float64))
    out = np.empty_like(fields)
    for by in range(-(-Ny // core)):
        for bx in range(-(-Nx // core)):
            ys = (np.arange(T) + by * core - halo) % Ny
            xs = (np.arange(T) + bx * core - halo) % Nx
            tile = fields[:, ys][:, :, xs].astype(np.float32).astype(np.float64)
            with torch.no_grad():
                y = forward(p, torch.tensor(tile[None]))[0].numpy()
            ye, xe = min(core, Ny - by * core), min(core, Nx - bx * core)
            out[:, by * core:by * core + ye, bx * core:bx * core + xe] = y[:, halo:halo + ye, halo:halo + xe]
    out -= (out - fields).mean(axis=(1, 2), keepdims=True)
    return out
