"""Pins the CPU oracle of the warm-start network before it judges the CUDA
kernels: autograd gradients against central finite differences, the
truncated spectral convolution against its definition as explicit Fourier
sums, the BF16 rounding of the weight file, and the parameter layout shared
with include/pfc_b200.h. Also the numpy heterostructure generator against the
stripe generator it extends. CPU only."""
import os
import re

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import fno_oracle as O  # noqa: E402
from pfc_b200 import fno, synth  # noqa: E402

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "pfc_b200.h")


def random_params(seed, spectral_scale=0.02):
    p = fno.init_params(seed, out_scale=1.0)
    rng = np.random.default_rng(seed + 1)
    for k, (o, s) in fno.layout().items():
        n = int(np.prod(s))
        if k[:2] in ("Rr", "Ri"):
            p[o:o + n] = rng.uniform(-1, 1, n) * spectral_scale
        if k in ("p", "q") or k[0] == "b":
            p[o:o + n] = rng.uniform(-0.1, 0.1, n)
    return p


def test_layout_matches_header():
    text = open(HEADER).read()
    consts = dict(re.findall(r"#define (PFCG_FNO_\w+) (\d+)", text))
    assert int(consts["PFCG_FNO_PARAMS"]) == fno.NPARAM
    assert int(consts["PFCG_FNO_CHANNELS"]) == fno.CHANNELS == O.C
    assert int(consts["PFCG_FNO_LAYERS"]) == fno.LAYERS == O.L
    assert int(consts["PFCG_FNO_MODES_X"]) == fno.MODES_X == O.MX
    assert int(consts["PFCG_FNO_MODES_Y"]) == fno.MODES_Y == O.MY
    assert 1.0e6 < fno.NPARAM < 1.1e6


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -7 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5e-3, 0.0, 65504.0],
                 dtype=np.float32)
    got = fno.bf16_round(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: even mantissa (1.0)
    assert got[0] == 1.0 and got[1] == 1.0
    # 1 + 2^-7 + 2^-8 ties between 1 + 2^-7 (odd) and 1 + 2^-6 (even)
    assert got[2] == np.float32(1.0 + 2 ** -6)
    assert got[3] == np.float32(1.0 + 2 ** -7)
    assert abs(got[4] - x[4]) <= abs(x[4]) * 2 ** -8
    assert got[5] == 0.0
    r = np.random.default_rng(0).normal(size=1000).astype(np.float32)
    assert np.all(np.abs(fno.bf16_round(r) - r) <= np.abs(r) * 2 ** -8)
    assert np.array_equal(fno.bf16_round(fno.bf16_round(r)), fno.bf16_round(r))


def test_spectral_convolution_matches_fourier_sums():
    """irfft2(R * rfft2(v)) on the retained modes == the explicit real sum
    sum_{kx, ky} w(kx) Re(Y(ky, kx) e^{2 pi i (kx x + ky y) / T}) / T^2."""
    T = 32
    rng = np.random.default_rng(3)
    v = rng.normal(size=(1, O.C, T, T))
    Rr = rng.normal(size=(O.C, O.C, O.MY, O.MX))
    Ri = rng.normal(size=(O.C, O.C, O.MY, O.MX))
    got = O.spectral(torch.tensor(v), torch.tensor(Rr), torch.tensor(Ri)).numpy()
    ys, xs = np.mgrid[0:T, 0:T]
    kys = list(range(O.MY // 2)) + list(range(T - O.MY // 2, T))
    want = np.zeros((O.C, T, T))
    R = Rr + 1j * Ri
    for r, ky in enumerate(kys):
        for kx in range(O.MX):
            e_fwd = np.exp(-2j * np.pi * (kx * xs + ky * ys) / T)
            X = (v[0] * e_fwd).sum(axis=(1, 2))               # [C]
            Yk = (R[:, :, r, kx] * X[:, None]).sum(axis=0)      # [out]
            w = 1.0 if kx == 0 else 2.0
            want += w * np.real(Yk[:, None, None] * np.conj(e_fwd)[None]) / T ** 2
    assert np.abs(got[0] - want).max() < 1e-9 * np.abs(want).max()


def test_oracle_gradient_matches_finite_differences():
    T = 32
    rng = np.random.default_rng(5)
    p = random_params(7).astype(np.float64)
    x = rng.normal(scale=0.3, size=(1, 2, T, T))
    t = x + rng.normal(scale=0.05, size=x.shape)
    _, g, _ = O.loss_and_grad(p, x, t)
    blocks = fno.layout()
    picks = []
    for k in ("P", "p", "W0", "b1", "Rr0", "Ri2", "Rr3", "W3", "Q", "q"):
        o, s = blocks[k]
        n = int(np.prod(s))
        picks += [o + int(i) for i in rng.choice(n, 2, replace=False)]
    h = 1e-6
    for i in picks:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (O.loss_and_grad(pp, x, t)[0] - O.loss_and_grad(pm, x, t)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1e-3, abs(g).max()), (i, fd, g[i])


def test_apply_tiled_on_one_tile_grid_is_the_network():
    """On a grid the size of one tile the tiled application is the network
    (periodic halo wraps onto the same tile) up to the mean restoration."""
    T = 32
    rng = np.random.default_rng(9)
    p = fno.bf16_round(random_params(11)).astype(np.float64)
    f = rng.normal(scale=0.3, size=(2, T, T)).astype(np.float32).astype(np.float64)
    got = O.apply_tiled(p, f, T)
    with torch.no_grad():
        y = O.forward(torch.tensor(p), torch.tensor(f[None]))[0].numpy()
    y -= (y - f).mean(axis=(1, 2), keepdims=True)
    assert np.abs(got - y).max() < 1e-10
    assert np.abs(got.mean(axis=(1, 2)) - f.mean(axis=(1, 2))).max() < 1e-13


def test_hetero2_extends_stripes2():
    a = synth.hetero2(96, 64, 0.7, 0.7, 0, 16, 0, (0.3, -0.3), (0.3, 0.3), (7.2552, 7.2552 * 1.04), 0.02, 5)
    b = synth.stripes2(96, 64, 0.7, 0.7, 16, (0.3, -0.3), (0.3, 0.3), (7.2552, 7.2552 * 1.04), 0.02, 5)
    assert np.array_equal(a, b)
    c = synth.hetero2(96, 64, 0.7, 0.7, 0, 16, 5, (0.3, -0.3), (0.3, 0.3), (7.2552, 7.2552), 0.0, 5)
    # stripes shifted by 5 columns: field 0 is disordered exactly where ((x + 5) // 16) is odd
    odd = ((np.arange(96) + 5) // 16) % 2 == 1
    assert np.all(c[0][:, odd] == 0.3) and np.all(c[1][:, ~odd] == -0.3)


def test_hetero2_voronoi_regions():
    g = synth.hetero2(80, 72, 0.7, 0.7, 6, 0, 0, (0.3, -0.3), (0.3, 0.3), (7.2552, 7.5), 0.0, 21)
    # every point has at least one field at its disordered mean
    at_mean = np.stack([g[0] == 0.3, g[1] == -0.3])
    assert np.all(at_mean.sum(axis=0) >= 1)
