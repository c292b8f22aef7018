"""The CPU oracle against numpy, the reference's golden runs and known answers
of the model (no GPU)."""
import math

import numpy as np
import pytest

import pyoracle
from helpers import golden_names, load_golden, params_of, rel
from pfc_b200 import params as P
from pfc_b200 import synth


@pytest.mark.parametrize("shape", [(8, 8), (16, 12), (15, 9), (64, 48), (30, 50), (7, 11), (96, 160)])
def test_fft_matches_numpy(shape):
    Ny, Nx = shape
    a = np.random.default_rng(1).standard_normal((Ny, Nx))
    S = pyoracle.rfft2_tr(a)
    ref = np.fft.rfft2(a).T
    assert np.abs(S - ref).max() <= 1e-13 * np.abs(ref).max()
    back = pyoracle.irfft2_tr(S, Nx) / (Nx * Ny)
    assert np.abs(back - a).max() <= 1e-13


@pytest.mark.parametrize("name", golden_names())
def test_oracle_matches_reference_binary(name):
    """The restatement reproduces the reference binary's .out rows and final
    fields (same FFT underneath, so to rounding)."""
    meta, z = load_golden(name)
    o = pyoracle.Oracle(params_of(meta), meta["Nx"], meta["Ny"], meta["dx"], meta["dy"])
    o.upload(z["fields"])
    rows = o.relax(meta["tend"], meta["Tprint"], meta["Topt"])
    ref = z["rows"]
    assert rows.shape[0] == ref.shape[0]
    # ref columns: t, seconds, dx, dy, <f>, <n_u>...
    np.testing.assert_allclose(rows[:, 0], ref[:, 0])
    np.testing.assert_allclose(rows[:, 1:3], ref[:, 2:4], rtol=1e-12, atol=0)
    np.testing.assert_allclose(rows[:, 3:], ref[:, 4:], rtol=1e-11, atol=1e-15)
    np.testing.assert_allclose(o.download(), z["final"], rtol=0, atol=1e-11)
    fave, nave, f = o.evaluate(want_f=True)
    np.testing.assert_allclose(f, z["f_final"], rtol=0, atol=1e-11)


def test_uniform_field_energy_known_answer():
    """Only k = 0 is non-zero: <f> = lambda n + (alpha + beta P(0))/2 n^2 + gamma/3 n^3 + delta/4 n^4."""
    d = P.honeycomb_1c(-0.25)
    d["gamma"] = [[0.3]]
    d["lambda"] = [0.1]
    p = P.make_params(d, 1.0, 1.0)
    o = pyoracle.Oracle(p, 16, 16, 0.7, 0.7)
    n = 0.2
    o.upload(np.full((1, 16, 16), n))
    fave, nave = o.evaluate()
    P0 = (1.0 - 0.0) ** 2  # (nu2 - 0)^2 with nu = 1
    expect = 0.1 * n + 0.5 * (-0.25 + 1.0 * P0) * n * n + 0.3 / 3 * n ** 3 + 0.25 * n ** 4
    assert rel(fave, expect) < 1e-14
    assert rel(nave[0], n) < 1e-14


def test_conserved_dynamics_keep_mean():
    p = P.make_params(P.honeycomb_1c(-0.25), 1.0, 1.0)
    o = pyoracle.Oracle(p, 32, 32, math.pi / 4, math.pi / 4)
    f0 = synth.noise_state(32, 32, 0.25, 0.05, 2)[None]
    o.upload(f0)
    o.step(50)
    assert abs(o.download().mean() - f0.mean()) < 1e-13


def test_linear_mode_grows_by_A():
    """gamma = delta = lambda = 0: a single Fourier mode is multiplied by exactly
    A(k) = exp(o a dt) per step (pfc-relax.c:946-952)."""
    d = P.honeycomb_1c(-0.25)
    d["delta"] = [0.0]
    p = P.make_params(d, 1.0, 0.5)
    Nx = Ny = 32
    dx = dy = 0.9
    o = pyoracle.Oracle(p, Nx, Ny, dx, dy)
    kxi, kyi = 3, 2
    x = np.arange(Nx) * dx
    y = np.arange(Ny) * dy
    kx = 2 * math.pi * kxi / (dx * Nx)
    ky = 2 * math.pi * kyi / (dy * Ny)
    f0 = 0.01 * np.cos(kx * x[None, :] + ky * y[:, None])
    o.upload(f0[None])
    o.step(3)
    k2 = kx * kx + ky * ky
    a = -0.25 + (1.0 - k2) ** 2
    A = math.exp(-k2 * a * 0.5)
    np.testing.assert_allclose(o.download()[0], f0 * A ** 3, atol=1e-15)


def test_semi_implicit_linear_mode_known_answer():
    """The oracle's semi-implicit variant (not in the reference): with gamma =
    delta = lambda = 0 a single Fourier mode is multiplied by exactly
    1 / (1 + dt k^2 a(k)) per step (conserved dynamics)."""
    d = P.honeycomb_1c(-0.25)
    d["delta"] = [0.0]
    p = P.make_params(d, 1.0, 0.5)
    Nx = Ny = 32
    dx = dy = 0.9
    o = pyoracle.Oracle(p, Nx, Ny, dx, dy)
    o.set_scheme("semi")
    x = np.arange(Nx) * dx
    y = np.arange(Ny) * dy
    kx = 2 * math.pi * 3 / (dx * Nx)
    ky = 2 * math.pi * 2 / (dy * Ny)
    f0 = 0.01 * np.cos(kx * x[None, :] + ky * y[:, None])
    o.upload(f0[None])
    o.step(3)
    k2 = kx * kx + ky * ky
    a = -0.25 + (1.0 - k2) ** 2
    g = 1.0 / (1.0 + 0.5 * k2 * a)
    np.testing.assert_allclose(o.download()[0], f0 * g ** 3, atol=1e-15)


def test_optimize_moves_toward_unstrained_lattice():
    """A one-mode triangular lattice strained by 2% relaxes dx back toward the
    lattice's own spacing (pfc-relax.c:1251-1290)."""
    Nx, Ny = 64, 64
    # 8 lattice periods across x and 5 rectangular cells (sqrt(3) a) across y
    a = synth.A_TRI
    dx0 = 8 * a / Nx
    dy0 = 5 * math.sqrt(3.0) * a / Ny
    d = P.honeycomb_1c(-0.25)
    p = P.make_params(d, 1.0, 1.0)
    X = np.arange(Nx)[None, :] * dx0
    Y = np.arange(Ny)[:, None] * dy0
    f0 = -0.25 - 0.2 * synth.oma(X, Y, 3, a)
    o = pyoracle.Oracle(p, Nx, Ny, dx0 * 1.02, dy0)
    o.upload(f0[None])
    o.step(20)
    dd = 1e-4
    for _ in range(6):
        dd = o.optimize(1, 0, dd)
        o.step(5)
    dx, _ = o.box()
    assert abs(dx - dx0) < abs(dx0 * 1.02 - dx0)
