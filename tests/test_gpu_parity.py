"""GPU path (libpfc_b200.so through the C ABI) against the reference's golden
runs and the CPU oracle.

Tolerances: the FP64 path follows the reference's arithmetic except for the
FFT (own Stockham on the GPU) and the Parseval form of the energy, so it agrees
to rounding amplified by the dynamics (fields 1e-9 absolute, energies 1e-9
relative; the box optimisation amplifies energy rounding into dx, dy at the
1e-10 level). The FP32 path is held to the FP32 accuracy bound: relative
difference of <f> against FP64 of at most 1e-6 while the field is near a
relaxed state, with max |dpsi| stated.
"""
import math

import numpy as np
import pytest

import pyoracle
from helpers import golden_names, load_golden, params_of, rel
from pfc_b200 import lib
from pfc_b200 import params as P
from pfc_b200 import synth

pytestmark = pytest.mark.gpu


def relax_gpu(meta, fields, precision):
    r = lib.Relaxation(params_of(meta), meta["Nx"], meta["Ny"], meta["dx"], meta["dy"], precision)
    r.upload(fields)
    rows = r.relax(meta["tend"], meta["Tprint"], meta["Topt"])
    return r, rows


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-14), ("fp32", 2e-6)])
@pytest.mark.parametrize("shape", [(32, 32), (64, 48), (40, 48), (56, 70), (512, 512), (128, 4096)])
def test_upload_download_roundtrip(precision, tol, shape):
    Ny, Nx = shape
    f = synth.noise_state(Nx, Ny, 0.3, 0.1, 4)[None]
    p = P.make_params(P.honeycomb_1c(), 1.0, 1.0)
    with lib.Relaxation(p, Nx, Ny, 0.7, 0.7, precision) as r:
        r.upload(f)
        back = r.download()
    assert np.abs(back - f).max() < tol


@pytest.mark.parametrize("name", golden_names())
def test_golden_fp64(name):
    meta, z = load_golden(name)
    r, rows = relax_gpu(meta, z["fields"], "fp64")
    ref = z["rows"]
    assert rows.shape[0] == ref.shape[0]
    np.testing.assert_allclose(rows[:, 1:3], ref[:, 2:4], rtol=1e-9, atol=0)
    np.testing.assert_allclose(rows[:, 3:], ref[:, 4:], rtol=1e-9, atol=1e-13)
    np.testing.assert_allclose(r.download(), z["final"], rtol=0, atol=1e-8)
    fave, nave, f = r.evaluate(want_f=True)
    np.testing.assert_allclose(f, z["f_final"], rtol=0, atol=1e-8)
    r.close()


# Runs whose first steps amplify rounding by orders of magnitude (deep quench,
# alpha_00 = -1.4: unstable modes grow x1.42 per step) follow a different
# trajectory in FP32; their FP32 check is the near-relaxed one below.
CHAOTIC = {"hetero2_opt_48"}


@pytest.mark.parametrize("name", [n for n in golden_names() if n not in CHAOTIC])
def test_golden_fp32(name):
    """FP32 FFT/pointwise with FP64 reductions and k = 0 mode, from the
    reference's initial states: energies and means against the reference run."""
    meta, z = load_golden(name)
    r, rows = relax_gpu(meta, z["fields"], "fp32")
    ref = z["rows"]
    np.testing.assert_allclose(rows[:, 3], ref[:, 4], rtol=2e-5, atol=1e-9)
    # means: exact (FP64) under conserved dynamics; with nonconserved dynamics
    # the k = 0 update sums FP32 nonlinear terms
    np.testing.assert_allclose(rows[:, 4:], ref[:, 5:], rtol=1e-12 if meta["c"] else 3e-6, atol=1e-14)
    np.testing.assert_allclose(r.download(), z["final"], rtol=0, atol=5e-3)
    r.close()


@pytest.mark.parametrize("name", golden_names())
def test_fp32_near_relaxed_energy_bound(name):
    """From the reference's final (near-relaxed) state, FP32 and FP64 GPU runs
    of 200 more steps agree on <f> to 1e-6 relative (the FP32 accuracy bound) and
    on the field to max |dpsi| < 1e-4."""
    meta, z = load_golden(name)
    out = {}
    for prec in ("fp64", "fp32"):
        with lib.Relaxation(params_of(meta), meta["Nx"], meta["Ny"], *z["box_final"], prec) as r:
            r.upload(z["final"])
            r.step(200)
            out[prec] = (r.evaluate()[0], r.download())
    assert rel(out["fp32"][0], out["fp64"][0]) < 1e-6
    assert np.abs(out["fp32"][1] - out["fp64"][1]).max() < 1e-4


@pytest.mark.parametrize("U,Nx,Ny", [(1, 128, 128), (2, 128, 96), (1, 256, 256), (2, 256, 256), (3, 96, 64)])
def test_fp64_matches_oracle_stepwise(U, Nx, Ny):
    dx = dy = 0.7
    if U == 1:
        p = P.make_params(P.honeycomb_1c(-0.25), 1.0, 1.0)
        f0 = synth.noise_state(Nx, Ny, 0.25, 0.05, 9)[None]
    elif U == 2:
        p = P.make_params(P.hetero_2c(0.04), 1.0, 0.25)
        f0 = synth.stripes2(Nx, Ny, dx, dy, 16, (0.3, -0.3), (0.3, 0.3), (7.2552, 7.2552 * 1.04), 0.02, 5)
    else:
        from golden.make_golden import hetero_3c
        p = P.make_params(hetero_3c(), 1.0, 0.25)
        f0 = np.array([synth.noise_state(Nx, Ny, m, 0.1, 7, stream=u) for u, m in enumerate((0.485, -0.32, -0.32))])
    o = pyoracle.Oracle(p, Nx, Ny, dx, dy)
    o.upload(f0)
    with lib.Relaxation(p, Nx, Ny, dx, dy, "fp64") as r:
        r.upload(f0)
        for chunk in (1, 9, 40, 70):
            assert o.step(chunk) == 0
            r.step(chunk)
            assert r.t == o.t
            np.testing.assert_allclose(r.download(), o.download(), rtol=0, atol=1e-11)
            fo, no = o.evaluate()
            fg, ng = r.evaluate()
            assert rel(fg, fo) < 1e-11
            np.testing.assert_allclose(ng, no, rtol=1e-12, atol=1e-14)


def test_nan_detection_returns_39():
    p = P.make_params(P.honeycomb_1c(), 1.0, 1.0)
    f = synth.noise_state(64, 64, 0.25, 0.05, 1)[None].copy()
    f[0, 10, 17] = np.nan
    with lib.Relaxation(p, 64, 64, 0.7, 0.7, "fp32") as r:
        r.upload(f)
        assert r.step_rc(3) == lib.NAN


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-14), ("fp32", 1e-6)])
def test_linear_mode_grows_by_A(precision, tol):
    """gamma = delta = lambda = 0: one Fourier mode is multiplied by A(k) per step."""
    d = P.honeycomb_1c(-0.25)
    d["delta"] = [0.0]
    p = P.make_params(d, 1.0, 0.5)
    Nx = Ny = 64
    dx = dy = 0.9
    kx = 2 * math.pi * 5 / (dx * Nx)
    ky = 2 * math.pi * 3 / (dy * Ny)
    x = np.arange(Nx) * dx
    y = np.arange(Ny) * dy
    f0 = 0.2 + 0.01 * np.cos(kx * x[None, :] + ky * y[:, None])
    k2 = kx * kx + ky * ky
    A = math.exp(-k2 * (-0.25 + (1 - k2) ** 2) * 0.5)
    with lib.Relaxation(p, Nx, Ny, dx, dy, precision) as r:
        r.upload(f0[None])
        r.step(4)
        got = r.download()[0]
    expect = 0.2 + (f0 - 0.2) * A ** 4
    assert np.abs(got - expect).max() < tol


def test_fp32_conserved_mean_is_exact():
    """Conserved dynamics: B(0) = 0, and the k = 0 mode is held in FP64, so the
    mean does not drift at all in FP32; the field's own mean stays within FP32
    rounding of it."""
    p = P.make_params(P.honeycomb_1c(-0.25), 1.0, 1.0)
    f0 = synth.noise_state(256, 256, 0.25, 0.05, 3)[None]
    with lib.Relaxation(p, 256, 256, math.pi / 4, math.pi / 4, "fp32") as r:
        r.upload(f0)
        _, n0 = r.evaluate()
        r.step(300)
        _, n1 = r.evaluate()
        field_mean = r.download().mean()
    assert n1[0] == n0[0]
    assert abs(n0[0] - f0.mean()) < 1e-15
    assert abs(field_mean - n1[0]) < 1e-9


def test_launches_per_step():
    p = P.make_params(P.honeycomb_1c(), 1.0, 1.0)
    with lib.Relaxation(p, 128, 128, 0.7, 0.7, "fp32") as r:
        r.upload(synth.noise_state(128, 128, 0.25, 0.05, 1)[None])
        c0 = r.launches
        r.step(200)
        assert r.launches - c0 == 2 * 200


@pytest.mark.parametrize("U,N,steps", [(1, 2048, 3), (2, 2048, 3), (1, 4096, 2), (2, 4096, 2)])
def test_specialised_sizes_match_oracle(U, N, steps):
    """The compile-time specialised STEP kernels of lengths 2048 and 4096 against
    the CPU oracle, FP64 and FP32."""
    dx = dy = 0.7
    if U == 1:
        p = P.make_params(P.honeycomb_1c(-0.25), 1.0, 1.0)
        f0 = synth.noise_state(N, N, 0.25, 0.05, 21)[None]
    else:
        p = P.make_params(P.hetero_2c(0.04), 1.0, 0.25)
        f0 = synth.stripes2(N, N, dx, dy, 256, (0.3, -0.3), (0.3, 0.3), (7.2552, 7.2552 * 1.04), 0.02, 22)
    o = pyoracle.Oracle(p, N, N, dx, dy)
    o.upload(f0)
    o.step(steps)
    ref = o.download()
    fo, _ = o.evaluate()
    o.close()
    for prec, tol, etol in (("fp64", 1e-12, 1e-12), ("fp32", 2e-5, 1e-6)):
        with lib.Relaxation(p, N, N, dx, dy, prec) as r:
            r.upload(f0)
            r.step(steps)
            got = r.download()
            fg, _ = r.evaluate()
        assert np.abs(got - ref).max() < tol, (prec, np.abs(got - ref).max())
        assert rel(fg, fo) < etol, (prec, rel(fg, fo))


@pytest.mark.parametrize("U", [1, 2])
@pytest.mark.parametrize("N", [256, 384, 512, 768, 1024, 1536])
def test_specialised_fp32_lengths_match_oracle(U, N, monkeypatch):
    """The FP32 STEP kernels specialised on the lengths below 2048 (radix 16 with
    a tail pass of radix 1, 2, 3, 4 or 6; 384 as radix 8, 6, 8) against the CPU
    oracle, beside the
    runtime-plan kernels (PFCG_GENERIC_KERNELS=1) on the same state. The two
    FP32 results differ in rounding only, which shows that a different
    transform ran."""
    dx = dy = 0.7
    steps = 5
    if U == 1:
        p = P.make_params(P.honeycomb_1c(-0.25), 1.0, 1.0)
        f0 = synth.noise_state(N, N, 0.25, 0.05, 31)[None]
    else:
        p = P.make_params(P.hetero_2c(0.04), 1.0, 0.25)
        f0 = synth.stripes2(N, N, dx, dy, N // 8, (0.3, -0.3), (0.3, 0.3), (7.2552, 7.2552 * 1.04), 0.02, 32)
    o = pyoracle.Oracle(p, N, N, dx, dy)
    o.upload(f0)
    o.step(steps)
    ref = o.download()
    fo, _ = o.evaluate()
    o.close()
    got = {}
    for generic in ("0", "1"):
        monkeypatch.setenv("PFCG_GENERIC_KERNELS", generic)
        with lib.Relaxation(p, N, N, dx, dy, "fp32") as r:
            r.upload(f0)
            r.step(steps)
            got[generic] = r.download()
            fg, _ = r.evaluate()
        assert np.abs(got[generic] - ref).max() < 2e-5, (generic, np.abs(got[generic] - ref).max())
        assert rel(fg, fo) < 1e-6, (generic, rel(fg, fo))
    assert not np.array_equal(got["0"], got["1"])


@pytest.mark.parametrize("U,Nx,Ny", [(2, 1024, 512), (1, 768, 1536), (2, 256, 4096), (1, 1536, 256)])
def test_specialised_fp32_rectangles_match_oracle(U, Nx, Ny):
    """Rectangular grids whose x and y lengths both have specialised kernels:
    the x-pass takes Nx's row tile, and the y-pass is specialised only where
    Ny's kernels use the same tile (1024 x 512, 768 x 1536, 1536 x 256), else
    the runtime-plan y-pass reads that layout (256 x 4096 at U = 2)."""
    dx, dy = 0.7, 0.75
    steps = 5
    if U == 1:
        p = P.make_params(P.honeycomb_1c(-0.25), 1.0, 1.0)
        f0 = synth.noise_state(Nx, Ny, 0.25, 0.05, 33)[None]
    else:
        p = P.make_params(P.hetero_2c(0.04), 1.0, 0.25)
        f0 = synth.stripes2(Nx, Ny, dx, dy, max(Nx // 8, 8), (0.3, -0.3), (0.3, 0.3), (7.2552, 7.2552 * 1.04), 0.02,
                            34)
    o = pyoracle.Oracle(p, Nx, Ny, dx, dy)
    o.upload(f0)
    o.step(steps)
    ref = o.download()
    fo, _ = o.evaluate()
    o.close()
    with lib.Relaxation(p, Nx, Ny, dx, dy, "fp32") as r:
        r.upload(f0)
        r.step(steps)
        got = r.download()
        fg, _ = r.evaluate()
    assert np.abs(got - ref).max() < 2e-5, np.abs(got - ref).max()
    assert rel(fg, fo) < 1e-6, rel(fg, fo)


@pytest.mark.parametrize("U,Nx,Ny", [(1, 8192, 8), (2, 8, 8192), (1, 7000, 12), (2, 10, 6174), (1, 8192, 40),
                                      (2, 7168, 8)])
def test_extreme_shapes_match_oracle(U, Nx, Ny):
    """The longest supported transforms (8192; 7168 with a factor 7), the
    shortest (8), ragged aspect ratios and the 5/7 radices against the CPU
    oracle, in each precision pfcg_size_supported_for accepts; where it refuses,
    pfcg_create refuses too."""
    dx, dy = 0.7, 0.65
    if U == 1:
        p = P.make_params(P.honeycomb_1c(-0.25), 1.0, 1.0)
        f0 = synth.noise_state(Nx, Ny, 0.25, 0.05, 31)[None]
    else:
        p = P.make_params(P.hetero_2c(0.04), 1.0, 0.25)
        f0 = np.array([synth.noise_state(Nx, Ny, m, 0.05, 32, stream=u) for u, m in enumerate((0.3, -0.3))])
    assert lib.size_supported(Nx, Ny)
    assert lib.size_supported_for(Nx, Ny, U, "fp32")  # every shape here fits in FP32
    o = pyoracle.Oracle(p, Nx, Ny, dx, dy)
    o.upload(f0)
    o.step(5)
    ref = o.download()
    fo, _ = o.evaluate()
    o.close()
    for prec, tol, etol in (("fp64", 1e-12, 1e-12), ("fp32", 2e-5, 1e-6)):
        if not lib.size_supported_for(Nx, Ny, U, prec):
            with pytest.raises(lib.PfcError) as e:
                lib.Relaxation(p, Nx, Ny, dx, dy, prec)
            assert e.value.code == lib.ESIZE
            continue
        with lib.Relaxation(p, Nx, Ny, dx, dy, prec) as r:
            r.upload(f0)
            r.step(5)
            assert np.abs(r.download() - ref).max() < tol, prec
            assert rel(r.evaluate()[0], fo) < etol, prec


def four_fields():
    """Four coupled fields (the most pfcg_params holds): the three-field
    heterostructure plus a fourth field with two modes, coupled to the first by
    smoothed-density (epsilon) and gradient (beta, mu) terms and to the third by
    alpha and gamma."""
    from golden.make_golden import hetero_3c

    d = hetero_3c()
    U = 4
    grow = lambda m, fill=0.0: [row + [fill] for row in m] + [[0.0] * U]  # noqa: E731
    d["alpha"] = grow(d["alpha"])
    d["alpha"][3][3] = -0.2
    d["alpha"][2][3] = 0.1
    d["beta"] = grow(d["beta"])
    d["beta"][3][3] = 1.0
    d["beta"][0][3] = 0.02
    d["gamma"] = grow(d["gamma"])
    d["gamma"][2][3] = 0.2
    d["epsilon"] = grow(d["epsilon"])
    d["epsilon"][0][3] = -0.5
    d["inv_mu"] = grow(d["inv_mu"])
    d["inv_mu"][0][3] = 1.05
    d["lambda"] = d["lambda"] + [0.0]
    d["delta"] = d["delta"] + [1.0]
    d["inv_nu"] = d["inv_nu"] + [[1.0, 2.0 ** 0.5]]
    d["omega"] = d["omega"] + [[1.0, 1.0]]
    d["phi"] = d["phi"] + [[0.0, 0.05]]
    return d


@pytest.mark.parametrize("Nx,Ny", [(64, 48), (80, 60)])
def test_four_fields_match_oracle(Nx, Ny):
    dx = dy = 0.7
    p = P.make_params(four_fields(), 1.0, 0.25)
    f0 = np.array([synth.noise_state(Nx, Ny, m, 0.1, 41, stream=u) for u, m in enumerate((0.485, -0.32, -0.32, 0.1))])
    o = pyoracle.Oracle(p, Nx, Ny, dx, dy)
    o.upload(f0)
    with lib.Relaxation(p, Nx, Ny, dx, dy, "fp64") as r64, lib.Relaxation(p, Nx, Ny, dx, dy, "fp32") as r32:
        r64.upload(f0)
        r32.upload(f0)
        for chunk in (1, 9, 20):
            assert o.step(chunk) == 0
            r64.step(chunk)
            r32.step(chunk)
            ref = o.download()
            np.testing.assert_allclose(r64.download(), ref, rtol=0, atol=1e-11)
            assert np.abs(r32.download() - ref).max() < 2e-5
            fo, no = o.evaluate()
            assert rel(r64.evaluate()[0], fo) < 1e-11
            assert rel(r32.evaluate()[0], fo) < 1e-6
            np.testing.assert_allclose(r64.evaluate()[1], no, rtol=1e-12, atol=1e-14)
