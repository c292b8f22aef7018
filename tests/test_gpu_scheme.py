"""The semi-implicit time integrator (pfcg_set_scheme), a selectable variant
beside the reference's ETD1 update (pfc-relax.c:947-953, applied at :1238):
N' = (N + dt o M) / (1 - dt o a), i.e. (N - dt k^2 M) / (1 + dt k^2 a) for
conserved dynamics.

Checked against the CPU oracle running the same update (FP64 to rounding, FP32
to the FP32 parity bound), against the exact growth factor of a single linear
mode, and against ETD1 on the relaxed end state: both schemes share the fixed
points of the dynamics, so from a relaxed state neither moves <f>, and a short
relaxation from the reference's near-relaxed golden state ends at the same <f>.
"""
import math

import numpy as np
import pytest

import pyoracle
from helpers import load_golden, params_of, rel
from pfc_b200 import lib
from pfc_b200 import params as P
from pfc_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("U,Nx,Ny", [(1, 128, 128), (2, 128, 96), (2, 256, 256)])
def test_semi_implicit_matches_oracle(U, Nx, Ny):
    dx = dy = 0.7
    if U == 1:
        p = P.make_params(P.honeycomb_1c(-0.25), 1.0, 1.0)
        f0 = synth.noise_state(Nx, Ny, 0.25, 0.05, 19)[None]
    else:
        p = P.make_params(P.hetero_2c(0.04), 1.0, 0.25)
        f0 = synth.stripes2(Nx, Ny, dx, dy, 16, (0.3, -0.3), (0.3, 0.3), (7.2552, 7.2552 * 1.04), 0.02, 15)
    # FP64 over 60 steps; FP32 over the first 20, before the ordering transient
    # of the two-field quench amplifies its rounding (the semi-implicit factor
    # 1/(1 - x) grows unstable modes faster than ETD1's exp(x))
    for prec, nsteps, tol, etol in (("fp64", 60, 1e-11, 1e-11), ("fp32", 20, 2e-5, 1e-6)):
        o = pyoracle.Oracle(p, Nx, Ny, dx, dy)
        o.set_scheme("semi")
        o.upload(f0)
        o.step(nsteps)
        ref = o.download()
        fo, no = o.evaluate()
        with lib.Relaxation(p, Nx, Ny, dx, dy, prec, scheme="semi") as r:
            assert r.scheme == "semi"
            r.upload(f0)
            r.step(nsteps)
            got = r.download()
            fg, ng = r.evaluate()
        assert np.abs(got - ref).max() < tol, (prec, np.abs(got - ref).max())
        assert rel(fg, fo) < etol, (prec, rel(fg, fo))
        np.testing.assert_allclose(ng, no, rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-14), ("fp32", 1e-6)])
@pytest.mark.parametrize("c", [1.0, 0.0])
def test_semi_implicit_linear_mode(precision, tol, c):
    """gamma = delta = lambda = 0: one Fourier mode is multiplied by exactly
    1 / (1 - o a dt) per step (o = -k^2 conserved, -1 nonconserved)."""
    d = P.honeycomb_1c(-0.25)
    d["delta"] = [0.0]
    p = P.make_params(d, c, 0.5)
    Nx = Ny = 64
    dx = dy = 0.9
    kx = 2 * math.pi * 5 / (dx * Nx)
    ky = 2 * math.pi * 3 / (dy * Ny)
    x = np.arange(Nx) * dx
    y = np.arange(Ny) * dy
    f0 = 0.2 + 0.01 * np.cos(kx * x[None, :] + ky * y[:, None])
    k2 = kx * kx + ky * ky
    a = -0.25 + (1 - k2) ** 2
    o = -k2 if c else -1.0
    g = 1.0 / (1.0 - o * a * 0.5)
    a0 = -0.25 + 1.0  # a(k = 0): the mean relaxes too when the dynamics are nonconserved
    g0 = 1.0 if c else 1.0 / (1.0 + a0 * 0.5)
    with lib.Relaxation(p, Nx, Ny, dx, dy, precision, scheme="semi") as r:
        r.upload(f0[None])
        r.step(4)
        got = r.download()[0]
    expect = 0.2 * g0 ** 4 + (f0 - 0.2) * g ** 4
    assert np.abs(got - expect).max() < tol


@pytest.mark.parametrize("name", ["hetero2_opt_48", "c1_noise_32"])
def test_semi_implicit_and_etd1_share_the_fixed_point(name):
    """The reference's final state of a golden run, relaxed further by ETD1
    until <f> changes by less than 1e-11 per step, is (nearly) a fixed point of
    both schemes: over 500 more steps neither lowers <f> by more than 1e-6
    relative, the semi-implicit run moves <f> by no more than three times what
    ETD1 does, and the two end fields agree to 1e-4."""
    meta, z = load_golden(name)
    with lib.Relaxation(params_of(meta), meta["Nx"], meta["Ny"], *z["box_final"], "fp64") as r:
        r.upload(z["final"])
        steps, _, _ = r.relax_until(1e-11, 100, 100000)
        assert steps is not None
        relaxed = r.download()
    out = {}
    for scheme in ("etd1", "semi"):
        with lib.Relaxation(params_of(meta), meta["Nx"], meta["Ny"], *z["box_final"], "fp64", scheme=scheme) as r:
            r.upload(relaxed)
            f0 = r.evaluate()[0]
            r.step(500)
            out[scheme] = (r.evaluate()[0], r.download())
        assert out[scheme][0] <= f0 * (1 + 1e-14) and rel(out[scheme][0], f0) < 1e-6, (scheme, out[scheme][0], f0)
    assert abs(out["semi"][0] - f0) <= 3 * abs(out["etd1"][0] - f0) + 1e-14 * abs(f0), (out["semi"][0], out["etd1"][0], f0)
    assert np.abs(out["semi"][1] - out["etd1"][1]).max() < 1e-4


def test_scheme_argument_checked():
    p = P.make_params(P.honeycomb_1c(-0.25), 1.0, 1.0)
    with lib.Relaxation(p, 32, 32, 0.7, 0.7, "fp64") as r:
        assert r.scheme == "etd1"
        assert r.L.pfcg_set_scheme(r.h, 7) == lib.EARG


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 1e-6)])
def test_semi_implicit_in_a_batch(precision, tol):
    """Problems of one batch on different schemes (set on the problems' handles
    after the batch was built, so the batch re-uploads their arguments) step
    like single handles on the same schemes."""
    p1 = P.make_params(P.honeycomb_1c(-0.25), 1.0, 1.0)
    p2 = P.make_params(P.hetero_2c(0.04), 1.0, 0.25)
    probs = []
    for k, (N, U) in enumerate([(256, 1), (384, 2), (96, 2), (256, 1)]):
        if U == 1:
            probs.append((p1, N, N, math.pi / 4, math.pi / 4, synth.noise_state(N, N, 0.25, 0.05, 70 + k)[None]))
        else:
            probs.append((p2, N, N, 0.7, 0.7, synth.stripes2(N, N, 0.7, 0.7, 16, (0.3, -0.3), (0.3, 0.3),
                                                             (7.2552, 7.2552 * 1.04), 0.02, 80 + k)))
    schemes = ["semi", "semi", "etd1", "etd1"]
    with lib.Batch([q[:5] for q in probs], precision, autotune=False) as b:
        for prob, q, s in zip(b.problems, probs, schemes):
            prob.upload(q[5])
            prob.set_scheme(s)
        b.step(12)
        got = [prob.download() for prob in b.problems]
    for q, s, g in zip(probs, schemes, got):
        with lib.Relaxation(*q[:5], precision, scheme=s) as r:
            r.upload(q[5])
            r.step(12)
            ref = r.download()
        assert np.abs(g - ref).max() < tol, s
    # the two schemes really differ on these states
    with lib.Relaxation(*probs[0][:5], precision) as r:
        r.upload(probs[0][5])
        r.step(12)
        assert np.abs(r.download() - got[0]).max() > 100 * tol
