"""Batched relaxation (pfcg_batch_*) against the same problems stepped one at a
time, and autotuned launch shapes against the default ones."""
import math

import numpy as np
import pytest

from pfc_b200 import lib
from pfc_b200 import params as P
from pfc_b200 import synth

pytestmark = pytest.mark.gpu


def problems():
    """Mixed sizes (radix 2, 3, 5), one and two fields, and box-size scalings of one
    state. 256 (twice), 384, 512 and 768 have specialised kernels in FP32 (a
    class of their own each in the batch, 768 with a radix-3 tail pass, 384 in
    radix 8); the rest run the runtime-plan kernels together."""
    out = []
    p1 = P.make_params(P.honeycomb_1c(-0.25), 1.0, 1.0)
    p2 = P.make_params(P.hetero_2c(0.04), 1.0, 0.25)
    base = synth.noise_state(96, 96, 0.25, 0.05, 40)[None]
    for k, (N, U) in enumerate([(256, 1), (96, 2), (160, 1), (384, 2), (128, 1), (512, 2), (768, 1), (256, 1)]):
        if U == 1:
            f = synth.noise_state(N, N, 0.25, 0.05, 50 + k)[None]
            out.append((p1, N, N, math.pi / 4, math.pi / 4, f))
        else:
            f = synth.stripes2(N, N, 0.7, 0.7, 16, (0.3, -0.3), (0.3, 0.3), (7.2552, 7.2552 * 1.04), 0.02, 60 + k)
            out.append((p2, N, N, 0.7, 0.7, f))
    for s in (0.98, 1.0, 1.02):
        out.append((p1, 96, 96, math.pi / 4 * s, math.pi / 4 * s, base))
    return out


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 1e-6)])
def test_batch_matches_single_problems(precision, tol):
    probs = problems()
    with lib.Batch([p[:5] for p in probs], precision, autotune=True) as b:
        for prob, p in zip(b.problems, probs):
            prob.upload(p[5])
        b.step(7)
        b.step(13)  # a second captured graph
        # FP32: classes (1, 256), (2, 384), (2, 512), (1, 768) and the runtime-plan rest
        assert b.launches(7) == (2 * 7 * (5 if precision == "fp32" else 1), 1)
        got = [prob.download() for prob in b.problems]
        energies = [prob.evaluate()[0] for prob in b.problems]
    for p, g, e in zip(probs, got, energies):
        with lib.Relaxation(*p[:5], precision) as r:
            r.upload(p[5])
            r.step(20)
            ref = r.download()
            fe = r.evaluate()[0]
        assert np.abs(g - ref).max() < tol
        assert abs(e - fe) <= tol * abs(fe)


@pytest.mark.parametrize("N", [384, 320])
def test_autotune_keeps_results(N):
    """320 has no specialised kernels: the autotuner picks the row tile and
    column group of the runtime-plan kernels. 384 has them and keeps their
    fixed shape."""
    p = P.make_params(P.honeycomb_1c(-0.25), 1.0, 1.0)
    f = synth.noise_state(N, N, 0.25, 0.05, 70)[None]
    out = []
    for tune in (False, True):
        with lib.Relaxation(p, N, N, 0.8, 0.8, "fp32") as r:
            if tune:
                r.autotune(3)
            r.upload(f)
            r.step(30)
            out.append(r.download())
    assert np.abs(out[0] - out[1]).max() < 1e-5


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 1e-6)])
def test_batch_specialised_2048(precision, tol):
    """2048² problems (specialised in both precisions: a class of their own, in
    FP64 on the same kernels as the persistent single-problem grid) beside a
    runtime-plan one, against the same problems stepped one at a time."""
    p1 = P.make_params(P.honeycomb_1c(-0.25), 1.0, 1.0)
    p2 = P.make_params(P.hetero_2c(0.04), 1.0, 0.25)
    probs = [(p1, 2048, 2048, math.pi / 4, math.pi / 4, synth.noise_state(2048, 2048, 0.25, 0.05, 80)[None]),
             (p2, 2048, 2048, 0.7, 0.7,
              synth.stripes2(2048, 2048, 0.7, 0.7, 256, (0.3, -0.3), (0.3, 0.3), (7.2552, 7.2552 * 1.04), 0.02, 81)),
             (p1, 96, 96, math.pi / 4, math.pi / 4, synth.noise_state(96, 96, 0.25, 0.05, 82)[None])]
    with lib.Batch([p[:5] for p in probs], precision, autotune=False) as b:
        for prob, p in zip(b.problems, probs):
            prob.upload(p[5])
        b.step(4)
        assert b.launches(4) == (2 * 4 * 3, 1)
        got = [prob.download() for prob in b.problems]
    for p, g in zip(probs, got):
        with lib.Relaxation(*p[:5], precision) as r:
            r.upload(p[5])
            r.step(4)
            ref = r.download()
        assert np.abs(g - ref).max() < tol
