"""Relaxation steps and energy evaluations are bit-reproducible: the x-pass
writes each row tile's sums of the nonlinear term to its own slot and the
y-pass adds the slots in a fixed order, and evaluate() adds its row tiles' and
Parseval blocks' sums the same way, so repeated runs from the same state give
the same fields, energies and optimised box bit for bit (the reference, a
serial CPU code, is reproducible the same way). Checked for the compile-time
specialised kernels (FP32 4096^2 and 512^2, FP64 2048^2), the runtime-plan
kernels (320^2) and the batch."""
import math

import numpy as np
import pytest

from pfc_b200 import lib
from pfc_b200 import params as P
from pfc_b200 import synth

pytestmark = pytest.mark.gpu


def _case(U, N):
    if U == 1:
        return P.make_params(P.honeycomb_1c(-0.25), 1.0, 1.0), math.pi / 4, synth.noise_state(N, N, 0.25, 0.05, 9)[None]
    return (P.make_params(P.hetero_2c(0.04), 1.0, 0.25), 0.7,
            synth.stripes2(N, N, 0.7, 0.7, max(N // 8, 8), (0.3, -0.3), (0.3, 0.3), (7.2552, 7.2552 * 1.04), 0.02, 8))


@pytest.mark.parametrize("U,N,prec", [(2, 4096, "fp32"), (1, 512, "fp32"), (2, 2048, "fp64"), (1, 320, "fp32")])
def test_repeated_runs_are_identical(U, N, prec):
    p, d, f0 = _case(U, N)
    out, en = [], []
    for _ in range(2):
        with lib.Relaxation(p, N, N, d, d, prec) as r:
            r.upload(f0)
            r.step(25)
            fave, nave = r.evaluate()
            dd = r.optimize(1, 1, 1e-4)
            r.step(5)
            out.append(r.download())
            en.append([fave] + list(nave) + [dd] + list(r.box()))
    assert np.all(np.isfinite(out[0])) and np.array_equal(out[0], out[1])
    assert en[0] == en[1]


def test_repeated_batches_are_identical():
    probs = []
    for k, (N, U) in enumerate([(256, 1), (384, 2), (96, 2), (512, 1)]):
        p, d, f = _case(U, N)
        probs.append((p, N, N, d, d, f))
    out = []
    for _ in range(2):
        with lib.Batch([q[:5] for q in probs], "fp32", autotune=False) as b:
            for prob, q in zip(b.problems, probs):
                prob.upload(q[5])
            b.step(15)
            out.append([prob.download() for prob in b.problems])
    for a, c in zip(out[0], out[1]):
        assert np.array_equal(a, c)
