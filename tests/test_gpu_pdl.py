"""Launch modes of the step kernels give the same results bit for bit: the x-
and y-pass kernels as programmatic dependent launches (the default) against
plain launches (PFCG_PDL=0), and runs of 16 steps replayed as one captured CUDA
graph (the default) against every kernel launched from the host
(PFCG_STEP_GRAPH=0), also across changes of the box and the scheme, which make
the graph be captured again. The switches are read once per process, so each
arm runs in its own interpreter.

Steps and evaluate() are bit-reproducible (every sum over CTAs is added in a
fixed order), so the fields and the energies must be equal."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SNIPPET = r"""
import sys
import numpy as np
sys.path.insert(0, {root!r})
from pfc_b200 import lib, synth
from pfc_b200 import params as P
U, N, prec, out, nsteps, changes = {U}, {N}, {prec!r}, {out!r}, {nsteps}, {changes}
if U == 1:
    p = P.make_params(P.honeycomb_1c(-0.25), 1.0, 1.0)
    f0 = synth.noise_state(N, N, 0.25, 0.05, 3)[None]
else:
    p = P.make_params(P.hetero_2c(0.04), 1.0, 0.25)
    f0 = synth.stripes2(N, N, 0.7, 0.7, max(N // 8, 8), (0.3, -0.3), (0.3, 0.3), (7.2552, 7.2552 * 1.04), 0.02, 4)
with lib.Relaxation(p, N, N, 0.7, 0.7, prec) as r:
    r.upload(f0)
    r.step(nsteps)
    if changes:
        # new arguments: the captured step graph must be recaptured each time
        r.set_box(0.7 * 1.01, 0.7 * 0.99)
        r.step(33)
        r.set_scheme("semi")
        r.step(20)
        r.set_scheme("etd1")
        r.set_box(0.7, 0.7)
        r.step(17)
    fave, nave = r.evaluate()
    np.savez(out, fields=r.download(), energy=np.array([fave] + list(nave)))
"""


@pytest.mark.parametrize("U,N,prec", [(2, 4096, "fp32"), (1, 512, "fp32"), (2, 256, "fp64"), (2, 384, "fp32")])
def test_dependent_launch_matches_plain_launch(U, N, prec, tmp_path):
    res = {}
    for mode in ("1", "0"):
        out = str(tmp_path / ("pdl%s.npz" % mode))
        env = dict(os.environ, PFCG_PDL=mode)
        code = SNIPPET.format(root=ROOT, U=U, N=N, prec=prec, out=out, nsteps=9, changes=False)
        r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        res[mode] = np.load(out)
    a, b = res["1"], res["0"]
    assert np.all(np.isfinite(a["fields"])) and np.array_equal(a["fields"], b["fields"])
    assert np.array_equal(a["energy"], b["energy"])


@pytest.mark.parametrize("U,N,prec", [(2, 4096, "fp32"), (1, 512, "fp32"), (2, 2048, "fp64"), (1, 320, "fp32")])
def test_step_graph_matches_host_launches(U, N, prec, tmp_path):
    res = {}
    for mode in ("1", "0"):
        out = str(tmp_path / ("graph%s.npz" % mode))
        env = dict(os.environ, PFCG_STEP_GRAPH=mode)
        code = SNIPPET.format(root=ROOT, U=U, N=N, prec=prec, out=out, nsteps=41, changes=True)
        r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        res[mode] = np.load(out)
    a, b = res["1"], res["0"]
    assert np.all(np.isfinite(a["fields"])) and np.array_equal(a["fields"], b["fields"])
    assert np.array_equal(a["energy"], b["energy"])
