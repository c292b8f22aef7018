"""The y-pass's TMA column loads: the same fields bit for bit as the plain
loads (PFCG_TMA=0), and the bounded mbarrier wait, made to run out on purpose
with the test hook PFCG_TMA_TEST_STALL (the wait then expects more bytes than
the loads bring, gives up after 1 ms and the step returns PFCG_ETIMEOUT; the
loads themselves are unchanged), after which a fresh handle steps normally."""
import numpy as np
import pytest

from pfc_b200 import lib
from pfc_b200 import params as P
from pfc_b200 import synth

pytestmark = pytest.mark.gpu


def _case(U, N):
    dx = 0.7
    if U == 1:
        return P.make_params(P.honeycomb_1c(-0.25), 1.0, 1.0), synth.noise_state(N, N, 0.25, 0.05, 3)[None]
    return (P.make_params(P.hetero_2c(0.04), 1.0, 0.25),
            synth.stripes2(N, N, dx, dx, max(N // 8, 8), (0.3, -0.3), (0.3, 0.3), (7.2552, 7.2552 * 1.04), 0.02, 4))


@pytest.mark.parametrize("U,N", [(2, 4096), (1, 2048), (2, 1024), (1, 256)])
def test_tma_loads_match_plain_loads(U, N, monkeypatch):
    p, f0 = _case(U, N)
    out = {}
    for mode in ("1", "0"):
        monkeypatch.setenv("PFCG_TMA", mode)
        with lib.Relaxation(p, N, N, 0.7, 0.7, "fp32") as r:
            r.upload(f0)
            r.step(7)
            out[mode] = r.download()
    assert np.array_equal(out["1"], out["0"])


def test_tma_wait_times_out_on_purpose(monkeypatch):
    p, f0 = _case(1, 256)
    monkeypatch.setenv("PFCG_TMA_TEST_STALL", "16")
    with lib.Relaxation(p, 256, 256, 0.7, 0.7, "fp32") as r:
        r.upload(f0)
        assert r.step_rc(2) == lib.ETIMEOUT
        assert "wait" in r.L.pfcg_last_error(r.h).decode()
    monkeypatch.delenv("PFCG_TMA_TEST_STALL")
    with lib.Relaxation(p, 256, 256, 0.7, 0.7, "fp32") as r:
        r.upload(f0)
        assert r.step_rc(3) == 0
