"""pfcg_relax_noalloc, the entry point for callers that cannot call cudaMalloc
(a host that hands out all device memory from its own pool, or a loop that
must not pay cudaMalloc's implicit device synchronisation): its workspace is a
static device array inside the library, and the caller passes only its own
device buffer of fields.

Checked through the C ABI against the allocating entry points (pfcg_create,
pfcg_upload, pfcg_step, pfcg_download) on two calls in a row, with different
inputs, so a call that leaked state from the previous one would show; against
the FP64 CPU oracle at the FP32 parity bound of the other tests; and on a NaN
input (return 39) followed by a clean call (return 0, so the NaN flag the
first call left in the shared workspace was cleared). The test allocates its
device buffers with torch; the entry point allocates nothing.
This file is collected last so that a run stopping at the first failure has
run every other test before it.
"""
import os
import sys

import numpy as np
import pytest

from pfc_b200 import lib
from pfc_b200 import params as P
from pfc_b200 import synth

pytestmark = pytest.mark.gpu


def reference_run(p, Nx, Ny, dx, dy, f0, n):
    with lib.Relaxation(p, Nx, Ny, dx, dy, "fp32") as r:
        r.upload(f0)
        r.step(n)
        return r.download()


@pytest.mark.parametrize("U,Nx,Ny", [(1, 256, 256), (2, 192, 160)])
def test_noalloc_matches_allocating_path_on_two_calls(U, Nx, Ny):
    import torch

    dx = dy = 0.7
    if U == 1:
        p = P.make_params(P.honeycomb_1c(-0.25), 1.0, 1.0)
        inputs = [synth.noise_state(Nx, Ny, 0.25, 0.05, s)[None] for s in (31, 32)]
    else:
        p = P.make_params(P.hetero_2c(0.04), 1.0, 0.25)
        inputs = [synth.stripes2(Nx, Ny, dx, dy, 32, (0.3, -0.3), (0.3, 0.3), (7.2552, 7.2552 * 1.04), 0.02, s)
                  for s in (33, 34)]
    nsteps = 40
    stream = torch.cuda.Stream()
    for f0 in inputs:
        expect = reference_run(p, Nx, Ny, dx, dy, f0, nsteps)
        dev = torch.tensor(np.ascontiguousarray(f0), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = lib.relax_noalloc(p, Nx, Ny, dx, dy, nsteps, dev.data_ptr(), stream.cuda_stream)
        assert rc == 0, lib.last_error()
        got = dev.cpu().numpy().reshape(expect.shape)
        assert np.abs(got - expect).max() < 1e-6


def test_noalloc_rejects_grids_beyond_its_workspace():
    import torch

    p = P.make_params(P.honeycomb_1c(-0.25), 1.0, 1.0)
    Nx = Ny = 2048  # 2 * 1025 * 2048 * 8 bytes > 32 MiB
    dev = torch.zeros((1, 8, 8), dtype=torch.float64, device="cuda")  # never touched: the size check comes first
    rc = lib.relax_noalloc(p, Nx, Ny, 0.7, 0.7, 1, dev.data_ptr(), 0)
    assert rc == lib.ESIZE
    assert "static workspace" in lib.last_error()


def test_noalloc_matches_oracle():
    """The no-alloc relaxation against the FP64 CPU oracle (test infrastructure),
    at the bounds the FP32 parity tests use: max |dpsi| < 2e-5, relative <f> 1e-6."""
    import torch

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
    import pyoracle

    # 20 steps: before the two-field quench's ordering transient amplifies FP32 rounding
    Nx, Ny, dx, dy, nsteps = 96, 80, 0.7, 0.7, 20
    p = P.make_params(P.hetero_2c(0.04), 1.0, 0.25)
    f0 = synth.stripes2(Nx, Ny, dx, dy, 24, (0.3, -0.3), (0.3, 0.3), (7.2552, 7.2552 * 1.04), 0.02, 41)
    o = pyoracle.Oracle(p, Nx, Ny, dx, dy)
    o.upload(f0)
    o.step(nsteps)
    ref = o.download()
    dev = torch.tensor(np.ascontiguousarray(f0), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    for _ in range(2):
        dev.copy_(torch.tensor(np.ascontiguousarray(f0), dtype=torch.float64))
        rc = lib.relax_noalloc(p, Nx, Ny, dx, dy, nsteps, dev.data_ptr(), 0)
        assert rc == 0, lib.last_error()
        got = dev.cpu().numpy().reshape(ref.shape)
        assert np.abs(got - ref).max() < 2e-5, np.abs(got - ref).max()


def test_noalloc_nan_then_clean_call():
    """A NaN in the input returns the reference's code 39; the next clean call
    returns 0, so the flag left in the shared workspace was cleared."""
    import torch

    Nx = Ny = 64
    p = P.make_params(P.honeycomb_1c(-0.25), 1.0, 1.0)
    bad = synth.noise_state(Nx, Ny, 0.25, 0.05, 51)[None].copy()
    bad[0, 3, 5] = np.nan
    dev = torch.tensor(bad, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    assert lib.relax_noalloc(p, Nx, Ny, 0.7, 0.7, 5, dev.data_ptr(), 0) == lib.NAN
    good = synth.noise_state(Nx, Ny, 0.25, 0.05, 52)[None]
    dev = torch.tensor(np.ascontiguousarray(good), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    assert lib.relax_noalloc(p, Nx, Ny, 0.7, 0.7, 5, dev.data_ptr(), 0) == 0, lib.last_error()
