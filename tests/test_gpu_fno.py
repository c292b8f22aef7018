"""Warm-start network kernels (pfcg_fno_*) against the CPU oracle, and the
device initial-state generator (pfcg_init_hetero) against its numpy
restatement.

Tolerances: the kernels compute in FP32 with BF16 weights, the oracle in
float64 with the same BF16 weights, so outputs agree to FP32 rounding of sums
of ~10^3-10^4 terms (1e-4 absolute on O(1) values) and gradients to 2e-3 in
relative L2 norm per parameter block."""
import os

import numpy as np
import pytest

from oracle import fno_oracle as O
from pfc_b200 import fno, lib, synth
from pfc_b200 import params as P

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


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


def inputs(B, T, seed):
    rng = np.random.default_rng(seed)
    x = np.stack([synth.hetero2(T, T, 0.7, 0.7, 0, T // 2, 3 + b, (0.3, -0.3), (0.3, 0.3), (7.2552, 7.5), 0.02,
                                seed + b) for b in range(B)]).astype(np.float32)
    t = (x + rng.normal(scale=0.05, size=x.shape)).astype(np.float32)
    return x, t


@pytest.mark.parametrize("T,B", [(32, 2), (64, 3)])
def test_forward_and_gradient_match_oracle(T, B):
    p = random_params(T + B)
    x, t = inputs(B, T, 100 + T)
    with fno.Network(T, 4) as net:
        net.set_params(p)
        dx = torch.tensor(x, device="cuda")
        dt = torch.tensor(t, device="cuda")
        dy = torch.empty_like(dx)
        torch.cuda.synchronize()
        net.forward(dx.data_ptr(), dy.data_ptr(), B)
        loss, g = net.loss_grad(dx.data_ptr(), dt.data_ptr(), B, want_grad=True)
        y = dy.cpu().numpy()
    pw = fno.bf16_round(p).astype(np.float64)
    loss_o, g_o, y_o = O.loss_and_grad(pw, x, t)
    assert np.abs(y - y_o).max() < 1e-4 * max(1.0, np.abs(y_o).max())
    assert abs(loss - loss_o) < 1e-4 * loss_o
    for k, (o, s) in fno.layout().items():
        n = int(np.prod(s))
        a, b = g[o:o + n].astype(np.float64), g_o[o:o + n]
        err = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        assert err < 2e-3, (k, err)


def test_adam_step_matches_its_formula():
    T, B = 32, 2
    p = random_params(3)
    x, t = inputs(B, T, 7)
    with fno.Network(T, B) as net:
        net.set_params(p)
        dx = torch.tensor(x, device="cuda")
        dt = torch.tensor(t, device="cuda")
        torch.cuda.synchronize()
        m = np.zeros_like(p, dtype=np.float64)
        v = np.zeros_like(p, dtype=np.float64)
        want = p.astype(np.float64)
        for step in range(1, 4):
            _, g = net.loss_grad(dx.data_ptr(), dt.data_ptr(), B, want_grad=True)
            net.adam_step(1e-3, 0.9, 0.999, 1e-8)
            g = g.astype(np.float64)
            m = 0.9 * m + 0.1 * g
            v = 0.999 * v + 0.001 * g * g
            want = want - 1e-3 * (m / (1 - 0.9 ** step)) / (np.sqrt(v / (1 - 0.999 ** step)) + 1e-8)
            got = net.get_params()
            assert np.abs(got - want).max() < 1e-6
            want = got.astype(np.float64)


def test_training_reduces_the_loss():
    """A learnable target (the input plus a smooth function of it) on a small
    tile: 150 Adam steps cut the loss by 10x or more."""
    T, B = 32, 4
    x, _ = inputs(8, T, 11)
    t = (x + 0.05 * np.tanh(4 * x)).astype(np.float32)
    with fno.Network(T, B) as net:
        net.set_params(fno.init_params(0))
        X = torch.tensor(x, device="cuda")
        Y = torch.tensor(t, device="cuda")
        first = None
        for it in range(150):
            k = (it * B) % 8
            xb, yb = X[k:k + B].contiguous(), Y[k:k + B].contiguous()
            torch.cuda.synchronize()
            loss = net.loss_grad(xb.data_ptr(), yb.data_ptr(), B)
            first = loss if first is None else first
            net.adam_step(3e-3)
        assert loss < first / 10, (first, loss)


@pytest.mark.parametrize("Nx,Ny", [(96, 64), (80, 40)])
def test_tiled_apply_matches_oracle_and_keeps_means(Nx, Ny):
    T = 32
    p = random_params(5)
    f = synth.hetero2(Nx, Ny, 0.7, 0.7, 4, 0, 0, (0.3, -0.3), (0.3, 0.3), (7.2552, 7.5), 0.02, 8)
    with fno.Network(T, 3) as net:  # several batches of tiles
        net.set_params(p)
        din = torch.tensor(f, device="cuda")
        dout = torch.empty_like(din)
        torch.cuda.synchronize()
        net.apply(din.data_ptr(), dout.data_ptr(), Nx, Ny)
        got = dout.cpu().numpy()
    want = O.apply_tiled(fno.bf16_round(p).astype(np.float64), f, T)
    assert np.abs(got - want).max() < 1e-4
    assert np.abs(got.mean(axis=(1, 2)) - f.mean(axis=(1, 2))).max() < 1e-12


def test_warmstart_through_the_handle():
    """pfcg_warmstart = download, tiled apply, upload, on the device; the step
    counter is kept and the state relaxes on from there."""
    N, T = 128, 64
    p = random_params(9)
    f = synth.hetero2(N, N, 0.7, 0.7, 0, 48, 5, (0.3, -0.3), (0.3, 0.3), (7.2552, 7.5), 0.02, 12)
    prm = P.make_params(P.hetero_2c(0.04), 1.0, 0.25)
    with fno.Network(T, 8) as net, lib.Relaxation(prm, N, N, 0.7, 0.7, "fp64") as r:
        net.set_params(p)
        r.upload(f)
        r.step(3)
        before = r.download()
        r.warmstart(net)
        assert r.t == 3
        after = r.download()
        din = torch.tensor(before, device="cuda")
        dout = torch.empty_like(din)
        torch.cuda.synchronize()
        net.apply(din.data_ptr(), dout.data_ptr(), N, N)
        assert np.abs(after - dout.cpu().numpy()).max() < 1e-12
        r.step(5)
        assert np.isfinite(r.evaluate()[0])


@pytest.mark.parametrize("grains,width,offset", [(0, 24, 0), (0, 40, 17), (5, 0, 0), (16, 0, 0)])
def test_init_hetero_matches_numpy(grains, width, offset):
    Nx, Ny = 112, 80
    spec = lib.make_hetero(grains, max(width, 1), offset, (0.3, -0.3), (0.25, 0.35), (7.2552, 7.2552 * 1.04),
                           0.02, 77 + grains, max_angle_deg=45.0)
    d = torch.empty((2, Ny, Nx), dtype=torch.float64, device="cuda")
    lib.init_hetero(d.data_ptr(), Nx, Ny, 0.7, 0.7, spec)
    got = d.cpu().numpy()
    want = synth.hetero2(Nx, Ny, 0.7, 0.7, grains, max(width, 1), offset, (0.3, -0.3), (0.25, 0.35),
                         (7.2552, 7.2552 * 1.04), 0.02, 77 + grains, max_angle_deg=45.0)
    assert np.abs(got - want).max() < 1e-12


def test_committed_weights_load_and_run():
    if not os.path.exists(fno.DEFAULT_WEIGHTS):
        pytest.skip("no trained weights in the tree")
    w = fno.load_weights()
    assert w.size == fno.NPARAM and np.all(np.isfinite(w))
    meta = fno.weights_meta()
    with fno.Network(meta["tile"], 2) as net:
        net.set_params(w)
        assert np.array_equal(net.get_params(), w)


def test_trained_network_gain_on_held_out_states():
    """What the shipped network gains over the plain method on states it was
    not trained on (seed 7; training used seed 1): from the state after the
    network's input step, its proposal is closer to the state the plain method
    reaches `horizon` steps later than the input state itself is (the plain
    method's own estimate without those steps). Measured on 8 held-out
    512 x 512 pairs; the trained model gave 0.81 of the no-network error on
    its validation set."""
    if not os.path.exists(fno.DEFAULT_WEIGHTS):
        pytest.skip("no trained weights in the tree")
    meta = fno.weights_meta()
    s0, s1 = meta["input_step"], meta["input_step"] + meta["horizon"]
    X0, Ys = fno.make_pairs(8, 512, (s0, s1), seed0=7, chunk=8, log=lambda *a: None)
    X, Y = Ys[s0], Ys[s1]
    with fno.Network(512, 8) as net:
        net.set_params(fno.load_weights())
        out = torch.empty_like(X)
        torch.cuda.synchronize()
        net.forward(X.data_ptr(), out.data_ptr(), 8)
    err_net = float(((out - Y) ** 2).mean())
    err_plain = float(((X - Y) ** 2).mean())
    print("held-out mean-square distance to the state %d steps on: network %.4f, without %.4f (ratio %.3f)"
          % (meta["horizon"], err_net, err_plain, err_net / err_plain))
    assert err_net < 0.92 * err_plain
