"""Learned warm start for two-field relaxations: a Fourier neural operator
trained on (initial, relaxed) pairs that the relaxation itself generates.

The network, its gradients, Adam and the tiled application are CUDA kernels
behind the pfcg_fno_* entry points of include/pfc_b200.h; this module holds
the parameter initialisation, the weight file, data generation (seeded
initial states from pfcg_init_hetero, relaxed by the batched FP32 path) and
the training loop. torch provides device buffers and index shuffling only.

The shipped weights (weights/fno_hetero2c_512.npz, made by `python -m
pfc_b200.fno`) map the state after `input_step` (500) plain FP32 steps to the
state `horizon` (4500) steps later; the seeded initial state itself is not a
usable input, because the lattice that forms in the first few hundred steps is
not predictable from it (the state after 2000 steps is as far from the initial
one as the fully relaxed state is).

Usage:
    net = Network(tile=512, max_batch=32)
    net.set_params(load_weights())
    relaxation.step(weights_meta()["input_step"])
    relaxation.warmstart(net)         # pfcg_warmstart on a U = 2 handle
    relaxation.relax_until(1e-9)      # the plain method finishes and judges
"""
from __future__ import annotations

import ctypes
import math
import os
import time

import numpy as np

from . import lib
from . import params as P

CHANNELS, LAYERS, MODES_X, MODES_Y = 32, 4, 8, 16
NK = MODES_X * MODES_Y
NPARAM = 2 * CHANNELS + CHANNELS + LAYERS * (CHANNELS * CHANNELS + CHANNELS + 2 * CHANNELS * CHANNELS * NK) \
    + 2 * CHANNELS + 2

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "weights", "fno_hetero2c_512.npz")


def layout() -> dict:
    """Offsets and shapes of each parameter block in the flat vector (the order
    of include/pfc_b200.h)."""
    C = CHANNELS
    out, off = {}, 0

    def put(name, shape):
        nonlocal off
        out[name] = (off, shape)
        off += int(np.prod(shape))

    put("P", (C, 2))
    put("p", (C,))
    for l in range(LAYERS):
        put("W%d" % l, (C, C))
        put("b%d" % l, (C,))
        put("Rr%d" % l, (C, C, MODES_Y, MODES_X))
        put("Ri%d" % l, (C, C, MODES_Y, MODES_X))
    put("Q", (2, C))
    put("q", (2,))
    assert off == NPARAM
    return out


def unpack(flat: np.ndarray) -> dict:
    return {k: flat[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in layout().items()}


def init_params(seed: int = 0, out_scale: float = 0.01) -> np.ndarray:
    """Uniform fan-in initialisation; spectral weights of size 1/C^2 and a small
    projection, so the untrained network is close to the identity map."""
    rng = np.random.default_rng(seed)
    C = CHANNELS
    flat = np.zeros(NPARAM, dtype=np.float32)
    for k, (o, s) in layout().items():
        n = int(np.prod(s))
        if k == "P":
            v = rng.uniform(-1, 1, n) / math.sqrt(2)
        elif k[0] == "W":
            v = rng.uniform(-1, 1, n) / math.sqrt(C)
        elif k[:2] in ("Rr", "Ri"):
            v = rng.uniform(-1, 1, n) / (C * C)
        elif k == "Q":
            v = rng.uniform(-1, 1, n) / math.sqrt(C) * out_scale
        else:
            v = np.zeros(n)
        flat[o:o + n] = v
    return flat


def to_bf16_bits(x: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even FP32 -> BF16 bit patterns."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = (b + 0x7FFF + ((b >> 16) & 1)) >> 16
    return r.astype(np.uint16)


def from_bf16_bits(h: np.ndarray) -> np.ndarray:
    return (h.astype(np.uint32) << 16).view(np.float32)


def bf16_round(x: np.ndarray) -> np.ndarray:
    """The weights the kernels read: FP32 rounded to BF16."""
    return from_bf16_bits(to_bf16_bits(x))


def save_weights(path: str, flat: np.ndarray, meta: dict) -> None:
    """BF16 weights (the precision the kernels read) plus training metadata."""
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez_compressed(path, bf16=to_bf16_bits(flat), meta=np.array(repr(meta)))


def load_weights(path: str = DEFAULT_WEIGHTS) -> np.ndarray:
    z = np.load(path)
    return from_bf16_bits(z["bf16"])


def weights_meta(path: str = DEFAULT_WEIGHTS) -> dict:
    import ast
    return ast.literal_eval(str(np.load(path)["meta"]))


class Network:
    """One pfcg_fno object: weights, Adam state and activation buffers for up to
    max_batch tiles of tile x tile points."""

    def __init__(self, tile: int = 512, max_batch: int = 16):
        self.L = lib.load()
        assert self.L.pfcg_fno_param_count() == NPARAM
        f = ctypes.c_void_p()
        rc = self.L.pfcg_fno_create(tile, max_batch, ctypes.byref(f))
        if rc:
            raise lib.PfcError(rc, self.L.pfcg_fno_last_error(None).decode())
        self.f = f
        self.tile, self.max_batch = tile, max_batch

    def _check(self, rc):
        if rc:
            raise lib.PfcError(rc, self.L.pfcg_fno_last_error(self.f).decode())

    def close(self):
        if getattr(self, "f", None):
            self.L.pfcg_fno_destroy(self.f)
            self.f = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_params(self, flat: np.ndarray) -> None:
        a = np.ascontiguousarray(flat, dtype=np.float32)
        assert a.size == NPARAM
        self._check(self.L.pfcg_fno_set_params(self.f, a.ctypes.data_as(ctypes.c_void_p)))

    def get_params(self) -> np.ndarray:
        a = np.empty(NPARAM, dtype=np.float32)
        self._check(self.L.pfcg_fno_get_params(self.f, a.ctypes.data_as(ctypes.c_void_p)))
        return a

    def forward(self, d_in: int, d_out: int, batch: int) -> None:
        """DEVICE [batch][2][tile][tile] FP32 in and out."""
        self._check(self.L.pfcg_fno_forward(self.f, ctypes.c_void_p(d_in), ctypes.c_void_p(d_out), batch))

    def loss_grad(self, d_in: int, d_target: int, batch: int, want_grad: bool = False):
        loss = ctypes.c_double()
        g = np.empty(NPARAM, dtype=np.float32) if want_grad else None
        self._check(self.L.pfcg_fno_loss_grad(self.f, ctypes.c_void_p(d_in), ctypes.c_void_p(d_target), batch,
                                              ctypes.byref(loss),
                                              g.ctypes.data_as(ctypes.c_void_p) if want_grad else None))
        return (loss.value, g) if want_grad else loss.value

    def adam_step(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8) -> None:
        self._check(self.L.pfcg_fno_adam_step(self.f, lr, beta1, beta2, eps))

    def apply(self, d_in: int, d_out: int, Nx: int, Ny: int, stream: int = 0) -> None:
        """Tiled application on a DEVICE grid of 2 x Ny x Nx doubles."""
        self._check(self.L.pfcg_fno_apply(self.f, ctypes.c_void_p(d_in), ctypes.c_void_p(d_out), Nx, Ny,
                                          ctypes.c_void_p(stream)))

    def launches(self) -> int:
        n = ctypes.c_longlong()
        self._check(self.L.pfcg_fno_launch_count(self.f, ctypes.byref(n)))
        return n.value


# ------------------------------------------------------------------ data ---

A0 = 7.2552  # lattice constant of the heterostructure workload's first field


def state_spec(i: int, seed0: int, N: int):
    """Initial state i of the training distribution: alternately stripes
    (width 32..N/2 columns, random offset) and Voronoi grains (2..16) of the
    two fields, lattice mismatch 2..6 %, amplitudes 0.2..0.4, noise 0.02."""
    u = np.random.default_rng(seed0 * 1000003 + i).uniform(size=6)
    mismatch = 1.02 + 0.04 * u[0]
    amp = 0.2 + 0.2 * u[1]
    if i % 2 == 0:
        width = int(32 * 2 ** (u[2] * math.log2(N / 64)))
        return lib.make_hetero(0, width, int(u[3] * 2 * width), (0.3, -0.3), (amp, amp), (A0, A0 * mismatch), 0.02,
                               seed0 * 100000 + i)
    grains = 2 + int(u[4] * 15)
    return lib.make_hetero(grains, 1, 0, (0.3, -0.3), (amp, amp), (A0, A0 * mismatch), 0.02, seed0 * 100000 + i,
                           max_angle_deg=60.0 * u[5])


def make_pairs(n: int, N: int = 512, steps=(10000,), seed0: int = 1, chunk: int = 400, dx: float = 0.7,
               log=print):
    """n pairs of N x N two-field heterostructure states: the seeded initial
    state and the state after each step count in `steps` of the batched FP32
    relaxation. Returns X [n, 2, N, N] and {steps: Y [n, 2, N, N]}, device FP32."""
    import torch
    p = P.make_params(P.hetero_2c(0.04), 1.0, 0.25)
    steps = sorted(steps)
    X = torch.empty((n, 2, N, N), dtype=torch.float32, device="cuda")
    Ys = {s: torch.empty_like(X) for s in steps}
    buf = torch.empty((2, N, N), dtype=torch.float64, device="cuda")
    t0 = time.time()
    for c0 in range(0, n, chunk):
        m = min(chunk, n - c0)
        with lib.Batch([(p, N, N, dx, dx)] * m, "fp32", autotune=True) as b:
            for j in range(m):
                lib.init_hetero(buf.data_ptr(), N, N, dx, dx, state_spec(c0 + j, seed0, N))
                X[c0 + j].copy_(buf)
                b.problems[j].upload_device(buf.data_ptr())
            torch.cuda.synchronize()
            done = 0
            for s in steps:
                while done < s:
                    k = min(1000, s - done)
                    b.step(k)
                    done += k
                for j in range(m):
                    b.problems[j].download_device(buf.data_ptr())
                    Ys[s][c0 + j].copy_(buf)
                torch.cuda.synchronize()
        log("pairs %d/%d  %.1f s" % (c0 + m, n, time.time() - t0))
    return X, Ys


def train(net: Network, X, Y, epochs: int = 20, batch: int = 16, lr: float = 1e-3, seed: int = 0, val=None,
          log=print) -> dict:
    """Adam on the mean-square error with a cosine learning-rate decay; random
    periodic shifts of each pair (a symmetry of the relaxation) as augmentation."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    n = X.shape[0]
    T = X.shape[-1]
    assert T == net.tile and batch <= net.max_batch
    xb = torch.empty((batch, 2, T, T), dtype=torch.float32, device="cuda")
    yb = torch.empty_like(xb)
    iters = epochs * (n // batch)
    it = 0
    hist = []
    t0 = time.time()
    for ep in range(epochs):
        perm = torch.randperm(n, generator=g)
        tot = 0.0
        for k in range(n // batch):
            idx = perm[k * batch:(k + 1) * batch].cuda()
            sx, sy = (int(v) for v in torch.randint(0, T, (2,), generator=g))
            xb.copy_(torch.roll(X.index_select(0, idx), (sy, sx), (2, 3)))
            yb.copy_(torch.roll(Y.index_select(0, idx), (sy, sx), (2, 3)))
            torch.cuda.synchronize()
            loss = net.loss_grad(xb.data_ptr(), yb.data_ptr(), batch)
            rate = lr * 0.5 * (1 + math.cos(math.pi * it / max(iters, 1)))
            net.adam_step(rate)
            tot += loss
            it += 1
        rec = {"epoch": ep, "train_mse": tot / (n // batch), "seconds": time.time() - t0}
        if val is not None:
            rec["val_mse"] = evaluate_mse(net, *val, batch)
        hist.append(rec)
        log(rec)
    return {"history": hist, "iters": iters, "seconds": time.time() - t0}


def evaluate_mse(net: Network, X, Y, batch: int = 16) -> float:
    """Mean-square error of the network's output over (X, Y), batch by batch."""
    tot, cnt = 0.0, 0
    for k in range(0, X.shape[0] - batch + 1, batch):
        xb = X[k:k + batch].contiguous()
        yb = Y[k:k + batch].contiguous()
        import torch
        torch.cuda.synchronize()
        tot += net.loss_grad(xb.data_ptr(), yb.data_ptr(), batch)
        cnt += 1
    return tot / max(cnt, 1)


def identity_mse(X, Y) -> float:
    return float(((X - Y) ** 2).mean())


def main(argv=None) -> None:
    """Regenerates the shipped weights: python -m pfc_b200.fno [--pairs 4000 ...].
    Input = the state after --input-step plain FP32 steps, target = the state
    after --target-step steps, 512 x 512 two-field heterostructures."""
    import argparse

    ap = argparse.ArgumentParser()
    ap.add_argument("--pairs", type=int, default=4000)
    ap.add_argument("--input-step", type=int, default=500)
    ap.add_argument("--target-step", type=int, default=5000)
    ap.add_argument("--epochs", type=int, default=12)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    a = ap.parse_args(argv)
    X0, Ys = make_pairs(a.pairs, 512, (a.input_step, a.target_step), seed0=a.seed, chunk=500)
    X, Y = Ys[a.input_step], Ys[a.target_step]
    del X0
    nval = 96
    with Network(512, a.batch) as net:
        net.set_params(init_params(0))
        tr = train(net, X[:-nval], Y[:-nval], epochs=a.epochs, batch=a.batch, lr=a.lr,
                   val=(X[-nval:], Y[-nval:]))
        save_weights(a.out, net.get_params(),
                     {"tile": 512, "input_step": a.input_step, "horizon": a.target_step - a.input_step,
                      "pairs": a.pairs, "epochs": a.epochs, "val_mse": tr["history"][-1]["val_mse"],
                      "identity_mse": identity_mse(X[-nval:], Y[-nval:]), "batch": a.batch, "lr": a.lr,
                      "data": "fno.make_pairs(%d, 512, (%d, %d), seed0=%d): state after %d FP32 steps -> state after %d"
                              % (a.pairs, a.input_step, a.target_step, a.seed, a.input_step, a.target_step),
                      "model": "hetero_2c(0.04), c=1, dt=0.25, dx=dy=0.7"})


if __name__ == "__main__":
    main()
