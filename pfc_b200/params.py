"""Model parameters: the ``pfcg_params`` struct of include/pfc_b200.h as a
ctypes Structure, built from input-file values the way pfc-relax.c's
read_input stores them (pfc-relax.c:542-705): 1/nu and 1/mu are read as
reciprocal lengths and stored squared-inverted (:655, :700), and mu2 is forced
to 0 where beta[u][v] == 0 (:699).

Also the parameter sets of the workloads this package measures.
"""
from __future__ import annotations

import ctypes
import math

MAX_U = 4
MAX_W = 4

_dU = ctypes.c_double * MAX_U
_dUU = (ctypes.c_double * MAX_U) * MAX_U
_dUW = (ctypes.c_double * MAX_W) * MAX_U


class Params(ctypes.Structure):
    _fields_ = [
        ("U", ctypes.c_int),
        ("W", ctypes.c_int * MAX_U),
        ("c", ctypes.c_double),
        ("sigma", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("lambda_", _dU),
        ("delta", _dU),
        ("alpha", _dUU),
        ("beta", _dUU),
        ("gamma", _dUU),
        ("epsilon", _dUU),
        ("mu2", _dUU),
        ("nu2", _dUW),
        ("omega", _dUW),
        ("phi", _dUW),
    ]


def make_params(d: dict, c: float, dt: float) -> Params:
    """``d`` holds input-file values (keys as in nfile.write_input)."""
    U = len(d["lambda"])
    if not 1 <= U <= MAX_U:
        raise ValueError("U must be in 1..%d" % MAX_U)
    p = Params()
    p.U = U
    p.c = c
    p.dt = dt
    p.sigma = d["sigma"]
    for u in range(U):
        p.lambda_[u] = d["lambda"][u]
        p.delta[u] = d["delta"][u]
        W = len(d["inv_nu"][u])
        if not 1 <= W <= MAX_W:
            raise ValueError("W[u] must be in 1..%d" % MAX_W)
        p.W[u] = W
        for w in range(W):
            inv = d["inv_nu"][u][w]
            p.nu2[u][w] = 1.0 / inv / inv
            p.omega[u][w] = d["omega"][u][w]
            p.phi[u][w] = d["phi"][u][w]
        for v in range(u, U):
            p.alpha[u][v] = d["alpha"][u][v]
            p.beta[u][v] = d["beta"][u][v]
            p.gamma[u][v] = d["gamma"][u][v]
        for v in range(u + 1, U):
            p.epsilon[u][v] = d["epsilon"][u][v]
            if d["beta"][u][v] == 0.0:
                p.mu2[u][v] = 0.0
            else:
                inv = d["inv_mu"][u][v]
                p.mu2[u][v] = 1.0 / inv / inv
    return p


def _zeros(U):
    return [[0.0] * U for _ in range(U)]


def honeycomb_1c(eps: float = -0.25) -> dict:
    """Single-component PFC, f = psi/2 (eps + (1 + lap)^2) psi + psi^4/4, in
    pfc-relax's form: alpha = eps, beta = 1, P = (nu^2 + lap)^2 with nu = 1,
    omega = 1, phi = 0, delta = 1, gamma = 0, lambda = 0."""
    return {
        "lambda": [0.0], "alpha": [[eps]], "beta": [[1.0]], "gamma": [[0.0]], "delta": [1.0],
        "epsilon": [[0.0]], "sigma": 0.2, "inv_nu": [[1.0]], "omega": [[1.0]], "phi": [[0.0]],
        "inv_mu": [[0.0]],
    }


def hetero_2c(mismatch: float = 0.04) -> dict:
    """Two-component lateral heterostructure: the first two fields of the
    reference's heterostructure demo (demos/hetero/hetero.in:20-63) with the
    second field's lattice length scaled by 1 + mismatch and the smoothed
    density coupling epsilon_01 = -0.8."""
    U = 2
    a = _zeros(U); b = _zeros(U); g = _zeros(U); e = _zeros(U); m = _zeros(U)
    a[0][0], a[0][1], a[1][1] = -1.4, -0.04, -0.3
    b[0][0], b[1][1] = 2.25, 1.0
    e[0][1] = -0.8
    return {
        "lambda": [0.0, 0.0], "alpha": a, "beta": b, "gamma": g, "delta": [2.25, 1.0],
        "epsilon": e, "sigma": 0.2, "inv_nu": [[1.0], [1.0 + mismatch]], "omega": [[1.0], [1.0]],
        "phi": [[0.0], [0.0]], "inv_mu": m,
    }


# lattice constant of the one-mode triangular state with wave number 1
A_TRI = 4.0 * math.pi / math.sqrt(3.0)
