"""Restatement of the reference's initial-state builder pieces that pfc-init
rebuilds (src/PFCInit.java), in plain Python/numpy.

TEST INFRASTRUCTURE ONLY: imported by tests/, never by the product package.

- java_random: java.util.Random as its API documentation specifies it (48-bit
  linear congruential generator, multiplier 0x5DEECE66D, addend 11; next(bits)
  the top bits; nextDouble = (next(26) * 2^27 + next(27)) * 2^-53; the seed
  scrambled by XOR with the multiplier).
- java_e: String.format("%.{prec}e", v) as java.util.Formatter produces it: the
  shortest decimal digits that read back to v, rounded half up to prec + 1
  significant digits, exponent with sign and at least two digits; NaN and
  Infinity spelled out. Python's repr gives the shortest digits.
- voronoi_step: the "V" step (:389-462) with closest() (:68-93) and OMA
  (:46-66), point by point in the Java loop order, one nextDouble per
  non-phantom point.
- write_n: the "O" step (:670-686).
"""
from __future__ import annotations

import decimal
import math

import numpy as np

_MASK = (1 << 48) - 1
_MULT = 0x5DEECE66D


class JavaRandom:
    def __init__(self, seed: int):
        self.state = (seed ^ _MULT) & _MASK

    def _next(self, bits: int) -> int:
        self.state = (self.state * _MULT + 0xB) & _MASK
        return self.state >> (48 - bits)

    def next_double(self) -> float:
        return ((self._next(26) << 27) + self._next(27)) * 2.0 ** -53


def java_e(v: float, prec: int) -> str:
    if math.isnan(v):
        return "NaN"
    if math.isinf(v):
        return "Infinity" if v > 0 else "-Infinity"
    neg = math.copysign(1.0, v) < 0
    if v == 0.0:
        digits, exp = "0" * (prec + 1), 0
    else:
        with decimal.localcontext() as ctx:
            ctx.prec = prec + 1
            ctx.rounding = decimal.ROUND_HALF_UP
            d = +decimal.Decimal(repr(abs(v)))
        sign, dg, e = d.as_tuple()
        digits = "".join(map(str, dg))
        exp = d.adjusted()
        digits = (digits + "0" * (prec + 1))[: prec + 1]
    mant = digits[0] + ("." + digits[1:] if prec > 0 else "")
    return "%s%se%s%02d" % ("-" if neg else "", mant, "-" if exp < 0 else "+", abs(exp))


def write_n(path: str, field: np.ndarray, dx: float, dy: float, prec: int) -> None:
    Ny, Nx = field.shape
    with open(path, "w", newline="\n") as fh:
        fh.write("%d %d " % (Nx, Ny))
        fh.write("%s %s\n" % (java_e(dx, prec), java_e(dy, prec)))
        for v in field.ravel():
            fh.write(java_e(float(v), prec) + "\n")


def oma(x: float, y: float, sym: int, a: float) -> float:
    q = 2.0 * math.pi / a
    if sym == 3:
        qx, qy = q, q / math.sqrt(3.0)
        return math.cos(qx * x) * math.cos(qy * y) + 0.5 * math.cos(2.0 * qy * y)
    if sym == 4:
        return math.cos(q * x) * math.cos(q * y)
    qx, qy = q, q / math.sqrt(3.0)
    return (- 2.0 * math.cos(qx * x - qy * y) - 2.0 * math.cos(2.0 * qy * y) - 2.0 * math.cos(- qx * x - qy * y)
            + math.cos(- qx * x - 3.0 * qy * y) + math.cos(2.0 * qx * x) + math.cos(- qx * x + 3.0 * qy * y))


def _wrap(d: float, L: float) -> float:
    while d < 0:
        d += L
    while d >= L:
        d -= L
    return d


def closest(u, v, x, y, W, H) -> int:
    n = 0
    d2 = None
    for m in range(len(x)):
        dx = u - x[m]
        if dx > 0.5 * W:
            dx -= W
        elif dx < -0.5 * W:
            dx += W
        dy = v - y[m]
        if dy > 0.5 * H:
            dy -= H
        elif dy < -0.5 * H:
            dy += H
        e = dx * dx + dy * dy
        if d2 is None or e < d2:
            n, d2 = m, e
    return n


def voronoi_step(arr: np.ndarray, dx: float, dy: float, grains: list, rng: JavaRandom) -> np.ndarray:
    """grains: dicts with the V step's fields (x, y, type, sym, a, nave, amp, namp,
    tx1, ty1, theta (degrees), xr, yr, tx2, ty2). arr is modified and returned."""
    Ny, Nx = arr.shape
    W, H = Nx * dx, Ny * dy
    x = [_wrap(g["x"], W) for g in grains]
    y = [_wrap(g["y"], H) for g in grains]
    th = [g["theta"] / 180.0 * math.pi for g in grains]
    for j in range(Ny):
        v = j * dy
        for i in range(Nx):
            u = i * dx
            n = closest(u, v, x, y, W, H)
            g = grains[n]
            if g["type"] == 2:
                continue
            uu = i * dx - g["tx2"] - g["xr"]
            vv = j * dy - g["ty2"] - g["yr"]
            sine, cosine = math.sin(-th[n]), math.cos(-th[n])
            rx = uu * cosine - vv * sine + g["xr"] - g["tx1"]
            ry = uu * sine + vv * cosine + g["yr"] - g["ty1"]
            arr[j, i] = (g["type"] * arr[j, i] + g["nave"] + g["amp"] * oma(rx, ry, g["sym"], g["a"])
                         + 2.0 * g["namp"] * (rng.next_double() - 0.5))
    return arr
