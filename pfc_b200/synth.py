"""Seeded synthetic initial states for the relaxation workloads.

Every input the tests and the benchmark use is generated here, so the CPU
oracle, the reference binary and the GPU path consume identical bytes.

Random numbers are counter based: value ``k`` of stream ``s`` under seed ``seed``
is the splitmix64 finaliser of ``(seed << 32) + (s << 56) + k`` (Steele, Lea and
Flood, "Fast splittable pseudorandom number generators", OOPSLA 2014). Two such
64-bit words give one standard normal by Box-Muller: u1 in (0, 1], u2 in [0, 1),
z = sqrt(-2 ln u1) cos(2 pi u2). The result depends only on (seed, stream, k),
never on how many values were drawn before, so a field can be generated in any
order or in pieces.

The lattice states restate the one-mode approximations of the reference's
initial-state builder (src/PFCInit.java:46-66, ``OMA``) and its periodic
nearest-centre Voronoi assignment (src/PFCInit.java:68-93 ``closest``,
:389-462).
"""
from __future__ import annotations

import math

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def _splitmix64(x: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = x + _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def uniform(seed: int, n: int, stream: int = 0, offset: int = 0) -> np.ndarray:
    """n uniforms in [0, 1) from words offset .. offset+n-1 of (seed, stream)."""
    key = (np.uint64(seed & 0xFFFFFF) << np.uint64(32)) + (np.uint64(stream & 0xFF) << np.uint64(56))
    idx = np.arange(offset, offset + n, dtype=np.uint64)
    with np.errstate(over="ignore"):
        w = _splitmix64(key + idx)
    return (w >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def normal(seed: int, n: int, stream: int = 0) -> np.ndarray:
    """n standard normals (Box-Muller over consecutive word pairs)."""
    key = (np.uint64(seed & 0xFFFFFF) << np.uint64(32)) + (np.uint64(stream & 0xFF) << np.uint64(56))
    idx = np.arange(n, dtype=np.uint64) * np.uint64(2)
    with np.errstate(over="ignore"):
        a = _splitmix64(key + idx)
        b = _splitmix64(key + idx + np.uint64(1))
    u1 = ((a >> np.uint64(11)).astype(np.float64) + 1.0) * (1.0 / 9007199254740992.0)
    u2 = (b >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * math.pi * u2)


def oma(x: np.ndarray, y: np.ndarray, sym: int, a: float) -> np.ndarray:
    """One-mode approximation of a 2-D lattice with lattice constant a
    (src/PFCInit.java:46-66): sym 3 triangular, 4 square, 6 honeycomb."""
    q = 2.0 * math.pi / a
    if sym == 3:
        qx, qy = q, q / math.sqrt(3.0)
        return np.cos(qx * x) * np.cos(qy * y) + 0.5 * np.cos(2.0 * qy * y)
    if sym == 4:
        return np.cos(q * x) * np.cos(q * y)
    if sym == 6:
        qx, qy = q, q / math.sqrt(3.0)
        return (-2.0 * np.cos(qx * x - qy * y) - 2.0 * np.cos(2.0 * qy * y) - 2.0 * np.cos(-qx * x - qy * y)
                + np.cos(-qx * x - 3.0 * qy * y) + np.cos(2.0 * qx * x) + np.cos(-qx * x + 3.0 * qy * y))
    raise ValueError("sym must be 3, 4 or 6")


# lattice constant of the triangular one-mode state whose wave number is 1 (nu = 1)
A_TRI = 4.0 * math.pi / math.sqrt(3.0)


def noise_state(Nx: int, Ny: int, mean: float, amp: float, seed: int, stream: int = 0) -> np.ndarray:
    """mean + amp * N(0, 1) white noise, shape (Ny, Nx)."""
    return mean + amp * normal(seed, Nx * Ny, stream).reshape(Ny, Nx)


def voronoi_labels(Nx: int, Ny: int, dx: float, dy: float, cx: np.ndarray, cy: np.ndarray) -> np.ndarray:
    """Index of the periodic-nearest centre for each grid point (src/PFCInit.java:68-93)."""
    W, H = Nx * dx, Ny * dy
    xs = np.arange(Nx) * dx
    ys = np.arange(Ny) * dy
    best = np.full((Ny, Nx), np.inf)
    lab = np.zeros((Ny, Nx), dtype=np.int64)
    for n in range(len(cx)):
        ddx = xs[None, :] - cx[n]
        ddx = np.where(ddx > 0.5 * W, ddx - W, np.where(ddx < -0.5 * W, ddx + W, ddx))
        ddy = ys[:, None] - cy[n]
        ddy = np.where(ddy > 0.5 * H, ddy - H, np.where(ddy < -0.5 * H, ddy + H, ddy))
        d2 = ddx * ddx + ddy * ddy
        closer = d2 < best
        best = np.where(closer, d2, best)
        lab = np.where(closer, n, lab)
    return lab


def polycrystal(Nx: int, Ny: int, dx: float, dy: float, grains: int, mean: float, amp: float,
                noise: float, seed: int, a: float = A_TRI, sym: int = 3,
                max_angle_deg: float = 60.0) -> np.ndarray:
    """Voronoi polycrystal: each grain is mean + amp * OMA(rotated r) with a
    uniform orientation in [0, max_angle), plus noise * N(0, 1). Shape (Ny, Nx)."""
    u = uniform(seed, 3 * grains, stream=1)
    cx = u[0::3] * Nx * dx
    cy = u[1::3] * Ny * dy
    theta = u[2::3] * math.radians(max_angle_deg)
    lab = voronoi_labels(Nx, Ny, dx, dy, cx, cy)
    X = np.broadcast_to(np.arange(Nx)[None, :] * dx, (Ny, Nx))
    Y = np.broadcast_to(np.arange(Ny)[:, None] * dy, (Ny, Nx))
    out = np.empty((Ny, Nx))
    for n in range(grains):
        sel = lab == n
        c, s = math.cos(-theta[n]), math.sin(-theta[n])
        xr = X[sel] * c - Y[sel] * s
        yr = X[sel] * s + Y[sel] * c
        out[sel] = mean + amp * oma(xr, yr, sym, a)
    if noise:
        out += noise * normal(seed, Nx * Ny, stream=2).reshape(Ny, Nx)
    return out


def stripes2(Nx: int, Ny: int, dx: float, dy: float, width: int, means: tuple, amps: tuple,
             lattice: tuple, noise: float, seed: int) -> np.ndarray:
    """Two-component lateral heterostructure: alternating vertical stripes of
    ``width`` grid columns; in the stripes of phase u field u carries
    means[u] + amps[u] * OMA(r; a = lattice[u]) and the other field sits at its
    disordered mean. Returns shape (2, Ny, Nx)."""
    X = np.broadcast_to(np.arange(Nx)[None, :] * dx, (Ny, Nx))
    Y = np.broadcast_to(np.arange(Ny)[:, None] * dy, (Ny, Nx))
    phase = (np.arange(Nx)[None, :] // width) % 2
    phase = np.broadcast_to(phase, (Ny, Nx))
    out = np.empty((2, Ny, Nx))
    for u in range(2):
        lat = means[u] + amps[u] * oma(X, Y, 3, lattice[u])
        out[u] = np.where(phase == u, lat, means[u])
        if noise:
            out[u] += noise * normal(seed, Nx * Ny, stream=3 + u).reshape(Ny, Nx)
    return out


def hetero2(Nx: int, Ny: int, dx: float, dy: float, grains: int, width: int, offset: int, means: tuple,
            amps: tuple, lattice: tuple, noise: float, seed: int, sym: int = 3,
            max_angle_deg: float = 60.0) -> np.ndarray:
    """Two-field heterostructure: each region belongs to one field, which carries
    means[u] + amps[u] * OMA(r rotated by the region's angle, sym, lattice[u])
    there, while the other field sits at its mean; noise * N(0, 1) is added to
    both (streams 3 and 4). grains > 0: periodic Voronoi grains whose centre,
    angle in [0, max_angle_deg) and field come from uniforms 4k..4k+3 of stream 1;
    grains <= 0: vertical stripes, field ((x + offset) // width) % 2, unrotated.
    With grains = 0 and offset = 0 this is stripes2. The device generator
    pfcg_init_hetero computes the same values. Shape (2, Ny, Nx)."""
    X = np.broadcast_to(np.arange(Nx)[None, :] * dx, (Ny, Nx))
    Y = np.broadcast_to(np.arange(Ny)[:, None] * dy, (Ny, Nx))
    if grains <= 0:
        phase = np.broadcast_to(((np.arange(Nx)[None, :] + offset) // width) % 2, (Ny, Nx))
        XR, YR = X, Y
    else:
        u = uniform(seed, 4 * grains, stream=1)
        cx = u[0::4] * Nx * dx
        cy = u[1::4] * Ny * dy
        theta = u[2::4] * math.radians(max_angle_deg)
        field = (u[3::4] >= 0.5).astype(np.int64)
        lab = voronoi_labels(Nx, Ny, dx, dy, cx, cy)
        phase = field[lab]
        XR = np.empty((Ny, Nx))
        YR = np.empty((Ny, Nx))
        for n in range(grains):
            sel = lab == n
            c, s = math.cos(-theta[n]), math.sin(-theta[n])
            XR[sel] = X[sel] * c - Y[sel] * s
            YR[sel] = X[sel] * s + Y[sel] * c
    out = np.empty((2, Ny, Nx))
    for f in range(2):
        lat = means[f] + amps[f] * oma(XR, YR, sym, lattice[f])
        out[f] = np.where(phase == f, lat, means[f])
        if noise:
            out[f] += noise * normal(seed, Nx * Ny, stream=3 + f).reshape(Ny, Nx)
    return out
