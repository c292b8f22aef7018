"""Generates the golden fixtures in this directory by running the reference
solver (demos/honey/pfc-relax.c compiled unchanged over the project's
FFTW/MPI shim: oracle/_ref/pfc-relax and, for beta_uv != 0, the same source
with the mu2 line of evaluate() corrected: oracle/_ref/pfc-relax-mu2fix).

Each case writes seeded synthetic input fields to .n files at 17 significant
digits (exact round trip), a .in file, runs the binary and stores the inputs,
the parameters, the .out rows and the final fields in <case>.npz.

Needs the reference tree (to build oracle/_ref with `make -C oracle ref`);
run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from pfc_b200 import nfile, synth  # noqa: E402
from pfc_b200 import params as P  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(ROOT, "oracle", "_ref")


def hetero_3c():
    """The reference's three-field heterostructure demo parameters
    (demos/hetero/hetero.in:20-63), beta_12 = 0.02 with 1/mu_12 = 1.018."""
    U = 3
    z = lambda: [[0.0] * U for _ in range(U)]  # noqa: E731
    a, b, g, e, m = z(), z(), z(), z(), z()
    a[0] = [-1.4, -0.04, -0.04]; a[1][1:] = [-0.3, 0.5]; a[2][2] = -0.3
    b[0][0] = 2.25; b[1][1:] = [1.0, 0.02]; b[2][2] = 1.0
    g[1][2] = 0.3
    e[0][1:] = [-0.8, -0.8]
    m[1][2] = 1.018
    return {"lambda": [0.0] * 3, "alpha": a, "beta": b, "gamma": g, "delta": [2.25, 1.0, 1.0], "epsilon": e,
            "sigma": 0.2, "inv_nu": [[1.0], [1.018], [1.018]], "omega": [[1.0]] * 3, "phi": [[0.0]] * 3,
            "inv_mu": m}


def two_mode():
    """Single field with a two-mode operator (square-lattice style): 1/nu = 1, sqrt(2)."""
    d = P.honeycomb_1c(-0.2)
    d["inv_nu"] = [[1.0, 2.0 ** 0.5]]
    d["omega"] = [[1.0, 1.0]]
    d["phi"] = [[0.0, 0.05]]
    d["gamma"] = [[0.1]]
    return d


def honey_nc():
    """demos/honey/honey.in:19-57: alpha -0.15, beta 1, gamma 0.8, delta 1, nonconserved."""
    d = P.honeycomb_1c(-0.15)
    d["gamma"] = [[0.8]]
    return d


CASES = [
    # name, params, Nx, Ny, dx, dy, dt, c, tend, Tprint, Topt, state, binary
    dict(name="c1_noise_32", params=P.honeycomb_1c(-0.25), Nx=32, Ny=32, dx=np.pi / 4, dy=np.pi / 4, dt=1.0, c=1.0,
         tend=200, Tprint=50, Topt=0, state=("noise", 0.25, 0.05, 0), binary="pfc-relax"),
    dict(name="honey_nc_48x32", params=honey_nc(), Nx=48, Ny=32, dx=0.7, dy=0.7, dt=0.5, c=0.0,
         tend=150, Tprint=50, Topt=0, state=("noise", 0.06, 0.2, 1), binary="pfc-relax"),
    dict(name="hetero2_opt_48", params=P.hetero_2c(0.04), Nx=48, Ny=48, dx=0.7, dy=0.7, dt=0.25, c=1.0,
         tend=300, Tprint=50, Topt=100, state=("stripes", 12, (0.3, -0.3), (0.3, 0.3), 0.02, 5), binary="pfc-relax"),
    dict(name="hetero3_mu_32", params=hetero_3c(), Nx=32, Ny=32, dx=0.7, dy=0.7, dt=0.25, c=1.0,
         tend=120, Tprint=40, Topt=0, state=("noise3", (0.485, -0.32, -0.32), 0.1, 7), binary="pfc-relax-mu2fix"),
    dict(name="twomode_40", params=two_mode(), Nx=40, Ny=40, dx=0.8, dy=0.8, dt=0.5, c=0.0,
         tend=100, Tprint=25, Topt=0, state=("noise", -0.1, 0.1, 3), binary="pfc-relax"),
    dict(name="mixed_48x40_opt", params=P.honeycomb_1c(-0.25), Nx=48, Ny=40, dx=0.78, dy=0.8, dt=1.0, c=1.0,
         tend=200, Tprint=50, Topt=50, state=("noise", 0.25, 0.05, 11), binary="pfc-relax"),
]


def make_state(spec, Nx, Ny, dx, dy, U):
    kind = spec[0]
    if kind == "noise":
        _, mean, amp, seed = spec
        return synth.noise_state(Nx, Ny, mean, amp, seed)[None]
    if kind == "noise3":
        _, means, amp, seed = spec
        return np.array([synth.noise_state(Nx, Ny, means[u], amp, seed, stream=u) for u in range(U)])
    if kind == "stripes":
        _, width, means, amps, noise, seed = spec
        return synth.stripes2(Nx, Ny, dx, dy, width, means, amps, (7.2552, 7.2552 * 1.04), noise, seed)
    raise ValueError(kind)


def run_case(cs):
    pd = cs["params"]
    U = len(pd["lambda"])
    Nx, Ny, dx, dy = cs["Nx"], cs["Ny"], cs["dx"], cs["dy"]
    fields = make_state(cs["state"], Nx, Ny, dx, dy, U)
    with tempfile.TemporaryDirectory() as d:
        ins = ["in%d.n" % u for u in range(U)]
        outs = ["out%d-#.n" % u for u in range(U)]
        for u in range(U):
            nfile.write_n(os.path.join(d, ins[u]), fields[u], dx, dy, 17)
        # exact round trip of the inputs
        fields = np.array([nfile.read_n(os.path.join(d, ins[u]))[0] for u in range(U)])
        tend = cs["tend"]
        nfile.write_input(os.path.join(d, "x.in"), ins, outs, "f-#.f", Tprint=cs["Tprint"], twrite=[0, tend],
                          pprint=17, pwrite=17, params=pd, c=cs["c"], tend=tend, dx=dx, dy=dy, dt=cs["dt"],
                          Topt=cs["Topt"], xopt=1, yopt=1)
        r = subprocess.run([os.path.join(REF, cs["binary"]), "x.in"], cwd=d, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("%s failed: %s %s" % (cs["name"], r.stdout, r.stderr))
        rows = nfile.read_out(os.path.join(d, "x.out"))
        final = np.array([nfile.read_n(os.path.join(d, "out%d-%d.n" % (u, tend)))[0] for u in range(U)])
        f_final = nfile.read_n(os.path.join(d, "f-%d.f" % tend))[0]
        _, dxo, dyo = nfile.read_n(os.path.join(d, "out0-%d.n" % tend))
    meta = {k: v for k, v in cs.items() if k not in ("state",)}
    meta["state"] = list(map(str, cs["state"]))
    np.savez_compressed(os.path.join(HERE, cs["name"] + ".npz"), fields=fields, rows=rows, final=final,
                        f_final=f_final, box_final=np.array([dxo, dyo]), meta=json.dumps(meta))
    print("%-18s U=%d %dx%d rows=%d <f>_end=%.15g" % (cs["name"], U, Nx, Ny, len(rows), rows[-1][4]))


def main():
    for b in ("pfc-relax", "pfc-relax-mu2fix"):
        if not os.path.exists(os.path.join(REF, b)):
            raise SystemExit("build the reference first: make -C oracle ref")
    for cs in CASES:
        run_case(cs)


if __name__ == "__main__":
    main()
