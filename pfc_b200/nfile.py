"""Readers and writers for pfc-relax's text files.

``.n`` / ``.f`` data files (pfc-relax.c:767-859 write_data / write_energy):
a header line ``"%d %d %.*lf %.*lf\\n"`` = Nx Ny dx dy at ``pwrite`` decimals,
then Nx*Ny values ``"%.*e\\n"`` in y-major order (j outer, i inner). Reading is
whitespace tolerant like the reference's fscanf (pfc-relax.c:747-752).

``.in`` parameter files (pfc-relax.c:414-726): labels I, M, R; see
``write_input``. This module is the host-side convenience layer used by the
tests and the benchmark; the drop-in ``pfc-relax`` executable has its own C
parser (pfc_b200/csrc/pfc_relax_main.c).
"""
from __future__ import annotations

import io
import os

import numpy as np


def format_n(field: np.ndarray, dx: float, dy: float, pwrite: int) -> str:
    """Text of a .n file, byte-identical to the reference's fprintf output."""
    Ny, Nx = field.shape
    out = io.StringIO()
    out.write("%d %d %.*f %.*f\n" % (Nx, Ny, pwrite, dx, pwrite, dy))
    fmt = "%.{}e\n".format(pwrite)
    out.write("".join(fmt % v for v in field.ravel()))
    return out.getvalue()


def write_n(path: str, field: np.ndarray, dx: float, dy: float, pwrite: int = 12) -> None:
    with open(path, "w") as f:
        f.write(format_n(np.asarray(field, dtype=np.float64), dx, dy, pwrite))


def write_n_header_only(path: str, Nx: int, Ny: int, dx: float, dy: float) -> None:
    """A .n file with only its header: enough for read_input (pfc-relax.c:463-470)."""
    with open(path, "w") as f:
        f.write("%d %d %.6f %.6f\n" % (Nx, Ny, dx, dy))


def read_n(path: str):
    """Returns (field (Ny, Nx) float64, dx, dy)."""
    with open(path) as f:
        toks = f.read().split()
    Nx, Ny = int(toks[0]), int(toks[1])
    dx, dy = float(toks[2]), float(toks[3])
    vals = np.array(toks[4:4 + Nx * Ny], dtype=np.float64)
    if vals.size != Nx * Ny:
        raise ValueError("%s: expected %d values, found %d" % (path, Nx * Ny, vals.size))
    return vals.reshape(Ny, Nx), dx, dy


def _row(vals):
    return "\t".join(repr(float(v)) for v in vals)


def write_input(path: str, innames, outnames, fname=None, *, Tprint: int, Twrite=None, twrite=None,
                pprint: int = 12, pwrite: int = 12, params: dict, c: float, tend: int, dx: float,
                dy: float, dt: float, Topt: int = 0, xopt: int = 1, yopt: int = 1) -> None:
    """Writes a pfc-relax .in file. ``params`` holds the input-file values:
    lambda (U), alpha/beta/gamma (UxU upper triangle), delta (U), epsilon (UxU,
    strict upper), sigma, inv_nu / omega / phi (U lists of W[u]), inv_mu (UxU,
    strict upper) — reciprocal lengths exactly as the file stores them."""
    U = len(innames)
    lines = ["# generated input for pfc-relax", "I\t" + "\t".join(innames)]
    outs = list(outnames) + ([fname] if fname else [])
    lines.append("\t" + "\t".join(outs))
    if twrite is not None:
        lines.append("\t%d\t[\t%s\t]\t%d\t%d" % (Tprint, "\t".join(str(t) for t in twrite), pprint, pwrite))
    else:
        lines.append("\t%d\t%d\t%d\t%d" % (Tprint, Twrite, pprint, pwrite))
    lines.append("M\t%d" % U)
    lines.append("l\t" + "\n\t".join(repr(float(v)) for v in params["lambda"]))
    for lab, key in (("a", "alpha"), ("b", "beta"), ("g", "gamma")):
        rows = [_row(params[key][u][u:]) for u in range(U)]
        lines.append(lab + "\t" + "\n\t".join(rows))
    lines.append("d\t" + "\n\t".join(repr(float(v)) for v in params["delta"]))
    erows = [_row(params["epsilon"][u][u + 1:]) for u in range(U - 1)]
    lines.append("e\t" + "\n\t".join(erows) if erows else "e\t")
    lines.append("s\t%r" % float(params["sigma"]))
    for lab, key in (("n", "inv_nu"), ("o", "omega"), ("p", "phi")):
        rows = [_row(params[key][u]) for u in range(U)]
        lines.append(lab + "\t" + "\n\t".join(rows))
    mrows = [_row(params["inv_mu"][u][u + 1:]) for u in range(U - 1)]
    lines.append("m\t" + "\n\t".join(mrows) if mrows else "m\t")
    lines.append("R\t%r\t%d\t%r\t%r\t%r\t%d\t%d\t%d" % (float(c), tend, float(dx), float(dy), float(dt), Topt, xopt, yopt))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def out_path(input_path: str) -> str:
    """Log file name: the input name with ".in" replaced by ".out", else ".out" appended (pfc-relax.c:888-893)."""
    base = input_path[:-3] if input_path.endswith(".in") else input_path
    return base + ".out"


def read_out(path: str):
    """Parses a .out log: rows of t, seconds, dx, dy, <f>, <n_0> .. <n_{U-1}>."""
    rows = []
    with open(path) as f:
        for line in f:
            if line.strip():
                rows.append([float(v) for v in line.split()])
    return np.array(rows)
