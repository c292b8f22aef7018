"""The initial-state builder pieces rebuilt from the reference's pfc-init
(src/PFCInit.java): the Voronoi step on the GPU (pfcg_init_voronoi), the
Java-format output writer (pfcg_write_n_pfcinit) and the pfc-init tool, checked
against oracle/pfcinit_oracle.py (a plain restatement of the Java code, with
java.util.Random as its API documentation specifies it)."""
import math
import os
import subprocess

import numpy as np
import pytest

import pfcinit_oracle as J
from pfc_b200 import lib, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOOL = os.path.join(ROOT, "pfc_b200", "pfc-init")


def test_java_format_restatement_known_cases():
    """Formatter rounds the shortest digits half up; C's printf would give
    1.2e-01, 2e+00 and 1.000e+00 for the first three."""
    assert J.java_e(0.125, 1) == "1.3e-01"
    assert J.java_e(2.5, 0) == "3e+00"
    assert J.java_e(1.0005, 3) == "1.001e+00"
    assert J.java_e(-0.0, 3) == "-0.000e+00"
    assert J.java_e(0.0, 2) == "0.00e+00"
    assert J.java_e(1e100, 2) == "1.00e+100"
    assert J.java_e(9.9996, 3) == "1.000e+01"
    assert J.java_e(float("nan"), 3) == "NaN" and J.java_e(-float("inf"), 3) == "-Infinity"
    assert J.java_e(0.7, 6) == "7.000000e-01"


def test_java_random_restatement():
    """new Random(42).nextDouble() and new Random(0).nextDouble() as the JVM gives them."""
    assert J.JavaRandom(42).next_double() == 0.7275636800328681
    assert J.JavaRandom(0).next_double() == 0.730967787376657
    L = lib.load()
    for s in (0, 42, 12345, -7, 2 ** 31 - 1):
        assert L.pfcg_java_random_seed(s) == J.JavaRandom(s).state


def _values():
    rng = np.random.default_rng(5)
    v = list(rng.standard_normal(3000) * 0.3) + list(10.0 ** rng.uniform(-300, 300, 500) * rng.choice([-1, 1], 500))
    # shortest digits that end in a 5 one place past the printed ones (Java and C round them differently)
    v += [0.125, 2.5, 1.0005, 0.0005, 1.25, -3.5, 4.45, 0.15, 1.0000005, 7.5e-8, 9.9996, 99.995, 0.7, -0.0, 0.0]
    return np.array(v, dtype=np.float64)


@pytest.mark.parametrize("prec", [0, 1, 3, 6, 12, 13])
def test_writer_matches_java_format(tmp_path, prec):
    """The bytes of pfcg_write_n_pfcinit against the restatement of the Java writer."""
    v = _values()
    Nx = 59
    Ny = len(v) // Nx
    f = np.ascontiguousarray(v[: Nx * Ny].reshape(Ny, Nx))
    a, b = str(tmp_path / "a.n"), str(tmp_path / "b.n")
    rc = lib.load().pfcg_write_n_pfcinit(a.encode(), Nx, Ny, 0.7, 0.125, lib._dptr(f), prec)
    assert rc == 0
    J.write_n(b, f, 0.7, 0.125, prec)
    assert open(a, "rb").read() == open(b, "rb").read()


def test_tool_load_transform_output(tmp_path):
    """pfc-init's L, T and O steps (no GPU work) against the restatement."""
    rng = np.random.default_rng(3)
    src = rng.standard_normal((12, 10))
    with open(tmp_path / "src.n", "w") as fh:
        fh.write("10 12 0.5 0.5\n")
        for x in src.ravel():
            fh.write("%.17e\n" % x)
    (tmp_path / "x.in").write_text(
        "# dims\nD\n\t16\t14\t0.5\t0.5\n\n# load\nL\tsrc.n\t0\n-3\t2\t7\t9\t5\t-1\n"
        "L\tsrc.n\t1\n0\t0\t10\t12\t0\t0\nT\t-0.25\t0.5\nO\tout.n\t6\n")
    r = subprocess.run([TOOL, "x.in"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    arr = np.zeros((14, 16))
    for (i0, j0, dNx, dNy, i1, j1, t) in ((-3, 2, 7, 9, 5, -1, 0), (0, 0, 10, 12, 0, 0, 1)):
        i0, j0, i1, j1 = i0 % 10, j0 % 12, i1 % 16, j1 % 14
        for j in range(dNy):
            for i in range(dNx):
                arr[(j1 + j) % 14, (i1 + i) % 16] = t * arr[(j1 + j) % 14, (i1 + i) % 16] + src[(j0 + j) % 12,
                                                                                                 (i0 + i) % 10]
    nave0 = 0.0
    for x in arr.ravel():
        nave0 += x
    nave0 *= 1.0 / 16 / 14
    arr = (arr - nave0) * 0.5 + -0.25
    J.write_n(str(tmp_path / "ref.n"), arr, 0.5, 0.5, 6)
    assert (tmp_path / "out.n").read_bytes() == (tmp_path / "ref.n").read_bytes()


def test_tool_errors():
    """Unknown labels and bad numbers stop with the reference's messages and exit code 1."""
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        for text, msg in (("D 8 8 0.7 0.7\nQ\n", 'Label expected instead of "Q"'),
                          ("D 8 x 0.7 0.7\n", 'Integer expected instead of "x"'),
                          ("D 8 8 0.7 z\n", 'Decimal number expected instead of "z"')):
            with open(os.path.join(d, "x.in"), "w") as fh:
                fh.write(text)
            r = subprocess.run([TOOL, "x.in"], cwd=d, capture_output=True, text=True)
            assert r.returncode == 1 and msg in r.stdout, (text, r.stdout)


def _grains():
    g = []
    rows = [(3.0, 5.0, 0, 3, 7.2552, 0.2, 0.5, 0.05, 0.0, 0.0, 12.0, 0.0, 0.0, 0.0, 0.0),
            (20.0, 4.0, 0, 6, 7.2552, -0.3, 1.0, 0.0, 1.5, -2.0, 33.0, 4.0, 5.0, 0.5, 0.25),
            (12.0, 20.0, 1, 4, 6.0, 0.1, 0.3, 0.1, 0.0, 0.0, -20.0, 10.0, 10.0, 0.0, 0.0),
            (-5.0, 30.0, 2, 3, 7.2552, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0),
            (31.0, 25.0, 0, 3, 8.1, 0.25, -0.4, 0.02, 0.3, 0.0, 59.0, 0.0, 0.0, 1.0, 2.0),
            (40.5, 1.0, 1, 6, 7.0, 0.0, 0.2, 0.0, 0.0, 0.0, 5.0, 0.0, 0.0, 0.0, 0.0)]
    keys = ("x", "y", "type", "sym", "a", "nave", "amp", "namp", "tx1", "ty1", "theta", "xr", "yr", "tx2", "ty2")
    for r in rows:
        g.append(dict(zip(keys, r)))
    return g


def _c_grains(gs):
    arr = (lib.Grain * len(gs))()
    for k, g in enumerate(gs):
        arr[k] = lib.Grain(g["x"], g["y"], g["type"], g["sym"], g["a"], g["nave"], g["amp"], g["namp"], g["tx1"],
                           g["ty1"], g["theta"], g["xr"], g["yr"], g["tx2"], g["ty2"])
    return arr


@pytest.mark.gpu
def test_voronoi_step_matches_java_restatement():
    """Two V steps in a row (the second superposes and continues the random
    sequence) on host memory, against the restatement point by point."""
    Nx, Ny, dx, dy = 48, 40, 0.9, 0.8
    gs = _grains()
    field = np.ascontiguousarray(np.full((Ny, Nx), 0.05))
    expect = field.copy()
    jr = J.JavaRandom(12345)
    state = lib.ctypes.c_longlong(lib.load().pfcg_java_random_seed(12345))
    for step in range(2):
        sub = gs if step == 0 else [dict(g, type=1 if g["type"] == 0 else g["type"]) for g in gs]
        rc = lib.load().pfcg_init_voronoi(lib._dptr(field), Nx, Ny, dx, dy, len(sub), _c_grains(sub),
                                          lib.ctypes.byref(state), None)
        assert rc == 0, lib.load().pfcg_init_last_error()
        J.voronoi_step(expect, dx, dy, sub, jr)
        assert np.abs(field - expect).max() < 1e-12
        assert state.value == jr.state


@pytest.mark.gpu
def test_voronoi_step_on_device_matches_polycrystal():
    """C2's single-field polycrystal state (32 grains, triangular one-mode
    lattice, orientations in [0, 60)) built by the V step on device memory
    equals synth.polycrystal's numpy construction without noise."""
    import torch

    N, dx = 256, math.pi / 4
    u = synth.uniform(0, 3 * 32, stream=1)
    gs = [dict(x=u[3 * k] * N * dx, y=u[3 * k + 1] * N * dx, type=0, sym=3, a=synth.A_TRI, nave=0.25, amp=-0.4,
               namp=0.0, tx1=0.0, ty1=0.0, theta=u[3 * k + 2] * 60.0, xr=0.0, yr=0.0, tx2=0.0, ty2=0.0)
          for k in range(32)]
    dev = torch.zeros((N, N), dtype=torch.float64, device="cuda")
    state = lib.ctypes.c_longlong(lib.load().pfcg_java_random_seed(1))
    torch.cuda.synchronize()
    rc = lib.load().pfcg_init_voronoi(dev.data_ptr(), N, N, dx, dx, 32, _c_grains(gs), lib.ctypes.byref(state), None)
    assert rc == 0, lib.load().pfcg_init_last_error()
    ref = synth.polycrystal(N, N, dx, dx, 32, 0.25, -0.4, 0.0, 0)
    assert np.abs(dev.cpu().numpy() - ref).max() < 1e-12


@pytest.mark.gpu
def test_tool_voronoi(tmp_path):
    """pfc-init with S, V (GPU), T and O against the restatement: same header
    bytes, same values to 1e-12 before formatting."""
    gs = _grains()
    lines = ["D", "48 40 0.9 0.8", "S 777", "V %d" % len(gs)]
    for g in gs:
        lines.append(" ".join(repr(float(g[k])) if k not in ("type", "sym") else str(g[k])
                              for k in ("x", "y", "type", "sym", "a", "nave", "amp", "namp", "tx1", "ty1", "theta",
                                        "xr", "yr", "tx2", "ty2")))
    lines += ["T 0.1 2.0", "O out.n 14"]
    (tmp_path / "x.in").write_text("\n".join(lines) + "\n")
    r = subprocess.run([TOOL, "x.in"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    arr = J.voronoi_step(np.zeros((40, 48)), 0.9, 0.8, gs, J.JavaRandom(777))
    nave0 = 0.0
    for x in arr.ravel():
        nave0 += x
    nave0 *= 1.0 / 48 / 40
    arr = (arr - nave0) * 2.0 + 0.1
    text = (tmp_path / "out.n").read_text().split("\n")
    assert text[0] == "48 40 %s %s" % (J.java_e(0.9, 14), J.java_e(0.8, 14))
    got = np.array([float(x) for x in text[1:] if x])
    assert got.shape == (48 * 40,) and np.abs(got - arr.ravel()).max() < 1e-12
