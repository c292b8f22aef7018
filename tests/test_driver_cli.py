"""The drop-in pfc-relax driver against the reference binary: the .in grammar,
error messages and exit codes (CPU: the driver stops after parsing when
PFC_B200_CHECK_ONLY=1), and whole runs on the GPU (marked gpu)."""
import os
import subprocess

import numpy as np
import pytest

from pfc_b200 import lib, nfile, synth
from pfc_b200 import params as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "pfc-relax")
DRV = lib.DRIVER_PATH

GOOD_1C = """# a comment line
I\tin0.n
\tout0-#.n\tf-#.f
\t10\t[\t0\t20\t]\t12\t6
M\t1
l\t0.0
a\t-0.25
b\t1.0
g\t0.0
d\t1.0
e\t
s\t0.2
n\t1.0
o\t1.0
p\t0.0
m\t
R\t1\t20\t0.785\t0.785\t1.0\t0\t1\t1
"""


def run(binary, cwd, args=("x.in",), env_extra=None):
    env = dict(os.environ)
    env["PFC_B200_CHECK_ONLY"] = "1"
    if env_extra:
        env.update(env_extra)
    r = subprocess.run([binary] + list(args), cwd=cwd, capture_output=True, text=True, env=env, timeout=120)
    return r.returncode, r.stdout


def setup_case(tmp_path, text, data=True, Nx=16, Ny=16, header=None, values=None):
    (tmp_path / "x.in").write_text(text)
    if data:
        f = synth.noise_state(Nx, Ny, 0.25, 0.05, 1)
        body = header if header is not None else "%d %d 0.785 0.785\n" % (Nx, Ny)
        vals = values if values is not None else "".join("%.12e\n" % v for v in f.ravel())
        (tmp_path / "in0.n").write_text(body + vals)


def mutate(old, new):
    assert old in GOOD_1C
    return GOOD_1C.replace(old, new)


CASES = [
    ("missing_input", None, 0),
    ("multichar", "XY\n" + GOOD_1C, 1),
    ("missing_data_file", mutate("I\tin0.n", "I\tnope.n"), 3),
    ("bad_outputs", mutate("\tout0-#.n\tf-#.f", "\ta\tb\tc"), 6),
    ("bad_write_params", mutate("\t10\t[\t0\t20\t]\t12\t6", "\t10\t20\t12\t6\t7"), 9),
    ("write_steps_not_increasing", mutate("[\t0\t20\t]", "[\t20\t0\t]"), 10),
    ("write_no_bracket", mutate("[\t0\t20\t]", "(\t0\t20\t]"), 9),
    ("field_count", mutate("M\t1", "M\t2"), 12),
    ("no_omega_label", mutate("o\t1.0\n", ""), 29),
    ("bad_lambda", mutate("l\t0.0", "l\tzero"), 14),
    ("bad_relax_line", mutate("R\t1\t20\t0.785\t0.785\t1.0\t0\t1\t1", "R\t1\t20\t0.785"), 35),
    ("unknown_label", GOOD_1C + "Z\n", 36),
]


@pytest.mark.parametrize("name,text,code", CASES)
def test_error_codes_match_reference(tmp_path, name, text, code):
    if text is not None:
        setup_case(tmp_path, text)
    got = run(DRV, tmp_path)
    ref = run(REF, tmp_path)
    assert ref[0] == code, (name, ref)
    assert got == ref, (name, got, ref)


@pytest.mark.parametrize("name,header,values,code", [
    ("bad_header", "16 x 0.785 0.785\n", None, 4),
    ("three_number_header", "16 16 0.785\n", None, 38),
    ("bad_value", None, "0.1\n" * 100 + "abc\n", 38),
    ("short_file", None, "0.1\n" * 100, 38),
])
def test_data_file_errors_match_reference(tmp_path, name, header, values, code):
    setup_case(tmp_path, GOOD_1C, header=header, values=values)
    got = run(DRV, tmp_path)
    ref = run(REF, tmp_path)
    assert ref[0] == code, (name, ref)
    assert got == ref, (name, got, ref)


def test_mismatched_dimensions(tmp_path):
    text = mutate("I\tin0.n", "I\tin0.n\tin1.n").replace("\tout0-#.n\tf-#.f", "\tout0-#.n\tout1-#.n")
    setup_case(tmp_path, text)
    (tmp_path / "in1.n").write_text("8 8 0.7 0.7\n" + "0.1\n" * 64)
    got = run(DRV, tmp_path)
    ref = run(REF, tmp_path)
    assert ref[0] == 5 and got == ref


def test_bad_argument_count(tmp_path):
    got = run(DRV, tmp_path, args=("a.in", "b.in"))
    ref = run(REF, tmp_path, args=("a.in", "b.in"))
    assert ref[0] == 41 and got == ref


def test_valid_input_parses(tmp_path):
    setup_case(tmp_path, GOOD_1C)
    code, out = run(DRV, tmp_path)
    assert code == 0 and out.startswith("ok U=1 Nx=16 Ny=16 tend=20 Tprint=10 nwrite=2")


def full_case(d, precision_env=None):
    pd = P.hetero_2c(0.04)
    Nx = Ny = 48
    dx = dy = 0.7
    f = synth.stripes2(Nx, Ny, dx, dy, 12, (0.3, -0.3), (0.3, 0.3), (7.2552, 7.2552 * 1.04), 0.02, 5)
    for u in range(2):
        nfile.write_n(os.path.join(d, "in%d.n" % u), f[u], dx, dy, 17)
    nfile.write_input(os.path.join(d, "case.in"), ["in0.n", "in1.n"], ["a-#.n0", "a-#.n1"], "a-#.f", Tprint=25,
                      twrite=[0, 30, 100, 150], pprint=12, pwrite=12, params=pd, c=1.0, tend=150, dx=dx, dy=dy,
                      dt=0.25, Topt=50, xopt=1, yopt=1)


@pytest.mark.gpu
def test_full_run_matches_reference(tmp_path):
    """Both binaries on the same input: the .out rows (t, dx, dy, <f>, <n_u>;
    the wall-seconds column aside), the names, headers and values of every
    written .n and .f file. The .f at t = 30 is the f(r) of the last evaluate
    (t = 25), as the reference writes it."""
    dirs = {}
    for name, exe in (("ref", REF), ("gpu", DRV)):
        d = tmp_path / name
        d.mkdir()
        full_case(str(d))
        env = dict(os.environ)
        env.pop("PFC_B200_CHECK_ONLY", None)
        r = subprocess.run([exe, "case.in"], cwd=d, capture_output=True, text=True, env=env, timeout=600)
        assert r.returncode == 0, (name, r.stdout, r.stderr)
        dirs[name] = d
    ro = nfile.read_out(str(dirs["ref"] / "case.out"))
    go = nfile.read_out(str(dirs["gpu"] / "case.out"))
    assert ro.shape == go.shape
    np.testing.assert_allclose(go[:, 0], ro[:, 0])
    np.testing.assert_allclose(go[:, 2:], ro[:, 2:], rtol=1e-9, atol=1e-12)
    names = sorted(p.name for p in dirs["ref"].iterdir() if p.suffix in (".n0", ".n1", ".f"))
    assert names == sorted(p.name for p in dirs["gpu"].iterdir() if p.suffix in (".n0", ".n1", ".f"))
    assert len(names) == 12
    for n in names:
        rt = (dirs["ref"] / n).read_text().splitlines()
        gt = (dirs["gpu"] / n).read_text().splitlines()
        assert len(rt) == len(gt) == 48 * 48 + 1
        rh, gh = rt[0].split(), gt[0].split()
        assert rh[:2] == gh[:2]
        np.testing.assert_allclose([float(x) for x in gh[2:]], [float(x) for x in rh[2:]], rtol=1e-9)
        np.testing.assert_allclose(np.array(gt[1:], float), np.array(rt[1:], float), rtol=0, atol=1e-8, err_msg=n)
        # number formatting: "%.12e" lines
        assert all(len(line.split("e")[0].split(".")[1]) == 12 for line in gt[1:50])


def big_case(tmp_path, Nx, Ny, prec, values_text):
    text = GOOD_1C.replace("\t10\t[\t0\t20\t]\t12\t6", "\t10\t[\t0\t20\t]\t12\t%d" % prec)
    (tmp_path / "x.in").write_text(text)
    (tmp_path / "in0.n").write_text("%d %d 0.785 0.785\n" % (Nx, Ny) + values_text)


@pytest.mark.parametrize("threads,prec", [(1, 6), (4, 6), (7, 17), (3, 1)])
def test_parallel_io_is_byte_identical_to_printf(tmp_path, threads, prec):
    """The multithreaded .n parser and writer give the bytes of one strtod and
    one fprintf("%.*e\\n") per value, for any thread count (values of every
    magnitude and sign, including zeros and subnormals)."""
    Nx, Ny = 96, 80
    rng = np.random.default_rng(threads * 100 + prec)
    v = rng.normal(size=Nx * Ny) * 10.0 ** rng.integers(-30, 30, size=Nx * Ny)
    v[:5] = [0.0, -0.0, 5e-324, -2.2250738585072014e-308, 1.7976931348623157e308]
    # irregular whitespace between values, as fscanf(" %lf") accepts
    seps = ["\n", " ", "\t", "  \n "]
    body = "".join("%.17g%s" % (x, seps[i % 4]) for i, x in enumerate(v))
    big_case(tmp_path, Nx, Ny, prec, body)
    code, out = run(DRV, tmp_path, env_extra={"PFC_B200_CHECK_ONLY": "2", "OMP_NUM_THREADS": str(threads)})
    assert code == 0, out
    parsed = np.array([float(t) for t in body.split()])
    want = "%d %d %.*f %.*f\n" % (Nx, Ny, prec, 0.785, prec, 0.785) + "".join("%.*e\n" % (prec, x) for x in parsed)
    assert (tmp_path / "in0.n.check").read_text() == want


@pytest.mark.parametrize("threads", [1, 5])
def test_parallel_parse_errors_follow_the_reference(tmp_path, threads):
    """A bad token among the first Nx*Ny values is error 38 (the reference's
    fscanf failure); values and garbage after the first Nx*Ny are never read."""
    Nx, Ny = 64, 64
    vals = ["%.12e" % x for x in synth.noise_state(Nx, Ny, 0.25, 0.05, 3).ravel()]
    env = {"OMP_NUM_THREADS": str(threads)}
    bad = list(vals)
    bad[3000] = "x1.0"
    big_case(tmp_path, Nx, Ny, 6, "\n".join(bad) + "\n")
    assert run(DRV, tmp_path, env_extra=env)[0] == 38
    big_case(tmp_path, Nx, Ny, 6, "\n".join(vals[:-1]) + "\n")
    assert run(DRV, tmp_path, env_extra=env)[0] == 38
    big_case(tmp_path, Nx, Ny, 6, "\n".join(vals + ["1.0", "junk", "2.0"]) + "\n")
    assert run(DRV, tmp_path, env_extra=env)[0] == 0


SMOOTH = os.path.join(ROOT, "pfc_b200", "smooth")
REF_SMOOTH = os.path.join(ROOT, "oracle", "_ref", "smooth")


def test_smooth_usage_and_missing_input(tmp_path):
    r = subprocess.run([SMOOTH], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "smooth" in r.stdout
    r = subprocess.run([SMOOTH, "nope.n", "out.n", "0.5"], cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "Input file not found!" in r.stdout


def smooth_numpy(f, dx, dy, sigma):
    """The smoothing of demos/honey/smooth.c:81-121 in numpy: r2c, multiply by
    exp(-k^2 / (2 sigma^2)), c2r (the kernel's real-space sum is 1)."""
    H, W = f.shape
    kx = 2 * np.pi / (dx * W) * np.arange(W // 2 + 1)
    ky = 2 * np.pi / (dy * H) * np.where(np.arange(H) < H // 2, np.arange(H), np.arange(H) - H)
    k2 = kx[None, :] ** 2 + ky[:, None] ** 2
    return np.fft.irfft2(np.fft.rfft2(f) * np.exp(-0.5 / sigma ** 2 * k2), s=f.shape)


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 2e-6)])
def test_smooth_matches_numpy_and_reference(tmp_path, precision, tol):
    W, H, dx, dy, sigma = 96, 64, 0.7, 0.65, 0.6
    f = synth.hetero2(W, H, dx, dy, 4, 0, 0, (0.3, -0.3), (0.3, 0.3), (7.2552, 7.5), 0.02, 4)[0]
    (tmp_path / "in.n").write_text("%d %d %.12f %.12f\n" % (W, H, dx, dy) + "".join("%.17e\n" % v for v in f.ravel()))
    env = dict(os.environ, PFC_B200_PRECISION=precision)
    r = subprocess.run([SMOOTH, "in.n", "out.n", str(sigma)], cwd=tmp_path, capture_output=True, text=True,
                       env=env, timeout=120)
    assert r.returncode == 0, r.stderr
    lines = (tmp_path / "out.n").read_text().splitlines()
    assert lines[0] == "%d %d %f %f" % (W, H, dx, dy)
    assert all(len(l.split("e")[0].split(".")[1]) == 12 for l in lines[1:])
    got = np.array([float(x) for x in lines[1:]]).reshape(H, W)
    want = smooth_numpy(f, dx, dy, sigma)
    assert np.abs(got - want).max() < tol * np.abs(want).max()
    if os.path.exists(REF_SMOOTH):
        r = subprocess.run([REF_SMOOTH, "in.n", "ref.n", str(sigma)], cwd=tmp_path, capture_output=True, timeout=120)
        assert r.returncode == 0
        ref = np.loadtxt(tmp_path / "ref.n", skiprows=1).reshape(H, W)
        assert np.abs(got - ref).max() < tol * np.abs(ref).max()


def test_numpy_smoothing_matches_reference_binary(tmp_path):
    """Pins smooth_numpy (the GPU test's oracle) to the reference smooth tool
    built from its own source over the FFT shim (CPU)."""
    if not os.path.exists(REF_SMOOTH):
        pytest.skip("reference smooth not built")
    W, H, dx, dy, sigma = 48, 40, 0.7, 0.65, 0.6
    f = synth.noise_state(W, H, 0.1, 0.3, 12)
    (tmp_path / "in.n").write_text("%d %d %.12f %.12f\n" % (W, H, dx, dy) + "".join("%.17e\n" % v for v in f.ravel()))
    r = subprocess.run([REF_SMOOTH, "in.n", "ref.n", str(sigma)], cwd=tmp_path, capture_output=True, timeout=120)
    assert r.returncode == 0
    ref = np.loadtxt(tmp_path / "ref.n", skiprows=1).reshape(H, W)
    assert np.abs(smooth_numpy(f, dx, dy, sigma) - ref).max() < 1e-12 * np.abs(ref).max()


FIELDS = os.path.join(ROOT, "pfc_b200", "fields")
REF_FIELDS = os.path.join(ROOT, "oracle", "_ref", "fields")


def polycrystal_file(path, W=128, H=96, seed=3):
    dx = dy = synth.A_TRI / 8
    p = synth.polycrystal(W, H, dx, dy, 5, 0.0, 0.5, 0.02, seed)
    path.write_text("%d %d %.12f %.12f\n" % (W, H, dx, dy) + "".join("%.17e\n" % v for v in p.ravel()))
    return p, dx, dy


@pytest.mark.parametrize("args,code,msg", [((), 0, "fields"), (("a", "b"), 1, "Error: Invalid syntax."),
                                           (("nope.n", "o.phi", "6", "0.2", "0.1"), 1, "Error: Input file not found.")])
def test_fields_cli_messages(tmp_path, args, code, msg):
    r = subprocess.run([FIELDS] + list(args), cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert r.returncode == code and msg in r.stdout
    if os.path.exists(REF_FIELDS) and args:
        rr = subprocess.run([REF_FIELDS] + list(args), cwd=tmp_path, capture_output=True, text=True, timeout=60)
        assert rr.returncode == code and msg in rr.stdout


def test_fields_oracle_matches_reference_binary(tmp_path):
    """Pins oracle/fields_oracle.py (the GPU test's checker) to the reference
    tool compiled over the FFT shim, to the reference's print precision."""
    if not os.path.exists(REF_FIELDS):
        pytest.skip("reference fields not built")
    import sys
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import fields_oracle as FO

    p, dx, dy = polycrystal_file(tmp_path / "d.n")
    r = subprocess.run([REF_FIELDS, "d.n", "o.phi", "o.chi", "6", "0.2", "0.1", "2.0"], cwd=tmp_path,
                       capture_output=True, timeout=120)
    assert r.returncode == 0
    ref = np.loadtxt(tmp_path / "o.phi", skiprows=1)
    refc = np.loadtxt(tmp_path / "o.chi", skiprows=1)
    psi, Z = FO.orientation(p, dx, dy, 6, 0.2, 0.1)
    chi = FO.deformation(Z, dx, dy, 2.0)
    # "%e" keeps 7 significant digits
    assert np.abs(ref[:, 0] - psi.real.ravel()).max() < 6e-7
    assert np.abs(ref[:, 1] - psi.imag.ravel()).max() < 6e-7
    assert np.abs(refc - chi.ravel()).max() < 6e-7 * np.abs(chi).max()


@pytest.mark.gpu
def test_fields_gpu_matches_oracle_and_reference(tmp_path):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import fields_oracle as FO

    p, dx, dy = polycrystal_file(tmp_path / "d.n")
    psi, chi = lib.fields(p, dx, dy, 6, 0.2, 0.1, 2.0)
    want_psi, Z = FO.orientation(p, dx, dy, 6, 0.2, 0.1)
    want_chi = FO.deformation(Z, dx, dy, 2.0)
    assert np.abs(psi - want_psi).max() < 1e-9
    assert np.abs(chi - want_chi).max() < 1e-9 * np.abs(want_chi).max()
    # the command-line tool writes the reference's format
    r = subprocess.run([FIELDS, "d.n", "o.phi", "o.chi", "6", "0.2", "0.1", "2.0"], cwd=tmp_path, capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    got = np.loadtxt(tmp_path / "o.phi", skiprows=1)
    assert np.abs(got[:, 0] - want_psi.real.ravel()).max() < 6e-7
    if os.path.exists(REF_FIELDS):
        subprocess.run([REF_FIELDS, "d.n", "r.phi", "r.chi", "6", "0.2", "0.1", "2.0"], cwd=tmp_path, timeout=120)
        assert (tmp_path / "o.phi").read_text().splitlines()[0] == (tmp_path / "r.phi").read_text().splitlines()[0]
        ref = np.loadtxt(tmp_path / "r.phi", skiprows=1)
        assert np.abs(got - ref).max() < 1.2e-6
        assert np.abs(np.loadtxt(tmp_path / "o.chi", skiprows=1) - np.loadtxt(tmp_path / "r.chi", skiprows=1)).max() \
            < 1.2e-6 * np.abs(want_chi).max()


@pytest.mark.gpu
def test_fields_rejects_odd_fold():
    p = synth.noise_state(32, 32, 0.0, 0.1, 1)
    with pytest.raises(lib.PfcError):
        lib.fields(p, 0.9, 0.9, 3, 0.2, 0.1)
