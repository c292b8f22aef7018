"""ctypes view of libpfc_b200.so (the C ABI in include/pfc_b200.h).

The shared library is built in-tree (``make -C pfc_b200``). There is no CPU
fallback: if the library or a CUDA device is missing, every entry point
raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .params import Params

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpfc_b200.so")
DRIVER_PATH = os.path.join(HERE, "pfc-relax")

FP32, FP64 = 0, 1

# time integration schemes of pfcg_set_scheme
SCHEMES = {"etd1": 0, "semi": 1}

OK = 0
NAN = 39
EARG, ECUDA, ESIZE, ENOMEM, ETIMEOUT, ENODEV = -1, -2, -3, -4, -5, -6

# size of pfcg_relax_noalloc's static device workspace (PFCG_NOALLOC_SCRATCH_BYTES)
NOALLOC_SCRATCH_BYTES = 32 << 20

class Grain(ctypes.Structure):
    """pfcg_grain: one grain of the builder's Voronoi step (include/pfc_b200.h)."""
    _fields_ = [("x", ctypes.c_double), ("y", ctypes.c_double), ("type", ctypes.c_int), ("sym", ctypes.c_int),
                ("a", ctypes.c_double), ("nave", ctypes.c_double), ("amp", ctypes.c_double),
                ("namp", ctypes.c_double), ("tx1", ctypes.c_double), ("ty1", ctypes.c_double),
                ("theta_deg", ctypes.c_double), ("xr", ctypes.c_double), ("yr", ctypes.c_double),
                ("tx2", ctypes.c_double), ("ty2", ctypes.c_double)]


# every entry point of include/pfc_b200.h with its ctypes signature
_vp, _ip, _dp = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)
SIGNATURES = {
    "pfcg_size_supported": (ctypes.c_int, [_ip, _ip]),
    "pfcg_size_supported_for": (ctypes.c_int, [_ip, _ip, _ip, _ip]),
    "pfcg_create": (ctypes.c_int, [ctypes.c_void_p, _ip, _ip, ctypes.c_double, ctypes.c_double, _ip,
                                   ctypes.POINTER(ctypes.c_void_p)]),
    "pfcg_upload": (ctypes.c_int, [_vp, _dp]),
    "pfcg_download": (ctypes.c_int, [_vp, _dp]),
    "pfcg_upload_device": (ctypes.c_int, [_vp, _vp]),
    "pfcg_download_device": (ctypes.c_int, [_vp, _vp]),
    "pfcg_init_hetero": (ctypes.c_int, [_vp, _ip, _ip, ctypes.c_double, ctypes.c_double, _vp, _vp]),
    "pfcg_init_last_error": (ctypes.c_char_p, []),
    "pfcg_init_voronoi": (ctypes.c_int, [_vp, _ip, _ip, ctypes.c_double, ctypes.c_double, _ip, _vp,
                                         ctypes.POINTER(ctypes.c_longlong), _vp]),
    "pfcg_java_random_seed": (ctypes.c_longlong, [ctypes.c_longlong]),
    "pfcg_write_n_pfcinit": (ctypes.c_int, [ctypes.c_char_p, _ip, _ip, ctypes.c_double, ctypes.c_double, _dp, _ip]),
    "pfcg_set_box": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double]),
    "pfcg_get_box": (ctypes.c_int, [_vp, _dp, _dp]),
    "pfcg_set_scheme": (ctypes.c_int, [_vp, _ip]),
    "pfcg_get_scheme": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int)]),
    "pfcg_set_time": (ctypes.c_int, [_vp, _ip]),
    "pfcg_get_time": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int)]),
    "pfcg_step": (ctypes.c_int, [_vp, _ip]),
    "pfcg_evaluate": (ctypes.c_int, [_vp, _dp, _dp, _dp]),
    "pfcg_optimize": (ctypes.c_int, [_vp, _ip, _ip, _dp]),
    "pfcg_smooth": (ctypes.c_int, [_vp, _ip, _dp]),
    "pfcg_fields": (ctypes.c_int, [_dp, _ip, _ip, ctypes.c_double, ctypes.c_double, _ip, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_double, _dp, _dp]),
    "pfcg_set_device": (ctypes.c_int, [_ip]),
    "pfcg_set_profiling": (ctypes.c_int, [_vp, _ip]),
    "pfcg_profile_read": (ctypes.c_int, [_vp, _dp, ctypes.POINTER(ctypes.c_longlong), _ip]),
    "pfcg_relax_noalloc": (ctypes.c_int, [ctypes.c_void_p, _ip, _ip, ctypes.c_double, ctypes.c_double, _ip,
                                          ctypes.c_void_p, ctypes.c_void_p]),
    "pfcg_autotune": (ctypes.c_int, [_vp, _ip]),
    "pfcg_batch_create": (ctypes.c_int, [_ip, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                         ctypes.POINTER(ctypes.c_int), _dp, _dp, _ip, _ip,
                                         ctypes.POINTER(ctypes.c_void_p)]),
    "pfcg_batch_problem": (ctypes.c_void_p, [_vp, _ip]),
    "pfcg_batch_step": (ctypes.c_int, [_vp, _ip]),
    "pfcg_batch_launches": (ctypes.c_int, [_vp, _ip, ctypes.POINTER(ctypes.c_longlong),
                                           ctypes.POINTER(ctypes.c_longlong)]),
    "pfcg_batch_destroy": (None, [_vp]),
    "pfcg_batch_stream": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_void_p)]),
    "pfcg_fno_param_count": (ctypes.c_size_t, []),
    "pfcg_fno_create": (ctypes.c_int, [_ip, _ip, ctypes.POINTER(ctypes.c_void_p)]),
    "pfcg_fno_set_params": (ctypes.c_int, [_vp, _vp]),
    "pfcg_fno_get_params": (ctypes.c_int, [_vp, _vp]),
    "pfcg_fno_forward": (ctypes.c_int, [_vp, _vp, _vp, _ip]),
    "pfcg_fno_loss_grad": (ctypes.c_int, [_vp, _vp, _vp, _ip, _dp, _vp]),
    "pfcg_fno_adam_step": (ctypes.c_int, [_vp, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float]),
    "pfcg_fno_apply": (ctypes.c_int, [_vp, _vp, _vp, _ip, _ip, _vp]),
    "pfcg_warmstart": (ctypes.c_int, [_vp, _vp]),
    "pfcg_fno_stream": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_void_p)]),
    "pfcg_fno_launch_count": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_longlong)]),
    "pfcg_fno_last_error": (ctypes.c_char_p, [_vp]),
    "pfcg_fno_destroy": (None, [_vp]),
    "pfcg_stream": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_void_p)]),
    "pfcg_launch_count": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_longlong)]),
    "pfcg_last_error": (ctypes.c_char_p, [_vp]),
    "pfcg_destroy": (None, [_vp]),
}

_lib = None


class PfcError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("pfcg error %d: %s" % (code, msg))
        self.code = code


def load():
    """Loads libpfc_b200.so once; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libpfc_b200.so is not built (run `make -C pfc_b200`); there is no CPU fallback")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def size_supported(Nx: int, Ny: int) -> bool:
    return bool(load().pfcg_size_supported(Nx, Ny))


def size_supported_for(Nx: int, Ny: int, U: int, precision: str) -> bool:
    return bool(load().pfcg_size_supported_for(Nx, Ny, U, {"fp32": FP32, "fp64": FP64}[precision]))


def set_device(device: int) -> None:
    """Device that later Relaxation objects on this thread use."""
    L = load()
    rc = L.pfcg_set_device(device)
    if rc:
        raise PfcError(rc, L.pfcg_last_error(None).decode())


class Relaxation:
    """One relaxation on the GPU: the state of pfc-relax's struct S for the hot
    path (fields, spectral state, box size, step counter)."""

    def __init__(self, params: Params, Nx: int, Ny: int, dx: float, dy: float, precision: str = "fp64",
                 scheme: str = "etd1"):
        self.L = load()
        self.params = params
        self.U = params.U
        self.Nx, self.Ny = Nx, Ny
        self.precision = precision
        prec = {"fp32": FP32, "fp64": FP64}[precision]
        h = ctypes.c_void_p()
        rc = self.L.pfcg_create(ctypes.byref(params), Nx, Ny, dx, dy, prec, ctypes.byref(h))
        if rc:
            raise PfcError(rc, self.L.pfcg_last_error(None).decode())
        self.h = h
        if scheme != "etd1":
            self.set_scheme(scheme)

    def set_scheme(self, scheme: str) -> None:
        """'etd1' (the reference's exponential update) or 'semi' (linear part implicit)."""
        self._check(self.L.pfcg_set_scheme(self.h, SCHEMES[scheme]))

    @property
    def scheme(self) -> str:
        v = ctypes.c_int()
        self._check(self.L.pfcg_get_scheme(self.h, ctypes.byref(v)))
        return {n: k for k, n in SCHEMES.items()}[v.value]

    def _check(self, rc: int):
        if rc:
            raise PfcError(rc, self.L.pfcg_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.L.pfcg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def upload(self, fields: np.ndarray) -> None:
        f = np.ascontiguousarray(fields, dtype=np.float64).reshape(self.U, self.Ny, self.Nx)
        self._check(self.L.pfcg_upload(self.h, _dptr(f)))

    def download(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty((self.U, self.Ny, self.Nx))
        self._check(self.L.pfcg_download(self.h, _dptr(out)))
        return out

    def upload_device(self, ptr: int) -> None:
        """Uploads U*Ny*Nx doubles from DEVICE memory at ptr."""
        self._check(self.L.pfcg_upload_device(self.h, ctypes.c_void_p(ptr)))

    def download_device(self, ptr: int) -> None:
        """Downloads the fields to U*Ny*Nx doubles of DEVICE memory at ptr."""
        self._check(self.L.pfcg_download_device(self.h, ctypes.c_void_p(ptr)))

    def smooth(self, u: int = 0) -> np.ndarray:
        """Field u smoothed by the model's kernel exp(-k^2 / (2 sigma^2))."""
        out = np.empty((self.Ny, self.Nx))
        self._check(self.L.pfcg_smooth(self.h, u, _dptr(out)))
        return out

    def warmstart(self, net) -> None:
        """Replaces the fields by the warm-start network's proposal (U = 2)."""
        self._check(self.L.pfcg_warmstart(self.h, net.f))

    def step(self, n: int = 1) -> int:
        """Advances n steps; returns 0, or raises PfcError (code 39 for NaN)."""
        rc = self.L.pfcg_step(self.h, n)
        self._check(rc)
        return rc

    def step_rc(self, n: int = 1) -> int:
        """Like step() but returns the status code instead of raising."""
        return self.L.pfcg_step(self.h, n)

    def evaluate(self, want_f: bool = False):
        fave = ctypes.c_double()
        nave = np.zeros(self.U)
        f = np.empty((self.Ny, self.Nx)) if want_f else None
        self._check(self.L.pfcg_evaluate(self.h, ctypes.byref(fave), _dptr(nave), _dptr(f) if want_f else None))
        return (fave.value, nave, f) if want_f else (fave.value, nave)

    def optimize(self, xopt: int, yopt: int, d: float) -> float:
        dd = ctypes.c_double(d)
        self._check(self.L.pfcg_optimize(self.h, xopt, yopt, ctypes.byref(dd)))
        return dd.value

    def set_box(self, dx: float, dy: float) -> None:
        self._check(self.L.pfcg_set_box(self.h, dx, dy))

    def box(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        self._check(self.L.pfcg_get_box(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    @property
    def t(self) -> int:
        v = ctypes.c_int()
        self._check(self.L.pfcg_get_time(self.h, ctypes.byref(v)))
        return v.value

    def set_time(self, t: int) -> None:
        self._check(self.L.pfcg_set_time(self.h, t))

    @property
    def stream(self) -> int:
        s = ctypes.c_void_p()
        self._check(self.L.pfcg_stream(self.h, ctypes.byref(s)))
        return s.value or 0

    def autotune(self, nsteps: int = 5) -> None:
        """Measure the runtime-plan launch shapes and keep the fastest (before upload)."""
        self._check(self.L.pfcg_autotune(self.h, nsteps))

    def set_profiling(self, on: bool) -> None:
        self._check(self.L.pfcg_set_profiling(self.h, 1 if on else 0))

    def profile(self):
        """{kind: (ms, launches)} for kinds 'xpass', 'ypass', 'other' since profiling was switched on."""
        ms = np.zeros(3)
        n = (ctypes.c_longlong * 3)()
        self._check(self.L.pfcg_profile_read(self.h, _dptr(ms), n, 3))
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(("xpass", "ypass", "other"))}

    @property
    def launches(self) -> int:
        c = ctypes.c_longlong()
        self._check(self.L.pfcg_launch_count(self.h, ctypes.byref(c)))
        return c.value

    def relax(self, tend: int, Tprint: int, Topt: int = 0, xopt: int = 1, yopt: int = 1, on_print=None):
        """pfc-relax.c:1293-1313 relax() schedule without file output, stepping
        in chunks between events. Returns the printed rows (t, dx, dy, <f>, <n_u>...)."""
        rows = []
        d = 1e-4
        t = self.t
        while t <= tend:
            if Topt > 0 and t > 0 and t % Topt == 0:
                d = self.optimize(xopt, yopt, d)
            if t % Tprint == 0:
                fave, nave = self.evaluate()
                dx, dy = self.box()
                row = [t, dx, dy, fave] + list(nave)
                rows.append(row)
                if on_print:
                    on_print(row)
            if t >= tend:
                break
            nxt = tend
            for T in (Tprint, Topt):
                if T > 0:
                    nxt = min(nxt, (t // T + 1) * T)
            self.step(nxt - t)
            t = nxt
        return np.array(rows)

    def relax_until(self, tol: float = 1e-9, every: int = 100, max_steps: int = 100000, Topt: int = 0,
                    xopt: int = 1, yopt: int = 1, d: float = 1e-4, on_print=None):
        """Steps until the free energy changes by less than tol per step, measured
        as |<f>(t) - <f>(t - every)| / every at every `every` steps. With Topt > 0
        the box is optimised every Topt steps first, in the order of relax()
        (pfc-relax.c:1297-1302: optimise, then evaluate, then step), starting
        from the sampling step d; the criterion then compares <f> of the current
        box. on_print(t, dx, dy, <f>) sees every evaluation. Returns (steps
        taken, final <f>, seconds); steps is None if max_steps ran out."""
        import time
        t0 = time.perf_counter()
        prev = self.evaluate()[0]
        if on_print:
            on_print(0, *self.box(), prev)
        done = 0
        while done < max_steps:
            self.step(every)
            done += every
            if Topt > 0 and done % Topt == 0:
                d = self.optimize(xopt, yopt, d)
            f = self.evaluate()[0]
            if on_print:
                on_print(done, *self.box(), f)
            if abs(f - prev) / every < tol:
                return done, f, time.perf_counter() - t0
            prev = f
        return None, prev, time.perf_counter() - t0


def relax_noalloc(params: Params, Nx: int, Ny: int, dx: float, dy: float, nsteps: int, fields_dev_ptr: int,
                  stream: int = 0) -> int:
    """pfcg_relax_noalloc on a caller-owned DEVICE buffer (U*Ny*Nx doubles,
    in/out). Returns the status code (0, 39 for NaN, negative on errors)."""
    L = load()
    return L.pfcg_relax_noalloc(ctypes.byref(params), Nx, Ny, dx, dy, nsteps, ctypes.c_void_p(fields_dev_ptr),
                                ctypes.c_void_p(stream))


class Hetero(ctypes.Structure):
    """pfcg_hetero: a seeded two-field heterostructure initial state."""
    _fields_ = [("grains", ctypes.c_int), ("stripe_width", ctypes.c_int), ("stripe_offset", ctypes.c_int),
                ("sym", ctypes.c_int), ("mean", ctypes.c_double * 2), ("amp", ctypes.c_double * 2),
                ("lattice", ctypes.c_double * 2), ("noise", ctypes.c_double), ("max_angle_deg", ctypes.c_double),
                ("seed", ctypes.c_uint)]


def make_hetero(grains: int, width: int, offset: int, means, amps, lattice, noise: float, seed: int,
                sym: int = 3, max_angle_deg: float = 60.0) -> Hetero:
    return Hetero(grains, width, offset, sym, (ctypes.c_double * 2)(*means), (ctypes.c_double * 2)(*amps),
                  (ctypes.c_double * 2)(*lattice), noise, max_angle_deg, seed)


def init_hetero(d_fields_ptr: int, Nx: int, Ny: int, dx: float, dy: float, spec: Hetero, stream: int = 0) -> None:
    """pfcg_init_hetero into 2*Ny*Nx doubles of DEVICE memory."""
    L = load()
    rc = L.pfcg_init_hetero(ctypes.c_void_p(d_fields_ptr), Nx, Ny, dx, dy, ctypes.byref(spec), ctypes.c_void_p(stream))
    if rc:
        raise PfcError(rc, L.pfcg_init_last_error().decode())


def fields(density: np.ndarray, dx: float, dy: float, fold: int, sk: float, sb: float, power: float | None = None):
    """pfcg_fields: (psi complex (Ny, Nx), chi (Ny, Nx) or None)."""
    L = load()
    d = np.ascontiguousarray(density, dtype=np.float64)
    Ny, Nx = d.shape
    psi = np.empty((2, Ny, Nx))
    chi = np.empty((Ny, Nx)) if power is not None else None
    rc = L.pfcg_fields(_dptr(d), Nx, Ny, dx, dy, fold, sk, sb, power or 0.0, _dptr(psi),
                       _dptr(chi) if chi is not None else None)
    if rc:
        raise PfcError(rc, L.pfcg_last_error(None).decode())
    return psi[0] + 1j * psi[1], chi


def last_error() -> str:
    return load().pfcg_last_error(None).decode()


class _Problem(Relaxation):
    """A problem owned by a Batch: an ordinary handle that the batch frees."""

    def __init__(self, L, h, params, Nx, Ny, precision):
        self.L = L
        self.h = ctypes.c_void_p(h)
        self.params = params
        self.U = params.U
        self.Nx, self.Ny = Nx, Ny
        self.precision = precision

    def close(self):
        self.h = None


class Batch:
    """Many relaxations stepped together (pfcg_batch_*): one CUDA graph per step
    count; per step, two batched kernels for each class of problems (one class
    per size and field count with specialised kernels, one for the rest)."""

    def __init__(self, problems, precision: str = "fp32", autotune: bool = True):
        """problems: list of (Params, Nx, Ny, dx, dy)."""
        self.L = load()
        n = len(problems)
        arr = (Params * n)(*[p[0] for p in problems])
        Nx = (ctypes.c_int * n)(*[p[1] for p in problems])
        Ny = (ctypes.c_int * n)(*[p[2] for p in problems])
        dx = np.array([p[3] for p in problems], dtype=np.float64)
        dy = np.array([p[4] for p in problems], dtype=np.float64)
        b = ctypes.c_void_p()
        rc = self.L.pfcg_batch_create(n, arr, Nx, Ny, _dptr(dx), _dptr(dy), {"fp32": FP32, "fp64": FP64}[precision],
                                      1 if autotune else 0, ctypes.byref(b))
        if rc:
            raise PfcError(rc, self.L.pfcg_last_error(None).decode())
        self.b = b
        self.problems = [_Problem(self.L, self.L.pfcg_batch_problem(b, i), p[0], p[1], p[2], precision)
                         for i, p in enumerate(problems)]

    def step(self, n: int = 1) -> int:
        rc = self.L.pfcg_batch_step(self.b, n)
        if rc:
            raise PfcError(rc, self.L.pfcg_last_error(None).decode())
        return rc

    @property
    def stream(self) -> int:
        """The cudaStream_t the batch launches on (for CUDA-event timing)."""
        s = ctypes.c_void_p()
        rc = self.L.pfcg_batch_stream(self.b, ctypes.byref(s))
        if rc:
            raise PfcError(rc, self.L.pfcg_last_error(None).decode())
        return s.value or 0

    def launches(self, nsteps: int = 1):
        """(kernel launches, graph launches) of pfcg_batch_step(nsteps)."""
        k, g = ctypes.c_longlong(), ctypes.c_longlong()
        rc = self.L.pfcg_batch_launches(self.b, nsteps, ctypes.byref(k), ctypes.byref(g))
        if rc:
            raise PfcError(rc, self.L.pfcg_last_error(None).decode())
        return k.value, g.value

    def close(self):
        if getattr(self, "b", None):
            for p in self.problems:
                p.close()
            self.L.pfcg_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
