"""ctypes wrapper of the CPU oracle (oracle/_build/libpfc_oracle.so) and of the
reference binaries built over the FFTW/MPI shim (oracle/_ref/).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product package.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libpfc_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("oracle not built: run `make -C oracle`")
        L = ctypes.CDLL(LIB_PATH)
        vp, ip, dp = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)
        L.pfco_create.restype = vp
        L.pfco_create.argtypes = [vp, ip, ip, ctypes.c_double, ctypes.c_double]
        L.pfco_destroy.argtypes = [vp]
        L.pfco_upload.argtypes = [vp, dp]
        L.pfco_download.argtypes = [vp, dp]
        L.pfco_spectrum.argtypes = [vp, dp]
        L.pfco_set_box.argtypes = [vp, ctypes.c_double, ctypes.c_double]
        L.pfco_get_box.argtypes = [vp, dp, dp]
        L.pfco_set_time.argtypes = [vp, ip]
        L.pfco_get_time.argtypes = [vp]
        L.pfco_get_time.restype = ip
        L.pfco_step.argtypes = [vp, ip]
        L.pfco_step.restype = ip
        L.pfco_evaluate.argtypes = [vp, dp, dp, dp]
        L.pfco_optimize.argtypes = [vp, ip, ip, dp]
        L.pfco_set_emulate_nu2.argtypes = [vp, ip]
        L.pfco_set_scheme.argtypes = [vp, ip]
        L.fft64_r2c_2d_tr.argtypes = [ip, ip, dp, ctypes.c_ssize_t, dp]
        L.fft64_c2r_2d_tr.argtypes = [ip, ip, dp, dp, ctypes.c_ssize_t]
        L.fft64_prepare_2d.argtypes = [ip, ip]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def rfft2_tr(field: np.ndarray) -> np.ndarray:
    """Oracle r2c of a (Ny, Nx) real field; returns (Nx/2+1, Ny) complex (transposed, unnormalised)."""
    L = lib()
    Ny, Nx = field.shape
    a = np.ascontiguousarray(field, dtype=np.float64)
    out = np.zeros((Nx // 2 + 1, Ny), dtype=np.complex128)
    L.fft64_prepare_2d(Ny, Nx)
    L.fft64_r2c_2d_tr(Ny, Nx, _dp(a), Nx, out.view(np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return out


def irfft2_tr(spec: np.ndarray, Nx: int) -> np.ndarray:
    """Oracle c2r of a (Nx/2+1, Ny) transposed spectrum; unnormalised."""
    L = lib()
    H, Ny = spec.shape
    s = np.ascontiguousarray(spec, dtype=np.complex128)
    out = np.zeros((Ny, Nx))
    L.fft64_prepare_2d(Ny, Nx)
    L.fft64_c2r_2d_tr(Ny, Nx, s.view(np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double)), _dp(out), Nx)
    return out


class Oracle:
    """FP64 CPU restatement of step / evaluate / optimize / update_AB."""

    def __init__(self, params, Nx: int, Ny: int, dx: float, dy: float):
        self.L = lib()
        self.params = params
        self.U = params.U
        self.Nx, self.Ny = Nx, Ny
        self.h = self.L.pfco_create(ctypes.byref(params), Nx, Ny, dx, dy)
        if not self.h:
            raise ValueError("pfco_create failed")

    def close(self):
        if self.h:
            self.L.pfco_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, fields: np.ndarray):
        f = np.ascontiguousarray(fields, dtype=np.float64).reshape(self.U, self.Ny, self.Nx)
        self.L.pfco_upload(self.h, _dp(f))

    def download(self) -> np.ndarray:
        out = np.zeros((self.U, self.Ny, self.Nx))
        self.L.pfco_download(self.h, _dp(out))
        return out

    def spectrum(self) -> np.ndarray:
        out = np.zeros((self.U, self.Nx // 2 + 1, self.Ny), dtype=np.complex128)
        self.L.pfco_spectrum(self.h, out.view(np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return out

    def step(self, n: int = 1) -> int:
        return self.L.pfco_step(self.h, n)

    def evaluate(self, want_f: bool = False):
        fave = ctypes.c_double()
        nave = np.zeros(self.U)
        f = np.zeros((self.Ny, self.Nx)) if want_f else None
        self.L.pfco_evaluate(self.h, ctypes.byref(fave), _dp(nave), _dp(f) if want_f else None)
        return (fave.value, nave, f) if want_f else (fave.value, nave)

    def optimize(self, xopt: int, yopt: int, d: float) -> float:
        dd = ctypes.c_double(d)
        self.L.pfco_optimize(self.h, xopt, yopt, ctypes.byref(dd))
        return dd.value

    def set_box(self, dx, dy):
        self.L.pfco_set_box(self.h, dx, dy)

    def box(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        self.L.pfco_get_box(self.h, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    @property
    def t(self):
        return self.L.pfco_get_time(self.h)

    def set_time(self, t):
        self.L.pfco_set_time(self.h, t)

    def emulate_nu2(self, on=True):
        self.L.pfco_set_emulate_nu2(self.h, 1 if on else 0)

    def set_scheme(self, scheme: str):
        """'etd1' (the reference) or 'semi' (the semi-implicit update, not in the reference)."""
        self.L.pfco_set_scheme(self.h, {"etd1": 0, "semi": 1}[scheme])

    def relax(self, tend: int, Tprint: int, Topt: int = 0, xopt: int = 1, yopt: int = 1):
        """The reference's relax() schedule (pfc-relax.c:1293-1313) without file
        output; returns the printed rows (t, dx, dy, <f>, <n_u>...)."""
        rows = []
        d = 1e-4
        for t in range(tend + 1):
            self.set_time(t)
            if Topt > 0 and t > 0 and t % Topt == 0:
                d = self.optimize(xopt, yopt, d)
            if t % Tprint == 0:
                fave, nave = self.evaluate()
                dx, dy = self.box()
                rows.append([t, dx, dy, fave] + list(nave))
            if t < tend:
                rc = self.step(1)
                if rc:
                    raise RuntimeError("oracle step failed with code %d" % rc)
        return np.array(rows)
