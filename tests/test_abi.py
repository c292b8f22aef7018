"""The C ABI library loads, exports every entry point of include/pfc_b200.h,
and refuses unsupported sizes; no kernel is launched (CPU only)."""
import os
import re

import pytest

from pfc_b200 import lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "pfc_b200.h")


def header_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(pfcg_[a-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert header_symbols() == sorted(lib.SIGNATURES)


def test_library_exports_every_symbol():
    L = lib.load()
    for name in header_symbols():
        assert hasattr(L, name), name


@pytest.mark.parametrize("Nx,Ny,ok", [(512, 512, 1), (4096, 4096, 1), (384, 1536, 1), (48, 40, 1), (56, 70, 1),
                                      (30, 42, 1), (11, 64, 0), (66, 64, 0), (64, 26, 0), (4, 8, 0), (16384, 64, 0)])
def test_size_supported(Nx, Ny, ok):
    assert lib.size_supported(Nx, Ny) == bool(ok)


def test_create_rejects_bad_arguments_without_gpu_work():
    from pfc_b200 import params as P
    p = P.make_params(P.honeycomb_1c(), 1.0, 1.0)
    with pytest.raises(lib.PfcError) as e:
        lib.Relaxation(p, 66, 64, 0.7, 0.7)
    assert e.value.code == lib.ESIZE


@pytest.mark.parametrize("Nx,Ny,U,prec,ok", [
    (8192, 8, 1, lib.FP64, 1), (8192, 8, 1, lib.FP32, 1), (7168, 8, 2, lib.FP64, 1),
    (8064, 8, 1, lib.FP32, 0),          # 8064 / 7 = 1152 butterflies: more than 512 threads x 2
    (8, 8192, 2, lib.FP64, 0),          # two FP64 columns of 8192 exceed shared memory
    (8, 8192, 2, lib.FP32, 1), (8192, 16, 4, lib.FP64, 0), (8192, 16, 4, lib.FP32, 1),
    (4096, 4096, 4, lib.FP64, 0),       # four FP64 columns of 4096 exceed shared memory
    (2048, 2048, 4, lib.FP64, 1), (30, 42, 3, lib.FP64, 1), (66, 64, 1, lib.FP32, 0), (64, 64, 0, lib.FP32, 0),
    (8192, 8192, 2, lib.FP32, 1), (8192, 8192, 2, lib.FP64, 0), (4096, 4096, 4, lib.FP32, 1),
    (1536, 1536, 2, lib.FP32, 1), (384, 384, 2, lib.FP32, 1), (998, 998, 1, lib.FP32, 0),  # 499 is prime
    (1001, 1000, 1, lib.FP32, 0)])  # odd lengths are refused: even 8..8192 only
def test_size_supported_for(Nx, Ny, U, prec, ok):
    """The exact host-side check of what pfcg_create accepts (no device work)."""
    assert lib.load().pfcg_size_supported_for(Nx, Ny, U, prec) == ok
