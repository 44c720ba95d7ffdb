"""Python handle on the CPU oracle (test infrastructure only).

Binds oracle/libicls_oracle.so with the same ``Solver`` class as the CUDA
library, so a test drives both with identical calls.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU legs import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ROOT = os.path.dirname(_HERE)
_PKG_PARENT = os.path.join(_ROOT, "icls-release_b200")
if _PKG_PARENT not in sys.path:
    sys.path.insert(0, _PKG_PARENT)

from icls_gpu.binding import Backend, Solver  # noqa: E402
from icls_gpu.config import IclsConfig  # noqa: E402

LIB = os.path.join(_HERE, "libicls_oracle.so")
_BACKEND = None


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB) or (
            os.path.getmtime(LIB) < os.path.getmtime(os.path.join(_HERE, "icls_oracle.cpp"))):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return LIB


def backend() -> Backend:
    global _BACKEND
    if _BACKEND is None:
        build()
        _BACKEND = Backend(LIB, "ora_")
        lib = _BACKEND.lib
        lib.ora_set_threads.argtypes = [C.c_int]
        lib.ora_set_threads.restype = C.c_int
        lib.ora_set_dt.argtypes = [C.c_void_p, C.c_double]
        lib.ora_vrfftf.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double)]
        lib.ora_vrfftb.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double)]
        lib.ora_vcosqf.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double)]
        lib.ora_vcosqb.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double)]
        lib.ora_get_pseudo_inv.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    return _BACKEND


def set_threads(n: int) -> int:
    return backend().lib.ora_set_threads(n)


class Oracle(Solver):
    def __init__(self, cfg: IclsConfig):
        super().__init__(cfg, backend())

    def pseudo_inv(self) -> np.ndarray:
        P = np.zeros(270)
        self.be.lib.ora_get_pseudo_inv(self.h, P.ctypes.data_as(C.POINTER(C.c_double)))
        return P.reshape(10, 27)

    def set_dt(self, dt: float):
        self.be.lib.ora_set_dt(self.h, dt)


def vrfftf(x: np.ndarray) -> np.ndarray:
    """VFFTPACK VRFFTF contract on each row of a C-contiguous 2-D array."""
    a = np.ascontiguousarray(x, dtype=np.float64).copy()
    m, n = a.shape
    backend().lib.ora_vrfftf(m, n, a.ctypes.data_as(C.POINTER(C.c_double)))
    return a


def vcosqf(x: np.ndarray) -> np.ndarray:
    """VFFTPACK VCOSQF contract (fft.f:68-216) on each row."""
    a = np.ascontiguousarray(x, dtype=np.float64).copy()
    m, n = a.shape
    backend().lib.ora_vcosqf(m, n, a.ctypes.data_as(C.POINTER(C.c_double)))
    return a


def vcosqb(x: np.ndarray) -> np.ndarray:
    """VFFTPACK VCOSQB contract (fft.f:218-372) on each row."""
    a = np.ascontiguousarray(x, dtype=np.float64).copy()
    m, n = a.shape
    backend().lib.ora_vcosqb(m, n, a.ctypes.data_as(C.POINTER(C.c_double)))
    return a


def vrfftb(x: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(x, dtype=np.float64).copy()
    m, n = a.shape
    backend().lib.ora_vrfftb(m, n, a.ctypes.data_as(C.POINTER(C.c_double)))
    return a
