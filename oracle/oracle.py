"""ctypes binding of the CPU FP64 oracle -- TEST INFRASTRUCTURE ONLY.

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg, always as the checker. Parity status: UNPINNED against reference runs
(see hercules_oracle.c); pinned by the known-answer tests in tests/.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from hercules_b200.params import HcDiag, Params, FIELD_IDS

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "libhercules_oracle.so")


def build(force: bool = False) -> str:
    src = os.path.join(_HERE, "hercules_oracle.c")
    if force or not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return _SO


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_SO)
        L.or_create.restype = ctypes.c_void_p
        L.or_create.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
        L.or_destroy.argtypes = [ctypes.c_void_p]
        for fn in ("or_set_field", "or_get_field"):
            getattr(L, fn).argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.or_initialize.argtypes = [ctypes.c_void_p]
        L.or_step.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.or_get_grid.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 5
        L.or_fft2d.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
        L.or_helmholtz_u.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double]
        L.or_set_threads.argtypes = [ctypes.c_int]
        L.or_set_body_force.argtypes = [ctypes.c_void_p] * 4
        _lib = L
    return _lib


def set_threads(n: int) -> None:
    lib().or_set_threads(int(n))


def fft2d(c: np.ndarray, direction: int) -> np.ndarray:
    """mpi_2d_fft on a complex (nz, ny, nx) array (x fastest); returns a copy."""
    a = np.ascontiguousarray(c, dtype=np.complex128).copy()
    nz, ny, nx = a.shape
    rc = lib().or_fft2d(nx, ny, nz, a.ctypes.data, direction)
    assert rc == 0
    return a


class Oracle:
    """One single-domain FP64 run of the reference time step on the CPU."""

    def __init__(self, p: Params):
        self.p = p
        err = ctypes.c_int(0)
        self._cp = p.to_c()
        self.h = lib().or_create(ctypes.byref(self._cp), ctypes.byref(err))
        if not self.h:
            raise ValueError(f"oracle rejected parameters (code {err.value})")

    def close(self):
        if self.h:
            lib().or_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set(self, name: str, arr: np.ndarray) -> None:
        a = np.ascontiguousarray(arr, dtype=np.float64)
        assert a.size == self.p.npoints
        rc = lib().or_set_field(self.h, FIELD_IDS[name], a.ctypes.data)
        assert rc == 0

    def get(self, name: str) -> np.ndarray:
        a = np.empty((self.p.nz, self.p.ny, self.p.nx), dtype=np.float64)
        rc = lib().or_get_field(self.h, FIELD_IDS[name], a.ctypes.data)
        assert rc == 0
        return a

    def load(self, fields: dict) -> None:
        for k, v in fields.items():
            self.set(k, v)

    def set_body_force(self, fx=None, fy=None, fz=None) -> None:
        """Body force added to ff, gg, hh (None: zero component; all None: off)."""
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (fx, fy, fz)]
        self._bf = arrs        # keep alive for the call
        ptrs = [None if a is None else a.ctypes.data for a in arrs]
        assert lib().or_set_body_force(self.h, *ptrs) == 0

    def initialize(self) -> None:
        assert lib().or_initialize(self.h) == 0

    def step(self, n: int = 1):
        diags = (HcDiag * n)()
        rc = lib().or_step(self.h, n, diags)
        return rc, [d.as_dict() for d in diags]

    def grid(self):
        nka = self.p.nz + 4
        arrs = [np.zeros(nka) for _ in range(5)]
        lib().or_get_grid(self.h, *[a.ctypes.data for a in arrs])
        return dict(zip(["dz", "l_t", "l_b", "dz_t", "dz_b"], arrs))

    def helmholtz_u(self, rhs: np.ndarray, rk_c: float) -> np.ndarray:
        a = np.ascontiguousarray(rhs, dtype=np.float64)
        out = np.empty_like(a)
        lib().or_helmholtz_u(self.h, a.ctypes.data, out.ctypes.data, rk_c)
        return out
