"""ctypes binding of libhercules_b200.so and the host-side `drive` mirror.

``Channel`` wraps one ``hc_handle``: the device-resident state of one HERCULES
run. Its methods mirror the reference's seam (src/module_navier_stokes.f90:31-218):
``upload`` replaces filling the module arrays (read_init_fields), ``initialize``
the set-up part of ``drive``, ``step`` the body of the time loop, ``download``
reading the module arrays for output.

There is no CPU fallback: if the CUDA library cannot be loaded the constructor
raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Dict, List, Optional

import numpy as np

from .params import HcDiag, HcParams, Params, FIELD_IDS, PREC_MIXED, check_parameters

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhercules_b200.so")

HC_ERRORS = {0: "ok", -1: "bad argument", -2: "parameter check failed", -3: "CUDA error",
             -4: "device allocation failed", -5: "NaN error", -6: "call out of order",
             -7: "option not supported", -8: "size beyond the documented maximum"}

# every entry point declared in include/hercules_b200.h
ABI_SYMBOLS = ["hc_create", "hc_set_grid", "hc_get_grid", "hc_upload", "hc_download",
               "hc_initialize", "hc_step", "hc_get_scalars", "hc_upload_dev", "hc_download_dev",
               "hc_last_step_ms", "hc_last_launch_count", "hc_set_profiling", "hc_kernel_profile",
               "hc_divergence_noalloc", "hc_set_body_force", "hc_set_graph", "hc_ensemble_create",
               "hc_ensemble_step", "hc_ensemble_last_ms", "hc_ensemble_destroy", "hc_adjoint_forward",
               "hc_adjoint_reverse", "hc_adjoint_reverse_t", "hc_adjoint", "hc_adjoint_last_ms", "hc_destroy", "hc_error_string"]


class HerculesError(RuntimeError):
    def __init__(self, code: int, what: str):
        super().__init__(f"{what}: {HC_ERRORS.get(code, code)} ({code})")
        self.code = code


_lib = None


def load_library(path: str = LIB_PATH):
    """Load the CUDA engine; raises if it is missing (no fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError(f"hercules_b200: CUDA library not built ({path}); run hercules_b200/build.py")
    L = ctypes.CDLL(path)
    vp, ip, dp = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    L.hc_create.argtypes = [ctypes.POINTER(HcParams), ctypes.POINTER(vp)]
    L.hc_set_grid.argtypes = [vp] + [ctypes.c_void_p] * 5
    L.hc_get_grid.argtypes = [vp] + [ctypes.c_void_p] * 5
    L.hc_upload.argtypes = [vp, ip, ctypes.c_void_p, ip, ip, ip]
    L.hc_download.argtypes = [vp, ip, ctypes.c_void_p, ip, ip, ip]
    L.hc_initialize.argtypes = [vp]
    L.hc_step.argtypes = [vp, ip, ctypes.c_void_p]
    L.hc_get_scalars.argtypes = [vp] + [ctypes.POINTER(dp)] * 5 + [ctypes.POINTER(ip)]
    L.hc_upload_dev.argtypes = [vp, ip, ctypes.c_void_p]
    L.hc_download_dev.argtypes = [vp, ip, ctypes.c_void_p]
    L.hc_last_step_ms.argtypes = [vp, ctypes.POINTER(dp)]
    L.hc_last_launch_count.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    L.hc_set_profiling.argtypes = [vp, ip]
    L.hc_kernel_profile.argtypes = [vp, ip, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ip)]
    L.hc_divergence_noalloc.argtypes = [ctypes.POINTER(HcParams), ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.hc_set_body_force.argtypes = [vp, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.hc_set_graph.argtypes = [vp, ip]
    L.hc_ensemble_create.argtypes = [ctypes.POINTER(vp), ip, ctypes.POINTER(vp)]
    L.hc_ensemble_step.argtypes = [vp, ip]
    L.hc_ensemble_last_ms.argtypes = [vp, ctypes.POINTER(dp), ctypes.POINTER(ctypes.c_longlong)]
    L.hc_ensemble_destroy.argtypes = [vp]
    L.hc_adjoint.argtypes = [vp, ip, ip] + [ctypes.c_void_p] * 9
    L.hc_adjoint_forward.argtypes = [vp, ip, ip]
    L.hc_adjoint_reverse.argtypes = [vp] + [ctypes.c_void_p] * 9
    L.hc_adjoint_reverse_t.argtypes = [vp] + [ctypes.c_void_p] * 11
    L.hc_adjoint_last_ms.argtypes = [vp, ctypes.POINTER(dp), ctypes.POINTER(dp),
                                     ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]
    L.hc_destroy.argtypes = [vp]
    L.hc_error_string.argtypes = [ip]
    L.hc_error_string.restype = ctypes.c_char_p
    for name in ABI_SYMBOLS:
        if name not in ("hc_error_string",):
            getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise HerculesError(rc, what)


class Channel:
    """One HERCULES channel / Ekman run resident on the current CUDA device."""

    def __init__(self, p: Params):
        check_parameters(p)
        self.p = p
        self._L = load_library()
        self._cp = p.to_c()
        h = ctypes.c_void_p()
        _check(self._L.hc_create(ctypes.byref(self._cp), ctypes.byref(h)), "hc_create")
        self.h = h

    # ---- lifetime -------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "h", None):
            self._L.hc_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- data -----------------------------------------------------------
    def _shape(self, ghost: int):
        p = self.p
        return (p.nz + 2 * ghost, p.ny + 2 * ghost, p.nx + 2 * ghost)

    def upload(self, name: str, arr: np.ndarray, ghost: int = 0) -> None:
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if a.shape != self._shape(ghost):
            raise ValueError(f"{name}: shape {a.shape} != {self._shape(ghost)}")
        _check(self._L.hc_upload(self.h, FIELD_IDS[name], a.ctypes.data,
                                 a.shape[2], a.shape[1], ghost), f"hc_upload({name})")

    def load(self, fields: Dict[str, np.ndarray]) -> None:
        for k, v in fields.items():
            self.upload(k, v)

    def download(self, name: str, ghost: int = 0, out: Optional[np.ndarray] = None) -> np.ndarray:
        """The field as a float64 array; `out` (C-contiguous float64 of the right
        shape, e.g. in pinned memory) is filled instead of a new array."""
        if out is not None:
            if out.shape != self._shape(ghost) or out.dtype != np.float64 or not out.flags["C_CONTIGUOUS"]:
                raise ValueError(f"download({name}): out must be C-contiguous float64 of shape {self._shape(ghost)}")
            a = out
        else:
            a = np.zeros(self._shape(ghost), dtype=np.float64)
        _check(self._L.hc_download(self.h, FIELD_IDS[name], a.ctypes.data,
                                   a.shape[2], a.shape[1], ghost), f"hc_download({name})")
        return a

    def upload_dev(self, name: str, ptr: int) -> None:
        _check(self._L.hc_upload_dev(self.h, FIELD_IDS[name], ctypes.c_void_p(ptr)), "hc_upload_dev")

    def download_dev(self, name: str, ptr: int) -> None:
        _check(self._L.hc_download_dev(self.h, FIELD_IDS[name], ctypes.c_void_p(ptr)), "hc_download_dev")

    def set_graph(self, enable: bool = True) -> None:
        """Replay each step from a captured CUDA graph (saves launch cost)."""
        _check(self._L.hc_set_graph(self.h, 1 if enable else 0), "hc_set_graph")

    def set_body_force(self, fx=None, fy=None, fz=None) -> None:
        """Body force (nz, ny, nx) added to ff, gg, hh; None components are zero,
        all None removes it. No counterpart in the reference."""
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (fx, fy, fz)]
        for a in arrs:
            if a is not None and a.shape != self._shape(0):
                raise ValueError(f"body force shape {a.shape} != {self._shape(0)}")
        ptrs = [None if a is None else ctypes.c_void_p(a.ctypes.data) for a in arrs]
        _check(self._L.hc_set_body_force(self.h, *ptrs), "hc_set_body_force")

    # ---- time stepping -------------------------------------------------
    def adjoint_forward(self, nsteps: int, ckpt: int = 10) -> None:
        """Advance nsteps (as step() would), keeping a checkpoint every ckpt steps
        for adjoint_reverse. No counterpart in the reference."""
        _check(self._L.hc_adjoint_forward(self.h, nsteps, ckpt), "hc_adjoint_forward")

    def adjoint_reverse(self, seeds: Dict[str, np.ndarray], body_force: bool = True) -> Dict[str, np.ndarray]:
        """Gradient of J = sum over f in seeds of <seeds[f], f_N> (f in u, v, w, p and,
        with temperature, t; the fields after the last adjoint_forward) with respect
        to the fields that pass started from (keys "u", "v", "w", "p"[, "t"]) and,
        with body_force, to the body force ("fx", "fy", "fz")."""
        shp = self._shape(0)
        names = ("u", "v", "w", "p") + (("t",) if self.p.isscalar else ())
        sd = {}
        for f in names:
            a = seeds.get(f)
            if a is not None:
                a = np.ascontiguousarray(a, dtype=np.float64)
                if a.shape != shp:
                    raise ValueError(f"seed {f}: shape {a.shape} != {shp}")
            sd[f] = a
        g = {f: np.zeros(shp) for f in names}
        gbf = np.zeros((3,) + shp) if body_force else None
        ptr = lambda a: None if a is None else ctypes.c_void_p(a.ctypes.data)
        if self.p.isscalar:
            _check(self._L.hc_adjoint_reverse_t(self.h, *[ptr(sd[f]) for f in names],
                                                *[ptr(g[f]) for f in names], ptr(gbf)),
                   "hc_adjoint_reverse_t")
        else:
            _check(self._L.hc_adjoint_reverse(self.h, *[ptr(sd[f]) for f in names],
                                              *[ptr(g[f]) for f in names], ptr(gbf)),
                   "hc_adjoint_reverse")
        if body_force:
            g.update(fx=gbf[0], fy=gbf[1], fz=gbf[2])
        return g

    def adjoint(self, nsteps: int, seeds: Dict[str, np.ndarray], ckpt: int = 10,
                body_force: bool = True) -> Dict[str, np.ndarray]:
        """adjoint_forward then adjoint_reverse."""
        self.adjoint_forward(nsteps, ckpt)
        return self.adjoint_reverse(seeds, body_force)

    def adjoint_timing(self) -> dict:
        """Device time (ms) and launches of the last adjoint(): forward pass and reverse sweep."""
        f, r = ctypes.c_double(), ctypes.c_double()
        lf, lr = ctypes.c_longlong(), ctypes.c_longlong()
        _check(self._L.hc_adjoint_last_ms(self.h, ctypes.byref(f), ctypes.byref(r), ctypes.byref(lf),
                                          ctypes.byref(lr)), "hc_adjoint_last_ms")
        return {"forward_ms": f.value, "reverse_ms": r.value, "forward_launches": lf.value,
                "reverse_launches": lr.value}

    def initialize(self) -> None:
        _check(self._L.hc_initialize(self.h), "hc_initialize")

    def step(self, n: int = 1, raise_on_nan: bool = True) -> List[dict]:
        diags = (HcDiag * max(n, 1))()
        rc = self._L.hc_step(self.h, n, diags)
        if rc == -5 and not raise_on_nan:
            return [d.as_dict() for d in diags[:n]]
        _check(rc, "hc_step")
        return [d.as_dict() for d in diags[:n]]

    def step_nodiag(self, n: int) -> int:
        """Advance n steps without copying diagnostics back; returns the status code."""
        return self._L.hc_step(self.h, n, None)

    def scalars(self) -> dict:
        d = [ctypes.c_double() for _ in range(5)]
        st = ctypes.c_int()
        _check(self._L.hc_get_scalars(self.h, *[ctypes.byref(x) for x in d], ctypes.byref(st)), "hc_get_scalars")
        names = ["time_sim", "dpx_drive", "ubar", "got", "div_hist_max"]
        out = {k: v.value for k, v in zip(names, d)}
        out["step"] = st.value
        return out

    def grid(self) -> Dict[str, np.ndarray]:
        nka = self.p.nz + 4
        arrs = [np.zeros(nka) for _ in range(5)]
        _check(self._L.hc_get_grid(self.h, *[a.ctypes.data for a in arrs]), "hc_get_grid")
        return dict(zip(["dz", "l_t", "l_b", "dz_t", "dz_b"], arrs))

    def set_grid(self, g: Dict[str, np.ndarray]) -> None:
        arrs = [np.ascontiguousarray(g[k], dtype=np.float64) for k in ["dz", "l_t", "l_b", "dz_t", "dz_b"]]
        _check(self._L.hc_set_grid(self.h, *[a.ctypes.data for a in arrs]), "hc_set_grid")

    @property
    def last_ms(self) -> float:
        v = ctypes.c_double()
        _check(self._L.hc_last_step_ms(self.h, ctypes.byref(v)), "hc_last_step_ms")
        return v.value

    @property
    def last_launches(self) -> int:
        v = ctypes.c_longlong()
        _check(self._L.hc_last_launch_count(self.h, ctypes.byref(v)), "hc_last_launch_count")
        return v.value

    def set_profiling(self, enable: bool) -> None:
        _check(self._L.hc_set_profiling(self.h, 1 if enable else 0), "hc_set_profiling")

    def kernel_profile(self) -> Dict[str, dict]:
        """Per-kernel launch count and total CUDA-event time since profiling was enabled."""
        mx = 32
        names = ctypes.create_string_buffer(32 * mx)
        ms = (ctypes.c_double * mx)()
        nl = (ctypes.c_longlong * mx)()
        cnt = ctypes.c_int()
        _check(self._L.hc_kernel_profile(self.h, mx, names, ms, nl, ctypes.byref(cnt)), "hc_kernel_profile")
        out = {}
        for q in range(cnt.value):
            nm = names.raw[32 * q:32 * q + 32].split(b"\0")[0].decode()
            out[nm] = {"launches": nl[q], "total_ms": ms[q]}
        return out

    @property
    def mixed(self) -> bool:
        return self.p.precision == PREC_MIXED


class Ensemble:
    """Independent channels advanced together through one CUDA graph per step
    (a branch per member). The channels stay owned by the caller; step them only
    through the ensemble while it exists."""

    def __init__(self, channels):
        self._L = load_library()
        self.channels = list(channels)
        arr = (ctypes.c_void_p * len(self.channels))(*[c.h for c in self.channels])
        h = ctypes.c_void_p()
        _check(self._L.hc_ensemble_create(arr, len(self.channels), ctypes.byref(h)), "hc_ensemble_create")
        self.h = h

    def step(self, n: int = 1) -> None:
        _check(self._L.hc_ensemble_step(self.h, int(n)), "hc_ensemble_step")

    @property
    def last_ms(self) -> float:
        ms = ctypes.c_double()
        self._L.hc_ensemble_last_ms(self.h, ctypes.byref(ms), None)
        return ms.value

    @property
    def launches_per_step(self) -> int:
        n = ctypes.c_longlong()
        self._L.hc_ensemble_last_ms(self.h, None, ctypes.byref(n))
        return n.value

    def close(self) -> None:
        if getattr(self, "h", None):
            self._L.hc_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

