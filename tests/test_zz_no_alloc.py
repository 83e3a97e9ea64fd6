"""hc_divergence_noalloc: the divergence check for callers that cannot allocate
device memory (a host that owns every device buffer itself, e.g. through its own
arena, and lets no library call cudaMalloc). It must reproduce the divergence
diagnostic that hc_step reports for the same fields, call after call, while
using only the fixed scratch array compiled into the library.

This file is named so that pytest collects it last; it also passes when run
alone in a fresh process (the entry point sets itself up on its first call).
"""
import ctypes

import numpy as np
import pytest

from hercules_b200 import inputs
from hercules_b200.params import PREC_FP64, PREC_MIXED, Params, config_channel_fd

TOL = 1e-10   # the FP64 parity tolerance of the GPU tests


def _field_dtype(p):
    import torch
    return torch.float32 if p.precision == PREC_MIXED else torch.float64


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [PREC_FP64, PREC_MIXED])
@pytest.mark.parametrize("cds", [1, 2])
def test_noalloc_divergence_matches_step_diagnostic(engine, prec, cds):
    import torch
    p = config_channel_fd(nx=32, ny=24, nz=17, precision=prec).replace(cds=cds)
    c = engine.Channel(p)
    c.load(inputs.poiseuille_noise(p, seed=5))
    c.initialize()
    diag = c.step(3)[-1]
    # the caller's own device copies of the final fields
    fields = {}
    for name in ("u", "v", "w"):
        t = torch.empty((p.nz, p.ny, p.nx), dtype=_field_dtype(p), device="cuda")
        c.download_dev(name, t.data_ptr())
        fields[name] = t
    dz = np.ascontiguousarray(c.grid()["dz"])
    L = engine.load_library()
    cp = p.to_c()
    for call in range(2):                     # two calls in a row share the scratch array
        out = torch.full((3,), np.nan, dtype=torch.float64, device="cuda")
        rc = L.hc_divergence_noalloc(ctypes.byref(cp), dz.ctypes.data, fields["u"].data_ptr(),
                                     fields["v"].data_ptr(), fields["w"].data_ptr(), out.data_ptr(), None)
        assert rc == 0, rc
        torch.cuda.synchronize()
        avg, mx, nan = out.cpu().tolist()
        assert nan == 0.0
        assert abs(avg - diag["div_avg"]) <= TOL * max(abs(diag["div_avg"]), 1e-300), (call, avg, diag["div_avg"])
        assert abs(mx - diag["div_max"]) <= TOL * max(abs(diag["div_max"]), 1e-300), (call, mx, diag["div_max"])
    c.close()


HC_ERR_ARG, HC_ERR_PARAM, HC_ERR_SIZE = -1, -2, -8

# Arguments the entry point refuses before it touches the GPU: the pointers are
# never dereferenced, so these cases run without a device.
REJECTED = {
    "odd_nx": (dict(nx=33), 4096, HC_ERR_PARAM),
    "odd_ny": (dict(ny=25), 4096, HC_ERR_PARAM),
    "odd_nx_fp64": (dict(nx=33, precision=PREC_FP64), 4096, HC_ERR_PARAM),
    "nz_too_small": (dict(nz=1), 4096, HC_ERR_PARAM),
    "spectral_cds": (dict(cds=3), 4096, HC_ERR_ARG),
    "unknown_precision": (dict(precision=7), 4096, HC_ERR_ARG),
    "misaligned_u": (dict(), 4096 + 4, HC_ERR_ARG),
    "misaligned_fp64": (dict(precision=PREC_FP64), 4096 + 4, HC_ERR_ARG),
    "nz_beyond_scratch": (dict(nx=8, ny=8, nz=5000), 4096, HC_ERR_SIZE),
    "points_beyond_2_31": (dict(nx=2048, ny=2048, nz=1024), 4096, HC_ERR_SIZE),
}


@pytest.mark.parametrize("case", list(REJECTED))
def test_noalloc_refuses_bad_arguments_without_device_work(case):
    from hercules_b200 import build, engine
    build.build()
    L = engine.load_library()
    kw, uaddr, code = REJECTED[case]
    base = dict(nx=32, ny=24, nz=17, cds=2, precision=PREC_MIXED)
    base.update(kw)
    p = Params(**base)
    cp = p.to_c()
    dz = np.ones(p.nz + 4)
    aligned = ctypes.c_void_p(4096)
    rc = L.hc_divergence_noalloc(ctypes.byref(cp), dz.ctypes.data, ctypes.c_void_p(uaddr), aligned, aligned,
                                 aligned, None)
    assert rc == code, (case, rc)
