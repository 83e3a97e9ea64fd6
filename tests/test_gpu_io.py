"""hc_upload / hc_download: the ghosted module-array layout of the reference
(leading dimensions nx+4, ny+4, ghost width 2) against the interior-only one, and
download into a caller's array, for FP64 and FP32 storage."""
import numpy as np
import pytest

from hercules_b200 import inputs
from hercules_b200.params import PREC_MIXED, Params


def _params(prec):
    return Params(lx=4.0, ly=3.0, lz=2.0, nx=16, ny=12, nz=9, zstretch=1.1, dt=2e-3, nu=1 / 300.0,
                  alpha=1 / 300.0 / 0.71, imax=10, precision=prec)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [0, PREC_MIXED], ids=["fp64", "mixed"])
def test_ghosted_and_interior_layouts_agree(engine, prec):
    p = _params(prec)
    f = inputs.small_random(p, seed=5)["u"]
    rng = np.random.default_rng(6)
    g = rng.standard_normal((p.nz + 4, p.ny + 4, p.nx + 4))        # ghost cells hold garbage
    g[2:-2, 2:-2, 2:-2] = f
    a, b = engine.Channel(p), engine.Channel(p)
    a.upload("u", f)
    b.upload("u", g, ghost=2)
    ua = a.download("u")
    assert np.array_equal(ua, b.download("u"))
    if prec == 0:
        assert np.array_equal(ua, f)
    else:
        assert np.array_equal(ua, f.astype(np.float32).astype(np.float64))
    # ghosted download: interior written, ghost cells left as they were
    out = np.full((p.nz + 4, p.ny + 4, p.nx + 4), 7.0)
    a.download("u", ghost=2, out=out)
    assert np.array_equal(out[2:-2, 2:-2, 2:-2], ua)
    inner = np.zeros_like(out, dtype=bool)
    inner[2:-2, 2:-2, 2:-2] = True
    assert np.all(out[~inner] == 7.0)
    # download into a caller's interior array
    buf = np.empty_like(ua)
    assert a.download("u", out=buf) is buf and np.array_equal(buf, ua)
    with pytest.raises(ValueError):
        a.download("u", out=np.empty((p.nz, p.ny, p.nx), dtype=np.float32))
    a.close()
    b.close()
