"""The PyTorch restatement of the FD step (the autograd reference of the
discrete adjoint) against the C oracle: same seeded start, a few steps, FP64."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from hercules_b200 import inputs
from hercules_b200.params import Params
from torch_step import TorchFD

FIELDS = ("u", "v", "w", "p")
CASES = [
    dict(cds=2, dts=2, dp_opt=3, ochannel=1, fc=0.5, ug=1.0, vg=0.2),
    dict(cds=1, dts=2, dp_opt=1, ochannel=0, u_mrf=0.3),
    dict(cds=2, dts=1, dp_opt=1, ochannel=0, u_mrf=-0.2),
]


def _params(case):
    return Params(lx=4.0, ly=3.0, lz=2.0, nx=16, ny=12, nz=17, zstretch=1.1, nu=1 / 300.0,
                  alpha=1 / 300.0 / 0.71, dt=2e-3, imax=100, isscalar=0, **case)


@pytest.mark.parametrize("case", CASES, ids=["fd4_rk3_ekman", "fd2_rk3_mrf", "fd4_ab2_mrf"])
def test_torch_step_matches_oracle(oracle_lib, case):
    p = _params(case)
    f0 = inputs.small_random(p, seed=7)
    bf = inputs.gaussian_body_force(p, seed=8, amp=0.02)
    o = oracle_lib.Oracle(p)
    o.load({k: f0[k] for k in FIELDS + (("ff", "gg", "hh") if p.dts == 1 else ())})
    o.set_body_force(*bf)
    o.initialize()
    rc, _ = o.step(3)
    assert rc == 0
    ref = {f: o.get(f) for f in FIELDS}
    o.close()
    t = TorchFD(p)
    T = lambda a: torch.tensor(a, dtype=torch.float64)
    hist = [T(f0[k]) if p.dts == 1 else T(np.zeros_like(f0["u"])) for k in ("ff", "gg", "hh")]
    st = tuple(T(f0[k]) for k in FIELDS) + tuple(hist)
    out = t.run(st, 3, tuple(T(b) for b in bf))
    for q, f in enumerate(FIELDS):
        a = out[q].numpy()
        b = ref[f]
        if f == "p":
            a, b = a - a.mean(), b - b.mean()
        assert np.max(np.abs(a - b)) <= 1e-11 * np.max(np.abs(b)), (f, np.max(np.abs(a - b)) / np.max(np.abs(b)))
