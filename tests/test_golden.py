"""The committed golden fixtures (tests/golden/, written by make_golden.py): the
oracle must still reproduce them (CPU), and the CUDA library must match them in
FP64 without the oracle running (GPU). Tolerances: oracle 1e-12 relative
(max-norm over the field's max: only the order of OpenMP-free sums can move),
CUDA FP64 1e-10, CUDA FP32-mixed u, v, w, t 1e-5."""
import glob
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402

from hercules_b200.params import PREC_MIXED  # noqa: E402
from parity_util import rel_err  # noqa: E402

FILES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))
NAMES = [os.path.splitext(os.path.basename(f))[0] for f in FILES]


def _load(name):
    z = np.load(os.path.join(HERE, "golden", name + ".npz"))
    p = make_golden.params_from_json(str(z["params"]))
    f = make_golden.start_state(p) if int(z["seed"]) == make_golden.SEED else None
    assert f is not None and make_golden.checksum(f) == str(z["start_sha256"]), "start state generator changed"
    return p, f, int(z["steps"]), {k: z[k] for k in make_golden.FIELDS}


def test_every_case_has_a_fixture():
    assert sorted(NAMES) == sorted(make_golden.CASES)


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_golden(name, oracle_lib):
    p, f, n, ref = _load(name)
    o = oracle_lib.Oracle(p)
    o.load(f)
    o.initialize()
    rc, _ = o.step(n)
    assert rc == 0
    for k, v in ref.items():
        if np.max(np.abs(v)) == 0:
            continue
        assert rel_err(o.get(k), v) <= 1e-12, k
    o.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("prec", [0, PREC_MIXED])
def test_cuda_matches_golden(name, prec, engine):
    p, f, n, ref = _load(name)
    c = engine.Channel(p.replace(precision=prec))
    c.load(f)
    c.initialize()
    c.step(n)
    for k, v in ref.items():
        if np.max(np.abs(v)) == 0 or (prec == PREC_MIXED and k == "p"):
            continue
        assert rel_err(c.download(k), v) <= (1e-10 if prec == 0 else 1e-5), k
    c.close()
