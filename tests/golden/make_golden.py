"""Regenerates the golden fixtures in this folder.

Each fixture holds a small seeded case of one branch of the time step (FD2/FD4,
RK3/AB2, pseudo-spectral, temperature under both bottom conditions, moving
frame, Ekman forcing, Rayleigh damping): its parameters, the checksum of its
start state (inputs.small_random with the stored seed) and the FP64 oracle's
u, v, w, p, t after the stored number of steps. They are regression fixtures of
the oracle, the CPU restatement of the reference (whose Fortran/MPI build is not
possible in this image, so no reference run backs them): tests/test_golden.py
checks that the oracle still reproduces them (CPU) and that the CUDA library
matches them without running the oracle (GPU).

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
from dataclasses import asdict

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

from hercules_b200 import inputs  # noqa: E402
from hercules_b200.params import Params  # noqa: E402

PI = 3.1415926535897932
FIELDS = ("u", "v", "w", "p", "t")
STEPS = 5


def _p(**kw):
    base = dict(lx=4.0, ly=3.0, lz=2.0, nx=16, ny=8, nz=9, zstretch=1.2, ochannel=0, dp_opt=1,
                cds=2, dts=2, nu=1.0 / 300.0, alpha=1.0 / 300.0 / 0.71, dt=2e-3, imax=100)
    base.update(kw)
    return Params(**base)


CASES = {
    "fd4_closed_rk3_dp2_scalar": _p(dp_opt=2, isscalar=1, got=0.4, tbot=-0.5, ttop=0.5),
    "fd2_open_ab2_umrf": _p(cds=1, dts=1, ochannel=1, u_mrf=0.3),
    "fd4_ekman_damp_scalar": _p(ochannel=1, dp_opt=3, fc=0.5, ug=1.0, vg=0.2, isdamp=1, nzdamp=3, cdamp=0.7,
                                isscalar=1, got=0.2, tbot=-1.0, ttop=0.0),
    "sp_open_skew_scalar_wall_flux": _p(lx=2 * PI, ly=PI, lz=1.0, cds=3, issk=1, ochannel=1, isscalar=1,
                                        got=0.5, tbc_bot=1, tbot=0.8, ttop=0.0, dt=1e-3),
    "sp_closed_ab2_dp2": _p(lx=2 * PI, ly=PI, lz=1.0, cds=3, dts=1, dp_opt=2, dt=1e-3),
}
SEED = 29


def start_state(p: Params):
    return inputs.small_random(p, seed=SEED)


def checksum(fields: dict) -> str:
    h = hashlib.sha256()
    for k in sorted(fields):
        h.update(k.encode())
        h.update(np.ascontiguousarray(fields[k], dtype=np.float64).tobytes())
    return h.hexdigest()


def params_json(p: Params) -> str:
    return json.dumps(asdict(p), sort_keys=True)


def params_from_json(s: str) -> Params:
    return Params(**json.loads(s))


def main():
    from oracle import oracle
    for name, p in CASES.items():
        f = start_state(p)
        o = oracle.Oracle(p)
        o.load(f)
        o.initialize()
        rc, _ = o.step(STEPS)
        assert rc == 0, (name, rc)
        out = {k: o.get(k) for k in FIELDS}
        o.close()
        np.savez(os.path.join(HERE, f"{name}.npz"), params=params_json(p), seed=SEED, steps=STEPS,
                 start_sha256=checksum(f), **out)
        print(name, "written")


if __name__ == "__main__":
    main()
