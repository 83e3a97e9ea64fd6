"""Seeded synthetic initial fields for the benchmark workloads.

The reference reads its initial state from results/init_{u,v,w,p,t}.dat
(raw float64, Fortran order, interior only; src/module_tools.f90:260-316) and
its own noise option is multiplicative and unseeded (src/module_tools.f90:321-357),
so the workloads here are generated from numpy's PCG64 with fixed seeds and
handed to both the GPU path and the CPU oracle. Arrays are returned in the
interior-only Fortran layout, i.e. numpy shape (nz, ny, nx) C-order, x fastest.
"""
from __future__ import annotations

import numpy as np

from .params import Params, mesh


def _rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def poiseuille_noise(p: Params, seed: int = 1, amp: float = 0.15):
    """Laminar Poiseuille u = 1.5(1-(z-1)^2) at cell centres plus uniform
    [-amp, amp] noise on u, v, w; w = 0 on the top wall face; p = t = 0."""
    g = _rng(seed)
    zc = mesh(p)["zc"]
    h = p.lz / 2.0
    base = 1.5 * (1.0 - ((zc - h) / h) ** 2)
    shape = (p.nz, p.ny, p.nx)
    u = base[:, None, None] + g.uniform(-amp, amp, size=shape)
    v = g.uniform(-amp, amp, size=shape)
    w = g.uniform(-amp, amp, size=shape)
    w[-1] = 0.0
    u = u - p.u_mrf
    return {"u": u, "v": v, "w": w, "p": np.zeros(shape), "t": np.zeros(shape)}


def loglaw_stratified(p: Params, seed: int = 10):
    """Open-channel log-law (u+ = z+ below 11, else 2.44 ln z+ + 5.2, z+ = 180 z)
    with 5% Gaussian noise on u and 5% of u_max on v, w; linear temperature
    between tbot and ttop plus 1% noise."""
    g = _rng(seed)
    zc = mesh(p)["zc"]
    zp = 180.0 * zc
    up = np.where(zp < 11.0, zp, 2.44 * np.log(np.maximum(zp, 1e-30)) + 5.2)
    shape = (p.nz, p.ny, p.nx)
    u = up[:, None, None] * (1.0 + 0.05 * g.standard_normal(shape))
    umax = float(up.max())
    v = 0.05 * umax * g.standard_normal(shape)
    w = 0.05 * umax * g.standard_normal(shape)
    w[-1] = 0.0
    dT = p.ttop - p.tbot
    tl = p.tbot + dT * zc / p.lz
    t = tl[:, None, None] + 0.01 * abs(dT) * g.standard_normal(shape)
    return {"u": u - p.u_mrf, "v": v, "w": w, "p": np.zeros(shape), "t": t}


def small_random(p: Params, seed: int = 0, amp: float = 0.1):
    """Generic seeded state for parity tests: a smooth mean profile plus noise on
    every prognostic field, including temperature and the AB2 histories."""
    g = _rng(seed)
    zc = mesh(p)["zc"]
    shape = (p.nz, p.ny, p.nx)
    base = 1.5 * (1.0 - ((zc - p.lz / 2) / (p.lz / 2)) ** 2) if p.ochannel == 0 else np.sqrt(np.maximum(zc / p.lz, 0))
    u = base[:, None, None] + amp * g.uniform(-1, 1, shape)
    v = amp * g.uniform(-1, 1, shape)
    w = amp * g.uniform(-1, 1, shape)
    w[-1] = 0.0
    pr = amp * g.uniform(-1, 1, shape)
    t = (p.tbot + (p.ttop - p.tbot) * zc / p.lz)[:, None, None] + amp * g.uniform(-1, 1, shape)
    out = {"u": u, "v": v, "w": w, "p": pr, "t": t}
    if p.dts == 1:
        for k in ("ff", "gg", "hh", "ss"):
            out[k] = amp * g.uniform(-1, 1, shape)
        out["hh"][-1] = 0.0
    return out
