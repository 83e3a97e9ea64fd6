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

from .params import Params, mesh, t_line


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
    with 5% Gaussian noise on u and 5% of u_max on v, w; the linear temperature
    between the walls (params.t_line) plus 1% of its range as noise."""
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
    tl = t_line(p, zc)
    dT = p.tbot * p.lz if p.tbc_bot else p.ttop - p.tbot
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
    t = t_line(p, zc)[:, None, None] + amp * g.uniform(-1, 1, shape)
    out = {"u": u, "v": v, "w": w, "p": pr, "t": t}
    if p.dts == 1:
        for k in ("ff", "gg", "hh", "ss"):
            out[k] = amp * g.uniform(-1, 1, shape)
        out["hh"][-1] = 0.0
    return out


def gaussian_body_force(p: Params, seed: int = 4, ell: float = 1.0, amp: float = 0.01):
    """Seeded smooth body force (fx, fy, fz) for the hc_set_body_force term: white
    noise filtered to a power spectrum proportional to exp(-k^2 ell^2 / 2), with
    the horizontal filter applied by FFT (periodic) and the wall-normal one as a
    Gaussian kernel over the cell centres of the stretched grid; scaled to RMS amp.
    fz vanishes on the top-wall level, where w is not advanced."""
    g = _rng(seed)
    zc = mesh(p)["zc"]
    shape = (p.nz, p.ny, p.nx)
    kx = 2 * np.pi * np.fft.fftfreq(p.nx, p.lx / p.nx)
    ky = 2 * np.pi * np.fft.fftfreq(p.ny, p.ly / p.ny)
    hfilt = np.exp(-(ky[:, None] ** 2 + kx[None, :] ** 2) * ell ** 2 / 4.0)
    dz = zc[:, None] - zc[None, :]
    zker = np.exp(-dz ** 2 / (ell ** 2))
    zker /= zker.sum(axis=1, keepdims=True)
    out = []
    for _ in range(3):
        x = g.standard_normal(shape)
        x = np.real(np.fft.ifft2(np.fft.fft2(x, axes=(1, 2)) * hfilt[None], axes=(1, 2)))
        x = np.tensordot(zker, x, axes=(1, 0))
        x *= amp / max(np.sqrt(np.mean(x ** 2)), 1e-300)
        out.append(x)
    out[2][-1] = 0.0
    return tuple(out)


ENSEMBLE_GRIDS = ((32, 32, 33), (48, 32, 49), (64, 48, 65), (96, 64, 65))


def ensemble_members(n: int = 64, seed: int = 1000, precision: int = 0, tune: bool = False,
                     tune_cache=None):
    """Seeded ensemble of independent closed channels: grid drawn uniformly from
    ENSEMBLE_GRIDS, Re_tau ~ U[100, 300] (nu = 1/Re_tau, constant pressure drive
    dp_opt=1), Richardson number ~ U[0, 1], Pr = 0.71, stable stratification
    (t: 0 at the bottom wall, 1 at the top), laminar Poiseuille plus 10% uniform
    noise. Member q uses seed + q. With tune=True the tile shapes of each distinct
    grid come from the autotuner (needs the GPU; tune_cache: optional JSON path).
    Returns a list of (Params, fields)."""
    from .params import config_channel_fd
    out = []
    for q in range(n):
        g = _rng(seed + q)
        nx, ny, nz = ENSEMBLE_GRIDS[int(g.integers(len(ENSEMBLE_GRIDS)))]
        re_tau = float(g.uniform(100.0, 300.0))
        ri = float(g.uniform(0.0, 1.0))
        nu = 1.0 / re_tau
        p = config_channel_fd(nx, ny, nz, precision=precision).replace(
            dp_opt=1, nu=nu, alpha=nu / 0.71, isscalar=1, got=ri, tbot=0.0, ttop=1.0, dt=2e-4, imax=500)
        zc = mesh(p)["zc"]
        shape = (p.nz, p.ny, p.nx)
        ul = zc * (p.lz - zc) / (2.0 * nu)
        amp = 0.1 * float(ul.max())
        u = ul[:, None, None] + amp * g.uniform(-1, 1, shape)
        v = amp * g.uniform(-1, 1, shape)
        w = amp * g.uniform(-1, 1, shape)
        w[-1] = 0.0
        t = (zc / p.lz)[:, None, None] + 0.01 * g.uniform(-1, 1, shape)
        out.append((p, {"u": u, "v": v, "w": w, "p": np.zeros(shape), "t": t}))
    if tune:
        from .autotune import tune_members
        tuned = tune_members([p for p, _ in out], tune_cache)
        out = [(q, f) for q, (_, f) in zip(tuned, out)]
    return out
