"""GPU parity: the CUDA engine against the CPU FP64 oracle on the same seeded
inputs, through the C-ABI (ctypes).

Tolerances (written per test): FP64 path <= 1e-10 relative (max-norm over the
field, divided by the field's max) after 10 steps; FP32-mixed path <= 1e-5 for
u, v, w, t and <= 2e-3 for p (parity_util.MIXED_P_TOL).
"""
import numpy as np
import pytest

from hercules_b200 import inputs
from hercules_b200.params import (Params, config_channel_fd, config_ekman, PREC_MIXED, MEAN_NAMES)
from parity_util import MIXED_TOL, MIXED_P_TOL, rel_err, run_pair

FP64_TOL = 1e-10


def small(**kw):
    base = dict(lx=4.0, ly=3.0, lz=2.0, nx=32, ny=24, nz=17, zstretch=1.0, ochannel=0, dp_opt=1,
                cds=2, dts=2, nu=1.0 / 300.0, alpha=1.0 / 300.0 / 0.71, dt=2e-3, imax=100)
    base.update(kw)
    return Params(**base)


CASES = {
    "fd4_closed_dp2": config_channel_fd(nx=32, ny=24, nz=17),
    "fd2_closed_dp1": small(cds=1),
    "fd4_open_scalar": small(ochannel=1, isscalar=1, got=0.5, tbot=-1.0, ttop=0.0),
    "fd2_open_scalar": small(cds=1, ochannel=1, isscalar=1, got=1.0, tbot=-1.0, ttop=0.0),
    "fd4_ab2_scalar": small(dts=1, isscalar=1, got=0.2),
    "fd4_ekman": config_ekman(nx=32, ny=32, nz=17),
    "fd4_umrf_scalar": small(u_mrf=0.4, isscalar=1, got=0.3, tbot=0.5, ttop=-0.25),
    "fd4_open_umrf_rivar": small(ochannel=1, u_mrf=-0.2, isscalar=1, is_ri_var=1, ri_str=0.1, ri_end=2.0, imax=20),
    "fd4_nonsquare_radix": small(nx=48, ny=40, nz=9),
    # Rayleigh damping: the undamped ghost cells of the reference (rayleigh_damping
    # touches the interior only) must be reproduced at the periodic seams
    "fd4_open_damp_scalar": small(ochannel=1, isscalar=1, got=0.3, tbot=-1.0, ttop=0.0,
                                  isdamp=1, nzdamp=6, cdamp=0.7),
    "fd2_closed_damp_full_depth": small(cds=1, isdamp=1, nzdamp=16, cdamp=1.0, isscalar=1, got=0.2),
    # fixed bottom-cooling flux (dT/dz = tbot at the wall) instead of a fixed wall temperature
    "fd4_open_scalar_wall_flux": small(ochannel=1, isscalar=1, got=0.5, tbc_bot=1, tbot=0.6, ttop=0.0),
    "fd2_ab2_damp_wall_flux": small(cds=1, dts=1, isscalar=1, got=0.3, tbc_bot=1, tbot=-0.2, ttop=0.5,
                                    isdamp=1, nzdamp=5, cdamp=0.6, u_mrf=0.2),
    "fd4_ab2_damp_umrf": small(dts=1, u_mrf=0.3, isdamp=1, nzdamp=3, cdamp=0.5),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_fd_fp64_parity_10_steps(name, oracle_lib, engine):
    p = CASES[name]
    fields = inputs.small_random(p, seed=7)
    o, od, rc, c, gd = run_pair(p, fields, 10, oracle_lib, engine)
    assert rc == 0
    names = ["u", "v", "w", "p"] + (["t", "ss"] if p.isscalar else []) + ["ff", "gg", "hh"]
    for f in names:
        e = rel_err(c.download(f), o.get(f))
        assert e <= FP64_TOL, f"{name}: field {f} rel err {e:.3e}"
    for f in MEAN_NAMES:
        b = o.get(f)
        if np.max(np.abs(b)) == 0:
            continue
        e = rel_err(c.download(f), b)
        assert e <= FP64_TOL, f"{name}: {f} rel err {e:.3e}"
    for a, b in zip(gd, od):
        assert a["step"] == b["step"]
        assert abs(a["time_sim"] - b["time_sim"]) <= 1e-12
        assert abs(a["cfl"] - b["cfl"]) <= FP64_TOL * max(1.0, abs(b["cfl"]))
        assert abs(a["dpx_drive"] - b["dpx_drive"]) <= FP64_TOL * max(1.0, abs(b["dpx_drive"]))
        assert abs(a["ubar"] - b["ubar"]) <= FP64_TOL * max(1.0, abs(b["ubar"]))
        assert abs(a["got"] - b["got"]) <= 1e-12 * max(1.0, abs(b["got"]))
        # divergence is round-off on both sides
        assert a["div_avg"] < 1e-9 and abs(a["div_max"]) < 1e-8
        assert a["nan_flag"] == 0
    c.close()
    o.close()


@pytest.mark.gpu
def test_config1_full_size_fp64_10_steps(oracle_lib, engine):
    """96x64x64 closed channel, FD4, RK3, dp_opt=2 from the seeded Poiseuille+10% start."""
    p = config_channel_fd()
    fields = inputs.poiseuille_noise(p, seed=1)
    o, od, rc, c, gd = run_pair(p, fields, 10, oracle_lib, engine)
    assert rc == 0
    for f in ["u", "v", "w", "p", "ff", "gg", "hh"] + MEAN_NAMES[:3] + MEAN_NAMES[4:9]:
        e = rel_err(c.download(f), o.get(f))
        assert e <= FP64_TOL, f"field {f} rel err {e:.3e}"
    assert abs(gd[-1]["ubar"] - od[-1]["ubar"]) <= 1e-12
    assert gd[-1]["div_avg"] < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["fd4_closed_dp2", "fd4_open_scalar", "fd4_open_damp_scalar", "fd4_open_scalar_wall_flux"])
def test_fd_mixed_precision_10_steps(name, oracle_lib, engine):
    p = CASES[name].replace(precision=PREC_MIXED)
    fields = inputs.small_random(p, seed=3)
    o, od, rc, c, gd = run_pair(p, fields, 10, oracle_lib, engine)
    assert rc == 0
    for f in ["u", "v", "w"] + (["t"] if p.isscalar else []):
        e = rel_err(c.download(f), o.get(f))
        assert e <= MIXED_TOL, f"{name}: field {f} rel err {e:.3e}"
    # Pressure: the FP32 round-off of u* reaches phi divided by dt at every
    # projection (not accumulated over steps); bound and measurements in
    # parity_util.MIXED_P_TOL
    pg, po = c.download("p"), o.get("p")
    e = rel_err(pg - pg.mean(), po - po.mean())
    assert e <= MIXED_P_TOL, f"{name}: p rel err {e:.3e}"
    assert gd[-1]["div_avg"] < 1e-3


@pytest.mark.gpu
def test_nan_is_reported_not_fatal(oracle_lib, engine):
    """A NaN planted in an input field ends hc_step with HC_ERR_NAN; the handle
    and the context stay usable (reference: print + stop, src/module_io.f90:135-140)."""
    p = small()
    fields = inputs.small_random(p, seed=1)
    fields["u"][3, 4, 5] = np.nan
    c = engine.Channel(p)
    c.load(fields)
    c.initialize()
    with pytest.raises(engine.HerculesError) as ei:
        c.step(2)
    assert ei.value.code == -5
    c.close()
    c2 = engine.Channel(p)
    c2.load(inputs.small_random(p, seed=1))
    c2.initialize()
    d = c2.step(1)
    assert d[0]["nan_flag"] == 0


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["fd4_ekman", "fd2_open_scalar", "fd4_open_damp_scalar"])
def test_fd_body_force_parity(name, oracle_lib, engine):
    """The body-force term (no reference counterpart) against the oracle's."""
    p = CASES[name]
    fields = inputs.small_random(p, seed=9)
    bf = inputs.gaussian_body_force(p, seed=4, amp=0.05)
    o = oracle_lib.Oracle(p)
    o.load(fields)
    o.set_body_force(*bf)
    o.initialize()
    rc, od = o.step(10)
    assert rc == 0
    c = engine.Channel(p)
    c.load(fields)
    c.set_body_force(*bf)
    c.initialize()
    c.step(10)
    for f in ["u", "v", "w", "p", "ff", "gg", "hh"]:
        e = rel_err(c.download(f), o.get(f))
        assert e <= FP64_TOL, f"{name}: field {f} rel err {e:.3e}"
    # the force changes the flow
    o2 = oracle_lib.Oracle(p)
    o2.load(fields)
    o2.initialize()
    o2.step(10)
    assert rel_err(o2.get("u"), o.get("u")) > 1e-6
    c.close()



@pytest.mark.gpu
@pytest.mark.parametrize("prec", [0, PREC_MIXED])
def test_neutral_temperature_statistics_deferred(prec, oracle_lib, engine):
    """Without a temperature equation T is frozen, and the engine adds the terms
    mean_t, mean_tt, mean_tw when they are read (from T and the growth of mean_w)
    instead of every step. Reads in between, a new T uploaded mid-run and a
    mean_w upload must give what the reference's per-step sums give (the oracle
    run through the same sequence)."""
    p = small(nz=9).replace(precision=prec)
    f0 = inputs.small_random(p, seed=12)
    t2 = f0["t"][::-1].copy() + 0.25
    tol = FP64_TOL if prec == 0 else MIXED_TOL
    o = oracle_lib.Oracle(p.replace(precision=0))
    o.load(f0)
    o.initialize()
    c = engine.Channel(p)
    c.load(f0)
    c.initialize()
    o.step(3); c.step(3)
    mid = {f: c.download(f) for f in ("mean_t", "mean_tt", "mean_tw")}
    for f, v in mid.items():
        assert rel_err(v, o.get(f)) <= tol, f
    o.step(2); c.step(2)
    o.set("t", t2); c.upload("t", t2)
    o.step(4); c.step(4)
    mw = o.get("mean_w")
    o.set("mean_w", mw); c.upload("mean_w", mw)
    o.step(3); c.step(3)
    for f in ("mean_t", "mean_tt", "mean_tw", "mean_w", "mean_ww"):
        assert rel_err(c.download(f), o.get(f)) <= tol, f
    c.close()
    o.close()
