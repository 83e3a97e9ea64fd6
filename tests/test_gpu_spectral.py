"""GPU parity of the pseudo-spectral time step (cds = 3, time_advancement_sp,
src/module_navier_stokes.f90:371-517) against the CPU FP64 oracle, through the
C-ABI.

Tolerances (written per test): FP64 <= 1e-10 relative (max-norm of the
difference over the max of the oracle field) after 10 steps; FP32-mixed
velocities <= 1e-5, pressure <= 1e-4 (parity_util.MIXED_P_TOL_SPECTRAL).
"""
import numpy as np
import pytest

from hercules_b200 import inputs
from hercules_b200.params import MEAN_NAMES, PREC_MIXED, Params, config_open_channel_spectral
from parity_util import MIXED_TOL, MIXED_P_TOL_SPECTRAL, rel_err, run_pair

MIXED_P_TOL = MIXED_P_TOL_SPECTRAL

FP64_TOL = 1e-10
PI = 3.1415926535897932


def sp(**kw):
    base = dict(lx=2 * PI, ly=PI, lz=1.0, nx=32, ny=24, nz=17, zstretch=1.0, ochannel=0, dp_opt=1,
                cds=3, dts=2, nu=1.0 / 180.0, alpha=1.0 / 180.0 / 0.71, dt=1e-3, imax=100)
    base.update(kw)
    return Params(**base)


SP_CASES = {
    # the stratified open channel, skew-symmetric advection
    "sp_open_scalar_skew": config_open_channel_spectral(nx=32, ny=24, nz=17),
    "sp_closed_dp2": sp(dp_opt=2),
    "sp_closed_scalar_umrf": sp(isscalar=1, got=0.4, tbot=0.5, ttop=-0.5, u_mrf=0.3),
    "sp_open_damp_scalar": sp(ochannel=1, isscalar=1, got=0.2, tbot=-1.0, ttop=0.0,
                              isdamp=1, nzdamp=6, cdamp=0.8),
    "sp_open_damp_skew_ekman": sp(ochannel=1, dp_opt=3, fc=0.5, ug=1.0, vg=0.2, issk=1,
                                  isdamp=1, nzdamp=4, cdamp=1.0),
    "sp_ab2_skew_scalar": sp(dts=1, issk=1, isscalar=1, got=0.3),
    "sp_radix_3_5": sp(nx=40, ny=36, nz=9, isscalar=1, got=0.1),
    "sp_ri_var": sp(ochannel=1, isscalar=1, is_ri_var=1, ri_str=0.1, ri_end=1.0, imax=20),
    # fixed bottom-cooling flux (dT/dz = tbot at the wall), the stratified open channel
    "sp_open_scalar_wall_flux": config_open_channel_spectral(nx=32, ny=24, nz=17).replace(
        tbc_bot=1, tbot=0.6, ttop=0.0),
    "sp_closed_ab2_wall_flux_umrf": sp(dts=1, isscalar=1, got=0.3, tbc_bot=1, tbot=0.3, ttop=0.5, u_mrf=0.2),
}


def _fields(p, seed):
    f = inputs.small_random(p, seed=seed)
    return f


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(SP_CASES))
def test_spectral_fp64_parity_10_steps(name, oracle_lib, engine):
    p = SP_CASES[name]
    o, od, rc, c, gd = run_pair(p, _fields(p, 11), 10, oracle_lib, engine)
    assert rc == 0
    names = ["u", "v", "w", "p", "phi", "ff", "gg", "hh"] + (["t", "ss"] if p.isscalar else [])
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
        # the spectral divergence is round-off on both sides, reported as |div|
        assert a["div_avg"] < 1e-9 and 0.0 <= a["div_max"] < 1e-8
        assert a["nan_flag"] == 0
    c.close()
    o.close()


@pytest.mark.gpu
def test_spectral_state_is_truncated(engine):
    """After a step the physical fields are images of 2/3-truncated spectra:
    their 2-D FFT has no energy at |l| >= nx/3 or |m| >= ny/3."""
    p = SP_CASES["sp_closed_dp2"]
    c = engine.Channel(p)
    c.load(_fields(p, 5))
    c.initialize()
    c.step(2)
    for name in ("u", "v", "p"):
        f = np.fft.fft2(c.download(name), axes=(1, 2))
        l = np.abs(np.fft.fftfreq(p.nx, 1.0 / p.nx))
        m = np.abs(np.fft.fftfreq(p.ny, 1.0 / p.ny))
        cut = (m[:, None] >= int(p.ny / 3.0)) | (l[None, :] >= int(p.nx / 3.0))
        assert np.abs(f[:, cut]).max() <= 1e-12 * np.abs(f).max(), name
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["sp_open_scalar_skew", "sp_open_damp_scalar", "sp_open_scalar_wall_flux"])
def test_spectral_mixed_precision_10_steps(name, oracle_lib, engine):
    p = SP_CASES[name].replace(precision=PREC_MIXED)
    o, od, rc, c, gd = run_pair(p, _fields(p, 3), 10, oracle_lib, engine)
    assert rc == 0
    for f in ["u", "v", "w"] + (["t"] if p.isscalar else []):
        e = rel_err(c.download(f), o.get(f))
        assert e <= MIXED_TOL, f"{name}: field {f} rel err {e:.3e}"
    pg, po = c.download("p"), o.get("p")
    e = rel_err(pg - pg.mean(), po - po.mean())
    assert e <= MIXED_P_TOL, f"{name}: p rel err {e:.3e}"
    assert gd[-1]["div_avg"] < 1e-3


@pytest.mark.gpu
def test_spectral_upload_after_initialize_is_refused(engine):
    p = SP_CASES["sp_closed_dp2"]
    c = engine.Channel(p)
    f = _fields(p, 1)
    c.load(f)
    c.initialize()
    with pytest.raises(engine.HerculesError) as ei:
        c.load({"u": f["u"]})
    assert ei.value.code == -6
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["sp_open_scalar_skew", "sp_open_damp_skew_ekman"])
def test_spectral_body_force_parity(name, oracle_lib, engine):
    p = SP_CASES[name]
    fields = _fields(p, 9)
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
    c.close()



@pytest.mark.gpu
@pytest.mark.parametrize("prec", [0, PREC_MIXED])
def test_products_fused_with_x_transform(prec, oracle_lib, engine):
    """The products (momentum and temperature) and their forward x transforms
    run as fused kernels (spec_products_fx) where nx/2 has an instantiation
    (32 x 24 here), and as the separate kernels otherwise (the radix-5 grid);
    both paths against the oracle, skew form with body force and temperature."""
    for name, fused in (("sp_open_scalar_skew", True), ("sp_radix_3_5", False)):
        p = SP_CASES[name].replace(issk=1, precision=prec)
        fields = _fields(p, 13)
        bf = inputs.gaussian_body_force(p, seed=2, amp=0.05)
        o = oracle_lib.Oracle(p)
        o.load(fields)
        o.set_body_force(*bf)
        o.initialize()
        rc, od = o.step(6)
        assert rc == 0
        c = engine.Channel(p)
        c.load(fields)
        c.set_body_force(*bf)
        c.initialize()
        c.set_profiling(True)
        c.step(6)
        prof = c.kernel_profile()
        # fused: the momentum and the temperature products both run fused
        assert (prof.get("spec_products_fx", {}).get("launches", 0) > 0) == fused, name
        assert (prof.get("spec_products", {}).get("launches", 0) > 0) == (not fused), name
        tol = FP64_TOL if prec == 0 else MIXED_TOL
        for f in ["u", "v", "w", "t"]:
            e = rel_err(c.download(f), o.get(f))
            assert e <= tol, f"{name}: field {f} rel err {e:.3e}"
        c.close()
        o.close()
