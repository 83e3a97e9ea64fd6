"""GPU parity of the kernels the production grids instantiate, against the CPU
FP64 oracle, through the C-ABI.

The transforms are compiled once per length (x half-lengths and y lengths 8 ...
512 of the form 2^a 3^b 5^c), each with its own passes, lines per block and
first-pass folding, and the column solves once per depth class K = ceil(nz/32).
The small parity cases of the other test files reach only the short lengths and
K <= 3, so here every compiled length and depth is run at a size the oracle
finishes in seconds: the transform length on one axis at full size with the
other axes small, the production planes (512 x 384 and 256 x 256) with 8
levels, and the column depths with a small plane.

Tolerances (per field, max-norm of the difference over the oracle field's max):
FP64 <= 1e-10 after the stated steps; FP32-mixed velocities (and temperature)
<= 1e-5. The reference's FFT is `mpi_2d_fft` (src/module_tools.f90:518-700),
its column solves `poisson_solver_fft` (src/module_poisson_solver.f90:483-658)
and `poisson_solver_fft_spec` (src/module_spectral.f90:602-746).
"""
import numpy as np
import pytest

from hercules_b200 import inputs
from hercules_b200.params import (PREC_MIXED, Params, config_channel_fd,
                                  config_open_channel_spectral)
from parity_util import rel_err

FP64_TOL = 1e-10
MIXED_TOL = 1e-5
PI = 3.1415926535897932

# every length with a compile-time transform (the x half-length nx/2 and ny)
FFT_LENGTHS = (8, 12, 16, 24, 32, 40, 48, 64, 80, 96, 128, 160, 192, 256, 320, 384, 512)


def _fd(nx, ny, nz, **kw):
    base = dict(lx=4.0, ly=3.0, lz=2.0, nx=nx, ny=ny, nz=nz, zstretch=1.0, ochannel=0, dp_opt=1,
                cds=2, dts=2, nu=1.0 / 300.0, alpha=1.0 / 300.0 / 0.71, dt=1e-3, imax=100)
    base.update(kw)
    return Params(**base)


def _sp(nx, ny, nz, **kw):
    base = dict(lx=2 * PI, ly=PI, lz=1.0, nx=nx, ny=ny, nz=nz, zstretch=1.0, ochannel=1, dp_opt=1,
                cds=3, issk=1, dts=2, nu=1.0 / 180.0, alpha=1.0 / 180.0 / 0.71, dt=1e-3, imax=100,
                isscalar=1, got=0.3, tbot=-1.0, ttop=0.0)
    base.update(kw)
    return Params(**base)


def _compare(p, fields, nsteps, oracle_lib, engine, precisions=(0, 1), extra=()):
    """One oracle run, then the GPU engine in each precision from the same state."""
    o = oracle_lib.Oracle(p)
    o.load(fields)
    o.initialize()
    rc, od = o.step(nsteps)
    assert rc == 0
    names = ["u", "v", "w", "p"] + (["t"] if p.isscalar else []) + list(extra)
    ref = {f: o.get(f) for f in names}
    o.close()
    errs = {}
    for prec in precisions:
        c = engine.Channel(p.replace(precision=prec))
        c.load(fields)
        c.initialize()
        gd = c.step(nsteps)
        assert gd[-1]["nan_flag"] == 0
        for f in names:
            errs[(prec, f)] = rel_err(c.download(f), ref[f])
        c.close()
    bad = []
    for (prec, f), e in errs.items():
        if prec == 0 and e > FP64_TOL:
            bad.append(f"FP64 {f} {e:.3e}")
        if prec == PREC_MIXED and f in ("u", "v", "w", "t") and e > MIXED_TOL:
            bad.append(f"mixed {f} {e:.3e}")
    assert not bad, "; ".join(bad)
    return errs


@pytest.mark.gpu
@pytest.mark.parametrize("n", FFT_LENGTHS)
@pytest.mark.parametrize("axis", ["x", "y"])
@pytest.mark.parametrize("method", ["fd4", "spectral"])
def test_every_transform_length(n, axis, method, oracle_lib, engine):
    """Each compiled transform length on one axis (the other axis at 16 points,
    5 levels), FD4 and pseudo-spectral, FP64 and mixed, 6 steps."""
    nx, ny = (2 * n, 16) if axis == "x" else (16, n)
    p = _fd(nx, ny, 5, isscalar=1, got=0.2) if method == "fd4" else _sp(nx, ny, 5)
    _compare(p, inputs.small_random(p, seed=21), 6, oracle_lib, engine)


PLANES = {
    # the config-3 plane (x half-length 256, y 384) in config-3 physics
    "fd4_512x384x8": config_channel_fd(nx=512, ny=384, nz=8),
    # the config-2 plane (x half-length 128, y 256) in config-2 physics
    "spectral_256x256x8": config_open_channel_spectral(nx=256, ny=256, nz=8),
    # the other method on each plane, with temperature on the FD one
    "fd4_256x256x8_scalar": _fd(256, 256, 8, ochannel=1, isscalar=1, got=0.5, tbot=-1.0, ttop=0.0),
    "spectral_512x384x8": _sp(512, 384, 8, ochannel=0, isscalar=0, lx=4 * PI, ly=4 * PI / 3, lz=2.0),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(PLANES))
def test_production_planes(name, oracle_lib, engine):
    """The production x-y planes with 8 levels, FP64 and mixed, 4 steps."""
    p = PLANES[name]
    _compare(p, inputs.small_random(p, seed=5), 4, oracle_lib, engine)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(PLANES) + ["fd4_256x192x9"])
def test_fused_2d_transforms(name, oracle_lib, engine):
    """tile[0] = -1: the fused 2-D transforms (thread-block clusters, the plane
    exchanged in distributed shared memory) on the planes that have a shape
    (512 x 384, 256 x 256, 256 x 192) against the oracle, FP64 and mixed."""
    p = PLANES[name] if name in PLANES else _fd(256, 192, 9, isscalar=1, got=0.3)
    p = p.replace(tile=[-1, 0, 0, 0])
    _compare(p, inputs.small_random(p, seed=6), 4, oracle_lib, engine)
    c = engine.Channel(p)
    c.load(inputs.small_random(p, seed=6))
    c.initialize()
    c.set_profiling(True)
    c.step(1)
    assert c.kernel_profile().get("fft2d_fwd", {}).get("launches", 0) > 0
    c.close()


DEPTHS = {
    # warp-per-column solves, K = ceil(nz/32) rows a lane
    "fd4_nz128": _fd(32, 24, 128, isscalar=1, got=0.3),
    "fd4_nz129": _fd(32, 24, 129, isscalar=1, got=0.3, ochannel=1, tbot=-1.0, ttop=0.0),
    "fd4_nz200": _fd(32, 24, 200),
    "fd4_nz256_config3_depth": config_channel_fd(nx=32, ny=24, nz=256),
    "fd2_nz256_scalar": _fd(16, 12, 256, cds=1, isscalar=1, got=0.2),
    # beyond 256 levels: one thread per column (k_column_fd, k_column_t)
    "fd4_nz300_thread_per_column": _fd(16, 12, 300, isscalar=1, got=0.2),
    # spectral column solves: the tiled kernel up to 128 levels, the warp kernel above
    "spectral_nz128_config2_depth": config_open_channel_spectral(nx=32, ny=24, nz=128),
    "spectral_nz129": _sp(16, 12, 129),
    "spectral_nz256": _sp(16, 12, 256, ochannel=0, dp_opt=2),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(DEPTHS))
def test_column_depths(name, oracle_lib, engine):
    """Every column-solve depth class the production grids use, FP64 and mixed,
    5 steps (histories and phi compared too in FP64)."""
    p = DEPTHS[name]
    extra = ("ff", "gg", "hh") if p.cds != 3 else ("phi",)
    _compare(p, inputs.small_random(p, seed=13), 5, oracle_lib, engine, extra=extra)


@pytest.mark.gpu
def test_config3_grid_statistics_and_diagnostics(oracle_lib, engine):
    """Config-3 plane: the statistics, bulk velocity and CFL of 3 FP64 steps."""
    p = config_channel_fd(nx=512, ny=384, nz=8)
    fields = inputs.poiseuille_noise(p, seed=3)
    o = oracle_lib.Oracle(p)
    o.load(fields)
    o.initialize()
    rc, od = o.step(3)
    assert rc == 0
    c = engine.Channel(p)
    c.load(fields)
    c.initialize()
    gd = c.step(3)
    for f in ("mean_u", "mean_v", "mean_w", "mean_uu", "mean_vv", "mean_ww", "mean_uw", "mean_vw"):
        b = o.get(f)
        assert rel_err(c.download(f), b) <= FP64_TOL, f
    for a, b in zip(gd, od):
        assert abs(a["cfl"] - b["cfl"]) <= FP64_TOL * abs(b["cfl"])
        assert abs(a["ubar"] - b["ubar"]) <= FP64_TOL
        assert abs(a["dpx_drive"] - b["dpx_drive"]) <= FP64_TOL * max(1.0, abs(b["dpx_drive"]))
    c.close()
    o.close()


# Grids of nx >= 64 and ny >= 32 run the strip momentum RHS (k_rhs_momentum_strip)
# in both precisions: partial tiles, several level chunks (tile[2]), both schemes,
# open/closed, temperature, AB2, and the body force
STRIP = {
    "fd4_closed_dp2_chunks": config_channel_fd(nx=96, ny=64, nz=40).replace(tile=[0, 0, 7, 0]),
    "fd2_open_scalar": _fd(64, 48, 17, cds=1, ochannel=1, isscalar=1, got=0.7, tbot=-1.0, ttop=0.0),
    "fd4_ab2_scalar_partial_tiles": _fd(160, 40, 9, dts=1, isscalar=1, got=0.3, tile=[0, 0, 4, 0]),
    "fd4_open_dp1": _fd(64, 32, 12, ochannel=1),
    "fd4_closed_scalar_wall_flux": _fd(64, 32, 17, isscalar=1, got=0.4, tbc_bot=1, tbot=0.5, ttop=1.0),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(STRIP))
def test_strip_rhs_against_oracle(name, oracle_lib, engine):
    """Both precisions through the strip RHS: FP64 <= 1e-10 and FP32-mixed
    velocities and temperature <= 1e-5 after 10 steps (histories too in FP64);
    the mixed divergence of every sub-step is reported and small."""
    p = STRIP[name]
    errs = _compare(p, inputs.small_random(p, seed=17), 10, oracle_lib, engine, extra=("ff", "gg", "hh"))
    assert max(e for (q, f), e in errs.items() if q == PREC_MIXED and f in ("u", "v", "w")) <= MIXED_TOL
    c = engine.Channel(p.replace(precision=PREC_MIXED))
    c.load(inputs.small_random(p, seed=17))
    c.initialize()
    d = c.step(2)[-1]
    nsub = 3 if p.dts == 2 else 1
    for s in range(nsub):
        assert 0.0 < d["div_avg_sub"][s] < 1e-3, (s, d["div_avg_sub"])
        assert abs(d["div_max_sub"][s]) >= d["div_avg_sub"][s]
    c.close()


@pytest.mark.gpu
def test_strip_rhs_body_force(oracle_lib, engine):
    p = config_channel_fd(nx=64, ny=32, nz=16).replace(dp_opt=1, nu=1.0 / 300.0)
    fields = inputs.small_random(p, seed=9)
    bf = inputs.gaussian_body_force(p, seed=4, amp=0.05)
    o = oracle_lib.Oracle(p)
    o.load(fields)
    o.set_body_force(*bf)
    o.initialize()
    rc, _ = o.step(10)
    assert rc == 0
    for prec, tol in ((0, FP64_TOL), (PREC_MIXED, MIXED_TOL)):
        c = engine.Channel(p.replace(precision=prec))
        c.load(fields)
        c.set_body_force(*bf)
        c.initialize()
        c.step(10)
        for f in ("u", "v", "w"):
            assert rel_err(c.download(f), o.get(f)) <= tol, (prec, f)
        c.close()
    o.close()


@pytest.mark.gpu
def test_strip_rhs_reports_nan(engine):
    """A NaN in the input reaches the check fused into the strip RHS (sub-step 2)
    or the final check, and hc_step returns HC_ERR_NAN."""
    p = config_channel_fd(nx=64, ny=32, nz=12, precision=PREC_MIXED)
    fields = inputs.small_random(p, seed=1)
    fields["v"][5, 7, 9] = np.nan
    c = engine.Channel(p)
    c.load(fields)
    c.initialize()
    with pytest.raises(engine.HerculesError) as ei:
        c.step(2)
    assert ei.value.code == -5
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name,prec", [("spectral_256x256x8", 0), ("spectral_256x256x8", PREC_MIXED),
                                       ("spectral_512x384x8", PREC_MIXED)])
def test_fused_products_are_deterministic(name, prec, engine):
    """The fused products + x transform kernels on production planes, where the
    product rows share a shared-memory buffer with the passes: two channels from
    the same state end bit-equal after 5 steps (a race between a level's
    unpacking and the next level's products would make them differ)."""
    p = PLANES[name].replace(precision=prec)
    fields = inputs.small_random(p, seed=17)
    out = []
    for _ in range(2):
        c = engine.Channel(p)
        c.load(fields)
        c.initialize()
        c.set_profiling(True)
        c.step(5)
        assert c.kernel_profile().get("spec_products_fx", {}).get("launches", 0) > 0
        out.append({f: c.download(f) for f in ("u", "v", "w", "p") + (("t",) if p.isscalar else ())})
        c.close()
    for f in out[0]:
        assert np.array_equal(out[0][f], out[1][f]), f
