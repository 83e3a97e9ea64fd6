"""Known-answer tests that pin the CPU oracle (the reference ships no tests or
golden vectors for its time step, so the oracle is pinned by results that follow
analytically from the reference's own discretisation). CPU only."""
import numpy as np
import pytest

from hercules_b200 import inputs
from hercules_b200.params import Params, config_channel_fd, mesh

PI = 3.1415926535897932


def small(**kw):
    base = dict(lx=4.0, ly=3.0, lz=2.0, nx=16, ny=12, nz=9, zstretch=1.0, ochannel=0, dp_opt=1,
                cds=2, dts=2, nu=1.0 / 300.0, alpha=1.0 / 300.0 / 0.71, dt=2e-3, imax=100)
    base.update(kw)
    return Params(**base)


def test_fft_matches_numpy_with_reference_conventions(oracle_lib):
    rng = np.random.default_rng(0)
    a = rng.standard_normal((3, 12, 24)) + 1j * rng.standard_normal((3, 12, 24))
    f = oracle_lib.fft2d(a, -1)
    ref = np.fft.fft2(a, axes=(1, 2)) / (12 * 24)
    ref[:, 6, :] = 0
    ref[:, :, 12] = 0
    assert np.abs(f - ref).max() < 1e-15
    b = oracle_lib.fft2d(f, 1)
    assert np.abs(b - np.fft.ifft2(ref, axes=(1, 2)) * (12 * 24)).max() < 1e-13


@pytest.mark.parametrize("n", [6, 10, 18, 30, 48, 96])
def test_fft_mixed_radix_lengths(oracle_lib, n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal((2, n, n)) + 0j
    f = oracle_lib.fft2d(a, -1)
    ref = np.fft.fft2(a, axes=(1, 2)) / (n * n)
    ref[:, n // 2, :] = 0
    ref[:, :, n // 2] = 0
    assert np.abs(f - ref).max() < 1e-14


@pytest.mark.parametrize("ochannel", [0, 1])
def test_mesh_matches_tanh_formula(oracle_lib, ochannel):
    p = small(ochannel=ochannel, zstretch=1.1, nz=17)
    o = oracle_lib.Oracle(p)
    g = o.grid()
    m = mesh(p)
    for k in ("dz", "l_t", "l_b", "dz_t", "dz_b"):
        assert np.allclose(g[k], m[k], rtol=1e-13, atol=1e-14)   # libm tanh may differ by an ulp
    dz = g["dz"][2:p.nz + 2]
    assert abs(dz.sum() - p.lz) < 1e-13
    if ochannel == 0:
        assert np.allclose(dz, dz[::-1], atol=1e-15)      # symmetric closed channel
    else:
        assert np.all(np.diff(dz) > 0)                     # refined at the bottom wall only


def _discrete_poiseuille(p):
    """Steady profile of the reference's discrete operator: nu * Lz u = -1 with the
    no-slip ghosts u(0) = -u(1), u(nz+1) = -u(nz)."""
    m = mesh(p)
    nz = p.nz
    dz, dzt, dzb = m["dz"][2:nz + 2], m["dz_t"][2:nz + 2], m["dz_b"][2:nz + 2]
    A = np.zeros((nz, nz))
    for k in range(nz):
        a, c = 1.0 / dzb[k] / dz[k], 1.0 / dzt[k] / dz[k]
        A[k, k] = -a - c
        if k > 0:
            A[k, k - 1] = a
        else:
            A[k, k] -= a
        if k < nz - 1:
            A[k, k + 1] = c
        else:
            A[k, k] -= c
    return np.linalg.solve(p.nu * A, -np.ones(nz))


@pytest.mark.parametrize("dts", [1, 2])
def test_discrete_poiseuille_is_a_fixed_point(oracle_lib, dts):
    """Constant-friction closed channel (dp_opt=1): the discrete Poiseuille profile
    satisfies nu Lz u + 1 = 0, the nonlinear terms vanish for u(z), and the RK3
    coefficients obey rk_a + rk_b = rk_c (AB2: 1.5 - 0.5 = 1), so the step must
    leave it unchanged."""
    p = small(dts=dts, dp_opt=1)
    uz = _discrete_poiseuille(p)
    shape = (p.nz, p.ny, p.nx)
    f = {"u": np.broadcast_to(uz[:, None, None], shape).copy(), "v": np.zeros(shape),
         "w": np.zeros(shape), "p": np.zeros(shape), "t": np.zeros(shape)}
    if dts == 1:
        f.update(ff=np.ones(shape), gg=np.zeros(shape), hh=np.zeros(shape), ss=np.zeros(shape))
    o = oracle_lib.Oracle(p)
    o.load(f)
    o.initialize()
    rc, d = o.step(4)
    assert rc == 0
    assert np.abs(o.get("u") - f["u"]).max() < 1e-12 * np.abs(f["u"]).max()
    for name in ("v", "w", "p"):
        assert np.abs(o.get(name)).max() < 1e-10
    assert d[-1]["div_avg"] < 1e-13


def _helm_numpy(p, rhs, rk_c):
    """Independent numpy restatement of poisson_solver_fft for the u equation
    (src/module_poisson_solver.f90:181-282, 483-658): FFT, per-mode tridiagonal
    with the builder's first-mode-only wall folds, inverse FFT."""
    nx, ny, nz = p.nx, p.ny, p.nz
    m = mesh(p)
    dz, dzt, dzb = m["dz"][2:nz + 2], m["dz_t"][2:nz + 2], m["dz_b"][2:nz + 2]
    dx2, dy2 = (p.lx / nx) ** 2, (p.ly / ny) ** 2
    aa0 = -0.5 * p.dt * p.nu / dz / dzb
    cc0 = -0.5 * p.dt * p.nu / dz / dzt
    th = lambda l, n: 2 * PI * l / n
    l = np.fft.fftfreq(nx, 1.0 / nx)
    mm = np.fft.fftfreq(ny, 1.0 / ny)
    kx = p.dt * (-2 * np.cos(2 * th(l, nx)) + 32 * np.cos(th(l, nx)) - 30) / 24 * p.nu / dx2
    ky = p.dt * (-2 * np.cos(2 * th(mm, ny)) + 32 * np.cos(th(mm, ny)) - 30) / 24 * p.nu / dy2
    src = np.fft.fft2(rhs, axes=(1, 2)) / (nx * ny)
    src[:, ny // 2, :] = 0
    src[:, :, nx // 2] = 0
    out = np.zeros_like(src)
    for j in range(ny):
        for i in range(nx):
            first = (i == 0 and j == 0)
            b = np.zeros(nz)
            a = rk_c * aa0.copy()
            c = rk_c * cc0.copy()
            for k in range(nz):
                diag = -kx[i] - ky[j]
                diag += -(aa0[k] if (k > 0 or first) else 0.0) - (cc0[k] if (k < nz - 1 or first) else 0.0)
                if first and k == 0:
                    diag -= aa0[k]
                if first and k == nz - 1:
                    diag -= cc0[k]
                b[k] = 1 + rk_c * diag
            a[0] = 0.0
            c[-1] = 0.0
            M = np.diag(b) + np.diag(a[1:], -1) + np.diag(c[:-1], 1)
            out[:, j, i] = np.linalg.solve(M, src[:, j, i])
    out[:, ny // 2, :] = 0
    out[:, :, nx // 2] = 0
    return np.real(np.fft.ifft2(out, axes=(1, 2)) * (nx * ny))


def test_helmholtz_solver_matches_numpy_restatement(oracle_lib):
    p = small(nx=8, ny=6, nz=7)
    rng = np.random.default_rng(3)
    rhs = rng.standard_normal((p.nz, p.ny, p.nx))
    o = oracle_lib.Oracle(p)
    got = o.helmholtz_u(rhs, 2.0 / 15.0)
    ref = _helm_numpy(p, rhs, 2.0 / 15.0)
    assert np.abs(got - ref).max() < 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("cds", [1, 2])
def test_projection_is_divergence_free(oracle_lib, cds):
    p = small(cds=cds, isscalar=1, got=0.5)
    o = oracle_lib.Oracle(p)
    o.load(inputs.small_random(p, seed=11))
    o.initialize()
    rc, d = o.step(3)
    assert rc == 0
    for dd in d:
        assert dd["div_avg"] < 1e-13
        assert max(abs(x) for x in dd["div_max_sub"]) < 1e-12


def test_constant_flow_rate_controller_drives_ubar_to_one(oracle_lib):
    """dp_opt=2: dpx_drive -= (ubar + u_mrf - 1) nu every sub-step
    (src/module_parameters.f90:594-613)."""
    p = config_channel_fd(nx=16, ny=12, nz=17)
    f = inputs.poiseuille_noise(p, seed=2)
    o = oracle_lib.Oracle(p)
    o.load(f)
    o.initialize()
    rc, d = o.step(3)
    assert rc == 0
    ub = [x["ubar"] for x in d]
    dp = [x["dpx_drive"] for x in d]
    assert all(abs(u - 1.0) < 0.02 for u in ub)
    # the controller pushes against the bulk-velocity excess
    assert (dp[1] - dp[0]) * (ub[0] - 1.0) < 0


def test_nan_input_stops_with_error(oracle_lib):
    p = small()
    f = inputs.small_random(p, seed=1)
    f["v"][2, 3, 4] = np.nan
    o = oracle_lib.Oracle(p)
    o.load(f)
    o.initialize()
    rc, d = o.step(2)
    assert rc == -5


def _linear_t(p, g, t0=0.3):
    """A wall-normal T profile with the discrete gradient g between all centres,
    T(k+1) = T(k) + g dz_t(k), and the top-wall value ttop that makes the ghost
    2 ttop - T(nz-1) continue it."""
    m = mesh(p)
    dzt = m["dz_t"][2:p.nz + 2]
    tz = t0 + g * np.concatenate([[0.0], np.cumsum(dzt[:-1])])
    return tz, tz[-1] + 0.5 * g * dzt[-1]


@pytest.mark.parametrize("dts", [1, 2])
@pytest.mark.parametrize("tbc_bot", [0, 1])
def test_conduction_profile_with_wall_gradient_is_steady(oracle_lib, dts, tbc_bot):
    """Poiseuille flow over a linear temperature profile on a stretched grid: the
    nonlinear terms vanish, the discrete diffusion of a linear profile vanishes
    at every level once the bottom ghost continues it, and the buoyancy of a
    horizontally uniform T is balanced by the pressure, so the step must leave
    T unchanged. tbc_bot = 1 prescribes the gradient itself (tbot = dT/dz), the
    reference's fixed wall temperature the wall value of the same line."""
    g = 0.8
    p = small(dts=dts, dp_opt=1, zstretch=1.5, isscalar=1, got=0.5, tbc_bot=tbc_bot)
    tz, ttop = _linear_t(p, g)
    dzb0 = mesh(p)["dz_b"][2]
    p = p.replace(ttop=ttop, tbot=g if tbc_bot else tz[0] - 0.5 * g * dzb0)
    uz = _discrete_poiseuille(p)
    shape = (p.nz, p.ny, p.nx)
    f = {"u": np.broadcast_to(uz[:, None, None], shape).copy(), "v": np.zeros(shape),
         "w": np.zeros(shape), "p": np.zeros(shape), "t": np.broadcast_to(tz[:, None, None], shape).copy()}
    if dts == 1:
        f.update(ff=np.ones(shape), gg=np.zeros(shape), hh=np.zeros(shape), ss=np.zeros(shape))
    o = oracle_lib.Oracle(p)
    o.load(f)
    o.initialize()
    rc, d = o.step(4)
    assert rc == 0
    assert np.abs(o.get("t") - f["t"]).max() < 1e-12 * np.abs(f["t"]).max()
    assert np.abs(o.get("w")).max() < 1e-10
    o.close()


def test_wall_gradient_condition_changes_the_mean_temperature(oracle_lib):
    """A uniform temperature under the two bottom conditions: a fixed wall value
    below it cools the first level, a fixed gradient g > 0 (heat leaving through
    the wall) cools it too, by a different amount, and levels far from the wall
    stay untouched after one step in both."""
    shape_p = small(isscalar=1, got=0.0, nz=17, ttop=1.0)
    shape = (shape_p.nz, shape_p.ny, shape_p.nx)
    f = {"u": np.zeros(shape), "v": np.zeros(shape), "w": np.zeros(shape), "p": np.zeros(shape),
         "t": np.ones(shape)}
    out = {}
    for tbc_bot, tbot in ((0, 0.0), (1, 0.5)):
        o = oracle_lib.Oracle(shape_p.replace(tbc_bot=tbc_bot, tbot=tbot, dp_opt=1))
        o.load(f)
        o.initialize()
        rc, _ = o.step(1)
        assert rc == 0
        out[tbc_bot] = o.get("t").mean(axis=(1, 2))
        o.close()
    for t in out.values():
        assert t[0] < 1.0 - 1e-6
        assert np.abs(t[6:11] - 1.0).max() < 1e-12
    assert abs(out[0][0] - out[1][0]) > 1e-6
