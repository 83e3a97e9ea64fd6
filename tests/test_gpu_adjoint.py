"""Discrete adjoint of the FD step (no reference counterpart): gradients from
hc_adjoint_forward / hc_adjoint_reverse against FP64 central finite differences
of the engine's own forward map, in random directions of the starting velocity,
pressure and body force."""
import numpy as np
import pytest

from hercules_b200 import adjoint, inputs
from hercules_b200.params import Params, config_ekman

FIELDS = ("u", "v", "w", "p")


def _run(engine, p, fields, bf, nsteps):
    c = engine.Channel(p)
    c.load(fields)
    c.set_body_force(*bf)
    c.initialize()
    c.step(nsteps)
    out = {f: c.download(f) for f in FIELDS}
    c.close()
    return out


def _objective(final, seeds):
    return sum(float(np.sum(seeds[f] * final[f])) for f in seeds)


def _direction(p, rng, with_p=True):
    shp = (p.nz, p.ny, p.nx)
    d = {f: rng.standard_normal(shp) for f in ("u", "v", "w", "p", "fx", "fy", "fz")}
    d["w"][-1] = 0.0
    d["fz"][-1] = 0.0
    if not with_p:
        d["p"][:] = 0.0
    return d


def _fd_check(engine, p, nsteps, ckpt, seeds, ndir=3, eps=1e-6, seed=11, amp_bf=0.02):
    fields = inputs.small_random(p, seed=seed)
    fields = {f: fields[f] for f in FIELDS}
    bf = inputs.gaussian_body_force(p, seed=seed + 1, amp=amp_bf)
    c = engine.Channel(p)
    c.load(fields)
    c.set_body_force(*bf)
    c.initialize()
    g = c.adjoint(nsteps, seeds, ckpt=ckpt)
    c.close()
    rng = np.random.default_rng(seed + 2)
    errs = []
    for _ in range(ndir):
        d = _direction(p, rng)
        plus = {f: fields[f] + eps * d[f] for f in FIELDS}
        minus = {f: fields[f] - eps * d[f] for f in FIELDS}
        bfp = tuple(bf[q] + eps * d[k] for q, k in enumerate(("fx", "fy", "fz")))
        bfm = tuple(bf[q] - eps * d[k] for q, k in enumerate(("fx", "fy", "fz")))
        jp = _objective(_run(engine, p, plus, bfp, nsteps), seeds)
        jm = _objective(_run(engine, p, minus, bfm, nsteps), seeds)
        fd = (jp - jm) / (2 * eps)
        ad = sum(float(np.sum(g[k] * d[k])) for k in ("u", "v", "w", "p", "fx", "fy", "fz"))
        errs.append(abs(ad - fd) / max(abs(fd), 1e-300))
    return errs


def _random_seeds(p, seed):
    rng = np.random.default_rng(seed)
    s = {f: rng.standard_normal((p.nz, p.ny, p.nx)) for f in FIELDS}
    s["w"][-1] = 0.0
    return s


SMALL = dict(lx=4.0, ly=3.0, lz=2.0, nx=16, ny=12, nz=17, zstretch=1.1, nu=1 / 300.0, alpha=1 / 300.0 / 0.71,
             dt=2e-3, imax=100, isscalar=0)


@pytest.mark.gpu
@pytest.mark.parametrize("case", [
    dict(cds=2, dts=2, dp_opt=1, ochannel=0),
    dict(cds=1, dts=2, dp_opt=1, ochannel=0, u_mrf=0.3),
    dict(cds=2, dts=1, dp_opt=1, ochannel=1),
    dict(cds=1, dts=1, dp_opt=3, ochannel=1, fc=0.5, ug=1.0, vg=0.2),
], ids=["fd4_rk3_closed", "fd2_rk3_mrf", "fd4_ab2_open", "fd2_ab2_coriolis"])
def test_adjoint_matches_central_differences(engine, case):
    p = Params(**{**SMALL, **case})
    errs = _fd_check(engine, p, nsteps=5, ckpt=2, seeds=_random_seeds(p, 5))
    assert max(errs) <= 1e-6, errs


@pytest.mark.gpu
def test_adjoint_small_ekman_wall_shear(engine):
    p = config_ekman(nx=16, ny=16, nz=17)
    errs = _fd_check(engine, p, nsteps=6, ckpt=4, seeds={"u": adjoint.wall_shear_seed(p)})
    assert max(errs) <= 1e-6, errs


@pytest.mark.gpu
def test_adjoint_leaves_the_forward_state_and_repeats(engine):
    """After the reverse sweep the handle holds the state of plain steps (bit for
    bit), and a second reverse sweep with the same seeds gives the same gradient."""
    p = Params(**{**SMALL, "cds": 2, "dts": 2, "dp_opt": 3, "ochannel": 1, "fc": 0.5, "ug": 1.0})
    fields = {f: v for f, v in inputs.small_random(p, seed=3).items() if f in FIELDS}
    bf = inputs.gaussian_body_force(p, seed=4, amp=0.02)
    ref = _run(engine, p, fields, bf, 7)
    c = engine.Channel(p)
    c.load(fields)
    c.set_body_force(*bf)
    c.initialize()
    c.adjoint_forward(7, ckpt=3)
    seeds = _random_seeds(p, 9)
    g1 = c.adjoint_reverse(seeds)
    for f in FIELDS:
        assert np.array_equal(c.download(f), ref[f]), f
    g2 = c.adjoint_reverse(seeds)
    for k in g1:
        assert np.array_equal(g1[k], g2[k]), k
    assert c.scalars()["step"] == 7
    t = c.adjoint_timing()
    assert t["forward_ms"] > 0 and t["reverse_ms"] > 0 and t["reverse_launches"] > 0
    c.step(1)                      # stepping invalidates the checkpoints
    with pytest.raises(engine.HerculesError):
        c.adjoint_reverse(seeds)
    c.close()


@pytest.mark.gpu
def test_adjoint_ekman_64_wall_shear_32_directions(engine):
    """The adjoint workload: Ekman layer 64x64x65, FP64, mean wall shear stress at
    step 50, checkpoint every 10 steps; gradient with respect to the starting
    velocity and a smooth body force, against central differences (eps = 1e-6)
    in 32 seeded random directions."""
    p = config_ekman()
    fields = {f: v for f, v in inputs.small_random(p, seed=21).items() if f in ("u", "v", "w")}
    fields["p"] = np.zeros_like(fields["u"])
    bf = inputs.gaussian_body_force(p, seed=22, ell=1.0, amp=0.01)
    seeds = {"u": adjoint.wall_shear_seed(p)}
    c = engine.Channel(p)
    c.load(fields)
    c.set_body_force(*bf)
    c.initialize()
    g = c.adjoint(50, seeds, ckpt=10)
    c.close()
    rng = np.random.default_rng(23)
    eps = 1e-6
    errs = []
    for _ in range(32):
        d = _direction(p, rng, with_p=False)
        plus = {f: fields[f] + eps * d[f] for f in FIELDS}
        minus = {f: fields[f] - eps * d[f] for f in FIELDS}
        bfp = tuple(bf[q] + eps * d[k] for q, k in enumerate(("fx", "fy", "fz")))
        bfm = tuple(bf[q] - eps * d[k] for q, k in enumerate(("fx", "fy", "fz")))
        jp = adjoint.wall_shear(_run(engine, p, plus, bfp, 50)["u"], p)
        jm = adjoint.wall_shear(_run(engine, p, minus, bfm, 50)["u"], p)
        fd = (jp - jm) / (2 * eps)
        ad = sum(float(np.sum(g[k] * d[k])) for k in ("u", "v", "w", "fx", "fy", "fz"))
        errs.append(abs(ad - fd) / max(abs(fd), 1e-300))
    assert max(errs) <= 1e-6, errs


@pytest.mark.gpu
def test_autograd_function_backward(engine):
    torch = pytest.importorskip("torch")
    p = Params(**{**SMALL, "cds": 2, "dts": 2, "dp_opt": 1, "ochannel": 0})
    f0 = inputs.small_random(p, seed=31)
    bf = inputs.gaussian_body_force(p, seed=32, amp=0.02)
    t = lambda a: torch.tensor(a, dtype=torch.float64, requires_grad=True)
    xs = [t(f0[f]) for f in FIELDS] + [t(b) for b in bf]
    c = engine.Channel(p)
    u, v, w, pr = adjoint.advance(c, 4, *xs, ckpt=2)
    j = adjoint.kinetic_energy(u, v, w) + 0.1 * pr.mean()
    j.backward()
    # the same gradient through the engine's entry points, seeds dJ/dx_N written out
    n = p.nx * p.ny * p.nz
    seeds = {"u": u.detach().numpy() / n, "v": v.detach().numpy() / n, "w": w.detach().numpy() / n,
             "p": np.full(u.shape, 0.1 / n)}
    c2 = engine.Channel(p)
    c2.load({f: f0[f] for f in FIELDS})
    c2.set_body_force(*bf)
    c2.initialize()
    g = c2.adjoint(4, seeds, ckpt=2)
    for x, k in zip(xs, ("u", "v", "w", "p", "fx", "fy", "fz")):
        assert np.allclose(x.grad.numpy(), g[k], rtol=1e-12, atol=1e-15), k
    c.close()
    c2.close()


@pytest.mark.gpu
@pytest.mark.parametrize("case", [
    dict(cds=2, dts=2, dp_opt=3, ochannel=1, fc=0.5, ug=1.0, vg=0.2),
    dict(cds=1, dts=2, dp_opt=1, ochannel=0, u_mrf=0.3),
    dict(cds=2, dts=1, dp_opt=1, ochannel=0, u_mrf=-0.2),
], ids=["fd4_rk3_ekman", "fd2_rk3_mrf", "fd4_ab2_mrf"])
def test_adjoint_matches_torch_autograd(engine, case):
    """The hand-written adjoint against autograd through the FP64 PyTorch
    restatement of the same discrete step (tests/torch_step.py)."""
    torch = pytest.importorskip("torch")
    from torch_step import TorchFD
    p = Params(**{**SMALL, **case})
    f0 = inputs.small_random(p, seed=41)
    bf = inputs.gaussian_body_force(p, seed=42, amp=0.02)
    seeds = _random_seeds(p, 43)
    nsteps = 3
    T = lambda a, g=False: torch.tensor(a, dtype=torch.float64, requires_grad=g)
    xs = [T(f0[f], True) for f in FIELDS] + [T(b, True) for b in bf]
    hist = tuple(T(np.zeros_like(f0["u"])) for _ in range(3))
    out = TorchFD(p).run(tuple(xs[:4]) + hist, nsteps, tuple(xs[4:]))
    j = sum((T(seeds[f]) * out[q]).sum() for q, f in enumerate(FIELDS))
    j.backward()
    c = engine.Channel(p)
    c.load({f: f0[f] for f in FIELDS})
    c.set_body_force(*bf)
    c.initialize()
    g = c.adjoint(nsteps, seeds, ckpt=2)
    c.close()
    for x, k in zip(xs, ("u", "v", "w", "p", "fx", "fy", "fz")):
        ref = x.grad.numpy()
        err = np.max(np.abs(g[k] - ref)) / np.max(np.abs(ref))
        assert err <= 1e-10, (k, err)


FIELDS_T = FIELDS + ("t",)


def _run_t(engine, p, fields, bf, nsteps):
    c = engine.Channel(p)
    c.load(fields)
    c.set_body_force(*bf)
    c.initialize()
    c.step(nsteps)
    out = {f: c.download(f) for f in FIELDS_T}
    c.close()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("case", [
    dict(cds=2, dts=2, dp_opt=1, ochannel=0, got=0.8),
    dict(cds=1, dts=2, dp_opt=3, ochannel=1, got=0.5, fc=0.5, ug=1.0, vg=0.2),
    dict(cds=2, dts=1, dp_opt=1, ochannel=0, got=0.8, u_mrf=0.3),
    dict(cds=1, dts=1, dp_opt=1, ochannel=1, got=-0.4),
    dict(cds=2, dts=2, dp_opt=1, ochannel=1, got=0.6, tbc_bot=1, tbot=0.4, ttop=0.0),
], ids=["fd4_rk3_closed", "fd2_rk3_ekman", "fd4_ab2_mrf", "fd2_ab2_unstable", "fd4_rk3_wall_flux"])
def test_adjoint_with_temperature_matches_central_differences(engine, case):
    """Stratified channels (constant Richardson number, buoyancy got T in the w
    equation): the gradient of <seeds, (u, v, w, p, T)_N> with respect to the
    starting u, v, w, p, T and the body force against FP64 central differences in
    random directions of all of them."""
    p = Params(**{**SMALL, **case, "isscalar": 1})
    fields = inputs.small_random(p, seed=51)
    fields = {f: fields[f] for f in FIELDS_T}
    bf = inputs.gaussian_body_force(p, seed=52, amp=0.02)
    seeds = _random_seeds(p, 53)
    seeds["t"] = np.random.default_rng(54).standard_normal((p.nz, p.ny, p.nx))
    nsteps, eps = 5, 1e-6
    c = engine.Channel(p)
    c.load(fields)
    c.set_body_force(*bf)
    c.initialize()
    g = c.adjoint(nsteps, seeds, ckpt=2)
    c.close()
    assert set(g) >= set(FIELDS_T)
    rng = np.random.default_rng(55)
    errs = []
    for _ in range(3):
        d = _direction(p, rng)
        d["t"] = rng.standard_normal((p.nz, p.ny, p.nx))
        plus = {f: fields[f] + eps * d[f] for f in FIELDS_T}
        minus = {f: fields[f] - eps * d[f] for f in FIELDS_T}
        bfp = tuple(bf[q] + eps * d[k] for q, k in enumerate(("fx", "fy", "fz")))
        bfm = tuple(bf[q] - eps * d[k] for q, k in enumerate(("fx", "fy", "fz")))
        jp = _objective(_run_t(engine, p, plus, bfp, nsteps), seeds)
        jm = _objective(_run_t(engine, p, minus, bfm, nsteps), seeds)
        fd = (jp - jm) / (2 * eps)
        ad = sum(float(np.sum(g[k] * d[k])) for k in FIELDS_T + ("fx", "fy", "fz"))
        errs.append(abs(ad - fd) / max(abs(fd), 1e-300))
    assert max(errs) <= 1e-6, errs


@pytest.mark.gpu
def test_adjoint_wall_heat_flux_per_field(engine):
    """The mean bottom-wall heat flux after 8 steps of a stably stratified closed
    channel: each of the T- and velocity-parts of the gradient separately against
    central differences (a direction in T alone, then in u, v, w alone), and the
    same gradient from two checkpoint spacings. The velocities move the wall flux
    about 1e-4 as much as T does, so their central difference takes eps = 1e-5
    (round-off of J over 2 eps |dJ| is then about 4e-6 of it) and a 1e-4 bound."""
    p = Params(**{**SMALL, "cds": 2, "dts": 2, "dp_opt": 1, "ochannel": 0, "got": 1.0, "isscalar": 1})
    fields = inputs.small_random(p, seed=61)
    fields = {f: fields[f] for f in FIELDS_T}
    bf = inputs.gaussian_body_force(p, seed=62, amp=0.02)
    seeds = {"t": adjoint.wall_heat_flux_seed(p)}
    gs = []
    for ckpt in (3, 8):
        c = engine.Channel(p)
        c.load(fields)
        c.set_body_force(*bf)
        c.initialize()
        gs.append(c.adjoint(8, seeds, ckpt=ckpt))
        c.close()
    for k in gs[0]:
        assert np.allclose(gs[0][k], gs[1][k], rtol=1e-12, atol=1e-16), k
    g = gs[0]
    rng = np.random.default_rng(63)
    for part, eps, tol in ((("t",), 1e-6, 1e-6), (("u", "v", "w"), 1e-5, 1e-4)):
        d = {f: (rng.standard_normal((p.nz, p.ny, p.nx)) if f in part else np.zeros((p.nz, p.ny, p.nx)))
             for f in FIELDS_T}
        d["w"][-1] = 0.0
        plus = {f: fields[f] + eps * d[f] for f in FIELDS_T}
        minus = {f: fields[f] - eps * d[f] for f in FIELDS_T}
        jp = adjoint.wall_heat_flux(_run_t(engine, p, plus, bf, 8)["t"], p)
        jm = adjoint.wall_heat_flux(_run_t(engine, p, minus, bf, 8)["t"], p)
        fd = (jp - jm) / (2 * eps)
        ad = sum(float(np.sum(g[k] * d[k])) for k in part)
        assert abs(ad - fd) <= tol * abs(fd), (part, ad, fd)
