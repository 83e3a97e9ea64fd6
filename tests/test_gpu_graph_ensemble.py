"""CUDA-graph stepping and the multi-channel ensemble (no reference counterpart):
both replay exactly the kernels of hc_step, so their results must equal eager
stepping bit for bit, member by member."""
import numpy as np
import pytest

from hercules_b200 import inputs
from hercules_b200.params import PREC_MIXED, Params, config_channel_fd
from parity_util import MIXED_P_TOL

PI = 3.1415926535897932


def _channel(engine, p, seed, graph=False, bf=None):
    c = engine.Channel(p)
    c.load(inputs.small_random(p, seed=seed))
    if bf is not None:
        c.set_body_force(*bf)
    c.initialize()
    if graph:
        c.set_graph(True)
    return c


@pytest.mark.gpu
@pytest.mark.parametrize("cds", [2, 3])
def test_graph_replay_equals_eager_across_diag_ring_wrap(engine, cds):
    p = Params(lx=4.0, ly=3.0, lz=2.0, nx=32, ny=24, nz=17, cds=cds, dts=2, dp_opt=2, nu=1 / 300.0,
               alpha=1 / 300.0 / 0.71, dt=1e-3, imax=1000, isscalar=1, got=0.2)
    a = _channel(engine, p, 3)
    b = _channel(engine, p, 3, graph=True)
    da = a.step(300)          # more steps than the 256-record diagnostics ring
    db = b.step(300)
    for f in ("u", "v", "w", "p", "t", "mean_uu"):
        assert np.array_equal(a.download(f), b.download(f)), f
    assert [d["step"] for d in db] == list(range(1, 301))
    for x, y in zip(da, db):
        assert x == y
    a.close()
    b.close()


@pytest.mark.gpu
def test_ensemble_members_equal_individual_runs(engine):
    members = [
        config_channel_fd(nx=32, ny=32, nz=33),
        config_channel_fd(nx=48, ny=32, nz=49, precision=PREC_MIXED),
        Params(lx=2 * PI, ly=PI, lz=1.0, nx=32, ny=24, nz=17, ochannel=1, cds=3, issk=1, dts=2, dp_opt=1,
               nu=1 / 180.0, alpha=1 / 180.0 / 0.71, dt=1e-3, isscalar=1, got=0.3),
        config_channel_fd(nx=64, ny=48, nz=65).replace(isscalar=1, got=0.5, dp_opt=1),
    ]
    bf = inputs.gaussian_body_force(members[0], seed=4, amp=0.02)
    ens_ch = [_channel(engine, p, 20 + q, bf=bf if q == 0 else None) for q, p in enumerate(members)]
    ref_ch = [_channel(engine, p, 20 + q, bf=bf if q == 0 else None) for q, p in enumerate(members)]
    e = engine.Ensemble(ens_ch)
    e.step(6)
    assert e.last_ms > 0 and e.launches_per_step > 4 * 20
    for c in ref_ch:
        c.step(6)
    for q, (x, y) in enumerate(zip(ens_ch, ref_ch)):
        prec = members[q].precision
        for f in ("u", "v", "w", "p", "t", "mean_u"):
            a, b = x.download(f), y.download(f)
            if prec == PREC_MIXED:
                tol = MIXED_P_TOL if f == "p" else 1e-5
                assert np.max(np.abs(a - b)) <= tol * max(float(np.max(np.abs(b))), 1e-30), (q, f)
            else:
                assert np.array_equal(a, b), (q, f)
        if prec != PREC_MIXED:
            assert x.scalars() == y.scalars()
    e.close()
    for c in ens_ch + ref_ch:
        c.close()


@pytest.mark.gpu
def test_ensemble_config_generator_runs(engine):
    """A few members of the seeded ensemble configuration step without NaN."""
    cases = inputs.ensemble_members(n=6, seed=1000)
    chans = []
    for p, fields in cases:
        c = engine.Channel(p)
        c.load(fields)
        c.initialize()
        chans.append(c)
    e = engine.Ensemble(chans)
    e.step(3)
    for c in chans:
        assert c.scalars()["step"] == 3
    e.close()
    for c in chans:
        c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [0, PREC_MIXED])
def test_grouped_ensemble_equals_individual_runs(engine, prec):
    """FD members advance through grouped launches (the i-th kernel of every member
    in one launch per kernel variant): a step of 12 members of four grids, with
    temperature, a body force and an AB2 member, takes far fewer launches than
    the members' own. With FP64 storage every member ends bit-equal to stepping
    it alone; with FP32 storage the grouped kernel is a separate compilation of
    the same body, whose FMA contractions may differ from the member's own
    kernel, so members agree to FP32 round-off (1e-5 relative, the mixed parity
    tolerance)."""
    grids = inputs.ENSEMBLE_GRIDS
    members = []
    for q in range(12):
        nx, ny, nz = grids[q % 4]
        p = config_channel_fd(nx, ny, nz, precision=prec).replace(
            dp_opt=1, nu=1.0 / (100.0 + 15 * q), alpha=1.0 / (71.0 + 10 * q), isscalar=1, got=0.05 * q,
            tbot=0.0, ttop=1.0, dt=2e-4)
        if q == 5:
            p = p.replace(dts=1)
        members.append(p)
    bf = inputs.gaussian_body_force(members[2], seed=4, amp=0.02)
    ens_ch = [_channel(engine, p, 40 + q, bf=bf if q == 2 else None) for q, p in enumerate(members)]
    ref_ch = [_channel(engine, p, 40 + q, bf=bf if q == 2 else None) for q, p in enumerate(members)]
    e = engine.Ensemble(ens_ch)
    e.step(5)
    solo = 0
    for c in ref_ch:
        c.step(5)
        solo = max(solo, c.last_launches // 5)
    # grouped: at most a few launches per kernel position, not one per member
    assert e.launches_per_step <= 5 * solo, (e.launches_per_step, solo)
    assert e.launches_per_step < len(members) * solo // 2
    for q, (x, y) in enumerate(zip(ens_ch, ref_ch)):
        for f in ("u", "v", "w", "p", "t", "ff", "mean_u", "mean_tw"):
            a, b = x.download(f), y.download(f)
            if prec == PREC_MIXED:
                # FP32 round-off of u* reaches p through phi = P^-1 div(u*) / dt,
                # amplified as in the mixed-vs-FP64 comparison (MIXED_P_TOL); the
                # history ff is the right-hand side itself, whose rounding no solve
                # damps (measured up to 1.0e-5 after 5 steps)
                tol = MIXED_P_TOL if f == "p" else (1e-4 if f == "ff" else 1e-5)
                assert np.max(np.abs(a - b)) <= tol * max(float(np.max(np.abs(b))), 1e-30), (q, f)
            else:
                assert np.array_equal(a, b), (q, f)
        if prec != PREC_MIXED:
            assert x.scalars() == y.scalars()
    e.close()
    for c in ens_ch + ref_ch:
        c.close()
