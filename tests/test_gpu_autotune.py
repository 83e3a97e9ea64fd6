"""The tile autotuner (no reference counterpart): the configuration it returns
is never slower than the built-in default over whole steps, and every tile it
may choose gives the same fields as the default (the tiles change only how the
work is split, except the transform kernels, whose runtime-plan variants agree
to round-off)."""
import numpy as np
import pytest

from hercules_b200 import autotune, inputs
from hercules_b200.params import PREC_MIXED, config_channel_fd
from parity_util import rel_err

GRIDS = {
    "ensemble_32x32x33_mixed": config_channel_fd(32, 32, 33, precision=PREC_MIXED).replace(
        dp_opt=1, nu=1 / 200.0, alpha=1 / 142.0, isscalar=1, got=0.5, tbot=0.0, ttop=1.0, dt=2e-4),
    "channel_96x64x64_fp64": config_channel_fd(96, 64, 64),
}


def _step_ms(engine, p, steps=20, reps=3):
    best = None
    for _ in range(reps):
        c = engine.Channel(p)
        c.load(inputs.small_random(p, seed=3))
        c.initialize()
        c.step_nodiag(3)
        c.step_nodiag(steps)
        t = c.last_ms / steps
        c.close()
        best = t if best is None else min(best, t)
    return best


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(GRIDS))
def test_tune_is_never_slower_than_default(name, engine):
    p = GRIDS[name]
    tile = autotune.tune(p)
    assert len(tile) == 4
    t_def = _step_ms(engine, p.replace(tile=[0, 0, 0, 0]))
    t_tun = _step_ms(engine, p.replace(tile=tile))
    # re-measured in a separate run: equal within timing noise or faster
    assert t_tun <= 1.05 * t_def, (tile, t_tun, t_def)


@pytest.mark.gpu
@pytest.mark.parametrize("slot,value", [(0, 4), (1, 4), (2, 8), (3, 2), (3, 1)])
def test_every_tile_choice_keeps_the_results(slot, value, engine):
    p = GRIDS["channel_96x64x64_fp64"].replace(nz=33)
    fields = inputs.small_random(p, seed=8)
    tile = [0, 0, 0, 0]
    tile[slot] = value
    out = []
    for t in ([0, 0, 0, 0], tile):
        c = engine.Channel(p.replace(tile=t))
        c.load(fields)
        c.initialize()
        c.step(4)
        out.append({f: c.download(f) for f in ("u", "v", "w", "p")})
        c.close()
    for f in ("u", "v", "w", "p"):
        assert rel_err(out[1][f], out[0][f]) <= 1e-10, (slot, value, f)


@pytest.mark.gpu
def test_ensemble_members_take_tuned_tiles(engine):
    cases = inputs.ensemble_members(n=4, seed=1000, precision=PREC_MIXED, tune=True)
    grids = {}
    for p, _ in cases:
        grids.setdefault((p.nx, p.ny, p.nz), tuple(p.tile))
        assert grids[(p.nx, p.ny, p.nz)] == tuple(p.tile)
    chans = []
    for p, f in cases:
        c = engine.Channel(p)
        c.load(f)
        c.initialize()
        chans.append(c)
    e = engine.Ensemble(chans)
    e.step(2)
    assert all(np.isfinite(c.download("u")).all() for c in chans)
    e.close()
    for c in chans:
        c.close()
