"""Tile-shape autotuner for the CUDA engine.

Each tunable kernel reads one entry of ``hc_params.tile`` (0 = the built-in
default):

* [0] x-transform rows per block. 0 keeps the kernels compiled for the length
  (lengths 2^a 3^b 5^c from 8 to 512, lines per block fixed at compile time); a
  positive value selects the runtime-plan kernels with that many rows a block,
  which can win on small grids where the compiled kernels leave SMs idle.
* [1] y-transform lines per block, the same way.
* [2] momentum-RHS levels per block (the same kernel; only its grid changes).
* [3] column solve: 0 the coalescing-tile kernel, 2 the warp-per-column kernel
  without tiles, 1 one thread per column.

The default (0) is always a candidate and is measured first. Every entry is
searched on its own with the others at 0, timing its kernels with the engine's
per-launch CUDA events; a non-default value is taken only if it beats the
default by ``margin``. The combined choice is then timed over whole steps
against the all-default configuration, and the default is returned unless the
combination is faster, so ``tune`` never returns a configuration that measured
slower than the default. Results can be cached in a JSON file keyed by grid,
method and precision.
"""
from __future__ import annotations

import json
import os
from typing import Dict, List, Optional

from .engine import Channel
from .params import Params
from . import inputs

CANDIDATES = {
    # tile[0]: -1 the fused 2-D transform instead of the separate x and y kernels
    0: ("fft_x", [0, -1, 1, 2, 4, 8, 16]),
    1: ("fft_y", [0, 1, 2, 4, 8, 16]),
    2: ("rhs_momentum", [0, 4, 8, 16, 32, 64]),
    3: ("column", [0, 2, 1]),
}
# the x slot is scored on every transform kernel: its choice can replace the
# separate x and y kernels by the fused 2-D transforms
KERNELS = {0: ("fft_x_r2c", "fft_x_c2r", "fft_y_fwd", "fft_y_inv", "fft2d_fwd", "fft2d_inv"),
           1: ("fft_y_fwd", "fft_y_inv"), 2: ("rhs_momentum",), 3: ("column_fd", "column_t")}


def _fields(p: Params):
    return inputs.small_random(p, seed=3)


def _run(p: Params, tile: List[int], steps: int, profile: bool):
    """Per-kernel average launch times (profile) or the device time of `steps`
    whole steps; None if the engine refuses the tile."""
    q = p.replace(tile=list(tile))
    try:
        c = Channel(q)
    except Exception:
        return None
    try:
        c.load(_fields(q))
        c.initialize()
        c.step_nodiag(2)
        if profile:
            c.set_profiling(True)
            c.step_nodiag(steps)
            prof = c.kernel_profile()
            return {k: v["total_ms"] / max(v["launches"], 1) for k, v in prof.items()}
        c.step_nodiag(steps)
        return c.last_ms
    finally:
        c.close()


def _score(times: Dict[str, float], slot: int) -> float:
    return sum(times.get(k, 0.0) for k in KERNELS[slot])


def tune(p: Params, steps: int = 3, margin: float = 0.03, verbose: bool = False) -> List[int]:
    """Tile choice for grid/method/precision `p` (its own tile entries are ignored)."""
    default = [0, 0, 0, 0]
    base = _run(p, default, steps, profile=True)
    if base is None:
        raise ValueError("the engine refuses this configuration")
    best = list(default)
    for slot, (_, cands) in CANDIDATES.items():
        if _score(base, slot) == 0.0:
            continue                      # the kernels of this slot do not run on this path
        ref = _score(base, slot)
        chosen, chosen_t = 0, ref
        for v in cands:
            if v == 0:
                continue
            tile = list(default)
            tile[slot] = v
            t = _run(p, tile, steps, profile=True)
            if t is None:
                continue
            s = _score(t, slot)
            if verbose:
                print(f"tile[{slot}]={v}: {s:.4f} ms (default {ref:.4f})")
            if s < chosen_t and s < ref * (1.0 - margin):
                chosen, chosen_t = v, s
        best[slot] = chosen
    if best == default:
        return best
    # the combination must beat the default over whole steps, measured back to back
    t_def = min(_run(p, default, steps, profile=False) for _ in range(2))
    t_best = min(_run(p, best, steps, profile=False) for _ in range(2))
    if verbose:
        print(f"whole step: default {t_def / steps:.4f} ms, tuned {best} {t_best / steps:.4f} ms")
    return best if t_best < t_def else default


def key_of(p: Params) -> str:
    return f"{p.nx}x{p.ny}x{p.nz}:prec{p.precision}:cds{p.cds}:scalar{p.isscalar}"


def cached(p: Params, path: Optional[str], **kw) -> List[int]:
    """tune(p) through a JSON cache at `path` (None: no cache)."""
    if path is None:
        return tune(p, **kw)
    db = json.load(open(path)) if os.path.exists(path) else {}
    key = key_of(p)
    if key not in db:
        db[key] = tune(p, **kw)
        with open(path, "w") as f:
            json.dump(db, f, indent=1)
    return db[key]


def tune_members(params: List[Params], path: Optional[str] = None, **kw) -> List[Params]:
    """Tile choice for each distinct grid/method/precision of an ensemble, applied
    to every member that shares it."""
    memo: Dict[str, List[int]] = {}
    out = []
    for p in params:
        k = key_of(p)
        if k not in memo:
            memo[k] = cached(p, path, **kw)
        out.append(p.replace(tile=list(memo[k])))
    return out
