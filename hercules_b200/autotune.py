"""Tile-shape autotuner for the CUDA engine.

Each tunable kernel reads one entry of ``hc_params.tile`` (0 = the built-in
default): [0] x-FFT rows per block, [1] y-FFT lines per block, [2] momentum-RHS
k levels per block, [3] column-solve threads per block (only used by the
thread-per-column kernel, nz > 256). The kernels are independent, so each
entry is searched on its own with the others left automatic, timing the
kernel with the engine's per-launch CUDA events over a couple of steps.
Results can be cached in a JSON file keyed by grid and precision.
"""
from __future__ import annotations

import json
import os
from typing import Dict, List, Optional

from .engine import Channel
from .params import Params
from . import inputs

CANDIDATES = {
    0: ("fft_x", [1, 2, 4, 8, 16]),
    1: ("fft_y", [1, 2, 4, 8, 16]),
    2: ("rhs_momentum", [4, 8, 16, 32, 64]),
}
KERNELS = {0: ("fft_x_r2c", "fft_x_c2r"), 1: ("fft_y_fwd", "fft_y_inv"), 2: ("rhs_momentum",)}


def _time(p: Params, tile: List[int], steps: int = 2) -> Optional[Dict[str, float]]:
    q = p.replace(tile=list(tile))
    try:
        c = Channel(q)
    except Exception:
        return None
    try:
        c.load(inputs.poiseuille_noise(q, seed=3))
        c.initialize()
        c.step_nodiag(1)
        c.set_profiling(True)
        c.step_nodiag(steps)
        prof = c.kernel_profile()
    finally:
        c.close()
    return {k: v["total_ms"] / max(v["launches"], 1) for k, v in prof.items()}


def tune(p: Params, steps: int = 2, verbose: bool = False) -> List[int]:
    best = [0, 0, 0, 0]
    for slot, (_, cands) in CANDIDATES.items():
        scores = {}
        for v in cands:
            tile = [0, 0, 0, 0]
            tile[slot] = v
            t = _time(p, tile, steps)
            if t is None:
                continue
            scores[v] = sum(t.get(k, 0.0) for k in KERNELS[slot])
            if verbose:
                print(f"tile[{slot}]={v}: {scores[v]:.4f} ms")
        if scores:
            best[slot] = min(scores, key=scores.get)
    return best


def cached(p: Params, path: str, **kw) -> List[int]:
    key = f"{p.nx}x{p.ny}x{p.nz}:prec{p.precision}:cds{p.cds}"
    db = json.load(open(path)) if os.path.exists(path) else {}
    if key not in db:
        db[key] = tune(p, **kw)
        with open(path, "w") as f:
            json.dump(db, f, indent=1)
    return db[key]
