"""Helpers shared by the GPU parity tests: run the same seeded state through
the CUDA engine and through the CPU oracle and compare."""
import numpy as np


def rel_err(a, b):
    den = float(np.max(np.abs(b)))
    num = float(np.max(np.abs(np.asarray(a) - np.asarray(b))))
    if den == 0.0:
        return num
    return num / den


def run_pair(p, fields, nsteps, oracle_mod, engine_mod):
    o = oracle_mod.Oracle(p)
    o.load(fields)
    o.initialize()
    rc_o, od = o.step(nsteps)
    c = engine_mod.Channel(p)
    c.load(fields)
    c.initialize()
    gd = c.step(nsteps)
    return o, od, rc_o, c, gd
