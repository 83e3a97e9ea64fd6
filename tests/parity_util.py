"""Helpers shared by the GPU parity tests: run the same seeded state through
the CUDA engine and through the CPU oracle and compare."""
import numpy as np

# FP32-mixed tolerances (relative, max-norm over the field's max). Velocities and
# temperature: 1e-5 after 10 steps (measured 1e-6 to 7e-6; they drift by about
# 2.5e-7 a step). Pressure: FP32 round-off of the right-hand side reaches u* and,
# through phi = P^-1 div(u*) / dt, the pressure, so its error is set afresh by
# every projection: it does not grow with the steps and scales as 1/dt (at
# 32x24x17, closed FD4 channel: 9.4e-4 after 1 step and 9.0e-4 after 40 at
# dt = 1e-3, 2.7e-3 and 4.8e-3 after 1 step at dt = 5e-4 and 2.5e-4). The bound
# is twice the largest error of the mixed parity cases after 10 steps (FD: 1.03e-3,
# closed channel fd4_closed_dp2; spectral: 4.8e-5).
MIXED_TOL = 1e-5
MIXED_P_TOL = 2e-3
MIXED_P_TOL_SPECTRAL = 1e-4


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
