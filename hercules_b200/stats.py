"""Statistics post-processing of the mean fields (the numpy counterpart of the
reference's misc/Post_Processing/Plot_Mean_Profiles.m, extended with the wall
friction and the wall-normal heat flux).

The mean_* files hold time averages of u + u_mrf, v, w, t and of the products
(u+u_mrf)^2, v^2, w^2, w_c (u_x + u_mrf), w_c v_y, t^2, t w_c, where w_c is w
averaged to the cell centre and u_x, v_y the interpolants of the last sub-step
(src/module_tools.f90:362-404). As in the Matlab script, second moments become
(co)variances point by point, <a b> - <a><b>, and every quantity is then
averaged over x and y (Plot_Mean_Profiles.m:46-61).
"""
from __future__ import annotations

import os
from typing import Dict

import numpy as np

from .params import Params, mesh

MEAN_FILES = ("mean_u", "mean_v", "mean_w", "mean_t", "mean_uu", "mean_vv", "mean_ww", "mean_uw",
              "mean_vw", "mean_tt", "mean_tw")


def read_mean_fields(results: str, p: Params) -> Dict[str, np.ndarray]:
    """The mean_*.dat files of a results directory (already divided by the step count)."""
    out = {}
    for name in MEAN_FILES:
        a = np.fromfile(os.path.join(results, f"{name}.dat"), dtype=np.float64)
        out[name] = a.reshape(p.nz, p.ny, p.nx)
    return out


def profiles(means: Dict[str, np.ndarray], p: Params) -> Dict[str, np.ndarray]:
    """Horizontally averaged mean profiles and (co)variances, one value per level.

    Keys: z (cell centres), U, V, W, T, uu, vv, ww, uw, vw, tt, tw, where
    uu = <u u> - <u>^2 etc. are formed point by point before the horizontal mean."""
    m = {k.replace("mean_", ""): np.asarray(v, dtype=np.float64) for k, v in means.items()}
    hz = lambda a: a.mean(axis=(1, 2))
    out = {"z": mesh(p)["zc"].copy()}
    out["U"], out["V"], out["W"], out["T"] = hz(m["u"]), hz(m["v"]), hz(m["w"]), hz(m["t"])
    out["uu"] = hz(m["uu"] - m["u"] ** 2)
    out["vv"] = hz(m["vv"] - m["v"] ** 2)
    out["ww"] = hz(m["ww"] - m["w"] ** 2)
    out["uw"] = hz(m["uw"] - m["u"] * m["w"])
    out["vw"] = hz(m["vw"] - m["v"] * m["w"])
    out["tt"] = hz(m["tt"] - m["t"] ** 2)
    out["tw"] = hz(m["tw"] - m["t"] * m["w"])
    return out


def wall_friction(prof: Dict[str, np.ndarray], p: Params) -> Dict[str, float]:
    """Wall shear stress and friction velocity from the first cell: with the no-slip
    ghost u(0) = -u(1) - 2 u_mrf (src/module_boundary.f90:53), the wall gradient of
    the absolute velocity U = u + u_mrf is U(1) / (dz(1) / 2). The closed channel
    averages both walls (the top wall of an open channel is free-slip)."""
    d = mesh(p)["dz"]
    tau_b = p.nu * prof["U"][0] / (0.5 * d[2])
    if p.ochannel == 0:
        tau_t = p.nu * prof["U"][-1] / (0.5 * d[p.nz + 1])
        tau = 0.5 * (tau_b + tau_t)
    else:
        tau_t = float("nan")
        tau = tau_b
    return {"tau_bottom": float(tau_b), "tau_top": float(tau_t), "tau_w": float(tau),
            "u_tau": float(np.sqrt(abs(tau)))}


def heat_flux(prof: Dict[str, np.ndarray], p: Params) -> Dict[str, np.ndarray]:
    """Wall-normal heat flux: the turbulent part <t'w'> per level, the molecular part
    -alpha dT/dz at the faces between levels, and the wall fluxes through the
    ghosts t(0) = 2 tbot - t(1), t(nz+1) = 2 ttop - t(nz) (src/module_boundary.f90:
    176-183); with a fixed bottom gradient (tbc_bot = 1) the bottom flux is the
    prescribed -alpha tbot and the bottom-wall temperature t(1) - tbot dz(1)/2 is
    the quantity the flow sets. Also the two wall temperatures."""
    m = mesh(p)
    T = prof["T"]
    dzt = m["dz_t"][2:p.nz + 1]               # distance between centres k and k+1
    mol_faces = -p.alpha * np.diff(T) / dzt
    if p.tbc_bot:
        q_bot = -p.alpha * p.tbot
        t_bot = T[0] - 0.5 * p.tbot * m["dz"][2]
    else:
        q_bot = -p.alpha * (T[0] - p.tbot) / (0.5 * m["dz"][2])
        t_bot = p.tbot
    q_top = -p.alpha * (p.ttop - T[-1]) / (0.5 * m["dz"][p.nz + 1])
    return {"turbulent": prof["tw"].copy(), "molecular_faces": mol_faces, "wall_bottom": float(q_bot),
            "wall_top": float(q_top), "t_wall_bottom": float(t_bot), "t_wall_top": float(p.ttop)}


def relative_difference(a: Dict[str, np.ndarray], b: Dict[str, np.ndarray], keys=("U", "uu", "vv", "ww", "uw")):
    """max |a - b| / max |b| per profile: the statistical comparison of two runs."""
    out = {}
    for k in keys:
        den = float(np.max(np.abs(b[k])))
        out[k] = float(np.max(np.abs(a[k] - b[k]))) / den if den > 0 else float(np.max(np.abs(a[k])))
    return out
