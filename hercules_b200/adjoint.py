"""Differentiable FD time advancement over the discrete adjoint kernels.

``Advance`` is a ``torch.autograd.Function``: its forward runs N steps of the
engine (``hc_adjoint_forward``, a checkpoint every ``ckpt`` steps) and returns
the final u, v, w, p; its backward hands the incoming gradients to
``hc_adjoint_reverse`` as seeds and returns the gradients with respect to the
starting u, v, w, p and the body force. PyTorch is only the autograd plumbing:
both passes run in the CUDA library; the tensors cross the C-ABI as host
float64 arrays.

The objectives of the adjoint workload are plain functions of the final fields:
the mean wall shear stress of the bottom wall (the first-cell gradient through
the no-slip ghost u(0) = -u(1) - 2 u_mrf, src/module_boundary.f90:53) and the
mean kinetic energy. No counterpart in the reference.
"""
from __future__ import annotations

from typing import Optional

import numpy as np

from .params import Params, mesh


def wall_shear(u, p: Params):
    """nu dU/dz at the bottom wall, averaged over the wall: nu (u(1) + u_mrf) / (dz(1)/2)."""
    dz1 = mesh(p)["dz"][2]
    return p.nu * ((u[0] + p.u_mrf).mean()) / (0.5 * dz1)


def wall_shear_seed(p: Params) -> np.ndarray:
    """d(wall_shear)/du as a field: nu / (dz(1)/2) / (nx ny) on the first level."""
    s = np.zeros((p.nz, p.ny, p.nx))
    s[0] = p.nu / (0.5 * mesh(p)["dz"][2]) / (p.nx * p.ny)
    return s


def wall_heat_flux(t, p: Params):
    """alpha dT/dz at the bottom wall, averaged over the wall, with the Dirichlet
    ghost T(0) = 2 tbot - T(1) (src/module_boundary.f90:180): alpha (T(1) - tbot) / (dz(1)/2)."""
    dz1 = mesh(p)["dz"][2]
    return p.alpha * ((t[0] - p.tbot).mean()) / (0.5 * dz1)


def wall_heat_flux_seed(p: Params) -> np.ndarray:
    """d(wall_heat_flux)/dT as a field: alpha / (dz(1)/2) / (nx ny) on the first level."""
    s = np.zeros((p.nz, p.ny, p.nx))
    s[0] = p.alpha / (0.5 * mesh(p)["dz"][2]) / (p.nx * p.ny)
    return s


def kinetic_energy(u, v, w):
    """Mean of (u^2 + v^2 + w^2) / 2 over the stored points."""
    return 0.5 * ((u ** 2).mean() + (v ** 2).mean() + (w ** 2).mean())


def _torch():
    import torch
    return torch


def make_advance():
    """The autograd Function (built lazily so that importing this module needs no torch)."""
    torch = _torch()

    class Advance(torch.autograd.Function):
        @staticmethod
        def forward(ctx, channel, nsteps: int, ckpt: int, u0, v0, w0, p0, fx, fy, fz):
            to_np = lambda t: t.detach().to("cpu", torch.float64).numpy()
            channel.load({"u": to_np(u0), "v": to_np(v0), "w": to_np(w0), "p": to_np(p0)})
            channel.set_body_force(to_np(fx), to_np(fy), to_np(fz))
            channel.initialize()
            channel.adjoint_forward(nsteps, ckpt)
            ctx.channel = channel
            ctx.device = u0.device
            out = [torch.from_numpy(channel.download(f)).to(u0.device) for f in ("u", "v", "w", "p")]
            return tuple(out)

        @staticmethod
        def backward(ctx, gu, gv, gw, gp):
            to_np = lambda t: None if t is None else t.detach().to("cpu", torch.float64).contiguous().numpy()
            g = ctx.channel.adjoint_reverse({"u": to_np(gu), "v": to_np(gv), "w": to_np(gw), "p": to_np(gp)})
            dev = ctx.device
            t = lambda a: torch.from_numpy(a).to(dev)
            return (None, None, None, t(g["u"]), t(g["v"]), t(g["w"]), t(g["p"]),
                    t(g["fx"]), t(g["fy"]), t(g["fz"]))

    return Advance


_ADVANCE = None


def advance(channel, nsteps: int, u0, v0, w0, p0, fx, fy, fz, ckpt: int = 10):
    """Differentiable (u_N, v_N, w_N, p_N) = N steps of `channel` from (u0, v0, w0,
    p0) under the body force (fx, fy, fz): float64 tensors of shape (nz, ny, nx)."""
    global _ADVANCE
    if _ADVANCE is None:
        _ADVANCE = make_advance()
    return _ADVANCE.apply(channel, nsteps, ckpt, u0, v0, w0, p0, fx, fy, fz)
