"""FP64 PyTorch restatement of the FD time step, differentiable by autograd.

Test infrastructure: the reference for the hand-written discrete adjoint. It
restates time_advancement_fd (src/module_navier_stokes.f90:290-354) for the
options the adjoint covers (cds = 1 or 2, RK3 or AB2, dp_opt = 1 or 3, no
temperature, no damping, body force) directly in physical space with torch
operations, so that autograd supplies the exact gradient of the same discrete
map:

* the momentum right-hand side of get_momentum_cnvdiff
  (src/module_cnvdiff.f90:35-374) over the interpolants of
  get_interp_fields_uvwhxyz (src/module_tools.f90:410-468) with the wall ghosts
  of update_boundary_uvwhxyz (src/module_boundary.f90:27-300);
* the implicit solves of poisson_solver_fft (src/module_poisson_solver.f90:483-658)
  on the full complex 2-D spectrum of mpi_2d_fft (src/module_tools.f90:518-700:
  forward e^{-i} divided by the length, both Nyquist modes zeroed), with the
  wall-normal matrices of get_u/w/p_eqn_coeff (src/module_poisson_solver.f90:32-477,
  the wall folds on the (0,0) mode only) as dense batched solves;
* the pressure source get_p_eqn_src (:127-176), the projection calculate_uvw
  (src/module_navier_stokes.f90:659-734) and calculate_new_p (:739-808).

The horizontal Fourier symbols are not written out: each is the DFT of its
physical stencil applied to a unit impulse, so the spectral solve uses exactly
the operators of the physical-space code.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from hercules_b200.params import Params, mesh

RK_A = (8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0)
RK_B = (0.0, -17.0 / 60.0, -5.0 / 12.0)
RK_C = (8.0 / 15.0, 2.0 / 15.0, 1.0 / 3.0)


def sx(a, s):
    """a(i + s) along x (periodic)."""
    return torch.roll(a, shifts=-s, dims=-1)


def sy(a, s):
    """a(j + s) along y (periodic)."""
    return torch.roll(a, shifts=-s, dims=-2)


class TorchFD:
    def __init__(self, p: Params):
        if p.cds not in (1, 2) or p.isscalar != 0 or p.isdamp != 0 or p.dp_opt not in (1, 3):
            raise ValueError("the restatement covers cds 1/2, dp_opt 1/3, no scalar, no damping")
        self.p = p
        m = mesh(p)
        t = lambda a: torch.tensor(np.asarray(a[2:p.nz + 2], dtype=np.float64))
        tg = lambda a: torch.tensor(np.asarray(a, dtype=np.float64))
        self.dz, self.dzt, self.dzb, self.lt = t(m["dz"]), t(m["dz_t"]), t(m["dz_b"]), t(m["l_t"])
        self.dz_all = tg(m["dz"])          # Fortran index k at [k-1], ghosts included
        self.dx, self.dy = p.lx / p.nx, p.ly / p.ny
        self._symbols()

    # ---------------------------------------------------------------- stencils
    def d1(self, a, dim, h):
        """Staggered first difference to the cell point: cds=2 (-a(+1) + 27 a(0) - 27 a(-1) + a(-2)) / 24h."""
        s = sx if dim == "x" else sy
        if self.p.cds == 1:
            return (a - s(a, -1)) / h
        return (-s(a, 1) + 27 * a - 27 * s(a, -1) + s(a, -2)) / 24.0 / h

    def g1(self, a, dim, h):
        """Staggered first difference to the face: (-a(+2) + 27 a(+1) - 27 a(0) + a(-1)) / 24h."""
        s = sx if dim == "x" else sy
        if self.p.cds == 1:
            return (s(a, 1) - a) / h
        return (-s(a, 2) + 27 * s(a, 1) - 27 * a + s(a, -1)) / 24.0 / h

    def d2(self, a, dim, h):
        s = sx if dim == "x" else sy
        if self.p.cds == 1:
            return (s(a, 1) - 2 * a + s(a, -1)) / (h * h)
        return (-s(a, 2) + 16 * s(a, 1) - 30 * a + 16 * s(a, -1) - s(a, -2)) / 12.0 / (h * h)

    def _symbol(self, op, n, axis):
        """DFT of op applied to a unit impulse: the symbol at every wavenumber index."""
        p = self.p
        d = torch.zeros((1, p.ny, p.nx), dtype=torch.float64)
        d[0, 0, 0] = 1.0
        r = op(d)
        line = r[0, 0, :] if axis == "x" else r[0, :, 0]
        return torch.fft.fft(line.to(torch.complex128))

    def _symbols(self):
        p = self.p
        self.sDx = self._symbol(lambda a: self.d1(a, "x", self.dx), p.nx, "x")
        self.sDy = self._symbol(lambda a: self.d1(a, "y", self.dy), p.ny, "y")
        self.sGx = self._symbol(lambda a: self.g1(a, "x", self.dx), p.nx, "x")
        self.sGy = self._symbol(lambda a: self.g1(a, "y", self.dy), p.ny, "y")
        self.sLx = self._symbol(lambda a: self.d2(a, "x", self.dx), p.nx, "x").real
        self.sLy = self._symbol(lambda a: self.d2(a, "y", self.dy), p.ny, "y").real
        # [ny, nx] mode grids
        self.Lxy = self.sLy[:, None] + self.sLx[None, :]
        self.Pxy = (self.sDy * self.sGy)[:, None].real + (self.sDx * self.sGx)[None, :].real
        nyq = torch.ones((p.ny, p.nx), dtype=torch.float64)
        nyq[p.ny // 2, :] = 0.0
        nyq[:, p.nx // 2] = 0.0
        self.nyq = nyq

    # ---------------------------------------------------------------- fft
    def fwd(self, a):
        p = self.p
        return torch.fft.fft2(a.to(torch.complex128)) / (p.nx * p.ny) * self.nyq

    def inv(self, c):
        p = self.p
        return (torch.fft.ifft2(c * self.nyq) * (p.nx * p.ny)).real

    # ---------------------------------------------------------------- rhs
    def rhs(self, u, v, w, pr, fp, bf, rk_a, rk_b, rk_c):
        p = self.p
        nz = p.nz
        um, dt, nu, fc = p.u_mrf, p.dt, p.nu, p.fc
        dx, dy = self.dx, self.dy
        closed = p.ochannel == 0
        cdif = rk_c * 0.5 * dt * nu
        dz, dzt, dzb, lt = (a[:, None, None] for a in (self.dz, self.dzt, self.dzb, self.lt))
        cds = p.cds

        def ih(a, d, lo):
            """4-point (cds=2) or 2-point mid-point interpolant over a(lo+3..lo) / a(lo+1..lo) along d."""
            s = sx if d == "x" else sy
            if cds == 1:
                return 0.5 * (s(a, lo + 1) + s(a, lo))
            return (-s(a, lo + 3) + 9 * s(a, lo + 2) + 9 * s(a, lo + 1) - s(a, lo)) * 0.0625

        def dflux(a, d, h, lo):
            """Staggered difference of a flux over offsets lo+3..lo (cds=2) or lo+1..lo."""
            s = sx if d == "x" else sy
            if cds == 1:
                return (s(a, lo + 1) - s(a, lo)) / h
            return (-s(a, lo + 3) + 27 * s(a, lo + 2) - 27 * s(a, lo + 1) + s(a, lo)) / 24.0 / h

        uhx = ih(u, "x", -2 if cds == 2 else -1)       # U(i+1), U(i), U(i-1), U(i-2)
        uhy = ih(u, "y", -1 if cds == 2 else 0)        # U(j+2) .. U(j-1)
        vhx = ih(v, "x", -1 if cds == 2 else 0)        # V(i+2) .. V(i-1)
        vhy = ih(v, "y", -2 if cds == 2 else -1)       # V(j+1) .. V(j-2)
        whx = ih(w, "x", -1 if cds == 2 else 0)
        why = ih(w, "y", -1 if cds == 2 else 0)
        zero = torch.zeros_like(u[:1])
        # z interpolants at the faces k = -1 .. nz-1 (nz+1 of them)
        uhz_in = u[1:] * lt[:-1] + u[:-1] * (1 - lt[:-1])
        vhz_in = v[1:] * lt[:-1] + v[:-1] * (1 - lt[:-1])
        uhz = torch.cat([zero - um, uhz_in, (zero - um) if closed else u[-1:]], 0)
        vhz = torch.cat([zero, vhz_in, zero if closed else v[-1:]], 0)
        whx_f = torch.cat([zero, whx[:-1], zero], 0)
        why_f = torch.cat([zero, why[:-1], zero], 0)
        # z ghosts of u, v
        ug = torch.cat([-u[:1] - 2 * um, u, (-u[-1:] - 2 * um) if closed else u[-1:]], 0)
        vg = torch.cat([-v[:1], v, -v[-1:] if closed else v[-1:]], 0)

        lo_c = -1 if cds == 2 else 0       # flux offsets i+2..i-1 (cds=2), i+1..i
        lo_s = -2 if cds == 2 else -1      # flux offsets i+1..i-2 (cds=2), i..i-1
        # ---- u
        uux = dflux(uhx * uhx, "x", dx, lo_c)
        ux = dflux(uhx, "x", dx, lo_c)
        uvy = dflux(uhy * vhx, "y", dy, lo_s)
        uwz = (uhz[1:] * whx_f[1:] - uhz[:-1] * whx_f[:-1]) / dz
        uzz = ((ug[2:] - u) / dzt - (u - ug[:-2]) / dzb) / dz
        if p.dp_opt == 3:
            fu = -uux - uvy - uwz - um * ux + fc * (0.5 * (vhx + sy(vhx, -1)) - p.vg)
        else:
            fu = -uux - uvy - uwz + 1.0 - um * ux
        fu = fu + bf[0]
        qu = u + dt * (rk_a * fu + rk_b * fp[0]) + cdif * (self.d2(u, "x", dx) + self.d2(u, "y", dy) + uzz) \
            - rk_c * dt * self.g1(pr, "x", dx)
        # ---- v
        vux = dflux(vhx * uhy, "x", dx, lo_s)
        vx = dflux(vhx, "x", dx, lo_s)
        vvy = dflux(vhy * vhy, "y", dy, lo_c)
        vwz = (vhz[1:] * why_f[1:] - vhz[:-1] * why_f[:-1]) / dz
        vzz = ((vg[2:] - v) / dzt - (v - vg[:-2]) / dzb) / dz
        if p.dp_opt == 3:
            fv = -vux - vvy - vwz - um * vx + fc * (p.ug - 0.5 * (uhy + sx(uhy, -1)) - um)
        else:
            fv = -vux - vvy - vwz - um * vx
        fv = fv + bf[1]
        qv = v + dt * (rk_a * fv + rk_b * fp[1]) + cdif * (self.d2(v, "x", dx) + self.d2(v, "y", dy) + vzz) \
            - rk_c * dt * self.g1(pr, "y", dy)
        # ---- w on the faces k = 0 .. nz-2
        wk, uhzk, vhzk = w[:-1], uhz[1:-1], vhz[1:-1]
        wux = dflux(whx[:-1] * uhzk, "x", dx, lo_s)
        wx = dflux(whx[:-1], "x", dx, lo_s)
        wvy = dflux(why[:-1] * vhzk, "y", dy, lo_s)
        wm = torch.cat([zero, w[:-2]], 0)
        wp = w[1:]
        wwz = ((0.5 * (wk + wp)) ** 2 - (0.5 * (wk + wm)) ** 2) / dzt[:-1]
        wzz = ((wp - wk) / dz[1:] - (wk - wm) / dz[:-1]) / dzt[:-1]
        fw = -wux - wvy - wwz - um * wx + bf[2][:-1]
        dpdz = (pr[1:] - pr[:-1]) / dzt[:-1]
        qw = wk + dt * (rk_a * fw + rk_b * fp[2][:-1]) + cdif * (self.d2(wk, "x", dx) + self.d2(wk, "y", dy) + wzz) \
            - rk_c * dt * dpdz
        fw_full = torch.cat([fw, fp[2][-1:]], 0)       # the top-wall level keeps its history
        return (qu, qv, qw), (fu, fv, fw_full)

    # ---------------------------------------------------------------- column
    def _tridiag(self, sub, diag, sup):
        """[..., n, n] from sub (row r, column r-1), diag, sup (row r, column r+1)."""
        return torch.diag_embed(diag) + torch.diag_embed(sub[..., 1:], offset=-1) + torch.diag_embed(sup[..., :-1], offset=1)

    def column(self, q, rk_c):
        p = self.p
        nz, ny, nx = p.nz, p.ny, p.nx
        dt, nu = p.dt, p.nu
        dz, dzt, dzb = self.dz, self.dzt, self.dzb
        closed = p.ochannel == 0
        cpl = torch.complex128
        # u, v: Helmholtz rows (get_u_eqn_coeff), wall folds on the (0,0) mode only
        a0 = -0.5 * dt * nu / dz / dzb
        c0 = -0.5 * dt * nu / dz / dzt
        kk = torch.arange(nz)
        au = torch.where(kk == 0, 0.0, a0)
        cu = torch.where(kk == nz - 1, 0.0, c0)
        dgu = -au - cu
        d0u = -a0 - c0
        d0u = d0u + torch.where(kk == 0, -a0, 0.0)
        d0u = d0u + torch.where(kk == nz - 1, (-c0 if closed else c0), 0.0)
        lam = 0.5 * dt * nu * self.Lxy                     # [ny, nx]
        is00 = torch.zeros((ny, nx), dtype=torch.bool)
        is00[0, 0] = True

        def helm(a, c, dg, d0, lam_):
            dgm = torch.where(is00[..., None], d0, dg)     # [ny, nx, n]
            diag = 1.0 + rk_c * (-lam_[..., None] + dgm)
            sub = (rk_c * a).expand_as(diag)
            sup = (rk_c * c).expand_as(diag)
            return self._tridiag(sub, diag, sup)

        Hu = helm(au, cu, dgu, d0u, lam).to(cpl)
        # w rows 0..nz-2 (get_w_eqn_coeff)
        dzp = self.dz_all[3:nz + 2]                        # dz(k+1)
        a0w = -0.5 * dt * nu / dz[:-1] / dzt[:-1]
        c0w = -0.5 * dt * nu / dzp / dzt[:-1]
        kw = torch.arange(nz - 1)
        aw = torch.where(kw == 0, 0.0, a0w)
        cw = torch.where(kw == nz - 2, 0.0, c0w)
        Hw = helm(aw, cw, -aw - cw, -a0w - c0w, lam).to(cpl)
        # p rows (get_p_eqn_coeff), pinned first row of the (0,0) mode
        a0p = 1.0 / dz / dzb
        c0p = 1.0 / dz / dzt
        ap = torch.where(kk == 0, 0.0, a0p)
        cp = torch.where(kk == nz - 1, 0.0, c0p)
        dgp = -ap - cp
        diagp = rk_c * (self.Pxy[..., None] + dgp)
        subp = (rk_c * ap).expand_as(diagp)
        supp = (rk_c * cp).expand_as(diagp).clone()
        supp[0, 0, 0] = 0.0
        Pm = self._tridiag(subp, diagp, supp).to(cpl)

        Q = [self.fwd(x) for x in q]                       # [nz', ny, nx]
        # (0,0)-mode source corrections of the moving frame (ubnd)
        bc = torch.zeros((nz, ny, nx), dtype=cpl)
        bc[0, 0, 0] = 2.0 * (-0.5 * rk_c * dt * nu / dz[0] / dzb[0]) * p.u_mrf
        if closed:
            bc[nz - 1, 0, 0] = 2.0 * (-0.5 * rk_c * dt * nu / dz[nz - 1] / dzt[nz - 1]) * p.u_mrf
        col = lambda a: a.permute(1, 2, 0)[..., None]      # [ny, nx, n, 1]
        uncol = lambda a: a[..., 0].permute(2, 0, 1)
        us = uncol(torch.linalg.solve(Hu, col(Q[0] + bc)))
        vs = uncol(torch.linalg.solve(Hu, col(Q[1])))
        ws = uncol(torch.linalg.solve(Hw, col(Q[2])))
        ws = torch.cat([ws, torch.zeros_like(ws[:1])], 0)  # w* = 0 on the top wall
        # pressure source: div(u*) / dt
        sDX = self.sDx[None, None, :]
        sDY = self.sDy[None, :, None]
        wprev = torch.cat([torch.zeros_like(ws[:1]), ws[:-1]], 0)
        s = (sDX * us + sDY * vs + (ws - wprev) / dz[:, None, None]) / dt
        mask = torch.ones_like(s.real)
        mask[0, 0, 0] = 0.0
        s = s * mask
        phi = uncol(torch.linalg.solve(Pm, col(s)))
        # projection and psi = phi - rk_c dt nu/2 lap(phi)
        cpr = rk_c * dt
        cps = rk_c * 0.5 * dt * nu
        sGX = self.sGx[None, None, :]
        sGY = self.sGy[None, :, None]
        un = us - cpr * sGX * phi
        vn = vs - cpr * sGY * phi
        gz = (phi[1:] - phi[:-1]) / dzt[:-1, None, None]
        wn = torch.cat([ws[:-1] - cpr * gz, torch.zeros_like(ws[:1])], 0)
        pu = torch.cat([phi[1:], phi[-1:]], 0)
        pd = torch.cat([phi[:1], phi[:-1]], 0)
        lz = ((pu - phi) / dzt[:, None, None] - (phi - pd) / dzb[:, None, None]) / dz[:, None, None]
        psi = phi - cps * (self.Lxy[None] * phi + lz)
        return self.inv(un), self.inv(vn), self.inv(wn), self.inv(psi)

    # ---------------------------------------------------------------- step
    def substep(self, st, sub, bf):
        p = self.p
        if p.dts == 2:
            ra, rb, rc = RK_A[sub], RK_B[sub], RK_C[sub]
        else:
            ra, rb, rc = 1.5, -0.5, 1.0
        u, v, w, pr, ff, gg, hh = st
        q, fnew = self.rhs(u, v, w, pr, (ff, gg, hh), bf, ra, rb, rc)
        un, vn, wn, psi = self.column(q, rc)
        return (un, vn, wn, pr + psi) + tuple(fnew)

    def run(self, st, nsteps, bf):
        nsub = 3 if self.p.dts == 2 else 1
        for _ in range(nsteps):
            for sub in range(nsub):
                st = self.substep(st, sub, bf)
        return st
