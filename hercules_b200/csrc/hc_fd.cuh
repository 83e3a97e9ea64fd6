// hc_fd.cuh -- finite-difference stencil kernels (cds = 1: 2nd order, cds = 2: 4th order).
//
// One thread per interior grid point. Every interpolant the reference stores in a
// separate array (uhx .. why, thx .. thz; src/module_tools.f90:410-512, with their
// ghost values from src/module_boundary.f90:202-355) is recomputed in registers
// from u, v, w, t, and every ghost cell is produced on load: periodic wrap in x, y
// and the wall / top conditions in z.
#pragma once
#include "hc_common.cuh"

template <typename R> struct FieldsIn {
    const R* u; const R* v; const R* w; const R* p; const R* t;
};

template <typename R> __device__ __forceinline__ R ldf(const R* f, const Geo& g, int i, int j, int k)
{
    return __ldg(f + ((long long)k * g.ny + wrapi(j, g.ny)) * g.nx + wrapi(i, g.nx));
}

// ---- z ghost cells on load (update_boundary_uvw/p/t, src/module_boundary.f90:33-196) ----
//
// Rayleigh damping (FD path) changes the interior of the top levels kd..nz-1 at
// the start of a sub-step but, in the reference, leaves every ghost cell as the
// previous boundary update wrote it (rayleigh_damping, src/module_tools.f90:
// 705-749, touches istr3..iend3 x jstr3..jend3 only). A value read outside the
// domain (a periodic neighbour or a z ghost) therefore still holds the undamped
// field. With the pre-damping copies s* of those levels set, every such read is
// served from the copy; interpolants are evaluated at the wrapped point, as the
// reference's interpolant ghosts are periodic copies of interior values.
template <typename R> struct Acc {
    FieldsIn<R> f;
    Geo g;
    R um, tbs, tba, ttop;   // bottom ghost of T: T(-1) = tbs T(0) + tba
    int closed;   // ochannel == 0
    // pre-damping copies of levels kd..nz-1 ([k-kd][j][i]); null: no damping
    const R* su; const R* sv; const R* sw; const R* sp; const R* st;
    int kd;

    // value of field f at (i, j, k) with k inside [0, nz): the current value
    // inside the domain, the undamped one across the periodic boundary
    __device__ __forceinline__ R raw(const R* fp, const R* sp_, int i, int j, int k) const {
        if (sp_ && k >= kd && !((unsigned)i < (unsigned)g.nx && (unsigned)j < (unsigned)g.ny))
            return __ldg(sp_ + ((long long)(k - kd) * g.ny + wrapi(j, g.ny)) * g.nx + wrapi(i, g.nx));
        return ldf(fp, g, i, j, k);
    }
    // source value of a z ghost (always the undamped field when damped)
    __device__ __forceinline__ R gsrc(const R* fp, const R* sp_, int i, int j, int k) const {
        if (sp_ && k >= kd) return __ldg(sp_ + ((long long)(k - kd) * g.ny + wrapi(j, g.ny)) * g.nx + wrapi(i, g.nx));
        return ldf(fp, g, i, j, k);
    }
    __device__ __forceinline__ R U(int i, int j, int k) const {
        if (k < 0) return -gsrc(f.u, su, i, j, 0) - R(2) * um;
        if (k >= g.nz) return closed ? -gsrc(f.u, su, i, j, g.nz - 1) - R(2) * um : gsrc(f.u, su, i, j, g.nz - 1);
        return raw(f.u, su, i, j, k);
    }
    __device__ __forceinline__ R V(int i, int j, int k) const {
        if (k < 0) return -gsrc(f.v, sv, i, j, 0);
        if (k >= g.nz) return closed ? -gsrc(f.v, sv, i, j, g.nz - 1) : gsrc(f.v, sv, i, j, g.nz - 1);
        return raw(f.v, sv, i, j, k);
    }
    __device__ __forceinline__ R W(int i, int j, int k) const {
        if (k < 0) return R(0);
        if (k >= g.nz) return -gsrc(f.w, sw, i, j, g.nz - 2);
        return raw(f.w, sw, i, j, k);          // level nz-1 is the top wall, stored as 0
    }
    __device__ __forceinline__ R P(int i, int j, int k) const {
        if (k < 0) return gsrc(f.p, sp, i, j, 0);
        if (k >= g.nz) return gsrc(f.p, sp, i, j, g.nz - 1);
        return raw(f.p, sp, i, j, k);
    }
    __device__ __forceinline__ R T(int i, int j, int k) const {
        if (k < 0) return tbs * gsrc(f.t, st, i, j, 0) + tba;
        if (k >= g.nz) return R(2) * ttop - gsrc(f.t, st, i, j, g.nz - 1);
        return raw(f.t, st, i, j, k);
    }
    __device__ __forceinline__ R lt(int k) const { return (R)ldz(g.z.l_t, k); }

    // ---- mid-point interpolants (get_interp_fields_uvwhxyz, src/module_tools.f90:410-468) ----
    template <int CDS> __device__ __forceinline__ R uhx(int i, int j, int k) const {
        i = wrapi(i, g.nx); j = wrapi(j, g.ny);
        if (CDS == 1) return R(0.5) * (U(i, j, k) + U(i - 1, j, k));
        return (-U(i + 1, j, k) + R(9) * U(i, j, k) + R(9) * U(i - 1, j, k) - U(i - 2, j, k)) * R(0.0625);
    }
    template <int CDS> __device__ __forceinline__ R uhy(int i, int j, int k) const {
        i = wrapi(i, g.nx); j = wrapi(j, g.ny);
        if (CDS == 1) return R(0.5) * (U(i, j + 1, k) + U(i, j, k));
        return (-U(i, j + 2, k) + R(9) * U(i, j + 1, k) + R(9) * U(i, j, k) - U(i, j - 1, k)) * R(0.0625);
    }
    template <int CDS> __device__ __forceinline__ R vhx(int i, int j, int k) const {
        i = wrapi(i, g.nx); j = wrapi(j, g.ny);
        if (CDS == 1) return R(0.5) * (V(i + 1, j, k) + V(i, j, k));
        return (-V(i + 2, j, k) + R(9) * V(i + 1, j, k) + R(9) * V(i, j, k) - V(i - 1, j, k)) * R(0.0625);
    }
    template <int CDS> __device__ __forceinline__ R vhy(int i, int j, int k) const {
        i = wrapi(i, g.nx); j = wrapi(j, g.ny);
        if (CDS == 1) return R(0.5) * (V(i, j, k) + V(i, j - 1, k));
        return (-V(i, j + 1, k) + R(9) * V(i, j, k) + R(9) * V(i, j - 1, k) - V(i, j - 2, k)) * R(0.0625);
    }
    // whx/why: 0 on the wall ghost below and on the top wall (update_boundary_uvwhxyz :232-235, :281-282)
    template <int CDS> __device__ __forceinline__ R whx(int i, int j, int k) const {
        i = wrapi(i, g.nx); j = wrapi(j, g.ny);
        if (k < 0 || k >= g.nz - 1) return R(0);
        if (CDS == 1) return R(0.5) * (W(i + 1, j, k) + W(i, j, k));
        return (-W(i + 2, j, k) + R(9) * W(i + 1, j, k) + R(9) * W(i, j, k) - W(i - 1, j, k)) * R(0.0625);
    }
    template <int CDS> __device__ __forceinline__ R why(int i, int j, int k) const {
        i = wrapi(i, g.nx); j = wrapi(j, g.ny);
        if (k < 0 || k >= g.nz - 1) return R(0);
        if (CDS == 1) return R(0.5) * (W(i, j + 1, k) + W(i, j, k));
        return (-W(i, j + 2, k) + R(9) * W(i, j + 1, k) + R(9) * W(i, j, k) - W(i, j - 1, k)) * R(0.0625);
    }
    // uhz/vhz: linear in z; wall value below, wall (closed) or surface value (open) on top
    __device__ __forceinline__ R uhz(int i, int j, int k) const {
        i = wrapi(i, g.nx); j = wrapi(j, g.ny);
        if (k < 0) return -um;
        if (k >= g.nz - 1) return closed ? -um : U(i, j, g.nz - 1);
        R l = lt(k);
        return U(i, j, k + 1) * l + U(i, j, k) * (R(1) - l);
    }
    __device__ __forceinline__ R vhz(int i, int j, int k) const {
        i = wrapi(i, g.nx); j = wrapi(j, g.ny);
        if (k < 0) return R(0);
        if (k >= g.nz - 1) return closed ? R(0) : V(i, j, g.nz - 1);
        R l = lt(k);
        return V(i, j, k + 1) * l + V(i, j, k) * (R(1) - l);
    }
    // temperature interpolants (get_interp_fields_thxyz :473-512, update_boundary_thxyz :311-355)
    template <int CDS> __device__ __forceinline__ R thx(int i, int j, int k) const {
        i = wrapi(i, g.nx); j = wrapi(j, g.ny);
        if (CDS == 1) return R(0.5) * (T(i + 1, j, k) + T(i, j, k));
        return (-T(i + 2, j, k) + R(9) * T(i + 1, j, k) + R(9) * T(i, j, k) - T(i - 1, j, k)) * R(0.0625);
    }
    template <int CDS> __device__ __forceinline__ R thy(int i, int j, int k) const {
        i = wrapi(i, g.nx); j = wrapi(j, g.ny);
        if (CDS == 1) return R(0.5) * (T(i, j + 1, k) + T(i, j, k));
        return (-T(i, j + 2, k) + R(9) * T(i, j + 1, k) + R(9) * T(i, j, k) - T(i, j - 1, k)) * R(0.0625);
    }
    __device__ __forceinline__ R thz(int i, int j, int k) const {
        i = wrapi(i, g.nx); j = wrapi(j, g.ny);
        if (k < 0) return tbs < R(0) ? R(0.5) * tba : R(0.5) * (T(i, j, -1) + T(i, j, 0));   // the wall value
        if (k >= g.nz - 1) return ttop;
        R l = lt(k);
        return T(i, j, k + 1) * l + T(i, j, k) * (R(1) - l);
    }
};

template <typename R> struct MomArgs {
    Acc<R> a;
    R* ff; R* gg; R* hh;          // histories, updated in place (old value read first)
    R* qu; R* qv; R* qw;
    R* uhx_s; R* vhy_s;           // stats snapshot of uhx, vhy (may be null)
    double rk_a, rk_b, rk_c;
    Phys ph;
    const DevScalars* sc;
    const R* bfx; const R* bfy; const R* bfz;   // body force (null: none)
};

// get_momentum_cnvdiff (src/module_cnvdiff.f90:35-374)
template <typename R, int CDS>
__global__ void __launch_bounds__(256) k_rhs_momentum(MomArgs<R> m)
{
    const Acc<R>& A = m.a;
    const Geo& g = A.g;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= g.nx || j >= g.ny) return;
    const long long id = ((long long)k * g.ny + j) * g.nx + i;

    const R dx = (R)g.dx, dy = (R)g.dy, dx2 = (R)g.dx2, dy2 = (R)g.dy2;
    const R dt = (R)m.ph.dt, nu = (R)m.ph.nu, um = A.um, fc = (R)m.ph.fc;
    const R rka = (R)m.rk_a, rkb = (R)m.rk_b, rkc = (R)m.rk_c;
    const R dz = (R)ldz(g.z.dz, k), dzt = (R)ldz(g.z.dz_t, k), dzb = (R)ldz(g.z.dz_b, k);
    const R cdif = rkc * R(0.5) * dt * nu;
    const R dpx = (R)m.sc->dpx_drive;

    // ---------------- U ----------------
    {
        R uux, uvy, ux, uxx, uyy, dpdx;
        if (CDS == 1) {
            R h1 = A.template uhx<1>(i + 1, j, k), h0 = A.template uhx<1>(i, j, k);
            uux = (h1 * h1 - h0 * h0) / dx;
            uvy = (A.template uhy<1>(i, j, k) * A.template vhx<1>(i, j, k) -
                   A.template uhy<1>(i, j - 1, k) * A.template vhx<1>(i, j - 1, k)) / dy;
            ux = (h1 - h0) / dx;
            uxx = (A.U(i + 1, j, k) - R(2) * A.U(i, j, k) + A.U(i - 1, j, k)) / dx2;
            uyy = (A.U(i, j + 1, k) - R(2) * A.U(i, j, k) + A.U(i, j - 1, k)) / dy2;
            dpdx = (A.P(i + 1, j, k) - A.P(i, j, k)) / dx;
        } else {
            R h2 = A.template uhx<2>(i + 2, j, k), h1 = A.template uhx<2>(i + 1, j, k);
            R h0 = A.template uhx<2>(i, j, k), hm = A.template uhx<2>(i - 1, j, k);
            uux = (-h2 * h2 + R(27) * h1 * h1 - R(27) * h0 * h0 + hm * hm) / R(24) / dx;
            uvy = (-A.template uhy<2>(i, j + 1, k) * A.template vhx<2>(i, j + 1, k) +
                   R(27) * A.template uhy<2>(i, j, k) * A.template vhx<2>(i, j, k) -
                   R(27) * A.template uhy<2>(i, j - 1, k) * A.template vhx<2>(i, j - 1, k) +
                   A.template uhy<2>(i, j - 2, k) * A.template vhx<2>(i, j - 2, k)) / R(24) / dy;
            ux = (-h2 + R(27) * h1 - R(27) * h0 + hm) / R(24) / dx;
            uxx = (-A.U(i + 2, j, k) + R(16) * A.U(i + 1, j, k) - R(30) * A.U(i, j, k) + R(16) * A.U(i - 1, j, k) - A.U(i - 2, j, k)) / R(12) / dx2;
            uyy = (-A.U(i, j + 2, k) + R(16) * A.U(i, j + 1, k) - R(30) * A.U(i, j, k) + R(16) * A.U(i, j - 1, k) - A.U(i, j - 2, k)) / R(12) / dy2;
            dpdx = (-A.P(i + 2, j, k) + R(27) * A.P(i + 1, j, k) - R(27) * A.P(i, j, k) + A.P(i - 1, j, k)) / R(24) / dx;
        }
        R uwz = (A.uhz(i, j, k) * A.template whx<CDS>(i, j, k) - A.uhz(i, j, k - 1) * A.template whx<CDS>(i, j, k - 1)) / dz;
        R uc = A.U(i, j, k);
        R uzz = ((A.U(i, j, k + 1) - uc) / dzt - (uc - A.U(i, j, k - 1)) / dzb) / dz;
        R f;
        if (m.ph.dp_opt == 3)
            f = -uux - uvy - uwz - um * ux + fc * (R(0.5) * (A.template vhx<CDS>(i, j, k) + A.template vhx<CDS>(i, j - 1, k)) - (R)m.ph.vg);
        else
            f = -uux - uvy - uwz + dpx - um * ux;
        if (m.bfx) f += m.bfx[id];
        R f0 = m.ff[id];
        m.ff[id] = f;
        m.qu[id] = uc + dt * (rka * f + rkb * f0) + cdif * (uxx + uyy + uzz) - rkc * dt * dpdx;
        if (m.uhx_s) m.uhx_s[id] = A.template uhx<CDS>(i, j, k);
    }
    // ---------------- V ----------------
    {
        R vux, vvy, vx, vxx, vyy, dpdy;
        if (CDS == 1) {
            R h0 = A.template vhx<1>(i, j, k), hm = A.template vhx<1>(i - 1, j, k);
            vux = (h0 * A.template uhy<1>(i, j, k) - hm * A.template uhy<1>(i - 1, j, k)) / dx;
            R y1 = A.template vhy<1>(i, j + 1, k), y0 = A.template vhy<1>(i, j, k);
            vvy = (y1 * y1 - y0 * y0) / dy;
            vx = (h0 - hm) / dx;
            vxx = (A.V(i + 1, j, k) - R(2) * A.V(i, j, k) + A.V(i - 1, j, k)) / dx2;
            vyy = (A.V(i, j + 1, k) - R(2) * A.V(i, j, k) + A.V(i, j - 1, k)) / dy2;
            dpdy = (A.P(i, j + 1, k) - A.P(i, j, k)) / dy;
        } else {
            R h1 = A.template vhx<2>(i + 1, j, k), h0 = A.template vhx<2>(i, j, k);
            R hm = A.template vhx<2>(i - 1, j, k), hm2 = A.template vhx<2>(i - 2, j, k);
            vux = (-h1 * A.template uhy<2>(i + 1, j, k) + R(27) * h0 * A.template uhy<2>(i, j, k) -
                   R(27) * hm * A.template uhy<2>(i - 1, j, k) + hm2 * A.template uhy<2>(i - 2, j, k)) / R(24) / dx;
            R y2 = A.template vhy<2>(i, j + 2, k), y1 = A.template vhy<2>(i, j + 1, k);
            R y0 = A.template vhy<2>(i, j, k), ym = A.template vhy<2>(i, j - 1, k);
            vvy = (-y2 * y2 + R(27) * y1 * y1 - R(27) * y0 * y0 + ym * ym) / R(24) / dy;
            vx = (-h1 + R(27) * h0 - R(27) * hm + hm2) / R(24) / dx;
            vxx = (-A.V(i + 2, j, k) + R(16) * A.V(i + 1, j, k) - R(30) * A.V(i, j, k) + R(16) * A.V(i - 1, j, k) - A.V(i - 2, j, k)) / R(12) / dx2;
            vyy = (-A.V(i, j + 2, k) + R(16) * A.V(i, j + 1, k) - R(30) * A.V(i, j, k) + R(16) * A.V(i, j - 1, k) - A.V(i, j - 2, k)) / R(12) / dy2;
            dpdy = (-A.P(i, j + 2, k) + R(27) * A.P(i, j + 1, k) - R(27) * A.P(i, j, k) + A.P(i, j - 1, k)) / R(24) / dy;
        }
        R vwz = (A.vhz(i, j, k) * A.template why<CDS>(i, j, k) - A.vhz(i, j, k - 1) * A.template why<CDS>(i, j, k - 1)) / dz;
        R vc = A.V(i, j, k);
        R vzz = ((A.V(i, j, k + 1) - vc) / dzt - (vc - A.V(i, j, k - 1)) / dzb) / dz;
        R f;
        if (m.ph.dp_opt == 3)
            f = -vux - vvy - vwz - um * vx + fc * ((R)m.ph.ug - R(0.5) * (A.template uhy<CDS>(i, j, k) + A.template uhy<CDS>(i - 1, j, k)) - um);
        else
            f = -vux - vvy - vwz - um * vx;
        if (m.bfx) f += m.bfy[id];
        R f0 = m.gg[id];
        m.gg[id] = f;
        m.qv[id] = vc + dt * (rka * f + rkb * f0) + cdif * (vxx + vyy + vzz) - rkc * dt * dpdy;
        if (m.vhy_s) m.vhy_s[id] = A.template vhy<CDS>(i, j, k);
    }
    // ---------------- W (k <= nz-2; the top-wall level keeps its old hh, qw) ----------------
    if (k <= g.nz - 2) {
        R wux, wvy, wx, wxx, wyy;
        if (CDS == 1) {
            R h0 = A.template whx<1>(i, j, k), hm = A.template whx<1>(i - 1, j, k);
            wux = (h0 * A.uhz(i, j, k) - hm * A.uhz(i - 1, j, k)) / dx;
            wvy = (A.template why<1>(i, j, k) * A.vhz(i, j, k) - A.template why<1>(i, j - 1, k) * A.vhz(i, j - 1, k)) / dy;
            wx = (h0 - hm) / dx;
            wxx = (A.W(i + 1, j, k) - R(2) * A.W(i, j, k) + A.W(i - 1, j, k)) / dx2;
            wyy = (A.W(i, j + 1, k) - R(2) * A.W(i, j, k) + A.W(i, j - 1, k)) / dy2;
        } else {
            R h1 = A.template whx<2>(i + 1, j, k), h0 = A.template whx<2>(i, j, k);
            R hm = A.template whx<2>(i - 1, j, k), hm2 = A.template whx<2>(i - 2, j, k);
            wux = (-h1 * A.uhz(i + 1, j, k) + R(27) * h0 * A.uhz(i, j, k) - R(27) * hm * A.uhz(i - 1, j, k) +
                   hm2 * A.uhz(i - 2, j, k)) / R(24) / dx;
            wvy = (-A.template why<2>(i, j + 1, k) * A.vhz(i, j + 1, k) + R(27) * A.template why<2>(i, j, k) * A.vhz(i, j, k) -
                   R(27) * A.template why<2>(i, j - 1, k) * A.vhz(i, j - 1, k) + A.template why<2>(i, j - 2, k) * A.vhz(i, j - 2, k)) / R(24) / dy;
            wx = (-h1 + R(27) * h0 - R(27) * hm + hm2) / R(24) / dx;
            wxx = (-A.W(i + 2, j, k) + R(16) * A.W(i + 1, j, k) - R(30) * A.W(i, j, k) + R(16) * A.W(i - 1, j, k) - A.W(i - 2, j, k)) / R(12) / dx2;
            wyy = (-A.W(i, j + 2, k) + R(16) * A.W(i, j + 1, k) - R(30) * A.W(i, j, k) + R(16) * A.W(i, j - 1, k) - A.W(i, j - 2, k)) / R(12) / dy2;
        }
        R wc = A.W(i, j, k), wp = A.W(i, j, k + 1), wm = A.W(i, j, k - 1);
        R a1 = R(0.5) * (wc + wp); a1 = a1 * a1;
        R a2 = R(0.5) * (wc + wm); a2 = a2 * a2;
        R wwz = (a1 - a2) / dzt;
        R dzp = (R)ldz(g.z.dz, k + 1);
        R wzz = ((wp - wc) / dzp - (wc - wm) / dz) / dzt;
        R f = -wux - wvy - wwz - um * wx;
        if (m.ph.isscalar == 1) {
            R l = A.lt(k);
            f = f + (R)m.sc->got * ((R(1) - l) * A.T(i, j, k) + l * A.T(i, j, k + 1) - (R)m.ph.t_ref);
        }
        R dpdz = (A.P(i, j, k + 1) - A.P(i, j, k)) / dzt;
        if (m.bfx) f += m.bfz[id];
        R f0 = m.hh[id];
        m.hh[id] = f;
        m.qw[id] = wc + dt * (rka * f + rkb * f0) + cdif * (wxx + wyy + wzz) - rkc * dt * dpdz;
    }
}

template <typename R> struct TempArgs {
    Acc<R> a;
    R* ss; R* qt;
    double rk_a, rk_b, rk_c;
    Phys ph;
    int kchunk;          // the strip kernel: levels a block
    const void* zm;      // the strip kernel: per-level metrics [5][nz] in the storage type
};

// get_temperature_cnvdiff (src/module_cnvdiff.f90:381-473); u, v, w are the
// projected velocities of this sub-step, t the one from before it.
template <typename R, int CDS>
__device__ __forceinline__ void k_rhs_temperature_body(const TempArgs<R>& m, const uint3 blockIdx, const dim3 gridDim)
{
    const Acc<R>& A = m.a;
    const Geo& g = A.g;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= g.nx || j >= g.ny) return;
    const long long id = ((long long)k * g.ny + j) * g.nx + i;
    const R dx = (R)g.dx, dy = (R)g.dy, dx2 = (R)g.dx2, dy2 = (R)g.dy2;
    const R dt = (R)m.ph.dt, al = (R)m.ph.alpha, um = A.um;
    const R dz = (R)ldz(g.z.dz, k), dzt = (R)ldz(g.z.dz_t, k), dzb = (R)ldz(g.z.dz_b, k);
    R tux, tvy, tx, txx, tyy;
    if (CDS == 1) {
        R h0 = A.template thx<1>(i, j, k), hm = A.template thx<1>(i - 1, j, k);
        tux = (h0 * A.U(i, j, k) - hm * A.U(i - 1, j, k)) / dx;
        tvy = (A.template thy<1>(i, j, k) * A.V(i, j, k) - A.template thy<1>(i, j - 1, k) * A.V(i, j - 1, k)) / dy;
        tx = (h0 - hm) / dx;
        txx = (A.T(i + 1, j, k) - R(2) * A.T(i, j, k) + A.T(i - 1, j, k)) / dx2;
        tyy = (A.T(i, j + 1, k) - R(2) * A.T(i, j, k) + A.T(i, j - 1, k)) / dy2;
    } else {
        R h1 = A.template thx<2>(i + 1, j, k), h0 = A.template thx<2>(i, j, k);
        R hm = A.template thx<2>(i - 1, j, k), hm2 = A.template thx<2>(i - 2, j, k);
        tux = (-h1 * A.U(i + 1, j, k) + R(27) * h0 * A.U(i, j, k) - R(27) * hm * A.U(i - 1, j, k) + hm2 * A.U(i - 2, j, k)) / R(24) / dx;
        tvy = (-A.template thy<2>(i, j + 1, k) * A.V(i, j + 1, k) + R(27) * A.template thy<2>(i, j, k) * A.V(i, j, k) -
               R(27) * A.template thy<2>(i, j - 1, k) * A.V(i, j - 1, k) + A.template thy<2>(i, j - 2, k) * A.V(i, j - 2, k)) / R(24) / dy;
        tx = (-h1 + R(27) * h0 - R(27) * hm + hm2) / R(24) / dx;
        txx = (-A.T(i + 2, j, k) + R(16) * A.T(i + 1, j, k) - R(30) * A.T(i, j, k) + R(16) * A.T(i - 1, j, k) - A.T(i - 2, j, k)) / R(12) / dx2;
        tyy = (-A.T(i, j + 2, k) + R(16) * A.T(i, j + 1, k) - R(30) * A.T(i, j, k) + R(16) * A.T(i, j - 1, k) - A.T(i, j - 2, k)) / R(12) / dy2;
    }
    R twz = (A.thz(i, j, k) * A.W(i, j, k) - A.thz(i, j, k - 1) * A.W(i, j, k - 1)) / dz;
    R tc = A.T(i, j, k);
    R tzz = ((A.T(i, j, k + 1) - tc) / dzt - (tc - A.T(i, j, k - 1)) / dzb) / dz;
    R s = -tux - tvy - twz - um * tx;
    R s0 = m.ss[id];
    m.ss[id] = s;
    m.qt[id] = tc + dt * ((R)m.rk_a * s + (R)m.rk_b * s0) + (R)m.rk_c * R(0.5) * dt * al * (txx + tyy + tzz);
}
template <typename R, int CDS>
__global__ void __launch_bounds__(256) k_rhs_temperature(TempArgs<R> m) { k_rhs_temperature_body<R, CDS>(m, blockIdx, gridDim); }

// ---------------------------------------------------------------------------
// block reductions
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
// keep the value of larger magnitude (ties: the larger value), so that the
// result does not depend on the reduction order
__device__ __forceinline__ double absmax_pick(double a, double b)
{
    double fa = fabs(a), fb = fabs(b);
    if (fb > fa || (fb == fa && b > a)) return b;
    return a;
}
__device__ __forceinline__ double warp_absmax(double v)
{
    for (int o = 16; o > 0; o >>= 1) v = absmax_pick(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_max(double v)
{
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Reductions use a fixed grid of at most RED_BLOCKS blocks that stride over the
// points, so the partial results (and the order they are combined in) depend on
// the grid size only: the sums are deterministic from run to run.
#define RED_BLOCKS 1184

// Divergence of the staggered fields at one point (get_p_eqn_src without the
// 1/dt, src/module_poisson_solver.f90:127-176; screen_div_error,
// src/module_io.f90:85-206). Every kernel that reports the divergence diagnostic
// goes through this one expression, so they agree bit for bit.
//   ux[0..3] = u(i+1), u(i), u(i-1), u(i-2); vy[0..3] likewise in j; w0, wm = w(k), w(k-1)
template <int CDS>
__device__ __forceinline__ double fd_div_point(const double* ux, const double* vy, double w0, double wm, double dx,
                                               double dy, double dzk)
{
    double dudx, dvdy;
    if (CDS == 1) {
        dudx = (ux[1] - ux[2]) * (1.0 / dx);
        dvdy = (vy[1] - vy[2]) * (1.0 / dy);
    } else {
        dudx = (-ux[0] + 27.0 * ux[1] - 27.0 * ux[2] + ux[3]) * (1.0 / (24.0 * dx));
        dvdy = (-vy[0] + 27.0 * vy[1] - 27.0 * vy[2] + vy[3]) * (1.0 / (24.0 * dy));
    }
    return dudx + dvdy + (w0 - wm) / dzk;
}

__device__ __forceinline__ void decode_pt(long long q, const Geo& g, int& i, int& j, int& k)
{
    i = (int)(q % g.nx);
    const long long r = q / g.nx;
    j = (int)(r % g.ny);
    k = (int)(r / g.ny);
}

// Divergence check (screen_div_error, src/module_io.f90:85-206): per block
// sum |div|, the signed div of largest magnitude, and a NaN flag.
// Work units are (256 consecutive (i,j) points) x (a chunk of levels); the
// blocks take the units in a fixed order, each thread walks its column up the
// chunk with the loads of two levels in flight and w(k-1) carried along.
// registers sized for four resident blocks with FP32 storage, three with FP64
// (at 512 x 384 x 256: 315 -> 239 us and 361 -> 309 us a launch; with the
// compiler's own budget too few warps had their loads in flight)
template <typename R> struct DivMinBlocks { static constexpr int v = sizeof(R) == sizeof(float) ? 4 : 3; };
template <typename R>
struct DivArgs {
    FieldsIn<R> f;
    Geo g;
    double* part;    // 3 doubles per block: sum |div|, signed div at max |div|, NaN flag
};
template <typename R, int CDS>
__device__ __forceinline__ void k_div_check_body(const DivArgs<R>& da, const uint3 blockIdx, const dim3 gridDim)
{
    const FieldsIn<R>& f = da.f;
    const Geo& g = da.g;
    double* part = da.part;
    __shared__ double s_sum[8], s_max[8];
    __shared__ int s_nan;
    const int tid = threadIdx.x;
    if (tid == 0) s_nan = 0;
    __syncthreads();
    double sm = 0.0, mx = 0.0;
    int nan = 0;
    if constexpr (sizeof(R) == sizeof(float)) {
        // FP32 storage: two x points a thread (nx is even), 8-byte loads
        const long long ncb2 = (g.nxy + 511) / 512;
        long long nch2 = (2LL * gridDim.x + ncb2 - 1) / ncb2;
        if (nch2 > g.nz) nch2 = g.nz;
        const int kc2 = (int)((g.nz + nch2 - 1) / nch2);
        for (long long un = blockIdx.x; un < ncb2 * nch2; un += gridDim.x) {
            const long long cb = un % ncb2;
            const int k0 = (int)(un / ncb2) * kc2, k1 = min(g.nz, k0 + kc2);
            const long long ij = cb * 512 + 2 * tid;
            if (ij >= g.nxy || k0 >= k1) continue;
            const int j = (int)(ij / g.nx), i = (int)(ij - (long long)j * g.nx);
            const int xm2 = wrapi(i - 2, g.nx) - i, xp2 = wrapi(i + 2, g.nx) - i;
            const long long yp1 = (long long)(wrapi(j + 1, g.ny) - j) * g.nx, ym1 = (long long)(wrapi(j - 1, g.ny) - j) * g.nx;
            const long long ym2 = (long long)(wrapi(j - 2, g.ny) - j) * g.nx;
            auto l2 = [](const R* p, long long q) { return *reinterpret_cast<const float2*>(p + q); };
            float2 wm = k0 > 0 ? l2(f.w, (long long)(k0 - 1) * g.nxy + ij) : make_float2(0.0f, 0.0f);
#pragma unroll 2
            for (int k = k0; k < k1; ++k) {
                const long long q = (long long)k * g.nxy + ij;
                const float2 um2 = l2(f.u, q + xm2), u0 = l2(f.u, q), up2 = l2(f.u, q + xp2);
                const float2 vp = l2(f.v, q + yp1), v0 = l2(f.v, q), vm = l2(f.v, q + ym1), vmm = l2(f.v, q + ym2);
                const float2 w0 = l2(f.w, q);
                const double dzk = ldz(g.z.dz, k);
                // x values i-2 .. i+3 of the pair
                const double xs[6] = {um2.x, um2.y, u0.x, u0.y, up2.x, up2.y};
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    double ux[4] = {xs[3 + s], xs[2 + s], xs[1 + s], xs[s]};
                    double vy[4] = {s ? vp.y : vp.x, s ? v0.y : v0.x, s ? vm.y : vm.x, s ? vmm.y : vmm.x};
                    const double wc = s ? w0.y : w0.x, wb = s ? wm.y : wm.x;
                    const double d = fd_div_point<CDS>(ux, vy, wc, wb, g.dx, g.dy, dzk);
                    if (ux[1] != ux[1] || vy[1] != vy[1] || wc != wc || d != d) {
                        nan = 1;
                    } else {
                        sm += fabs(d);
                        mx = absmax_pick(mx, d);
                    }
                }
                wm = w0;
            }
        }
    } else {
    const long long ncb = (g.nxy + 255) / 256;
    long long nch = (2LL * gridDim.x + ncb - 1) / ncb;
    if (nch > g.nz) nch = g.nz;
    const int kc = (int)((g.nz + nch - 1) / nch);
    for (long long un = blockIdx.x; un < ncb * nch; un += gridDim.x) {
        const long long cb = un % ncb;
        const int k0 = (int)(un / ncb) * kc, k1 = min(g.nz, k0 + kc);
        const long long ij = cb * 256 + tid;
        if (ij >= g.nxy || k0 >= k1) continue;
        const int j = (int)(ij / g.nx), i = (int)(ij - (long long)j * g.nx);
        const int xp1 = wrapi(i + 1, g.nx) - i, xm1 = wrapi(i - 1, g.nx) - i, xm2 = wrapi(i - 2, g.nx) - i;
        const long long yp1 = (long long)(wrapi(j + 1, g.ny) - j) * g.nx, ym1 = (long long)(wrapi(j - 1, g.ny) - j) * g.nx;
        const long long ym2 = (long long)(wrapi(j - 2, g.ny) - j) * g.nx;
        double wm = k0 > 0 ? (double)f.w[(long long)(k0 - 1) * g.nxy + ij] : 0.0;
        for (int kb = k0; kb < k1; kb += 2) {
            double ux[2][4], vy[2][4], wc[2];
            bool in[2];
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                in[e] = kb + e < k1;
                const long long q = (long long)(in[e] ? kb + e : kb) * g.nxy + ij;
                ux[e][1] = (double)f.u[q]; ux[e][2] = (double)f.u[q + xm1];
                vy[e][1] = (double)f.v[q]; vy[e][2] = (double)f.v[q + ym1];
                if (CDS == 2) {
                    ux[e][0] = (double)f.u[q + xp1]; ux[e][3] = (double)f.u[q + xm2];
                    vy[e][0] = (double)f.v[q + yp1]; vy[e][3] = (double)f.v[q + ym2];
                } else {
                    ux[e][0] = ux[e][3] = vy[e][0] = vy[e][3] = 0.0;
                }
                wc[e] = (double)f.w[q];
            }
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                if (!in[e]) continue;
                const double w_below = e == 0 ? wm : wc[0];
                const double d = fd_div_point<CDS>(ux[e], vy[e], wc[e], w_below, g.dx, g.dy, ldz(g.z.dz, kb + e));
                if (ux[e][1] != ux[e][1] || vy[e][1] != vy[e][1] || wc[e] != wc[e] || d != d) {
                    nan = 1;
                } else {
                    sm += fabs(d);
                    mx = absmax_pick(mx, d);
                }
            }
            wm = wc[1];
        }
    }
    }
    if (nan) s_nan = 1;
    sm = warp_sum(sm);
    mx = warp_absmax(mx);
    const int lane = tid & 31, wid = tid >> 5;
    if (lane == 0) { s_sum[wid] = sm; s_max[wid] = mx; }
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
        sm = lane < nw ? s_sum[lane] : 0.0;
        mx = lane < nw ? s_max[lane] : 0.0;
        sm = warp_sum(sm);
        mx = warp_absmax(mx);
        if (lane == 0) {
            part[3 * blockIdx.x + 0] = sm;
            part[3 * blockIdx.x + 1] = mx;
            part[3 * blockIdx.x + 2] = s_nan ? 1.0 : 0.0;
        }
    }
}
template <typename R, int CDS>
__global__ void __launch_bounds__(256, DivMinBlocks<R>::v) k_div_check(DivArgs<R> a) { k_div_check_body<R, CDS>(a, blockIdx, gridDim); }

template <typename R> struct StatsArgs {
    FieldsIn<R> f;
    Geo g;
    const R* uhx_s; const R* vhy_s;     // null on the spectral path: u, v used directly
    double* mean[11];
    // FP32 storage: the step's products go into FP32 sums of the current window
    // of `window` steps, folded into the FP64 sums after every step whose number
    // is a multiple of the window (null: straight into the FP64 sums)
    float* win[11];
    const int* step;                     // completed steps, this one included
    int window;
    int accumulate;
    // non-null (no temperature equation, T frozen): the temperature terms (mean_t,
    // mean_tt, mean_tw) are not accumulated; the kernel counts the steps here and
    // k_tstat_flush adds them later from T and the growth of mean_w
    int* tdefer;
    double um, dt;
    double* part;                        // per block: sum u*dz, CFL max
};

// accumulators of the temperature terms (mean_t, mean_tt, mean_tw)
__host__ __device__ constexpr bool stats_is_t(int a) { return a == 3 || a == 9 || a == 10; }

// The deferred temperature terms of n statistics steps with T frozen:
// mean_t += n T, mean_tt += n T^2, mean_tw += T (Sw(k) + Sw(k-1)) / 2, where Sw is
// the growth of the mean_w sums since the last flush (w below the wall is 0).
template <typename R>
__global__ void k_tstat_flush(const R* __restrict__ t, double* mt, double* mtt, double* mtw,
                              const double* __restrict__ mw, const float* __restrict__ ww,
                              const double* __restrict__ mw0, const int* cnt, long long nxy, long long n)
{
    const double nd = (double)*cnt;
    if (nd == 0.0) return;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const double tv = (double)t[q];
        const double s0 = mw[q] + (ww ? (double)ww[q] : 0.0) - mw0[q];
        const double s1 = q >= nxy ? mw[q - nxy] + (ww ? (double)ww[q - nxy] : 0.0) - mw0[q - nxy] : 0.0;
        mt[q] += nd * tv;
        mtt[q] += nd * (tv * tv);
        mtw[q] += tv * 0.5 * (s0 + s1);
    }
}
// after a flush: the mean_w sums it started from, and no step pending
static __global__ void k_tstat_snap(double* mw0, const double* __restrict__ mw, const float* __restrict__ ww,
                                    int* cnt, long long n)
{
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        mw0[q] = mw[q] + (ww ? (double)ww[q] : 0.0);
    if (blockIdx.x == 0 && threadIdx.x == 0) *cnt = 0;
}

// FP64 sums plus the pending FP32 window: what the mean accumulators hold
static __global__ void k_mean_combine(double* __restrict__ dst, const double* __restrict__ tot,
                               const float* __restrict__ win, long long n)
{
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        dst[q] = tot[q] + (double)win[q];
}

// calculate_mean_fields (src/module_tools.f90:362-404 / src/module_spectral.f90:1012-1052)
// fused with the bulk velocity sum of calculate_ubar (src/module_parameters.f90:513-546)
// and the CFL of screen_cpu_time (src/module_io.f90:43-61) for the next step.
// A thread walks its (i,j) column through a chunk of levels, G levels at a time:
// every load of a group (fields, then accumulators) is issued before its first
// store, so the read-modify-writes of consecutive levels overlap in flight.
// FP32 storage: registers sized for three resident blocks
template <typename R> struct StatsMinBlocks { static constexpr int v = sizeof(R) == sizeof(float) ? 3 : 2; };

template <typename R>
__device__ __forceinline__ void k_stats_body(const StatsArgs<R>& s, const uint3 blockIdx, const dim3 gridDim)
{
    // blockIdx.x: 256 consecutive (i,j) points of a plane; blockIdx.y: a chunk of levels
    constexpr int G = 2;
    __shared__ double s_sum[8], s_cfl[8];
    const Geo& g = s.g;
    const int tid = threadIdx.x;
    const double rdx = 1.0 / g.dx, rdy = 1.0 / g.dy;
    const long long ij = (long long)blockIdx.x * blockDim.x + tid;
    const int kc = (g.nz + gridDim.y - 1) / gridDim.y;
    const int k0 = blockIdx.y * kc, k1 = min(g.nz, k0 + kc);
    double ub = 0.0, cfl = 0.0;
    if constexpr (sizeof(R) == sizeof(float)) {
        // FP32 storage: a thread owns two adjacent points (nxy is even), so every
        // field and window access is an 8-byte load or store; 512 points a block
        const long long p2 = ij * 2;
        if (p2 < g.nxy) {
            auto l2 = [](const float* p, long long q) { return *reinterpret_cast<const float2*>(p + q); };
            const double um = s.um;
            const bool fold = s.accumulate && (*s.step % s.window) == 0;
            const bool skt = s.tdefer != nullptr;
            if (skt && s.accumulate && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) ++*s.tdefer;
            // ceil(nz / gridDim.y) levels a chunk: the last chunks can start at or past
            // nz, and then read nothing (w below the chunk included)
            float2 wm = (k0 > 0 && k0 < k1) ? l2(s.f.w, (long long)(k0 - 1) * g.nxy + p2) : make_float2(0.0f, 0.0f);
#pragma unroll 2
            for (int k = k0; k < k1; ++k) {
                const long long q = (long long)k * g.nxy + p2;
                const float2 u = l2(s.f.u, q), v = l2(s.f.v, q), w = l2(s.f.w, q);
                const double dzk = ldz(g.z.dz, k);
                ub += (double)u.x * dzk;
                cfl = fmax(cfl, s.dt * fabs((double)u.x) * rdx + s.dt * fabs((double)v.x) * rdy + s.dt * fabs((double)w.x) / dzk);
                ub += (double)u.y * dzk;
                cfl = fmax(cfl, s.dt * fabs((double)u.y) * rdx + s.dt * fabs((double)v.y) * rdy + s.dt * fabs((double)w.y) / dzk);
                if (s.accumulate) {
                    const float2 t = skt ? make_float2(0.0f, 0.0f) : l2(s.f.t, q);
                    const float2 ux = s.uhx_s ? l2(s.uhx_s, q) : u;
                    const float2 vy = s.vhy_s ? l2(s.vhy_s, q) : v;
                    auto c = [&](int a, int e) -> double {
                        const double U = e ? u.y : u.x, V = e ? v.y : v.x, Wc = e ? w.y : w.x, T = e ? t.y : t.x;
                        const double WP = e ? wm.y : wm.x;
                        const double wc = 0.5 * (Wc + WP);
                        switch (a) {
                        case 0: return U + um;
                        case 1: return V;
                        case 2: return Wc;
                        case 3: return T;
                        case 4: return (U + um) * (U + um);
                        case 5: return V * V;
                        case 6: return Wc * Wc;
                        case 7: return wc * ((double)(e ? ux.y : ux.x) + um);
                        case 8: return wc * (double)(e ? vy.y : vy.x);
                        case 9: return T * T;
                        default: return T * 0.5 * (Wc + WP);
                        }
                    };
                    if (!fold) {
                        float2 m[11];
#pragma unroll
                        for (int a = 0; a < 11; ++a)
                            if (!(skt && stats_is_t(a))) m[a] = l2(s.win[a], q);
#pragma unroll
                        for (int a = 0; a < 11; ++a)
                            if (!(skt && stats_is_t(a)))
                                *reinterpret_cast<float2*>(s.win[a] + q) =
                                    make_float2((float)((double)m[a].x + c(a, 0)), (float)((double)m[a].y + c(a, 1)));
                    } else {
                        // end of a window: FP64 sum += window + this step, the window restarts at 0
#pragma unroll
                        for (int a = 0; a < 11; ++a) {
                            if (skt && stats_is_t(a)) continue;
                            double2* mp = reinterpret_cast<double2*>(s.mean[a] + q);
                            const float2 wv = l2(s.win[a], q);
                            double2 mv = *mp;
                            mv.x += (double)wv.x + c(a, 0);
                            mv.y += (double)wv.y + c(a, 1);
                            *mp = mv;
                            *reinterpret_cast<float2*>(s.win[a] + q) = make_float2(0.0f, 0.0f);
                        }
                    }
                }
                wm = w;
            }
        }
    } else if (ij < g.nxy) {
        const R* __restrict__ fu = s.f.u; const R* __restrict__ fv = s.f.v;
        const R* __restrict__ fw = s.f.w; const R* __restrict__ ft = s.f.t;
        const R* __restrict__ fux = s.uhx_s; const R* __restrict__ fvy = s.vhy_s;
        const double um = s.um;
        // FP32 storage always keeps the FP32 window sums (allocated with the handle)
        const bool fold = sizeof(R) == sizeof(float) && s.accumulate && (*s.step % s.window) == 0;
        const bool skt = s.tdefer != nullptr;
        if (skt && s.accumulate && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) ++*s.tdefer;
        double wm = (k0 > 0 && k0 < k1) ? (double)fw[(long long)(k0 - 1) * g.nxy + ij] : 0.0;
        for (int kb = k0; kb < k1; kb += G) {
            // the fields stay in the storage type in registers; products in FP64
            R u[G], v[G], w[G], t[G], ux[G], vy[G];
            bool in[G];
#pragma unroll
            for (int e = 0; e < G; ++e) {
                in[e] = kb + e < k1;
                const long long q = (long long)(in[e] ? kb + e : kb) * g.nxy + ij;
                u[e] = fu[q]; v[e] = fv[q]; w[e] = fw[q];
                if (s.accumulate) {
                    t[e] = skt ? R(0) : ft[q];
                    ux[e] = fux ? fux[q] : u[e];
                    vy[e] = fvy ? fvy[q] : v[e];
                } else {
                    t[e] = R(0); ux[e] = R(0); vy[e] = R(0);
                }
            }
            double wp[G];                   // w one level below each of the group's levels
#pragma unroll
            for (int e = 0; e < G; ++e) {
                wp[e] = e == 0 ? wm : (double)w[e - 1];
                const double dzk = ldz(g.z.dz, in[e] ? kb + e : kb);
                if (in[e]) {
                    const double ue = u[e];
                    ub += ue * dzk;
                    cfl = fmax(cfl, s.dt * fabs(ue) * rdx + s.dt * fabs((double)v[e]) * rdy + s.dt * fabs((double)w[e]) / dzk);
                }
            }
            wm = w[G - 1];
            if (!s.accumulate) continue;
            // this step's product a at level kb + e
            auto c = [&](int a, int e) -> double {
                const double U = u[e], V = v[e], Wc = w[e], T = t[e];
                const double wc = 0.5 * (Wc + wp[e]);
                switch (a) {
                case 0: return U + um;
                case 1: return V;
                case 2: return Wc;
                case 3: return T;
                case 4: return (U + um) * (U + um);
                case 5: return V * V;
                case 6: return Wc * Wc;
                case 7: return wc * ((double)ux[e] + um);
                case 8: return wc * (double)vy[e];
                case 9: return T * T;
                default: return T * 0.5 * (Wc + wp[e]);
                }
            };
            if (sizeof(R) == sizeof(double)) {
                // FP64 storage: straight into the FP64 sums
                double m[11][G];
#pragma unroll
                for (int a = 0; a < 11; ++a)
#pragma unroll
                    for (int e = 0; e < G; ++e)
                        if (in[e] && !(skt && stats_is_t(a))) m[a][e] = s.mean[a][(long long)(kb + e) * g.nxy + ij];
#pragma unroll
                for (int a = 0; a < 11; ++a)
#pragma unroll
                    for (int e = 0; e < G; ++e)
                        if (in[e] && !(skt && stats_is_t(a))) s.mean[a][(long long)(kb + e) * g.nxy + ij] = m[a][e] + c(a, e);
            } else if (!fold) {
                float m[11][G];
#pragma unroll
                for (int a = 0; a < 11; ++a)
#pragma unroll
                    for (int e = 0; e < G; ++e)
                        if (in[e] && !(skt && stats_is_t(a))) m[a][e] = s.win[a][(long long)(kb + e) * g.nxy + ij];
#pragma unroll
                for (int a = 0; a < 11; ++a)
#pragma unroll
                    for (int e = 0; e < G; ++e)
                        if (in[e] && !(skt && stats_is_t(a))) s.win[a][(long long)(kb + e) * g.nxy + ij] = (float)((double)m[a][e] + c(a, e));
            } else {
                // end of a window: FP64 sum += window + this step, the window restarts at 0
#pragma unroll
                for (int a = 0; a < 11; ++a)
#pragma unroll
                    for (int e = 0; e < G; ++e)
                        if (in[e] && !(skt && stats_is_t(a))) {
                            const long long q = (long long)(kb + e) * g.nxy + ij;
                            s.mean[a][q] += (double)s.win[a][q] + c(a, e);
                            s.win[a][q] = 0.0f;
                        }
            }
        }
    }
    ub = warp_sum(ub);
    cfl = warp_max(cfl);
    const int lane = tid & 31, wid = tid >> 5;
    if (lane == 0) { s_sum[wid] = ub; s_cfl[wid] = cfl; }
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
        ub = lane < nw ? s_sum[lane] : 0.0;
        cfl = lane < nw ? s_cfl[lane] : 0.0;
        ub = warp_sum(ub);
        cfl = warp_max(cfl);
        if (lane == 0) {
            const long long b = (long long)blockIdx.y * gridDim.x + blockIdx.x;
            s.part[2 * b + 0] = ub;
            s.part[2 * b + 1] = cfl;
        }
    }
}
template <typename R>
__global__ void __launch_bounds__(256, StatsMinBlocks<R>::v) k_stats(StatsArgs<R> s) { k_stats_body<R>(s, blockIdx, gridDim); }

// ---------------------------------------------------------------------------
// rayleigh_damping (src/module_tools.f90:705-749) of u, v, w, p, t on levels
// kd..nz-1: x -= sigma(k) (x - <x>_plane). The plane means come first (fixed
// reduction order), then one pass keeps the undamped values of those levels
// (the reference's ghost cells still hold them, see Acc) and damps the fields.
// ---------------------------------------------------------------------------
template <typename R> struct FdDampArgs {
    R* f[5];
    R* stale[5];          // [k-kd][j][i]
    double* mean;         // [5][nz]
    const double* sig;    // [nz], 0 below the layer
    Geo g;
    int kd;
};

template <typename R>
__global__ void __launch_bounds__(256) k_fd_damp_mean(FdDampArgs<R> a)
{
    __shared__ double sh[8];
    const int k = a.kd + blockIdx.x, f = blockIdx.y;
    const R* src = a.f[f] + (long long)k * a.g.nxy;
    double sm = 0.0;
    for (long long q = threadIdx.x; q < a.g.nxy; q += blockDim.x) sm += (double)src[q];
    sm = warp_sum(sm);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = sm;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
        a.mean[f * a.g.nz + k] = t / (double)a.g.nx / (double)a.g.ny;
    }
}

template <typename R>
__global__ void __launch_bounds__(256) k_fd_damp_apply(FdDampArgs<R> a)
{
    const long long per = (long long)(a.g.nz - a.kd) * a.g.nxy;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < 5 * per; q += (long long)gridDim.x * blockDim.x) {
        const int f = (int)(q / per);
        const long long r = q - f * per;
        const int k = a.kd + (int)(r / a.g.nxy);
        R* x = a.f[f] + (long long)a.kd * a.g.nxy + r;
        const double v = (double)*x;
        a.stale[f][r] = (R)v;
        const double sg = __ldg(a.sig + k);
        *x = (R)(v - sg * (v - a.mean[f * a.g.nz + k]));
    }
}
