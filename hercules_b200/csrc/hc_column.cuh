// hc_column.cuh -- the per-wavenumber wall-normal solves.
//
// For every horizontal wavenumber pair (l, m) of the half spectrum one thread
// walks its z column. The FD kernel fuses what the reference does in eleven
// separate passes of time_advancement_fd (src/module_navier_stokes.f90:290-354):
//   three Helmholtz solves for u*, v*, w* (poisson_solver_fft with the ubnd and
//   zstagger flags, src/module_poisson_solver.f90:483-658), the pressure source
//   (get_p_eqn_src :127-176, a circulant stencil, so its spectral symbol applied
//   to the solved modes), the phi Poisson solve with the null-space pin, the
//   projection (calculate_uvw, src/module_navier_stokes.f90:659-734) and the phi
//   part of the pressure update (calculate_new_p :739-808), whose physical
//   p += psi is applied by the inverse-FFT epilogue.
// The Thomas elimination, the (0,0) mean mode and every coefficient stay in FP64
// for both precision modes.
//
// Thomas coefficients follow the reference's builders (get_*_eqn_coeff,
// src/module_poisson_solver.f90:32-477) including their first-mode-only wall
// folds: dg00[k] is the diagonal part for the (0,0) mode, dgen[k] for all others.
#pragma once
#include "hc_common.cuh"

struct ColCoef {
    // per l (nxh) and m (ny)
    const double* hx;    // Helmholtz symbol (momentum, nu), includes 0.5 dt nu
    const double* hy;
    const double* hxt;   // Helmholtz symbol (temperature, alpha)
    const double* hyt;
    const double* px;    // Poisson symbol
    const double* py;
    const double2* dx;   // divergence symbols
    const double2* dy;
    const double2* gx;   // gradient symbols
    const double2* gy;
    const double* lx;    // second-derivative symbols (pressure update)
    const double* ly;
    // per k (nz): sub/super diagonals and diagonal parts
    const double* au; const double* cu; const double* dgu; const double* d0u;
    const double* aw; const double* cw; const double* dgw; const double* d0w;
    const double* ap; const double* cp; const double* dgp; const double* d0p;
    const double* at; const double* ct; const double* dgt; const double* d0t;
    // per k reciprocals of dz, dz_t, dz_b
    const double* rdz; const double* rdzt; const double* rdzb;
};

struct ColScratch {
    double* bu;   // [nz][ncol] eliminated diagonals
    double* bw;
    double* bp;
    double2* su;  // [nz][ncol] eliminated right-hand sides, then solutions
    double2* sv;
    double2* sw;
    double2* sp;
};

template <typename R> struct ColArgs {
    typename V2<R>::T* qu;   // in: q^u, out: u^(n+1) modes (in place)
    typename V2<R>::T* qv;
    typename V2<R>::T* qw;
    typename V2<R>::T* psi;  // out: phi - rk_c dt nu/2 lap(phi)
    ColCoef c;
    ColScratch s;
    Geo g;
    double rk_c, dt, nu;
    double bcu0, bcu1;       // (0,0)-mode source corrections of the u equation (ubnd)
    const int* halt;
};

template <typename R> __device__ __forceinline__ double2 ld2(const typename V2<R>::T* p, long long i)
{
    typename V2<R>::T v = p[i];
    return make_double2((double)v.x, (double)v.y);
}
template <typename R> __device__ __forceinline__ void st2(typename V2<R>::T* p, long long i, double2 v)
{
    p[i] = mk2<R>((R)v.x, (R)v.y);
}
__device__ __forceinline__ double2 zsub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 zadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 zscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 zmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }

template <typename R>
__device__ __forceinline__ void k_column_fd_body(const ColArgs<R>& a, const uint3 blockIdx, const dim3 gridDim)
{
    if (a.halt && *a.halt) return;
    const long long ncol = a.g.ncol;
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncol) return;
    const int nz = a.g.nz;
    const int l = (int)(c % a.g.nxh);
    const int m = (int)(c / a.g.nxh);
    const bool is00 = (c == 0);
    const double rk = a.rk_c, dt = a.dt;
    const double lam = __ldg(a.c.hx + l) + __ldg(a.c.hy + m);
    const double lamp = __ldg(a.c.px + l) + __ldg(a.c.py + m);
    const double* dgu = is00 ? a.c.d0u : a.c.dgu;
    const double* dgw = is00 ? a.c.d0w : a.c.dgw;
    const double* dgp = is00 ? a.c.d0p : a.c.dgp;

    // ---- forward elimination: u and v share one matrix, w has its own (k <= nz-2)
    double bu_p = 0.0, bw_p = 0.0;
    double2 su_p = make_double2(0, 0), sv_p = su_p, sw_p = su_p;
    for (int k = 0; k < nz; ++k) {
        const long long id = (long long)k * ncol + c;
        double2 su = ld2<R>(a.qu, id), sv = ld2<R>(a.qv, id);
        if (is00) {
            if (k == 0) su.x += a.bcu0;
            if (k == nz - 1) su.x += a.bcu1;
        }
        double bu = 1.0 + rk * (-lam + __ldg(dgu + k));
        if (k > 0) {
            const double t = rk * __ldg(a.c.au + k) / bu_p;
            bu = bu - rk * __ldg(a.c.cu + k - 1) * t;
            su = zsub(su, zscale(su_p, t));
            sv = zsub(sv, zscale(sv_p, t));
        }
        a.s.bu[id] = bu; a.s.su[id] = su; a.s.sv[id] = sv;
        bu_p = bu; su_p = su; sv_p = sv;
        if (k <= nz - 2) {
            double2 sw = ld2<R>(a.qw, id);
            double bw = 1.0 + rk * (-lam + __ldg(dgw + k));
            if (k > 0) {
                const double t = rk * __ldg(a.c.aw + k) / bw_p;
                bw = bw - rk * __ldg(a.c.cw + k - 1) * t;
                sw = zsub(sw, zscale(sw_p, t));
            }
            a.s.bw[id] = bw; a.s.sw[id] = sw;
            bw_p = bw; sw_p = sw;
        }
    }
    // ---- back substitution: u*, v*, w* (w* = 0 on the top wall)
    {
        double2 xu = make_double2(0, 0), xv = xu, xw = xu;
        for (int k = nz - 1; k >= 0; --k) {
            const long long id = (long long)k * ncol + c;
            const double b = a.s.bu[id];
            if (k == nz - 1) {
                xu = zscale(a.s.su[id], 1.0 / b); xv = zscale(a.s.sv[id], 1.0 / b);
                xu = make_double2(a.s.su[id].x / b, a.s.su[id].y / b);
                xv = make_double2(a.s.sv[id].x / b, a.s.sv[id].y / b);
            } else {
                const double cc = rk * __ldg(a.c.cu + k);
                double2 su = a.s.su[id], sv = a.s.sv[id];
                xu = make_double2((su.x - cc * xu.x) / b, (su.y - cc * xu.y) / b);
                xv = make_double2((sv.x - cc * xv.x) / b, (sv.y - cc * xv.y) / b);
            }
            a.s.su[id] = xu; a.s.sv[id] = xv;
            if (k <= nz - 2) {
                const double bw = a.s.bw[id];
                double2 sw = a.s.sw[id];
                if (k == nz - 2) xw = make_double2(sw.x / bw, sw.y / bw);
                else {
                    const double cc = rk * __ldg(a.c.cw + k);
                    xw = make_double2((sw.x - cc * xw.x) / bw, (sw.y - cc * xw.y) / bw);
                }
                a.s.sw[id] = xw;
            } else {
                a.s.sw[id] = make_double2(0, 0);
            }
        }
    }
    // ---- phi: source = div(u*)/dt, forward elimination
    const double2 DX = __ldg(a.c.dx + l), DY = __ldg(a.c.dy + m);
    {
        double bp_p = 0.0;
        double2 sp_p = make_double2(0, 0), w_prev = sp_p;
        for (int k = 0; k < nz; ++k) {
            const long long id = (long long)k * ncol + c;
            const double2 us = a.s.su[id], vs = a.s.sv[id], ws = a.s.sw[id];
            const double dzk = ldz(a.g.z.dz, k);
            double2 div = zadd(zmul(DX, us), zmul(DY, vs));
            div = zadd(div, make_double2((ws.x - w_prev.x) / dzk, (ws.y - w_prev.y) / dzk));
            double2 src = make_double2(div.x / dt, div.y / dt);
            w_prev = ws;
            if (is00 && k == 0) src = make_double2(0, 0);             // null-space pin
            double bp = rk * (lamp + __ldg(dgp + k));
            if (k > 0) {
                const double cprev = (is00 && k == 1) ? 0.0 : rk * __ldg(a.c.cp + k - 1);
                const double t = rk * __ldg(a.c.ap + k) / bp_p;
                bp = bp - cprev * t;
                src = zsub(src, zscale(sp_p, t));
            }
            a.s.bp[id] = bp; a.s.sp[id] = src;
            bp_p = bp; sp_p = src;
        }
    }
    // ---- phi back substitution + projection + psi
    {
        const double2 GX = __ldg(a.c.gx + l), GY = __ldg(a.c.gy + m);
        const double lxy = __ldg(a.c.lx + l) + __ldg(a.c.ly + m);
        const double cpr = rk * dt, cps = rk * 0.5 * dt * a.nu;
        double2 ph_n = make_double2(0, 0);   // phi(k+1)
        double2 ph_nn = ph_n;                // phi(k+2)
        double2 ph = ph_n;
        for (int k = nz - 1; k >= -1; --k) {
            if (k >= 0) {
                const long long id = (long long)k * ncol + c;
                const double b = a.s.bp[id];
                const double2 s = a.s.sp[id];
                if (k == nz - 1) ph = make_double2(s.x / b, s.y / b);
                else {
                    const double cc = (is00 && k == 0) ? 0.0 : rk * __ldg(a.c.cp + k);
                    ph = make_double2((s.x - cc * ph_n.x) / b, (s.y - cc * ph_n.y) / b);
                }
                // projection at level k
                const double2 us = a.s.su[id], vs = a.s.sv[id], ws = a.s.sw[id];
                st2<R>(a.qu, id, zsub(us, zscale(zmul(GX, ph), cpr)));
                st2<R>(a.qv, id, zsub(vs, zscale(zmul(GY, ph), cpr)));
                if (k <= nz - 2) {
                    const double dzt = ldz(a.g.z.dz_t, k);
                    st2<R>(a.qw, id, make_double2(ws.x - cpr * (ph_n.x - ph.x) / dzt, ws.y - cpr * (ph_n.y - ph.y) / dzt));
                } else {
                    st2<R>(a.qw, id, make_double2(0, 0));
                }
            }
            // psi at level k+1 (needs phi(k), phi(k+1), phi(k+2); Neumann ghosts)
            const int kp = k + 1;
            if (kp <= nz - 1) {
                const double2 pc = ph_n;
                const double2 pu = (kp == nz - 1) ? pc : ph_nn;
                const double2 pd = (k >= 0) ? ph : pc;
                const double dzt = ldz(a.g.z.dz_t, kp), dzb = ldz(a.g.z.dz_b, kp), dzk = ldz(a.g.z.dz, kp);
                double2 lz;
                lz.x = ((pu.x - pc.x) / dzt - (pc.x - pd.x) / dzb) / dzk;
                lz.y = ((pu.y - pc.y) / dzt - (pc.y - pd.y) / dzb) / dzk;
                double2 ps;
                ps.x = pc.x - cps * (lxy * pc.x + lz.x);
                ps.y = pc.y - cps * (lxy * pc.y + lz.y);
                st2<R>(a.psi, (long long)kp * ncol + c, ps);
            }
            ph_nn = ph_n;
            ph_n = ph;
        }
    }
}
template <typename R>
__global__ void __launch_bounds__(256) k_column_fd(ColArgs<R> a) { k_column_fd_body<R>(a, blockIdx, gridDim); }

// Temperature Helmholtz solve (poisson_solver_fft with tbnd=1), in place.
template <typename R> struct ColTArgs {
    typename V2<R>::T* qt;
    ColCoef c;
    ColScratch s;
    Geo g;
    double rk_c;
    double bct0, bct1;       // (0,0)-mode Dirichlet source corrections (tbnd)
    typename V2<R>::T* out;  // solution (may equal qt)
    int ltr, mtr;            // > 0: spectral truncation, modes |l| >= ltr or |m| >= mtr set to 0
    const int* halt;
};

// 2/3-rule truncation test (spectral_truncation, src/module_spectral.f90:1222-1268)
// for half-spectrum column (l, m); m in FFT order.
__device__ __forceinline__ bool spec_truncated(int l, int m, int ny, int ltr, int mtr)
{
    if (ltr <= 0) return false;
    const int ms = m < ny / 2 ? m : m - ny;
    return l >= ltr || ms >= mtr || ms <= -mtr;
}

template <typename R>
__device__ __forceinline__ void k_column_t_body(const ColTArgs<R>& a, const uint3 blockIdx, const dim3 gridDim)
{
    if (a.halt && *a.halt) return;
    const long long ncol = a.g.ncol;
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncol) return;
    const int nz = a.g.nz;
    const int l = (int)(c % a.g.nxh);
    const int m = (int)(c / a.g.nxh);
    const bool is00 = (c == 0);
    const double rk = a.rk_c;
    const double lam = __ldg(a.c.hxt + l) + __ldg(a.c.hyt + m);
    const double* dg = is00 ? a.c.d0t : a.c.dgt;
    double b_p = 0.0;
    double2 s_p = make_double2(0, 0);
    for (int k = 0; k < nz; ++k) {
        const long long id = (long long)k * ncol + c;
        double2 s = ld2<R>(a.qt, id);
        if (is00) {
            if (k == 0) s.x += a.bct0;
            if (k == nz - 1) s.x += a.bct1;
        }
        double b = 1.0 + rk * (-lam + __ldg(dg + k));
        if (k > 0) {
            const double t = rk * __ldg(a.c.at + k) / b_p;
            b = b - rk * __ldg(a.c.ct + k - 1) * t;
            s = zsub(s, zscale(s_p, t));
        }
        a.s.bu[id] = b; a.s.su[id] = s;
        b_p = b; s_p = s;
    }
    double2 x = make_double2(0, 0);
    const bool tr = spec_truncated(l, m, a.g.ny, a.ltr, a.mtr);
    for (int k = nz - 1; k >= 0; --k) {
        const long long id = (long long)k * ncol + c;
        const double b = a.s.bu[id];
        const double2 s = a.s.su[id];
        if (k == nz - 1) x = make_double2(s.x / b, s.y / b);
        else {
            const double cc = rk * __ldg(a.c.ct + k);
            x = make_double2((s.x - cc * x.x) / b, (s.y - cc * x.y) / b);
        }
        st2<R>(a.out, id, tr ? make_double2(0, 0) : x);
    }
}
template <typename R>
__global__ void __launch_bounds__(256) k_column_t(ColTArgs<R> a) { k_column_t_body<R>(a, blockIdx, gridDim); }
