// hc_rhs_tiled.cuh -- SMEM-tiled momentum right-hand side (get_momentum_cnvdiff,
// src/module_cnvdiff.f90:35-374), the hot stencil of the FD step.
//
// A block owns a TX x TY tile of (x, y) and marches up a chunk of k levels.
// Per level it keeps
//   * raw planes of u, v, w at k-1, k, k+1 and p, t at k, k+1 in a rolling SMEM
//     window with a 4-point halo (periodic wrap and the z wall/top conditions of
//     update_boundary_uvw/p/t are applied while loading), and
//   * the products that the flux differences need -- uhx, uhy, vhx, vhy, whx and
//     uhy*vhx, uhz*whx, vhz*why (get_interp_fields_uvwhxyz + the ghost values of
//     update_boundary_uvwhxyz) -- computed once per point on a 2-point halo,
// so every interpolant is evaluated once per point instead of once per use. The
// level-(k-1) products a thread needs for the z differences stay in registers.
#pragma once
#include "hc_fd.cuh"

#define RT_TX 32
#define RT_TY 8
#define RT_W4 (RT_TX + 8)
#define RT_H4 (RT_TY + 8)
#define RT_P4 (RT_W4 * RT_H4)
#define RT_W2 (RT_TX + 4)
#define RT_H2 (RT_TY + 4)
#define RT_P2 (RT_W2 * RT_H2)
#define RT_NFLUX 8

template <typename R> struct RhsTArgs {
    FieldsIn<R> f;
    Geo g;
    R* ff; R* gg; R* hh;
    R* qu; R* qv; R* qw;
    R* uhx_s; R* vhy_s;
    double rk_a, rk_b, rk_c;
    Phys ph;
    const DevScalars* sc;
    int kchunk;
    int with_t;
    // divergence check of the incoming u, v, w (screen_div_error of the previous
    // sub-step, src/module_io.f90:85-206), per block: sum |div|, signed div of
    // largest magnitude, NaN flag; null when not wanted
    double* part_div;
    const R* bfx; const R* bfy; const R* bfz;   // body force added to ff, gg, hh (null: none)
    const void* zm;      // per-level metrics [5][nz] in the storage type (the strip kernel)
};

#define RT_KMAX 64
template <typename R> __host__ size_t rhs_tiled_smem(int with_t)
{
    return sizeof(R) * ((size_t)(9 + 2 + (with_t ? 2 : 0)) * RT_P4 + (size_t)RT_NFLUX * RT_P2) +
           sizeof(R) * 6 * (RT_KMAX + 1);
}

#define RT_NLD ((RT_P4 + 255) / 256)

// Load one raw plane (level lvl, possibly the ghost level -1 or nz) into SMEM.
// off[] holds this thread's wrapped (x, y) offsets, computed once per block.
template <typename R>
__device__ __forceinline__ void rt_load_plane(R* dst, const R* src, const Geo& g, const int* off, int lvl, int kind,
                                              R um, R tbot, R ttop, int closed)
{
    // kind: 0 u, 1 v, 2 w, 3 p, 4 t
    const int nz = g.nz;
    int sl = lvl;
    R sgn = R(1), add = R(0);
    if (lvl < 0) {
        sl = 0;
        if (kind == 0) { sgn = R(-1); add = -R(2) * um; }
        else if (kind == 1) { sgn = R(-1); }
        else if (kind == 2) { sgn = R(0); }
        else if (kind == 4) { sgn = R(-1); add = R(2) * tbot; }
    } else if (lvl >= nz) {
        sl = nz - 1;
        if (kind == 0) { if (closed) { sgn = R(-1); add = -R(2) * um; } }
        else if (kind == 1) { if (closed) sgn = R(-1); }
        else if (kind == 2) { sl = nz - 2; sgn = R(-1); }
        else if (kind == 4) { sgn = R(-1); add = R(2) * ttop; }
    }
    const R* base = src + (long long)sl * g.nxy;
#pragma unroll
    for (int r = 0; r < RT_NLD; ++r) {
        const int e = threadIdx.x + 256 * r;
        if (e < RT_P4) dst[e] = sgn * __ldg(base + off[r]) + add;
    }
}

// Register-staged variant used to overlap the next level's loads with the
// current level's arithmetic: fetch issues the loads, put stores to SMEM.
template <typename R>
__device__ __forceinline__ void rt_fetch(R* v, const R* src, const Geo& g, const int* off, int lvl, int kind,
                                         R um, R tbot, R ttop, int closed)
{
    const int nz = g.nz;
    int sl = lvl;
    R sgn = R(1), add = R(0);
    if (lvl >= nz) {
        sl = nz - 1;
        if (kind == 0) { if (closed) { sgn = R(-1); add = -R(2) * um; } }
        else if (kind == 1) { if (closed) sgn = R(-1); }
        else if (kind == 2) { sl = nz - 2; sgn = R(-1); }
        else if (kind == 4) { sgn = R(-1); add = R(2) * ttop; }
    }
    const R* base = src + (long long)sl * g.nxy;
#pragma unroll
    for (int r = 0; r < RT_NLD; ++r) {
        const int e = threadIdx.x + 256 * r;
        v[r] = (e < RT_P4) ? sgn * __ldg(base + off[r]) + add : R(0);
    }
}
template <typename R>
__device__ __forceinline__ void rt_put(R* dst, const R* v)
{
#pragma unroll
    for (int r = 0; r < RT_NLD; ++r) {
        const int e = threadIdx.x + 256 * r;
        if (e < RT_P4) dst[e] = v[r];
    }
}

// blocks per SM the register budget is sized for: FP32 fits three (80 registers,
// no spills), FP64 two
template <typename R> struct RhsMinBlocks { static constexpr int v = sizeof(R) == sizeof(float) ? 3 : 2; };

template <typename R, int CDS>
__device__ __forceinline__ void k_rhs_momentum_tiled_body(const RhsTArgs<R>& a, const uint3 blockIdx, const dim3 gridDim)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* sm = reinterpret_cast<R*>(smem_raw);
    R* SU = sm;                  // [3][P4]
    R* SV = SU + 3 * RT_P4;
    R* SW = SV + 3 * RT_P4;
    R* SP = SW + 3 * RT_P4;      // [2][P4]
    R* ST = SP + 2 * RT_P4;      // [2][P4] if with_t
    R* FX = ST + (a.with_t ? 2 * RT_P4 : 0);
    R* F_UHX = FX;
    R* F_UHY = FX + 1 * RT_P2;
    R* F_VHX = FX + 2 * RT_P2;
    R* F_VHY = FX + 3 * RT_P2;
    R* F_WHX = FX + 4 * RT_P2;
    R* F_B = FX + 5 * RT_P2;     // uhy * vhx
    R* F_CZ = FX + 6 * RT_P2;    // uhz * whx
    R* F_EZ = FX + 7 * RT_P2;    // vhz * why
    R* ZM = FX + RT_NFLUX * RT_P2;   // per level of the chunk: 1/dz, 1/dz_t, 1/dz_b, l_t, 1/dz(k+1)

    const Geo& g = a.g;
    const int nz = g.nz;
    const int x0 = blockIdx.x * RT_TX, y0 = blockIdx.y * RT_TY;
    const int kb = blockIdx.z * a.kchunk;
    const int ke = min(nz, kb + a.kchunk);
    const int tx = threadIdx.x % RT_TX, ty = threadIdx.x / RT_TX;
    const int xi = x0 + tx, yj = y0 + ty;
    const bool active = xi < g.nx && yj < g.ny;
    const R um = (R)a.ph.um, tbot = (R)a.ph.tbot, ttop = (R)a.ph.ttop;
    const int closed = a.ph.ochannel == 0;

    const R rdx = R(1) / (R)g.dx, rdy = R(1) / (R)g.dy;
    const R r24dx = R(1) / (R(24) * (R)g.dx), r24dy = R(1) / (R(24) * (R)g.dy);
    const R r12dx2 = R(1) / (R(12) * (R)g.dx2), r12dy2 = R(1) / (R(12) * (R)g.dy2);
    const R rdx2 = R(1) / (R)g.dx2, rdy2 = R(1) / (R)g.dy2;
    const R dt = (R)a.ph.dt, nu = (R)a.ph.nu, fc = (R)a.ph.fc;
    const R rka = (R)a.rk_a, rkb = (R)a.rk_b, rkc = (R)a.rk_c;
    const R cdif = rkc * R(0.5) * dt * nu;
    const R dpx = (R)a.sc->dpx_drive;
    const R got = (R)a.sc->got;
    const R h16 = R(0.0625);

    auto slot3 = [](int lvl) { return (lvl + 3) % 3; };
    for (int q = threadIdx.x; q < ke - kb; q += blockDim.x) {
        const int k = kb + q;
        ZM[q] = R(1) / (R)ldz(g.z.dz, k);
        ZM[(RT_KMAX + 1) + q] = R(1) / (R)ldz(g.z.dz_t, k);
        ZM[2 * (RT_KMAX + 1) + q] = R(1) / (R)ldz(g.z.dz_b, k);
        ZM[3 * (RT_KMAX + 1) + q] = (R)ldz(g.z.l_t, k);
        ZM[4 * (RT_KMAX + 1) + q] = R(1) / (R)ldz(g.z.dz, k + 1);
    }
    int off[RT_NLD];
#pragma unroll
    for (int r = 0; r < RT_NLD; ++r) {
        const int e = threadIdx.x + 256 * r;
        const int ry = e / RT_W4, rx = e - ry * RT_W4;
        int x = (x0 - 4 + rx) % g.nx; if (x < 0) x += g.nx;
        int y = (y0 - 4 + ry) % g.ny; if (y < 0) y += g.ny;
        off[r] = y * g.nx + x;
    }
    // initial window: u, v, w at kb-1, kb, kb+1; p, t at kb, kb+1
    for (int L = kb - 1; L <= kb + 1; ++L) {
        rt_load_plane<R>(SU + slot3(L) * RT_P4, a.f.u, g, off, L, 0, um, tbot, ttop, closed);
        rt_load_plane<R>(SV + slot3(L) * RT_P4, a.f.v, g, off, L, 1, um, tbot, ttop, closed);
        rt_load_plane<R>(SW + slot3(L) * RT_P4, a.f.w, g, off, L, 2, um, tbot, ttop, closed);
    }
    for (int L = kb; L <= kb + 1; ++L) {
        rt_load_plane<R>(SP + (L & 1) * RT_P4, a.f.p, g, off, L, 3, um, tbot, ttop, closed);
        if (a.with_t) rt_load_plane<R>(ST + (L & 1) * RT_P4, a.f.t, g, off, L, 4, um, tbot, ttop, closed);
    }
    __syncthreads();

    // own-point products of level kb-1 (uhz*whx, vhz*why); zero below the wall
    const int rc = (ty + 4) * RT_W4 + (tx + 4);     // own raw index
    const int fc0 = (ty + 2) * RT_W2 + (tx + 2);    // own flux index
    R cz_prev = R(0), ez_prev = R(0);
    if (kb > 0) {
        const int L = kb - 1;
        const R* u0 = SU + slot3(L) * RT_P4; const R* u1 = SU + slot3(L + 1) * RT_P4;
        const R* v0 = SV + slot3(L) * RT_P4; const R* v1 = SV + slot3(L + 1) * RT_P4;
        const R* w0 = SW + slot3(L) * RT_P4;
        const R l = (R)ldz(g.z.l_t, L);
        const R uhz = u1[rc] * l + u0[rc] * (R(1) - l);
        const R vhz = v1[rc] * l + v0[rc] * (R(1) - l);
        R whx, why;
        if (CDS == 1) { whx = R(0.5) * (w0[rc + 1] + w0[rc]); why = R(0.5) * (w0[rc + RT_W4] + w0[rc]); }
        else {
            whx = (-w0[rc + 2] + R(9) * w0[rc + 1] + R(9) * w0[rc] - w0[rc - 1]) * h16;
            why = (-w0[rc + 2 * RT_W4] + R(9) * w0[rc + RT_W4] + R(9) * w0[rc] - w0[rc - RT_W4]) * h16;
        }
        cz_prev = uhz * whx;
        ez_prev = vhz * why;
    }

    double dv_sum = 0.0, dv_max = 0.0;
    int dv_nan = 0;
    for (int k = kb; k < ke; ++k) {
        const bool more = k + 1 < ke;
        R nu_[RT_NLD], nv_[RT_NLD], nw_[RT_NLD], np_[RT_NLD], nt_[RT_NLD];
        if (more) {
            const int L = k + 2;
            rt_fetch<R>(nu_, a.f.u, g, off, L, 0, um, tbot, ttop, closed);
            rt_fetch<R>(nv_, a.f.v, g, off, L, 1, um, tbot, ttop, closed);
            rt_fetch<R>(nw_, a.f.w, g, off, L, 2, um, tbot, ttop, closed);
            rt_fetch<R>(np_, a.f.p, g, off, L, 3, um, tbot, ttop, closed);
            if (a.with_t) rt_fetch<R>(nt_, a.f.t, g, off, L, 4, um, tbot, ttop, closed);
        }
        const long long id = ((long long)k * g.ny + yj) * g.nx + xi;
        R f0u = R(0), f0v = R(0), f0w = R(0);
        if (active) {
            f0u = a.ff[id];
            f0v = a.gg[id];
            if (k < nz - 1) f0w = a.hh[id];
        }
        const R* um1 = SU + slot3(k - 1) * RT_P4; const R* u0 = SU + slot3(k) * RT_P4; const R* up1 = SU + slot3(k + 1) * RT_P4;
        const R* vm1 = SV + slot3(k - 1) * RT_P4; const R* v0 = SV + slot3(k) * RT_P4; const R* vp1 = SV + slot3(k + 1) * RT_P4;
        const R* wm1 = SW + slot3(k - 1) * RT_P4; const R* w0 = SW + slot3(k) * RT_P4; const R* wp1 = SW + slot3(k + 1) * RT_P4;
        const R* p0 = SP + (k & 1) * RT_P4; const R* pp1 = SP + ((k + 1) & 1) * RT_P4;
        const R lt = ZM[3 * (RT_KMAX + 1) + (k - kb)];
        const bool wface = k < nz - 1;   // whx, why vanish on the top wall level
        // ---- level-k products on the 2-point halo
        for (int e = threadIdx.x; e < RT_P2; e += blockDim.x) {
            const int fy = e / RT_W2, fx = e - fy * RT_W2;
            const int r = (fy + 2) * RT_W4 + (fx + 2);
            R uhx, uhy, vhx, vhy, whx = R(0), why = R(0);
            if (CDS == 1) {
                uhx = R(0.5) * (u0[r] + u0[r - 1]);
                uhy = R(0.5) * (u0[r + RT_W4] + u0[r]);
                vhx = R(0.5) * (v0[r + 1] + v0[r]);
                vhy = R(0.5) * (v0[r] + v0[r - RT_W4]);
                if (wface) { whx = R(0.5) * (w0[r + 1] + w0[r]); why = R(0.5) * (w0[r + RT_W4] + w0[r]); }
            } else {
                uhx = (-u0[r + 1] + R(9) * u0[r] + R(9) * u0[r - 1] - u0[r - 2]) * h16;
                uhy = (-u0[r + 2 * RT_W4] + R(9) * u0[r + RT_W4] + R(9) * u0[r] - u0[r - RT_W4]) * h16;
                vhx = (-v0[r + 2] + R(9) * v0[r + 1] + R(9) * v0[r] - v0[r - 1]) * h16;
                vhy = (-v0[r + RT_W4] + R(9) * v0[r] + R(9) * v0[r - RT_W4] - v0[r - 2 * RT_W4]) * h16;
                if (wface) {
                    whx = (-w0[r + 2] + R(9) * w0[r + 1] + R(9) * w0[r] - w0[r - 1]) * h16;
                    why = (-w0[r + 2 * RT_W4] + R(9) * w0[r + RT_W4] + R(9) * w0[r] - w0[r - RT_W4]) * h16;
                }
            }
            R uhz, vhz;
            if (wface) { uhz = up1[r] * lt + u0[r] * (R(1) - lt); vhz = vp1[r] * lt + v0[r] * (R(1) - lt); }
            else { uhz = closed ? -um : u0[r]; vhz = closed ? R(0) : v0[r]; }
            F_UHX[e] = uhx; F_UHY[e] = uhy; F_VHX[e] = vhx; F_VHY[e] = vhy; F_WHX[e] = whx;
            F_B[e] = uhy * vhx;
            F_CZ[e] = uhz * whx;
            F_EZ[e] = vhz * why;
        }
        __syncthreads();

        if (active && a.part_div) {
            // FP64 divergence of the stored fields, as k_div_check computes it
            const double uc = (double)u0[rc], vc = (double)v0[rc], wc = (double)w0[rc];
            double ux[4] = {(double)u0[rc + 1], uc, (double)u0[rc - 1], (double)u0[rc - 2]};
            double vy[4] = {(double)v0[rc + RT_W4], vc, (double)v0[rc - RT_W4], (double)v0[rc - 2 * RT_W4]};
            const double d = fd_div_point<CDS>(ux, vy, wc, k > 0 ? (double)wm1[rc] : 0.0, g.dx, g.dy, ldz(g.z.dz, k));
            if (uc != uc || vc != vc || wc != wc || d != d) dv_nan = 1;
            else { dv_sum += fabs(d); dv_max = absmax_pick(dv_max, d); }
        }
        if (active) {
            const R rdz = ZM[k - kb], rdzt = ZM[(RT_KMAX + 1) + (k - kb)], rdzb = ZM[2 * (RT_KMAX + 1) + (k - kb)];
            const int f = fc0;
            // ---------------- U ----------------
            {
                R uux, uvy, ux, uxx, uyy, dpdx;
                const R uc = u0[rc];
                if (CDS == 1) {
                    const R h1 = F_UHX[f + 1], h0 = F_UHX[f];
                    uux = (h1 * h1 - h0 * h0) * rdx;
                    uvy = (F_B[f] - F_B[f - RT_W2]) * rdy;
                    ux = (h1 - h0) * rdx;
                    uxx = (u0[rc + 1] - R(2) * uc + u0[rc - 1]) * rdx2;
                    uyy = (u0[rc + RT_W4] - R(2) * uc + u0[rc - RT_W4]) * rdy2;
                    dpdx = (p0[rc + 1] - p0[rc]) * rdx;
                } else {
                    const R h2 = F_UHX[f + 2], h1 = F_UHX[f + 1], h0 = F_UHX[f], hm = F_UHX[f - 1];
                    uux = (-h2 * h2 + R(27) * h1 * h1 - R(27) * h0 * h0 + hm * hm) * r24dx;
                    uvy = (-F_B[f + RT_W2] + R(27) * F_B[f] - R(27) * F_B[f - RT_W2] + F_B[f - 2 * RT_W2]) * r24dy;
                    ux = (-h2 + R(27) * h1 - R(27) * h0 + hm) * r24dx;
                    uxx = (-u0[rc + 2] + R(16) * u0[rc + 1] - R(30) * uc + R(16) * u0[rc - 1] - u0[rc - 2]) * r12dx2;
                    uyy = (-u0[rc + 2 * RT_W4] + R(16) * u0[rc + RT_W4] - R(30) * uc + R(16) * u0[rc - RT_W4] - u0[rc - 2 * RT_W4]) * r12dy2;
                    dpdx = (-p0[rc + 2] + R(27) * p0[rc + 1] - R(27) * p0[rc] + p0[rc - 1]) * r24dx;
                }
                const R cz = F_CZ[f];
                const R uwz = (cz - cz_prev) * rdz;
                cz_prev = cz;
                const R uzz = ((up1[rc] - uc) * rdzt - (uc - um1[rc]) * rdzb) * rdz;
                R fu;
                if (a.ph.dp_opt == 3) fu = -uux - uvy - uwz - um * ux + fc * (R(0.5) * (F_VHX[f] + F_VHX[f - RT_W2]) - (R)a.ph.vg);
                else fu = -uux - uvy - uwz + dpx - um * ux;
                if (a.bfx) fu += a.bfx[id];
                a.ff[id] = fu;
                a.qu[id] = uc + dt * (rka * fu + rkb * f0u) + cdif * (uxx + uyy + uzz) - rkc * dt * dpdx;
                if (a.uhx_s) a.uhx_s[id] = F_UHX[f];
            }
            // ---------------- V ----------------
            {
                R vux, vvy, vx, vxx, vyy, dpdy;
                const R vc = v0[rc];
                if (CDS == 1) {
                    const R h0 = F_VHX[f], hm = F_VHX[f - 1];
                    vux = (F_B[f] - F_B[f - 1]) * rdx;
                    const R y1 = F_VHY[f + RT_W2], y0v = F_VHY[f];
                    vvy = (y1 * y1 - y0v * y0v) * rdy;
                    vx = (h0 - hm) * rdx;
                    vxx = (v0[rc + 1] - R(2) * vc + v0[rc - 1]) * rdx2;
                    vyy = (v0[rc + RT_W4] - R(2) * vc + v0[rc - RT_W4]) * rdy2;
                    dpdy = (p0[rc + RT_W4] - p0[rc]) * rdy;
                } else {
                    const R h1 = F_VHX[f + 1], h0 = F_VHX[f], hm = F_VHX[f - 1], hm2 = F_VHX[f - 2];
                    vux = (-F_B[f + 1] + R(27) * F_B[f] - R(27) * F_B[f - 1] + F_B[f - 2]) * r24dx;
                    const R y2 = F_VHY[f + 2 * RT_W2], y1 = F_VHY[f + RT_W2], y0v = F_VHY[f], ym = F_VHY[f - RT_W2];
                    vvy = (-y2 * y2 + R(27) * y1 * y1 - R(27) * y0v * y0v + ym * ym) * r24dy;
                    vx = (-h1 + R(27) * h0 - R(27) * hm + hm2) * r24dx;
                    vxx = (-v0[rc + 2] + R(16) * v0[rc + 1] - R(30) * vc + R(16) * v0[rc - 1] - v0[rc - 2]) * r12dx2;
                    vyy = (-v0[rc + 2 * RT_W4] + R(16) * v0[rc + RT_W4] - R(30) * vc + R(16) * v0[rc - RT_W4] - v0[rc - 2 * RT_W4]) * r12dy2;
                    dpdy = (-p0[rc + 2 * RT_W4] + R(27) * p0[rc + RT_W4] - R(27) * p0[rc] + p0[rc - RT_W4]) * r24dy;
                }
                const R ez = F_EZ[f];
                const R vwz = (ez - ez_prev) * rdz;
                ez_prev = ez;
                const R vzz = ((vp1[rc] - vc) * rdzt - (vc - vm1[rc]) * rdzb) * rdz;
                R fv;
                if (a.ph.dp_opt == 3) fv = -vux - vvy - vwz - um * vx + fc * ((R)a.ph.ug - R(0.5) * (F_UHY[f] + F_UHY[f - 1]) - um);
                else fv = -vux - vvy - vwz - um * vx;
                if (a.bfx) fv += a.bfy[id];
                a.gg[id] = fv;
                a.qv[id] = vc + dt * (rka * fv + rkb * f0v) + cdif * (vxx + vyy + vzz) - rkc * dt * dpdy;
                if (a.vhy_s) a.vhy_s[id] = F_VHY[f];
            }
            // ---------------- W (k <= nz-2) ----------------
            if (wface) {
                R wux, wvy, wx, wxx, wyy;
                const R wc = w0[rc], wp = wp1[rc], wm = wm1[rc];
                if (CDS == 1) {
                    wux = (F_CZ[f] - F_CZ[f - 1]) * rdx;
                    wvy = (F_EZ[f] - F_EZ[f - RT_W2]) * rdy;
                    wx = (F_WHX[f] - F_WHX[f - 1]) * rdx;
                    wxx = (w0[rc + 1] - R(2) * wc + w0[rc - 1]) * rdx2;
                    wyy = (w0[rc + RT_W4] - R(2) * wc + w0[rc - RT_W4]) * rdy2;
                } else {
                    wux = (-F_CZ[f + 1] + R(27) * F_CZ[f] - R(27) * F_CZ[f - 1] + F_CZ[f - 2]) * r24dx;
                    wvy = (-F_EZ[f + RT_W2] + R(27) * F_EZ[f] - R(27) * F_EZ[f - RT_W2] + F_EZ[f - 2 * RT_W2]) * r24dy;
                    wx = (-F_WHX[f + 1] + R(27) * F_WHX[f] - R(27) * F_WHX[f - 1] + F_WHX[f - 2]) * r24dx;
                    wxx = (-w0[rc + 2] + R(16) * w0[rc + 1] - R(30) * wc + R(16) * w0[rc - 1] - w0[rc - 2]) * r12dx2;
                    wyy = (-w0[rc + 2 * RT_W4] + R(16) * w0[rc + RT_W4] - R(30) * wc + R(16) * w0[rc - RT_W4] - w0[rc - 2 * RT_W4]) * r12dy2;
                }
                R a1 = R(0.5) * (wc + wp); a1 = a1 * a1;
                R a2 = R(0.5) * (wc + wm); a2 = a2 * a2;
                const R wwz = (a1 - a2) * rdzt;
                const R rdzp = ZM[4 * (RT_KMAX + 1) + (k - kb)];
                const R wzz = ((wp - wc) * rdzp - (wc - wm) * rdz) * rdzt;
                R fw = -wux - wvy - wwz - um * wx;
                if (a.ph.isscalar == 1) {
                    const R* t0 = ST + (k & 1) * RT_P4; const R* tp1 = ST + ((k + 1) & 1) * RT_P4;
                    fw = fw + got * ((R(1) - lt) * t0[rc] + lt * tp1[rc] - (R)a.ph.t_ref);
                }
                const R dpdz = (pp1[rc] - p0[rc]) * rdzt;
                if (a.bfx) fw += a.bfz[id];
                a.hh[id] = fw;
                a.qw[id] = wc + dt * (rka * fw + rkb * f0w) + cdif * (wxx + wyy + wzz) - rkc * dt * dpdz;
            }
        }
        if (!more) break;
        __syncthreads();
        // advance the window: level k+2 replaces k-1 (u, v, w) and k (p, t)
        {
            const int L = k + 2;
            rt_put<R>(SU + slot3(L) * RT_P4, nu_);
            rt_put<R>(SV + slot3(L) * RT_P4, nv_);
            rt_put<R>(SW + slot3(L) * RT_P4, nw_);
            rt_put<R>(SP + (L & 1) * RT_P4, np_);
            if (a.with_t) rt_put<R>(ST + (L & 1) * RT_P4, nt_);
        }
        __syncthreads();
    }
    if (a.part_div) {
        __shared__ double s_sum[8], s_max[8];
        __shared__ int s_nan;
        __syncthreads();
        if (threadIdx.x == 0) s_nan = 0;
        __syncthreads();
        if (dv_nan) s_nan = 1;
        dv_sum = warp_sum(dv_sum);
        dv_max = warp_absmax(dv_max);
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        if (lane == 0) { s_sum[wid] = dv_sum; s_max[wid] = dv_max; }
        __syncthreads();
        if (wid == 0) {
            dv_sum = lane < 8 ? s_sum[lane] : 0.0;
            dv_max = lane < 8 ? s_max[lane] : 0.0;
            dv_sum = warp_sum(dv_sum);
            dv_max = warp_absmax(dv_max);
            if (lane == 0) {
                const long long b = ((long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
                a.part_div[3 * b + 0] = dv_sum;
                a.part_div[3 * b + 1] = dv_max;
                a.part_div[3 * b + 2] = s_nan ? 1.0 : 0.0;
            }
        }
    }
}
template <typename R, int CDS>
__global__ void __launch_bounds__(256, RhsMinBlocks<R>::v) k_rhs_momentum_tiled(RhsTArgs<R> a) { k_rhs_momentum_tiled_body<R, CDS>(a, blockIdx, gridDim); }
