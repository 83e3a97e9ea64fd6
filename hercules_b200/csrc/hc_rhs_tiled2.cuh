// hc_rhs_tiled2.cuh -- FP32 momentum right-hand side with two x points a thread.
//
// The same computation as k_rhs_momentum_tiled (get_momentum_cnvdiff,
// src/module_cnvdiff.f90:35-374, over the rolling SMEM window of raw planes and
// per-level interpolant products), for the FP32 storage of the mixed mode: a
// thread owns the points (2 tx, ty) and (2 tx + 1, ty) of a 64 x 8 tile, so that
// every shared-memory read of a stencil is an 8-byte load serving both points
// (the x neighbours i-2 .. i+3 of the pair are three float2 loads, a y
// neighbour one). nx is even, so a pair is always inside or outside the domain
// together and its global accesses are 8-byte aligned.
#pragma once
#include "hc_rhs_tiled.cuh"

#define R2_TX 64                      // points in x (32 threads x 2)
#define R2_TY 8
#define R2_W4 (R2_TX + 8)
#define R2_H4 (R2_TY + 8)
#define R2_P4 (R2_W4 * R2_H4)
#define R2_W2 (R2_TX + 4)
#define R2_H2 (R2_TY + 4)
#define R2_P2 (R2_W2 * R2_H2)
#define R2_NLD ((R2_P4 + 255) / 256)

__host__ inline size_t rhs_tiled2_smem(int with_t)
{
    return sizeof(float) * ((size_t)(9 + 2 + (with_t ? 2 : 0)) * R2_P4 + (size_t)RT_NFLUX * R2_P2) +
           sizeof(float) * 6 * (RT_KMAX + 1);
}

__device__ __forceinline__ float2 ld2s(const float* p, int i) { return *reinterpret_cast<const float2*>(p + i); }
__device__ __forceinline__ void st2s(float* p, int i, float a, float b) { *reinterpret_cast<float2*>(p + i) = make_float2(a, b); }

// six consecutive values p[i-2 .. i+3] (i even) as v[0..5]
__device__ __forceinline__ void ld6(const float* p, int i, float* v)
{
    const float2 a = ld2s(p, i - 2), b = ld2s(p, i), c = ld2s(p, i + 2);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y; v[4] = c.x; v[5] = c.y;
}

__device__ __forceinline__ void r2_plane_src(const Geo& g, int lvl, int kind, float um, float tbot, float ttop,
                                             int closed, int& sl, float& sgn, float& add)
{
    const int nz = g.nz;
    sl = lvl; sgn = 1.0f; add = 0.0f;
    if (lvl < 0) {
        sl = 0;
        if (kind == 0) { sgn = -1.0f; add = -2.0f * um; }
        else if (kind == 1) { sgn = -1.0f; }
        else if (kind == 2) { sgn = 0.0f; }
        else if (kind == 4) { sgn = -1.0f; add = 2.0f * tbot; }
    } else if (lvl >= nz) {
        sl = nz - 1;
        if (kind == 0) { if (closed) { sgn = -1.0f; add = -2.0f * um; } }
        else if (kind == 1) { if (closed) sgn = -1.0f; }
        else if (kind == 2) { sl = nz - 2; sgn = -1.0f; }
        else if (kind == 4) { sgn = -1.0f; add = 2.0f * ttop; }
    }
}

__device__ __forceinline__ void r2_fetch(float* v, const float* src, const Geo& g, const int* off, int lvl, int kind,
                                         float um, float tbot, float ttop, int closed)
{
    int sl; float sgn, add;
    r2_plane_src(g, lvl, kind, um, tbot, ttop, closed, sl, sgn, add);
    const float* base = src + (long long)sl * g.nxy;
#pragma unroll
    for (int r = 0; r < R2_NLD; ++r) {
        const int e = threadIdx.x + 256 * r;
        v[r] = (e < R2_P4) ? sgn * __ldg(base + off[r]) + add : 0.0f;
    }
}
__device__ __forceinline__ void r2_put(float* dst, const float* v)
{
#pragma unroll
    for (int r = 0; r < R2_NLD; ++r) {
        const int e = threadIdx.x + 256 * r;
        if (e < R2_P4) dst[e] = v[r];
    }
}

template <int CDS>
__device__ __forceinline__ void k_rhs_momentum_tiled2_body(const RhsTArgs<float>& a, const uint3 blockIdx, const dim3 gridDim)
{
    typedef float R;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* sm = reinterpret_cast<R*>(smem_raw);
    R* SU = sm;                  // [3][P4]
    R* SV = SU + 3 * R2_P4;
    R* SW = SV + 3 * R2_P4;
    R* SP = SW + 3 * R2_P4;      // [2][P4]
    R* ST = SP + 2 * R2_P4;      // [2][P4] if with_t
    R* FX = ST + (a.with_t ? 2 * R2_P4 : 0);
    R* F_UHX = FX;
    R* F_UHY = FX + 1 * R2_P2;
    R* F_VHX = FX + 2 * R2_P2;
    R* F_VHY = FX + 3 * R2_P2;
    R* F_WHX = FX + 4 * R2_P2;
    R* F_B = FX + 5 * R2_P2;     // uhy * vhx
    R* F_CZ = FX + 6 * R2_P2;    // uhz * whx
    R* F_EZ = FX + 7 * R2_P2;    // vhz * why
    R* ZM = FX + RT_NFLUX * R2_P2;

    const Geo& g = a.g;
    const int nz = g.nz;
    const int x0 = blockIdx.x * R2_TX, y0 = blockIdx.y * R2_TY;
    const int kb = blockIdx.z * a.kchunk;
    const int ke = min(nz, kb + a.kchunk);
    const int tx = threadIdx.x % 32, ty = threadIdx.x / 32;
    const int xi = x0 + 2 * tx, yj = y0 + ty;
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
    int off[R2_NLD];
#pragma unroll
    for (int r = 0; r < R2_NLD; ++r) {
        const int e = threadIdx.x + 256 * r;
        const int ry = e / R2_W4, rx = e - ry * R2_W4;
        int x = (x0 - 4 + rx) % g.nx; if (x < 0) x += g.nx;
        int y = (y0 - 4 + ry) % g.ny; if (y < 0) y += g.ny;
        off[r] = y * g.nx + x;
    }
    {
        float v[R2_NLD];
        for (int L = kb - 1; L <= kb + 1; ++L) {
            r2_fetch(v, a.f.u, g, off, L, 0, um, tbot, ttop, closed); r2_put(SU + slot3(L) * R2_P4, v);
            r2_fetch(v, a.f.v, g, off, L, 1, um, tbot, ttop, closed); r2_put(SV + slot3(L) * R2_P4, v);
            r2_fetch(v, a.f.w, g, off, L, 2, um, tbot, ttop, closed); r2_put(SW + slot3(L) * R2_P4, v);
        }
        for (int L = kb; L <= kb + 1; ++L) {
            r2_fetch(v, a.f.p, g, off, L, 3, um, tbot, ttop, closed); r2_put(SP + (L & 1) * R2_P4, v);
            if (a.with_t) { r2_fetch(v, a.f.t, g, off, L, 4, um, tbot, ttop, closed); r2_put(ST + (L & 1) * R2_P4, v); }
        }
    }
    __syncthreads();

    const int rc = (ty + 4) * R2_W4 + (2 * tx + 4);     // own raw index (even)
    const int fc0 = (ty + 2) * R2_W2 + (2 * tx + 2);    // own flux index (even)
    R cz_prev[2] = {R(0), R(0)}, ez_prev[2] = {R(0), R(0)};
    if (kb > 0) {
        const int L = kb - 1;
        const R* u0 = SU + slot3(L) * R2_P4; const R* u1 = SU + slot3(L + 1) * R2_P4;
        const R* v0 = SV + slot3(L) * R2_P4; const R* v1 = SV + slot3(L + 1) * R2_P4;
        const R* w0 = SW + slot3(L) * R2_P4;
        const R l = (R)ldz(g.z.l_t, L);
        float wx[6];
        ld6(w0, rc, wx);
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            const R uhz = u1[rc + s] * l + u0[rc + s] * (R(1) - l);
            const R vhz = v1[rc + s] * l + v0[rc + s] * (R(1) - l);
            R whx, why;
            const int r = rc + s;
            if (CDS == 1) { whx = R(0.5) * (wx[3 + s] + wx[2 + s]); why = R(0.5) * (w0[r + R2_W4] + w0[r]); }
            else {
                whx = (-wx[4 + s] + R(9) * wx[3 + s] + R(9) * wx[2 + s] - wx[1 + s]) * h16;
                why = (-w0[r + 2 * R2_W4] + R(9) * w0[r + R2_W4] + R(9) * w0[r] - w0[r - R2_W4]) * h16;
            }
            cz_prev[s] = uhz * whx;
            ez_prev[s] = vhz * why;
        }
    }

    double dv_sum = 0.0, dv_max = 0.0;
    int dv_nan = 0;
    for (int k = kb; k < ke; ++k) {
        const bool more = k + 1 < ke;
        R nu_[R2_NLD], nv_[R2_NLD], nw_[R2_NLD], np_[R2_NLD];
        if (more) {
            const int L = k + 2;
            r2_fetch(nu_, a.f.u, g, off, L, 0, um, tbot, ttop, closed);
            r2_fetch(nv_, a.f.v, g, off, L, 1, um, tbot, ttop, closed);
            r2_fetch(nw_, a.f.w, g, off, L, 2, um, tbot, ttop, closed);
            r2_fetch(np_, a.f.p, g, off, L, 3, um, tbot, ttop, closed);
        }
        const long long id = ((long long)k * g.ny + yj) * g.nx + xi;
        // the thread's history values, loaded here so that their latency overlaps
        // the products below (loaded in the U, V and W blocks right before their
        // use, they stalled those blocks: 1612 -> 1381 us a launch at 512 x 384 x 256)
        float2 f0u = make_float2(0, 0), f0v = f0u, f0w = f0u;
        if (active) {
            f0u = *reinterpret_cast<const float2*>(a.ff + id);
            f0v = *reinterpret_cast<const float2*>(a.gg + id);
            if (k < nz - 1) f0w = *reinterpret_cast<const float2*>(a.hh + id);
        }
        const R* um1 = SU + slot3(k - 1) * R2_P4; const R* u0 = SU + slot3(k) * R2_P4; const R* up1 = SU + slot3(k + 1) * R2_P4;
        const R* vm1 = SV + slot3(k - 1) * R2_P4; const R* v0 = SV + slot3(k) * R2_P4; const R* vp1 = SV + slot3(k + 1) * R2_P4;
        const R* wm1 = SW + slot3(k - 1) * R2_P4; const R* w0 = SW + slot3(k) * R2_P4; const R* wp1 = SW + slot3(k + 1) * R2_P4;
        const R* p0 = SP + (k & 1) * R2_P4; const R* pp1 = SP + ((k + 1) & 1) * R2_P4;
        const R lt = ZM[3 * (RT_KMAX + 1) + (k - kb)];
        const bool wface = k < nz - 1;
        // ---- level-k products on the 2-point halo, two x points per thread
        for (int e2 = threadIdx.x; e2 < R2_P2 / 2; e2 += blockDim.x) {
            const int fy = e2 / (R2_W2 / 2), fx = 2 * (e2 - fy * (R2_W2 / 2));
            const int e = fy * R2_W2 + fx;
            const int r = (fy + 2) * R2_W4 + (fx + 2);
            float ux[6], vx[6], wx[6];
            ld6(u0, r, ux); ld6(v0, r, vx);
            const float2 uy2 = ld2s(u0, r + 2 * R2_W4), uy1 = ld2s(u0, r + R2_W4), uym = ld2s(u0, r - R2_W4);
            const float2 vy1 = ld2s(v0, r + R2_W4), vym = ld2s(v0, r - R2_W4), vym2 = ld2s(v0, r - 2 * R2_W4);
            float2 wy2 = make_float2(0, 0), wy1 = wy2, wym = wy2;
            if (wface) {
                ld6(w0, r, wx);
                wy2 = ld2s(w0, r + 2 * R2_W4); wy1 = ld2s(w0, r + R2_W4); wym = ld2s(w0, r - R2_W4);
            } else {
#pragma unroll
                for (int q = 0; q < 6; ++q) wx[q] = 0.0f;
            }
            float2 up = make_float2(0, 0), vp = up;
            if (wface) { up = ld2s(up1, r); vp = ld2s(vp1, r); }
            R o_uhx[2], o_uhy[2], o_vhx[2], o_vhy[2], o_whx[2], o_b[2], o_cz[2], o_ez[2];
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                // x values of this point: index 2 + s is the point, ux[1+s] its i-1 ...
                const R c_u = ux[2 + s], c_v = vx[2 + s], c_w = wx[2 + s];
                const R u_y2 = s ? uy2.y : uy2.x, u_y1 = s ? uy1.y : uy1.x, u_ym = s ? uym.y : uym.x;
                const R v_y1 = s ? vy1.y : vy1.x, v_ym = s ? vym.y : vym.x, v_ym2 = s ? vym2.y : vym2.x;
                const R w_y2 = s ? wy2.y : wy2.x, w_y1 = s ? wy1.y : wy1.x, w_ym = s ? wym.y : wym.x;
                R uhx, uhy, vhx, vhy, whx = R(0), why = R(0);
                if (CDS == 1) {
                    uhx = R(0.5) * (c_u + ux[1 + s]);
                    uhy = R(0.5) * (u_y1 + c_u);
                    vhx = R(0.5) * (vx[3 + s] + c_v);
                    vhy = R(0.5) * (c_v + v_ym);
                    if (wface) { whx = R(0.5) * (wx[3 + s] + c_w); why = R(0.5) * (w_y1 + c_w); }
                } else {
                    uhx = (-ux[3 + s] + R(9) * c_u + R(9) * ux[1 + s] - ux[0 + s]) * h16;
                    uhy = (-u_y2 + R(9) * u_y1 + R(9) * c_u - u_ym) * h16;
                    vhx = (-vx[4 + s] + R(9) * vx[3 + s] + R(9) * c_v - vx[1 + s]) * h16;
                    vhy = (-v_y1 + R(9) * c_v + R(9) * v_ym - v_ym2) * h16;
                    if (wface) {
                        whx = (-wx[4 + s] + R(9) * wx[3 + s] + R(9) * c_w - wx[1 + s]) * h16;
                        why = (-w_y2 + R(9) * w_y1 + R(9) * c_w - w_ym) * h16;
                    }
                }
                R uhz, vhz;
                const R upv = s ? up.y : up.x, vpv = s ? vp.y : vp.x;
                if (wface) { uhz = upv * lt + c_u * (R(1) - lt); vhz = vpv * lt + c_v * (R(1) - lt); }
                else { uhz = closed ? -um : c_u; vhz = closed ? R(0) : c_v; }
                o_uhx[s] = uhx; o_uhy[s] = uhy; o_vhx[s] = vhx; o_vhy[s] = vhy; o_whx[s] = whx;
                o_b[s] = uhy * vhx; o_cz[s] = uhz * whx; o_ez[s] = vhz * why;
            }
            st2s(F_UHX, e, o_uhx[0], o_uhx[1]); st2s(F_UHY, e, o_uhy[0], o_uhy[1]);
            st2s(F_VHX, e, o_vhx[0], o_vhx[1]); st2s(F_VHY, e, o_vhy[0], o_vhy[1]);
            st2s(F_WHX, e, o_whx[0], o_whx[1]); st2s(F_B, e, o_b[0], o_b[1]);
            st2s(F_CZ, e, o_cz[0], o_cz[1]); st2s(F_EZ, e, o_ez[0], o_ez[1]);
        }
        __syncthreads();

        if (active) {
            const R rdz = ZM[k - kb], rdzt = ZM[(RT_KMAX + 1) + (k - kb)], rdzb = ZM[2 * (RT_KMAX + 1) + (k - kb)];
            const int f = fc0;
            auto sel = [](float2 v, int s) { return s ? v.y : v.x; };
            // ---------------- divergence of the incoming fields (FP64) ----------------
            if (a.part_div) {
                float ux[6];
                ld6(u0, rc, ux);
                const float2 vc2 = ld2s(v0, rc), vym = ld2s(v0, rc - R2_W4), vym2 = ld2s(v0, rc - 2 * R2_W4);
                const float2 vy1 = ld2s(v0, rc + R2_W4), wc2 = ld2s(w0, rc), wzm = ld2s(wm1, rc);
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const int c = 2 + s;
                    const double uc = (double)ux[c], vc = (double)sel(vc2, s), wc = (double)sel(wc2, s);
                    double dux[4] = {(double)ux[c + 1], uc, (double)ux[c - 1], (double)ux[c - 2]};
                    double dvy[4] = {(double)sel(vy1, s), vc, (double)sel(vym, s), (double)sel(vym2, s)};
                    const double d = fd_div_point<CDS>(dux, dvy, wc, k > 0 ? (double)sel(wzm, s) : 0.0, g.dx, g.dy,
                                                       ldz(g.z.dz, k));
                    if (uc != uc || vc != vc || wc != wc || d != d) dv_nan = 1;
                    else { dv_sum += fabs(d); dv_max = absmax_pick(dv_max, d); }
                }
            }
            // ---------------- U ----------------
            {
                float ux[6], px[6], fuhx[6];
                ld6(u0, rc, ux); ld6(p0, rc, px); ld6(F_UHX, f, fuhx);
                const float2 uy2 = ld2s(u0, rc + 2 * R2_W4), uy1 = ld2s(u0, rc + R2_W4);
                const float2 uym = ld2s(u0, rc - R2_W4), uym2 = ld2s(u0, rc - 2 * R2_W4);
                const float2 uzp = ld2s(up1, rc), uzm = ld2s(um1, rc);
                const float2 fb0 = ld2s(F_B, f), fb_y1 = ld2s(F_B, f + R2_W2), fb_ym = ld2s(F_B, f - R2_W2);
                const float2 fb_ym2 = ld2s(F_B, f - 2 * R2_W2);
                const float2 fcz0 = ld2s(F_CZ, f), fvhx0 = ld2s(F_VHX, f), fvhx_ym = ld2s(F_VHX, f - R2_W2);
                const float2 bfu = a.bfx ? *reinterpret_cast<const float2*>(a.bfx + id) : make_float2(0, 0);
                float out_f[2], out_q[2];
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const int c = 2 + s;
                    R uux, uvy, uxv, uxx, uyy, dpdx;
                    const R uc = ux[c];
                    if (CDS == 1) {
                        const R h1 = fuhx[c + 1], h0 = fuhx[c];
                        uux = (h1 * h1 - h0 * h0) * rdx;
                        uvy = (sel(fb0, s) - sel(fb_ym, s)) * rdy;
                        uxv = (h1 - h0) * rdx;
                        uxx = (ux[c + 1] - R(2) * uc + ux[c - 1]) * rdx2;
                        uyy = (sel(uy1, s) - R(2) * uc + sel(uym, s)) * rdy2;
                        dpdx = (px[c + 1] - px[c]) * rdx;
                    } else {
                        const R h2 = fuhx[c + 2], h1 = fuhx[c + 1], h0 = fuhx[c], hm = fuhx[c - 1];
                        uux = (-h2 * h2 + R(27) * h1 * h1 - R(27) * h0 * h0 + hm * hm) * r24dx;
                        uvy = (-sel(fb_y1, s) + R(27) * sel(fb0, s) - R(27) * sel(fb_ym, s) + sel(fb_ym2, s)) * r24dy;
                        uxv = (-h2 + R(27) * h1 - R(27) * h0 + hm) * r24dx;
                        uxx = (-ux[c + 2] + R(16) * ux[c + 1] - R(30) * uc + R(16) * ux[c - 1] - ux[c - 2]) * r12dx2;
                        uyy = (-sel(uy2, s) + R(16) * sel(uy1, s) - R(30) * uc + R(16) * sel(uym, s) - sel(uym2, s)) * r12dy2;
                        dpdx = (-px[c + 2] + R(27) * px[c + 1] - R(27) * px[c] + px[c - 1]) * r24dx;
                    }
                    const R cz = sel(fcz0, s);
                    const R uwz = (cz - cz_prev[s]) * rdz;
                    cz_prev[s] = cz;
                    const R uzz = ((sel(uzp, s) - uc) * rdzt - (uc - sel(uzm, s)) * rdzb) * rdz;
                    R fu;
                    if (a.ph.dp_opt == 3) fu = -uux - uvy - uwz - um * uxv + fc * (R(0.5) * (sel(fvhx0, s) + sel(fvhx_ym, s)) - (R)a.ph.vg);
                    else fu = -uux - uvy - uwz + dpx - um * uxv;
                    fu += sel(bfu, s);
                    out_f[s] = fu;
                    out_q[s] = uc + dt * (rka * fu + rkb * sel(f0u, s)) + cdif * (uxx + uyy + uzz) - rkc * dt * dpdx;
                }
                *reinterpret_cast<float2*>(a.ff + id) = make_float2(out_f[0], out_f[1]);
                *reinterpret_cast<float2*>(a.qu + id) = make_float2(out_q[0], out_q[1]);
                if (a.uhx_s) *reinterpret_cast<float2*>(a.uhx_s + id) = make_float2(fuhx[2], fuhx[3]);
            }
            // ---------------- V ----------------
            {
                float vx[6], fvhx[6], fb[6], fuhy[6];
                ld6(v0, rc, vx); ld6(F_VHX, f, fvhx); ld6(F_B, f, fb); ld6(F_UHY, f, fuhy);
                const float2 vy2 = ld2s(v0, rc + 2 * R2_W4), vy1 = ld2s(v0, rc + R2_W4);
                const float2 vym = ld2s(v0, rc - R2_W4), vym2 = ld2s(v0, rc - 2 * R2_W4);
                const float2 vzp = ld2s(vp1, rc), vzm = ld2s(vm1, rc);
                const float2 p0c = ld2s(p0, rc), py2 = ld2s(p0, rc + 2 * R2_W4), py1 = ld2s(p0, rc + R2_W4);
                const float2 pym = ld2s(p0, rc - R2_W4);
                const float2 fvy2 = ld2s(F_VHY, f + 2 * R2_W2), fvy1 = ld2s(F_VHY, f + R2_W2), fvy0 = ld2s(F_VHY, f);
                const float2 fvym = ld2s(F_VHY, f - R2_W2), fez0 = ld2s(F_EZ, f);
                const float2 bfv = a.bfx ? *reinterpret_cast<const float2*>(a.bfy + id) : make_float2(0, 0);
                float out_f[2], out_q[2];
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const int c = 2 + s;
                    R vux, vvy, vxv, vxx, vyy, dpdy;
                    const R vc = vx[c];
                    if (CDS == 1) {
                        const R h0 = fvhx[c], hm = fvhx[c - 1];
                        vux = (fb[c] - fb[c - 1]) * rdx;
                        const R y1 = sel(fvy1, s), y0v = sel(fvy0, s);
                        vvy = (y1 * y1 - y0v * y0v) * rdy;
                        vxv = (h0 - hm) * rdx;
                        vxx = (vx[c + 1] - R(2) * vc + vx[c - 1]) * rdx2;
                        vyy = (sel(vy1, s) - R(2) * vc + sel(vym, s)) * rdy2;
                        dpdy = (sel(py1, s) - sel(p0c, s)) * rdy;
                    } else {
                        const R h1 = fvhx[c + 1], h0 = fvhx[c], hm = fvhx[c - 1], hm2 = fvhx[c - 2];
                        vux = (-fb[c + 1] + R(27) * fb[c] - R(27) * fb[c - 1] + fb[c - 2]) * r24dx;
                        const R y2 = sel(fvy2, s), y1 = sel(fvy1, s), y0v = sel(fvy0, s), ym = sel(fvym, s);
                        vvy = (-y2 * y2 + R(27) * y1 * y1 - R(27) * y0v * y0v + ym * ym) * r24dy;
                        vxv = (-h1 + R(27) * h0 - R(27) * hm + hm2) * r24dx;
                        vxx = (-vx[c + 2] + R(16) * vx[c + 1] - R(30) * vc + R(16) * vx[c - 1] - vx[c - 2]) * r12dx2;
                        vyy = (-sel(vy2, s) + R(16) * sel(vy1, s) - R(30) * vc + R(16) * sel(vym, s) - sel(vym2, s)) * r12dy2;
                        dpdy = (-sel(py2, s) + R(27) * sel(py1, s) - R(27) * sel(p0c, s) + sel(pym, s)) * r24dy;
                    }
                    const R ez = sel(fez0, s);
                    const R vwz = (ez - ez_prev[s]) * rdz;
                    ez_prev[s] = ez;
                    const R vzz = ((sel(vzp, s) - vc) * rdzt - (vc - sel(vzm, s)) * rdzb) * rdz;
                    R fv;
                    if (a.ph.dp_opt == 3) fv = -vux - vvy - vwz - um * vxv + fc * ((R)a.ph.ug - R(0.5) * (fuhy[c] + fuhy[c - 1]) - um);
                    else fv = -vux - vvy - vwz - um * vxv;
                    fv += sel(bfv, s);
                    out_f[s] = fv;
                    out_q[s] = vc + dt * (rka * fv + rkb * sel(f0v, s)) + cdif * (vxx + vyy + vzz) - rkc * dt * dpdy;
                }
                *reinterpret_cast<float2*>(a.gg + id) = make_float2(out_f[0], out_f[1]);
                *reinterpret_cast<float2*>(a.qv + id) = make_float2(out_q[0], out_q[1]);
                if (a.vhy_s) *reinterpret_cast<float2*>(a.vhy_s + id) = fvy0;
            }
            // ---------------- W (k <= nz-2) ----------------
            if (wface) {
                float wx[6], fcz[6], fwhx[6];
                ld6(w0, rc, wx); ld6(F_CZ, f, fcz); ld6(F_WHX, f, fwhx);
                const float2 wy2 = ld2s(w0, rc + 2 * R2_W4), wy1 = ld2s(w0, rc + R2_W4);
                const float2 wym = ld2s(w0, rc - R2_W4), wym2 = ld2s(w0, rc - 2 * R2_W4);
                const float2 wzp = ld2s(wp1, rc), wzm = ld2s(wm1, rc), pzp = ld2s(pp1, rc), p0c = ld2s(p0, rc);
                const float2 fez0 = ld2s(F_EZ, f), fez1 = ld2s(F_EZ, f + R2_W2), fezm = ld2s(F_EZ, f - R2_W2);
                const float2 fezm2 = ld2s(F_EZ, f - 2 * R2_W2);
                const float2 bfw = a.bfx ? *reinterpret_cast<const float2*>(a.bfz + id) : make_float2(0, 0);
                float2 tt0 = make_float2(0, 0), tt1 = tt0;
                if (a.ph.isscalar == 1) { tt0 = ld2s(ST + (k & 1) * R2_P4, rc); tt1 = ld2s(ST + ((k + 1) & 1) * R2_P4, rc); }
                float out_f[2], out_q[2];
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const int c = 2 + s;
                    R wux, wvy, wxv, wxx, wyy;
                    const R wc = wx[c], wp = sel(wzp, s), wm = sel(wzm, s);
                    if (CDS == 1) {
                        wux = (fcz[c] - fcz[c - 1]) * rdx;
                        wvy = (sel(fez0, s) - sel(fezm, s)) * rdy;
                        wxv = (fwhx[c] - fwhx[c - 1]) * rdx;
                        wxx = (wx[c + 1] - R(2) * wc + wx[c - 1]) * rdx2;
                        wyy = (sel(wy1, s) - R(2) * wc + sel(wym, s)) * rdy2;
                    } else {
                        wux = (-fcz[c + 1] + R(27) * fcz[c] - R(27) * fcz[c - 1] + fcz[c - 2]) * r24dx;
                        wvy = (-sel(fez1, s) + R(27) * sel(fez0, s) - R(27) * sel(fezm, s) + sel(fezm2, s)) * r24dy;
                        wxv = (-fwhx[c + 1] + R(27) * fwhx[c] - R(27) * fwhx[c - 1] + fwhx[c - 2]) * r24dx;
                        wxx = (-wx[c + 2] + R(16) * wx[c + 1] - R(30) * wc + R(16) * wx[c - 1] - wx[c - 2]) * r12dx2;
                        wyy = (-sel(wy2, s) + R(16) * sel(wy1, s) - R(30) * wc + R(16) * sel(wym, s) - sel(wym2, s)) * r12dy2;
                    }
                    R a1 = R(0.5) * (wc + wp); a1 = a1 * a1;
                    R a2 = R(0.5) * (wc + wm); a2 = a2 * a2;
                    const R wwz = (a1 - a2) * rdzt;
                    const R rdzp = ZM[4 * (RT_KMAX + 1) + (k - kb)];
                    const R wzz = ((wp - wc) * rdzp - (wc - wm) * rdz) * rdzt;
                    R fw = -wux - wvy - wwz - um * wxv;
                    if (a.ph.isscalar == 1)
                        fw = fw + got * ((R(1) - lt) * sel(tt0, s) + lt * sel(tt1, s) - (R)a.ph.t_ref);
                    const R dpdz = (sel(pzp, s) - sel(p0c, s)) * rdzt;
                    fw += sel(bfw, s);
                    out_f[s] = fw;
                    out_q[s] = wc + dt * (rka * fw + rkb * sel(f0w, s)) + cdif * (wxx + wyy + wzz) - rkc * dt * dpdz;
                }
                *reinterpret_cast<float2*>(a.hh + id) = make_float2(out_f[0], out_f[1]);
                *reinterpret_cast<float2*>(a.qw + id) = make_float2(out_q[0], out_q[1]);
            }
        }
        if (!more) break;
        __syncthreads();
        {
            const int L = k + 2;
            r2_put(SU + slot3(L) * R2_P4, nu_);
            r2_put(SV + slot3(L) * R2_P4, nv_);
            r2_put(SW + slot3(L) * R2_P4, nw_);
            r2_put(SP + (L & 1) * R2_P4, np_);
            if (a.with_t) {
                float nt_[R2_NLD];
                r2_fetch(nt_, a.f.t, g, off, L, 4, um, tbot, ttop, closed);
                r2_put(ST + (L & 1) * R2_P4, nt_);
            }
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
template <int CDS>
__global__ void __launch_bounds__(256, 2) k_rhs_momentum_tiled2(RhsTArgs<float> a) { k_rhs_momentum_tiled2_body<CDS>(a, blockIdx, gridDim); }
