// hc_column_warp.cuh -- warp-per-wavenumber column solves (nz <= 32*8).
//
// Same mathematics as hc_column.cuh (the reference's FFT-Thomas solves,
// src/module_poisson_solver.f90:483-658, fused with the projection and the phi
// part of the pressure update), but one warp owns one (l, m) column:
//   * lane `ln` holds rows ln*K .. ln*K+K-1 in registers (K = ceil(nz/32));
//   * each lane eliminates its K-1 interior rows locally, leaving every interior
//     unknown as an affine function of the last unknowns of its own and of the
//     previous lane's block (partition method);
//   * the 32 block-last unknowns satisfy a tridiagonal system that is solved by
//     parallel cyclic reduction over warp shuffles (5 steps);
//   * u*, v*, w* live in per-warp shared memory (FP64) between the Helmholtz
//     solves and the projection, so nothing but the inputs and the four outputs
//     crosses HBM.
// Rows beyond the system size are identity rows. The elimination order differs
// from the reference's sequential Thomas sweep; for these diagonally dominant
// systems the results agree to round-off.
#pragma once
#include "hc_column.cuh"

__device__ __forceinline__ double2 shfl_up2(double2 v, int s)
{
    return make_double2(__shfl_up_sync(0xffffffffu, v.x, s), __shfl_up_sync(0xffffffffu, v.y, s));
}
__device__ __forceinline__ double2 shfl_dn2(double2 v, int s)
{
    return make_double2(__shfl_down_sync(0xffffffffu, v.x, s), __shfl_down_sync(0xffffffffu, v.y, s));
}

// Reciprocal by Newton-Raphson iteration on f(y) = 1/y - x, i.e.
// y <- y + y (1 - x y), seeded with the single-precision reciprocal. Each step
// doubles the number of correct bits (about 23 -> 46 -> 92), so two steps reach
// FP64 round-off. The pivots of the diagonally dominant column systems stay far
// inside the FP32 range; anything outside it (and NaN) takes the IEEE division.
__device__ __forceinline__ double rcp_nr(double x)
{
    const double ax = fabs(x);
    if (!(ax > 1e-30 && ax < 1e30)) return 1.0 / x;
    double y = (double)__frcp_rn((float)x);
    double e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    e = fma(-x, y, 1.0);
    return fma(y, e, y);
}

// Solve sum_j A(r,j) x_j = d_r for NR right-hand sides. coef(r, a, b, c) gives row
// r's sub-diagonal, diagonal and super-diagonal (identity rows past the end).
template <int K, int NR, typename CF>
__device__ __forceinline__ void warp_partition_solve(const CF& coef, double2 (&d)[NR][K], int ln)
{
    const int r0 = ln * K;
    double vv[K], ww[K], ib[K];     // ib: reciprocal of the eliminated diagonal
    if (K >= 2) {
        double a0, b0, c0;
        coef(r0, a0, b0, c0);
        ib[0] = rcp_nr(b0);
        vv[0] = -a0;
        ww[0] = (K == 2) ? -c0 : 0.0;
        double cprev = c0;
#pragma unroll
        for (int i = 1; i <= K - 2; ++i) {
            double ai, bi, ci;
            coef(r0 + i, ai, bi, ci);
            const double mlt = ai * ib[i - 1];
            ib[i] = rcp_nr(bi - mlt * cprev);
#pragma unroll
            for (int q = 0; q < NR; ++q) d[q][i] = zsub(d[q][i], zscale(d[q][i - 1], mlt));
            vv[i] = -mlt * vv[i - 1];
            ww[i] = (i == K - 2 ? -ci : 0.0) - mlt * ww[i - 1];
            cprev = ci;
        }
#pragma unroll
        for (int q = 0; q < NR; ++q) d[q][K - 2] = zscale(d[q][K - 2], ib[K - 2]);
        vv[K - 2] *= ib[K - 2];
        ww[K - 2] *= ib[K - 2];
#pragma unroll
        for (int i = K - 3; i >= 0; --i) {
            double ai, bi, ci;
            coef(r0 + i, ai, bi, ci);
#pragma unroll
            for (int q = 0; q < NR; ++q) d[q][i] = zscale(zsub(d[q][i], zscale(d[q][i + 1], ci)), ib[i]);
            vv[i] = (vv[i] - ci * vv[i + 1]) * ib[i];
            ww[i] = (ww[i] - ci * ww[i + 1]) * ib[i];
        }
    }
    // reduced row of this block's last unknown y_ln:
    //   A y_{ln-1} + B y_ln + C y_{ln+1} = D
    double aK, bK, cK;
    coef(r0 + K - 1, aK, bK, cK);
    const double xm_v = K >= 2 ? vv[K - 2] : 1.0;
    const double xm_w = K >= 2 ? ww[K - 2] : 0.0;
    const double f_v = K >= 2 ? vv[0] : 0.0;
    const double f_w = K >= 2 ? ww[0] : 1.0;
    const double nf_v = __shfl_down_sync(0xffffffffu, f_v, 1);
    const double nf_w = __shfl_down_sync(0xffffffffu, f_w, 1);
    double A = aK * xm_v;
    double B = aK * xm_w + bK + cK * nf_v;
    double C = cK * nf_w;
    double2 D[NR];
#pragma unroll
    for (int q = 0; q < NR; ++q) {
        const double2 xm_g = K >= 2 ? d[q][K - 2 < 0 ? 0 : K - 2] : make_double2(0, 0);
        const double2 f_g = K >= 2 ? d[q][0] : make_double2(0, 0);
        const double2 nf_g = shfl_dn2(f_g, 1);
        D[q] = zsub(zsub(d[q][K - 1], zscale(xm_g, aK)), zscale(nf_g, cK));
    }
    // parallel cyclic reduction across the 32 lanes
#pragma unroll
    for (int s = 1; s < 32; s <<= 1) {
        double Am = __shfl_up_sync(0xffffffffu, A, s), Bm = __shfl_up_sync(0xffffffffu, B, s);
        double Cm = __shfl_up_sync(0xffffffffu, C, s);
        double Ap = __shfl_down_sync(0xffffffffu, A, s), Bp = __shfl_down_sync(0xffffffffu, B, s);
        double Cp = __shfl_down_sync(0xffffffffu, C, s);
        const bool lo = ln < s, hi = ln + s > 31;
        if (lo) { Am = 0.0; Bm = 1.0; Cm = 0.0; }
        if (hi) { Ap = 0.0; Bp = 1.0; Cp = 0.0; }
        const double k1 = A * rcp_nr(Bm), k2 = C * rcp_nr(Bp);
#pragma unroll
        for (int q = 0; q < NR; ++q) {
            double2 Dm = shfl_up2(D[q], s), Dp = shfl_dn2(D[q], s);
            if (lo) Dm = make_double2(0, 0);
            if (hi) Dp = make_double2(0, 0);
            D[q] = zsub(zsub(D[q], zscale(Dm, k1)), zscale(Dp, k2));
        }
        const double nA = -Am * k1, nC = -Cp * k2, nB = B - Cm * k1 - Ap * k2;
        A = nA; B = nB; C = nC;
    }
    const double iB = rcp_nr(B);
#pragma unroll
    for (int q = 0; q < NR; ++q) {
        const double2 y = zscale(D[q], iB);
        double2 yp = shfl_up2(y, 1);
        if (ln == 0) yp = make_double2(0, 0);
#pragma unroll
        for (int i = 0; i < K - 1; ++i)
            d[q][i] = zadd(d[q][i], make_double2(vv[i] * yp.x + ww[i] * y.x, vv[i] * yp.y + ww[i] * y.y));
        d[q][K - 1] = y;
    }
}

#define CW_WARPS 4

template <int K> __host__ size_t column_warp_smem() { return (size_t)CW_WARPS * 3 * K * 32 * sizeof(double2); }

template <typename R, int K>
__global__ void __launch_bounds__(CW_WARPS * 32, 4) k_column_fd_warp(ColArgs<R> a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (a.halt && *a.halt) return;
    const int ln = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const long long ncol = a.g.ncol;
    const long long c = (long long)blockIdx.x * CW_WARPS + wp;
    if (c >= ncol) return;                       // uniform per warp
    double2* SU = reinterpret_cast<double2*>(smem_raw) + (size_t)wp * 3 * K * 32;
    double2* SV = SU + K * 32;
    double2* SW = SV + K * 32;
    const int nz = a.g.nz;
    const int l = (int)(c % a.g.nxh), m = (int)(c / a.g.nxh);
    const bool is00 = (c == 0);
    const double rk = a.rk_c, dt = a.dt;
    const double lam = __ldg(a.c.hx + l) + __ldg(a.c.hy + m);
    const double lamp = __ldg(a.c.px + l) + __ldg(a.c.py + m);
    const double* dgu = is00 ? a.c.d0u : a.c.dgu;
    const double* dgw = is00 ? a.c.d0w : a.c.dgw;
    const double* dgp = is00 ? a.c.d0p : a.c.dgp;
    const int r0 = ln * K;

    // ---- u*, v*: one matrix, two right-hand sides
    {
        double2 d[2][K];
#pragma unroll
        for (int i = 0; i < K; ++i) {
            const int r = r0 + i;
            if (r < nz) {
                const long long id = (long long)r * ncol + c;
                d[0][i] = ld2<R>(a.qu, id);
                d[1][i] = ld2<R>(a.qv, id);
                if (is00 && r == 0) d[0][i].x += a.bcu0;
                if (is00 && r == nz - 1) d[0][i].x += a.bcu1;
            } else {
                d[0][i] = make_double2(0, 0);
                d[1][i] = make_double2(0, 0);
            }
        }
        auto cf = [&](int r, double& aa, double& bb, double& cc) {
            if (r < nz) {
                aa = rk * __ldg(a.c.au + r);
                cc = rk * __ldg(a.c.cu + r);
                bb = 1.0 + rk * (-lam + __ldg(dgu + r));
            } else { aa = 0.0; bb = 1.0; cc = 0.0; }
        };
        warp_partition_solve<K, 2>(cf, d, ln);
#pragma unroll
        for (int i = 0; i < K; ++i) { SU[i * 32 + ln] = d[0][i]; SV[i * 32 + ln] = d[1][i]; }
    }
    // ---- w*: rows 0..nz-2 (the top-wall row is an identity row with zero source)
    {
        double2 dw[1][K];
#pragma unroll
        for (int i = 0; i < K; ++i) {
            const int r = r0 + i;
            dw[0][i] = r < nz - 1 ? ld2<R>(a.qw, (long long)r * ncol + c) : make_double2(0, 0);
        }
        auto cf = [&](int r, double& aa, double& bb, double& cc) {
            if (r < nz - 1) {
                aa = rk * __ldg(a.c.aw + r);
                cc = rk * __ldg(a.c.cw + r);
                bb = 1.0 + rk * (-lam + __ldg(dgw + r));
            } else { aa = 0.0; bb = 1.0; cc = 0.0; }
        };
        warp_partition_solve<K, 1>(cf, dw, ln);
#pragma unroll
        for (int i = 0; i < K; ++i) SW[i * 32 + ln] = dw[0][i];
    }
    __syncwarp();
    // ---- phi: source div(u*)/dt, Poisson with the null-space pin on (0,0)
    const double2 DX = __ldg(a.c.dx + l), DY = __ldg(a.c.dy + m);
    const double rdt = 1.0 / dt;
    double2 ph[1][K];
    {
        const double2 wlast = SW[(K - 1) * 32 + ln];
        double2 wprev0 = shfl_up2(wlast, 1);
        if (ln == 0) wprev0 = make_double2(0, 0);
#pragma unroll
        for (int i = 0; i < K; ++i) {
            const int r = r0 + i;
            if (r < nz) {
                const double2 us = SU[i * 32 + ln], vs = SV[i * 32 + ln], ws = SW[i * 32 + ln];
                const double2 wm = i > 0 ? SW[(i - 1) * 32 + ln] : wprev0;
                const double rdz = __ldg(a.c.rdz + r);
                double2 div = zadd(zmul(DX, us), zmul(DY, vs));
                div = zadd(div, make_double2((ws.x - wm.x) * rdz, (ws.y - wm.y) * rdz));
                ph[0][i] = make_double2(div.x * rdt, div.y * rdt);
                if (is00 && r == 0) ph[0][i] = make_double2(0, 0);
            } else {
                ph[0][i] = make_double2(0, 0);
            }
        }
        auto cf = [&](int r, double& aa, double& bb, double& cc) {
            if (r < nz) {
                aa = rk * __ldg(a.c.ap + r);
                cc = (is00 && r == 0) ? 0.0 : rk * __ldg(a.c.cp + r);
                bb = rk * (lamp + __ldg(dgp + r));
            } else { aa = 0.0; bb = 1.0; cc = 0.0; }
        };
        warp_partition_solve<K, 1>(cf, ph, ln);
    }
    // ---- projection and psi = phi - rk_c dt nu/2 lap(phi)
    {
        const double2 GX = __ldg(a.c.gx + l), GY = __ldg(a.c.gy + m);
        const double lxy = __ldg(a.c.lx + l) + __ldg(a.c.ly + m);
        const double cpr = rk * dt, cps = rk * 0.5 * dt * a.nu;
        double2 nxt0 = shfl_dn2(ph[0][0], 1);            // phi of the next lane's first row
        double2 prv0 = shfl_up2(ph[0][K - 1], 1);        // phi of the previous lane's last row
#pragma unroll
        for (int i = 0; i < K; ++i) {
            const int r = r0 + i;
            if (r >= nz) continue;
            const long long id = (long long)r * ncol + c;
            const double2 pc = ph[0][i];
            const double2 pu = (r == nz - 1) ? pc : (i < K - 1 ? ph[0][i + 1] : nxt0);
            const double2 pd = (r == 0) ? pc : (i > 0 ? ph[0][i - 1] : prv0);
            const double2 us = SU[i * 32 + ln], vs = SV[i * 32 + ln], ws = SW[i * 32 + ln];
            st2<R>(a.qu, id, zsub(us, zscale(zmul(GX, pc), cpr)));
            st2<R>(a.qv, id, zsub(vs, zscale(zmul(GY, pc), cpr)));
            const double rdzt = __ldg(a.c.rdzt + r), rdzb = __ldg(a.c.rdzb + r), rdz = __ldg(a.c.rdz + r);
            if (r <= nz - 2) {
                st2<R>(a.qw, id, make_double2(ws.x - cpr * (pu.x - pc.x) * rdzt, ws.y - cpr * (pu.y - pc.y) * rdzt));
            } else {
                st2<R>(a.qw, id, make_double2(0, 0));
            }
            double2 lz;
            lz.x = ((pu.x - pc.x) * rdzt - (pc.x - pd.x) * rdzb) * rdz;
            lz.y = ((pu.y - pc.y) * rdzt - (pc.y - pd.y) * rdzb) * rdz;
            st2<R>(a.psi, id, make_double2(pc.x - cps * (lxy * pc.x + lz.x), pc.y - cps * (lxy * pc.y + lz.y)));
        }
    }
}

// Temperature Helmholtz solve (tbnd), warp per column.
template <typename R, int K>
__global__ void __launch_bounds__(CW_WARPS * 32) k_column_t_warp(ColTArgs<R> a)
{
    if (a.halt && *a.halt) return;
    const int ln = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const long long ncol = a.g.ncol;
    const long long c = (long long)blockIdx.x * CW_WARPS + wp;
    if (c >= ncol) return;
    const int nz = a.g.nz;
    const int l = (int)(c % a.g.nxh), m = (int)(c / a.g.nxh);
    const bool is00 = (c == 0);
    const double rk = a.rk_c;
    const double lam = __ldg(a.c.hxt + l) + __ldg(a.c.hyt + m);
    const double* dg = is00 ? a.c.d0t : a.c.dgt;
    const int r0 = ln * K;
    double2 d[1][K];
#pragma unroll
    for (int i = 0; i < K; ++i) {
        const int r = r0 + i;
        if (r < nz) {
            d[0][i] = ld2<R>(a.qt, (long long)r * ncol + c);
            if (is00 && r == 0) d[0][i].x += a.bct0;
            if (is00 && r == nz - 1) d[0][i].x += a.bct1;
        } else {
            d[0][i] = make_double2(0, 0);
        }
    }
    auto cf = [&](int r, double& aa, double& bb, double& cc) {
        if (r < nz) {
            aa = rk * __ldg(a.c.at + r);
            cc = rk * __ldg(a.c.ct + r);
            bb = 1.0 + rk * (-lam + __ldg(dg + r));
        } else { aa = 0.0; bb = 1.0; cc = 0.0; }
    };
    warp_partition_solve<K, 1>(cf, d, ln);
    const bool tr = spec_truncated(l, m, a.g.ny, a.ltr, a.mtr);
#pragma unroll
    for (int i = 0; i < K; ++i) {
        const int r = r0 + i;
        if (r < nz) st2<R>(a.out, (long long)r * ncol + c, tr ? make_double2(0, 0) : d[0][i]);
    }
}

// ---------------------------------------------------------------------------
// Same fused FD column work as k_column_fd_warp, but the block stages the
// columns of CT_COLS adjacent wavenumber pairs in shared memory, so that every
// global load and store is a coalesced row segment of CT_COLS modes instead of
// one scattered 16-byte access per lane. Tile layout per column: [i][lane]
// (row r = lane*K + i), columns padded by one slot so that the row-wise global
// loads land in distinct banks.
// ---------------------------------------------------------------------------
#define CT_COLS 8

template <int K> __host__ __device__ constexpr int ct_stride() { return K * 32 + 1; }
template <int K> __host__ size_t column_tile_smem() { return (size_t)3 * CT_COLS * ct_stride<K>() * sizeof(double2); }

// rows [0, nrows) of CT_COLS columns starting at c0: global [r][c] <-> tile [c][r%K][r/K]
template <typename R, int K>
__device__ __forceinline__ void ct_load(const typename V2<R>::T* __restrict__ q, double2* T, long long c0, long long ncol,
                                        int nrows)
{
    for (int idx = threadIdx.x; idx < nrows * CT_COLS; idx += blockDim.x) {
        const int r = idx / CT_COLS, cb = idx - r * CT_COLS;
        const long long c = c0 + cb;
        T[cb * ct_stride<K>() + (r % K) * 32 + r / K] = c < ncol ? ld2<R>(q, (long long)r * ncol + c) : make_double2(0, 0);
    }
}
template <typename R, int K>
__device__ __forceinline__ void ct_store(typename V2<R>::T* __restrict__ q, const double2* T, long long c0, long long ncol,
                                         int nrows)
{
    for (int idx = threadIdx.x; idx < nrows * CT_COLS; idx += blockDim.x) {
        const int r = idx / CT_COLS, cb = idx - r * CT_COLS;
        const long long c = c0 + cb;
        if (c < ncol) st2<R>(q, (long long)r * ncol + c, T[cb * ct_stride<K>() + (r % K) * 32 + r / K]);
    }
}

template <typename R, int K>
__global__ void __launch_bounds__(CT_COLS * 32, 2) k_column_fd_tile(ColArgs<R> a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (a.halt && *a.halt) return;
    const int ln = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const long long ncol = a.g.ncol;
    const long long c0 = (long long)blockIdx.x * CT_COLS;
    const long long c = c0 + wp;
    const bool active = c < ncol;
    const int nz = a.g.nz;
    double2* TU = reinterpret_cast<double2*>(smem_raw);
    double2* TV = TU + CT_COLS * ct_stride<K>();
    double2* TW = TV + CT_COLS * ct_stride<K>();
    ct_load<R, K>(a.qu, TU, c0, ncol, nz);
    ct_load<R, K>(a.qv, TV, c0, ncol, nz);
    ct_load<R, K>(a.qw, TW, c0, ncol, nz - 1);
    __syncthreads();
    double2* SU = TU + wp * ct_stride<K>();
    double2* SV = TV + wp * ct_stride<K>();
    double2* SW = TW + wp * ct_stride<K>();
    const int l = (int)(c % a.g.nxh), m = (int)(c / a.g.nxh);
    const bool is00 = (c == 0);
    const double rk = a.rk_c, dt = a.dt;
    const int r0 = ln * K;
    double2 ph[1][K];
    if (active) {
        const double lam = __ldg(a.c.hx + l) + __ldg(a.c.hy + m);
        const double lamp = __ldg(a.c.px + l) + __ldg(a.c.py + m);
        const double* dgu = is00 ? a.c.d0u : a.c.dgu;
        const double* dgw = is00 ? a.c.d0w : a.c.dgw;
        const double* dgp = is00 ? a.c.d0p : a.c.dgp;
        // ---- u*, v*: one matrix, two right-hand sides
        {
            double2 d[2][K];
#pragma unroll
            for (int i = 0; i < K; ++i) {
                const int r = r0 + i;
                if (r < nz) {
                    d[0][i] = SU[i * 32 + ln];
                    d[1][i] = SV[i * 32 + ln];
                    if (is00 && r == 0) d[0][i].x += a.bcu0;
                    if (is00 && r == nz - 1) d[0][i].x += a.bcu1;
                } else {
                    d[0][i] = make_double2(0, 0);
                    d[1][i] = make_double2(0, 0);
                }
            }
            auto cf = [&](int r, double& aa, double& bb, double& cc) {
                if (r < nz) {
                    aa = rk * __ldg(a.c.au + r);
                    cc = rk * __ldg(a.c.cu + r);
                    bb = 1.0 + rk * (-lam + __ldg(dgu + r));
                } else { aa = 0.0; bb = 1.0; cc = 0.0; }
            };
            warp_partition_solve<K, 2>(cf, d, ln);
#pragma unroll
            for (int i = 0; i < K; ++i) { SU[i * 32 + ln] = d[0][i]; SV[i * 32 + ln] = d[1][i]; }
        }
        // ---- w*: rows 0..nz-2 (the top-wall row is an identity row with zero source)
        {
            double2 dw[1][K];
#pragma unroll
            for (int i = 0; i < K; ++i) dw[0][i] = r0 + i < nz - 1 ? SW[i * 32 + ln] : make_double2(0, 0);
            auto cf = [&](int r, double& aa, double& bb, double& cc) {
                if (r < nz - 1) {
                    aa = rk * __ldg(a.c.aw + r);
                    cc = rk * __ldg(a.c.cw + r);
                    bb = 1.0 + rk * (-lam + __ldg(dgw + r));
                } else { aa = 0.0; bb = 1.0; cc = 0.0; }
            };
            warp_partition_solve<K, 1>(cf, dw, ln);
#pragma unroll
            for (int i = 0; i < K; ++i) SW[i * 32 + ln] = dw[0][i];
        }
        __syncwarp();
        // ---- phi: source div(u*)/dt, Poisson with the null-space pin on (0,0)
        const double2 DX = __ldg(a.c.dx + l), DY = __ldg(a.c.dy + m);
        const double rdt = 1.0 / dt;
        {
            const double2 wlast = SW[(K - 1) * 32 + ln];
            double2 wprev0 = shfl_up2(wlast, 1);
            if (ln == 0) wprev0 = make_double2(0, 0);
#pragma unroll
            for (int i = 0; i < K; ++i) {
                const int r = r0 + i;
                if (r < nz) {
                    const double2 us = SU[i * 32 + ln], vs = SV[i * 32 + ln], ws = SW[i * 32 + ln];
                    const double2 wm = i > 0 ? SW[(i - 1) * 32 + ln] : wprev0;
                    const double rdz = __ldg(a.c.rdz + r);
                    double2 div = zadd(zmul(DX, us), zmul(DY, vs));
                    div = zadd(div, make_double2((ws.x - wm.x) * rdz, (ws.y - wm.y) * rdz));
                    ph[0][i] = make_double2(div.x * rdt, div.y * rdt);
                    if (is00 && r == 0) ph[0][i] = make_double2(0, 0);
                } else {
                    ph[0][i] = make_double2(0, 0);
                }
            }
            auto cf = [&](int r, double& aa, double& bb, double& cc) {
                if (r < nz) {
                    aa = rk * __ldg(a.c.ap + r);
                    cc = (is00 && r == 0) ? 0.0 : rk * __ldg(a.c.cp + r);
                    bb = rk * (lamp + __ldg(dgp + r));
                } else { aa = 0.0; bb = 1.0; cc = 0.0; }
            };
            warp_partition_solve<K, 1>(cf, ph, ln);
        }
        // ---- projection of u*, v*, w* in place in the tiles
        {
            const double2 GX = __ldg(a.c.gx + l), GY = __ldg(a.c.gy + m);
            const double cpr = rk * dt;
            const double2 nxt0 = shfl_dn2(ph[0][0], 1);
#pragma unroll
            for (int i = 0; i < K; ++i) {
                const int r = r0 + i;
                if (r >= nz) continue;
                const double2 pc = ph[0][i];
                const double2 pu = (r == nz - 1) ? pc : (i < K - 1 ? ph[0][i + 1] : nxt0);
                const double2 us = SU[i * 32 + ln], vs = SV[i * 32 + ln], ws = SW[i * 32 + ln];
                const double rdzt = __ldg(a.c.rdzt + r);
                SU[i * 32 + ln] = zsub(us, zscale(zmul(GX, pc), cpr));
                SV[i * 32 + ln] = zsub(vs, zscale(zmul(GY, pc), cpr));
                SW[i * 32 + ln] = r <= nz - 2 ? make_double2(ws.x - cpr * (pu.x - pc.x) * rdzt, ws.y - cpr * (pu.y - pc.y) * rdzt)
                                              : make_double2(0, 0);
            }
        }
    } else {
#pragma unroll
        for (int i = 0; i < K; ++i) ph[0][i] = make_double2(0, 0);
    }
    __syncthreads();
    ct_store<R, K>(a.qu, TU, c0, ncol, nz);
    ct_store<R, K>(a.qv, TV, c0, ncol, nz);
    ct_store<R, K>(a.qw, TW, c0, ncol, nz);
    __syncthreads();
    // ---- psi = phi - rk_c dt nu/2 lap(phi), staged through the u tile
    {
        const double2 nxt0 = shfl_dn2(ph[0][0], 1);
        const double2 prv0 = shfl_up2(ph[0][K - 1], 1);
        if (active) {
            const double lxy = __ldg(a.c.lx + l) + __ldg(a.c.ly + m);
            const double cps = rk * 0.5 * dt * a.nu;
#pragma unroll
            for (int i = 0; i < K; ++i) {
                const int r = r0 + i;
                if (r >= nz) continue;
                const double2 pc = ph[0][i];
                const double2 pu = (r == nz - 1) ? pc : (i < K - 1 ? ph[0][i + 1] : nxt0);
                const double2 pd = (r == 0) ? pc : (i > 0 ? ph[0][i - 1] : prv0);
                const double rdzt = __ldg(a.c.rdzt + r), rdzb = __ldg(a.c.rdzb + r), rdz = __ldg(a.c.rdz + r);
                double2 lz;
                lz.x = ((pu.x - pc.x) * rdzt - (pc.x - pd.x) * rdzb) * rdz;
                lz.y = ((pu.y - pc.y) * rdzt - (pc.y - pd.y) * rdzb) * rdz;
                SU[i * 32 + ln] = make_double2(pc.x - cps * (lxy * pc.x + lz.x), pc.y - cps * (lxy * pc.y + lz.y));
            }
        }
    }
    __syncthreads();
    ct_store<R, K>(a.psi, TU, c0, ncol, nz);
}
