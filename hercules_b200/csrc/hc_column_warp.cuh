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

// The hardware's single-precision reciprocal approximation (PTX rcp.approx.ftz:
// within about one FP32 ulp; subnormal inputs flush to zero, and no pivot of the
// column systems comes near that range).
__device__ __forceinline__ float rcp_approx(float x)
{
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Reciprocal by Newton-Raphson iteration on f(y) = 1/y - x, i.e.
// y <- y + y (1 - x y), seeded with the single-precision approximation. Each step
// squares the relative error (about 2^-23 -> 2^-46 -> 2^-92), so two steps reach
// FP64 round-off. The pivots of the diagonally dominant column systems stay far
// inside the FP32 range; anything outside it (and NaN) takes the IEEE division.
__device__ __forceinline__ double rcp_nr(double x)
{
    const double ax = fabs(x);
    if (!(ax > 1e-30 && ax < 1e30)) return 1.0 / x;
    double y = (double)rcp_approx((float)x);
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
__device__ __forceinline__ void k_column_fd_warp_body(const ColArgs<R>& a, const uint3 blockIdx, const dim3 gridDim)
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
template <typename R, int K>
__global__ void __launch_bounds__(CW_WARPS * 32, 4) k_column_fd_warp(ColArgs<R> a) { k_column_fd_warp_body<R, K>(a, blockIdx, gridDim); }

// ---------------------------------------------------------------------------
// Columns of CT_COLS adjacent wavenumber pairs staged in shared memory, so that
// every global load and store is a coalesced row segment of CT_COLS modes
// instead of one scattered access per lane. Tile layout per column: [i][lane]
// (row r = lane*K + i), rows of RP slots (the per-lane accesses of the solves
// are consecutive), columns padded so that the row-wise global loads, whose 32
// lanes write 4 rows r of 8 columns, spread over the banks: 16-byte elements
// (FP64) rows of 32 and one pad slot a column; 8-byte elements (FP32) rows of 33
// and two (rows of 32 put the 4 rows on one bank group: 4-way conflicts in every
// load and store of the tiles, 2-way with 33).
// ---------------------------------------------------------------------------
#define CT_COLS 8

template <typename TT> struct CtLayout {
    static constexpr int rp = sizeof(TT) == 8 ? 33 : 32;
    template <int K> __host__ __device__ static constexpr int stride() { return K * rp + (sizeof(TT) == 8 ? 2 : 1); }
};
template <int K> __host__ __device__ constexpr int ct_stride_e(size_t elem)
{
    return elem == 8 ? CtLayout<float2>::stride<K>() : CtLayout<double2>::stride<K>();
}

// ---------------------------------------------------------------------------
// The partition + PCR solve on a chosen arithmetic type T (float or double):
// the mixed-precision column kernel runs its Helmholtz solves in FP32 and keeps
// the Poisson solve and the (0,0) mean mode in FP64.
// ---------------------------------------------------------------------------
// FP32 solves (the mixed mode's Helmholtz systems): the approximation alone; its
// error is of the order of the elimination's own FP32 rounding
__device__ __forceinline__ float rcp_t(float x) { return rcp_approx(x); }
__device__ __forceinline__ double rcp_t(double x) { return rcp_nr(x); }

template <typename T> __device__ __forceinline__ typename V2<T>::T t2sub(typename V2<T>::T a, typename V2<T>::T b)
{
    return mk2<T>(a.x - b.x, a.y - b.y);
}
template <typename T> __device__ __forceinline__ typename V2<T>::T t2axpy(typename V2<T>::T a, typename V2<T>::T b, T s)
{
    return mk2<T>(a.x - s * b.x, a.y - s * b.y);           // a - s b
}
template <typename T> __device__ __forceinline__ typename V2<T>::T t2scale(typename V2<T>::T a, T s)
{
    return mk2<T>(a.x * s, a.y * s);
}
template <typename T> __device__ __forceinline__ typename V2<T>::T t2shfl_up(typename V2<T>::T v, int s)
{
    return mk2<T>(__shfl_up_sync(0xffffffffu, v.x, s), __shfl_up_sync(0xffffffffu, v.y, s));
}
template <typename T> __device__ __forceinline__ typename V2<T>::T t2shfl_dn(typename V2<T>::T v, int s)
{
    return mk2<T>(__shfl_down_sync(0xffffffffu, v.x, s), __shfl_down_sync(0xffffffffu, v.y, s));
}

// The partition + PCR solve of one system on the arithmetic type T (float or
// double), in three phases: the lane's local elimination and the reduced row of
// its last unknown (elim), one PCR level (pcr), the back-substitution (finish).
// warp_partition_solve_t runs them for one system; warp_partition_solve2_t for two
// independent systems phase by phase, so that the dependent chains of the one
// fill the latency of the other's.
template <typename T, int K, int NR> struct PartSys {
    typedef typename V2<T>::T T2;
    T vv[K], ww[K], ib[K];
    T A, B, C;
    T2 D[NR];
    template <typename CF> __device__ __forceinline__ void elim(const CF& coef, T2 (&d)[NR][K], int ln)
    {
        const int r0 = ln * K;
        if (K >= 2) {
            T a0, b0, c0;
            coef(r0, a0, b0, c0);
            ib[0] = rcp_t(b0);
            vv[0] = -a0;
            ww[0] = (K == 2) ? -c0 : T(0);
            T cprev = c0;
#pragma unroll
            for (int i = 1; i <= K - 2; ++i) {
                T ai, bi, ci;
                coef(r0 + i, ai, bi, ci);
                const T mlt = ai * ib[i - 1];
                ib[i] = rcp_t(bi - mlt * cprev);
#pragma unroll
                for (int q = 0; q < NR; ++q) d[q][i] = t2axpy<T>(d[q][i], d[q][i - 1], mlt);
                vv[i] = -mlt * vv[i - 1];
                ww[i] = (i == K - 2 ? -ci : T(0)) - mlt * ww[i - 1];
                cprev = ci;
            }
#pragma unroll
            for (int q = 0; q < NR; ++q) d[q][K - 2] = t2scale<T>(d[q][K - 2], ib[K - 2]);
            vv[K - 2] *= ib[K - 2];
            ww[K - 2] *= ib[K - 2];
#pragma unroll
            for (int i = K - 3; i >= 0; --i) {
                T ai, bi, ci;
                coef(r0 + i, ai, bi, ci);
#pragma unroll
                for (int q = 0; q < NR; ++q) d[q][i] = t2scale<T>(t2axpy<T>(d[q][i], d[q][i + 1], ci), ib[i]);
                vv[i] = (vv[i] - ci * vv[i + 1]) * ib[i];
                ww[i] = (ww[i] - ci * ww[i + 1]) * ib[i];
            }
        }
        T aK, bK, cK;
        coef(r0 + K - 1, aK, bK, cK);
        const T xm_v = K >= 2 ? vv[K - 2] : T(1);
        const T xm_w = K >= 2 ? ww[K - 2] : T(0);
        const T f_v = K >= 2 ? vv[0] : T(0);
        const T f_w = K >= 2 ? ww[0] : T(1);
        const T nf_v = __shfl_down_sync(0xffffffffu, f_v, 1);
        const T nf_w = __shfl_down_sync(0xffffffffu, f_w, 1);
        A = aK * xm_v;
        B = aK * xm_w + bK + cK * nf_v;
        C = cK * nf_w;
#pragma unroll
        for (int q = 0; q < NR; ++q) {
            const T2 z = mk2<T>(T(0), T(0));
            const T2 xm_g = K >= 2 ? d[q][K - 2 < 0 ? 0 : K - 2] : z;
            const T2 f_g = K >= 2 ? d[q][0] : z;
            const T2 nf_g = t2shfl_dn<T>(f_g, 1);
            D[q] = t2axpy<T>(t2axpy<T>(d[q][K - 1], xm_g, aK), nf_g, cK);
        }
    }
    __device__ __forceinline__ void pcr(int s, int ln)
    {
        T Am = __shfl_up_sync(0xffffffffu, A, s), Bm = __shfl_up_sync(0xffffffffu, B, s);
        T Cm = __shfl_up_sync(0xffffffffu, C, s);
        T Ap = __shfl_down_sync(0xffffffffu, A, s), Bp = __shfl_down_sync(0xffffffffu, B, s);
        T Cp = __shfl_down_sync(0xffffffffu, C, s);
        const bool lo = ln < s, hi = ln + s > 31;
        if (lo) { Am = T(0); Bm = T(1); Cm = T(0); }
        if (hi) { Ap = T(0); Bp = T(1); Cp = T(0); }
        const T k1 = A * rcp_t(Bm), k2 = C * rcp_t(Bp);
#pragma unroll
        for (int q = 0; q < NR; ++q) {
            T2 Dm = t2shfl_up<T>(D[q], s), Dp = t2shfl_dn<T>(D[q], s);
            if (lo) Dm = mk2<T>(T(0), T(0));
            if (hi) Dp = mk2<T>(T(0), T(0));
            D[q] = t2axpy<T>(t2axpy<T>(D[q], Dm, k1), Dp, k2);
        }
        const T nA = -Am * k1, nC = -Cp * k2, nB = B - Cm * k1 - Ap * k2;
        A = nA; B = nB; C = nC;
    }
    __device__ __forceinline__ void finish(T2 (&d)[NR][K], int ln)
    {
        const T iB = rcp_t(B);
#pragma unroll
        for (int q = 0; q < NR; ++q) {
            const T2 y = t2scale<T>(D[q], iB);
            T2 yp = t2shfl_up<T>(y, 1);
            if (ln == 0) yp = mk2<T>(T(0), T(0));
#pragma unroll
            for (int i = 0; i < K - 1; ++i)
                d[q][i] = mk2<T>(d[q][i].x + vv[i] * yp.x + ww[i] * y.x, d[q][i].y + vv[i] * yp.y + ww[i] * y.y);
            d[q][K - 1] = y;
        }
    }
};

template <typename T, int K, int NR, typename CF>
__device__ __forceinline__ void warp_partition_solve_t(const CF& coef, typename V2<T>::T (&d)[NR][K], int ln)
{
    PartSys<T, K, NR> a;
    a.elim(coef, d, ln);
#pragma unroll
    for (int s = 1; s < 32; s <<= 1) a.pcr(s, ln);
    a.finish(d, ln);
}

template <typename T, int K, int NR1, int NR2, typename CF1, typename CF2>
__device__ __forceinline__ void warp_partition_solve2_t(const CF1& coef1, typename V2<T>::T (&d1)[NR1][K],
                                                        const CF2& coef2, typename V2<T>::T (&d2)[NR2][K], int ln)
{
    PartSys<T, K, NR1> a;
    PartSys<T, K, NR2> b;
    a.elim(coef1, d1, ln);
    b.elim(coef2, d2, ln);
#pragma unroll
    for (int s = 1; s < 32; s <<= 1) { a.pcr(s, ln); b.pcr(s, ln); }
    a.finish(d1, ln);
    b.finish(d2, ln);
}

// ---------------------------------------------------------------------------
// The fused FD column work of k_column_fd_warp over column tiles in the storage
// type, with the Helmholtz solves in the storage precision: in the mixed mode
// the u, v, w solves run in FP32 (the (0,0) mean mode, with its forcing, and the
// phi Poisson solve stay FP64); in FP64 mode everything is FP64.
// ---------------------------------------------------------------------------
// FP32 storage: per-level tables after the tiles, six FP32 ones (u and w
// Helmholtz rows) and six FP64 ones (Poisson rows, 1/dz, 1/dz_t, 1/dz_b). FP64
// storage reads those coefficients through the read-only cache (its tiles
// already fill the shared memory of two blocks).
// the three tiles; FP32 storage: the level tables and 16 wavenumber constants
// of each column
template <int K> __host__ size_t column_tile_smem_r(size_t elem)
{
    return (size_t)3 * CT_COLS * ct_stride_e<K>(elem) * elem +
           (elem == sizeof(float2) ? (size_t)6 * K * 32 * (sizeof(float) + sizeof(double)) +
                                         (size_t)CT_COLS * 16 * sizeof(double) : 0);
}

template <typename R, int K>
__device__ __forceinline__ void k_column_fd_tile_r_body(const ColArgs<R>& a, const uint3 blockIdx, const dim3 gridDim)
{
    typedef typename V2<R>::T TT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (a.halt && *a.halt) return;
    const int ln = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const long long ncol = a.g.ncol;
    const long long c0 = (long long)blockIdx.x * CT_COLS;
    const long long c = c0 + wp;
    const bool active = c < ncol;
    const int nz = a.g.nz;
    constexpr int STR = CtLayout<TT>::template stride<K>();
    constexpr int RP = CtLayout<TT>::rp;
    TT* TU = reinterpret_cast<TT*>(smem_raw);
    TT* TV = TU + CT_COLS * STR;
    TT* TW = TV + CT_COLS * STR;
    // FP32 storage: the per-level tables follow the tiles
    float* HT = reinterpret_cast<float*>(TW + CT_COLS * STR);
    double* DT = reinterpret_cast<double*>(HT + 6 * K * 32);
    // FP32 storage: 16 wavenumber constants of each column (hx, hy, px, py, the
    // divergence and gradient symbols, lx, ly), loaded together with the tiles so
    // that no warp waits on them later: entry q of column cb at CW[cb * 16 + q]
    // (904 -> 884 us a launch at 512 x 384 x 256). With FP64 storage the same
    // staging was slower (1613 -> 1680 us): there the warps load them when needed.
    constexpr bool kCW = sizeof(R) == sizeof(float);
    double* CW = DT + 6 * K * 32;
    double cwv = 0.0;
    if (kCW) {
        const int cq = threadIdx.x & 15, cb = threadIdx.x >> 4;
        const long long cc = c0 + cb;
        if (cb < CT_COLS && cc < ncol && cq < 14) {
            const int l = (int)(cc % a.g.nxh), m = (int)(cc / a.g.nxh);
            const double* q2l = nullptr;
            switch (cq) {
            case 0: q2l = a.c.hx + l; break;
            case 1: q2l = a.c.hy + m; break;
            case 2: q2l = a.c.px + l; break;
            case 3: q2l = a.c.py + m; break;
            case 4: case 5: q2l = reinterpret_cast<const double*>(a.c.dx + l) + (cq - 4); break;
            case 6: case 7: q2l = reinterpret_cast<const double*>(a.c.dy + m) + (cq - 6); break;
            case 8: case 9: q2l = reinterpret_cast<const double*>(a.c.gx + l) + (cq - 8); break;
            case 10: case 11: q2l = reinterpret_cast<const double*>(a.c.gy + m) + (cq - 10); break;
            case 12: q2l = a.c.lx + l; break;
            default: q2l = a.c.ly + m; break;
            }
            cwv = __ldg(q2l);
        }
    }
    // nrows * CT_COLS <= 32 K * CT_COLS = K * blockDim: at most K elements per
    // thread, all loads issued before the first shared-memory store
    auto load = [&](const TT* __restrict__ q, TT* T, int nrows) {
        TT v[K];
#pragma unroll
        for (int it = 0; it < K; ++it) {
            const int idx = threadIdx.x + it * CT_COLS * 32;
            const int r = idx / CT_COLS, cb = idx - r * CT_COLS;
            const long long cc = c0 + cb;
            v[it] = (idx < nrows * CT_COLS && cc < ncol) ? q[(long long)r * ncol + cc] : mk2<R>(R(0), R(0));
        }
#pragma unroll
        for (int it = 0; it < K; ++it) {
            const int idx = threadIdx.x + it * CT_COLS * 32;
            const int r = idx / CT_COLS, cb = idx - r * CT_COLS;
            if (idx < nrows * CT_COLS) T[cb * STR + (r % K) * RP + r / K] = v[it];
        }
    };
    auto store = [&](TT* __restrict__ q, const TT* T, int nrows) {
        for (int idx = threadIdx.x; idx < nrows * CT_COLS; idx += blockDim.x) {
            const int r = idx / CT_COLS, cb = idx - r * CT_COLS;
            const long long cc = c0 + cb;
            if (cc < ncol) q[(long long)r * ncol + cc] = T[cb * STR + (r % K) * RP + r / K];
        }
    };
    load(a.qu, TU, nz);
    load(a.qv, TV, nz);
    load(a.qw, TW, nz - 1);
    if (kCW && (threadIdx.x >> 4) < CT_COLS) CW[threadIdx.x] = cwv;
    // FP32 storage: the per-level Helmholtz coefficients of the rk_c of this
    // sub-step in FP32 (sub, super, and the diagonal without its -rk lam part),
    // computed once per block instead of per row and lane; tables in the tiles' [i][lane] order (row r = lane*K + i at i*32 + lane),
    // so that the 32 lanes of a warp read 32 consecutive entries
    auto tpos = [](int r) { return (r % K) * 32 + r / K; };
    // table q (0..5: rk ap, rk cp, rk dgp, 1/dz, 1/dz_t, 1/dz_b) at level r
    auto dtab = [&](int q, int r) -> double {
        if constexpr (sizeof(R) == sizeof(float)) return DT[q * K * 32 + tpos(r)];
        const double* src[6] = {a.c.ap, a.c.cp, a.c.dgp, a.c.rdz, a.c.rdzt, a.c.rdzb};
        return q < 3 ? a.rk_c * __ldg(src[q] + r) : __ldg(src[q] + r);
    };
    if constexpr (sizeof(R) == sizeof(float)) {
        for (int r = threadIdx.x; r < nz; r += blockDim.x) {
            const int t = tpos(r);
            DT[t] = a.rk_c * __ldg(a.c.ap + r);
            DT[K * 32 + t] = a.rk_c * __ldg(a.c.cp + r);
            DT[2 * K * 32 + t] = a.rk_c * __ldg(a.c.dgp + r);
            DT[3 * K * 32 + t] = __ldg(a.c.rdz + r);
            DT[4 * K * 32 + t] = __ldg(a.c.rdzt + r);
            DT[5 * K * 32 + t] = __ldg(a.c.rdzb + r);
        }
    }
    if constexpr (sizeof(R) == sizeof(float)) {
        const double rkc = a.rk_c;
        for (int r = threadIdx.x; r < nz; r += blockDim.x) {
            const int t = tpos(r);
            HT[t] = (float)(rkc * __ldg(a.c.au + r));
            HT[K * 32 + t] = (float)(rkc * __ldg(a.c.cu + r));
            HT[2 * K * 32 + t] = (float)(1.0 + rkc * __ldg(a.c.dgu + r));
            if (r < nz - 1) {
                HT[3 * K * 32 + t] = (float)(rkc * __ldg(a.c.aw + r));
                HT[4 * K * 32 + t] = (float)(rkc * __ldg(a.c.cw + r));
                HT[5 * K * 32 + t] = (float)(1.0 + rkc * __ldg(a.c.dgw + r));
            }
        }
    }
    __syncthreads();
    TT* SU = TU + wp * STR;
    TT* SV = TV + wp * STR;
    TT* SW = TW + wp * STR;
    const int l = (int)(c % a.g.nxh), m = (int)(c / a.g.nxh);
    const bool is00 = (c == 0);
    const double rk = a.rk_c, dt = a.dt;
    const int r0 = ln * K;
    const double* cw = CW + wp * 16;
    double2 ph[1][K];
    if (active) {
        const double lam = kCW ? cw[0] + cw[1] : __ldg(a.c.hx + l) + __ldg(a.c.hy + m);
        const double lamp = kCW ? cw[2] + cw[3] : __ldg(a.c.px + l) + __ldg(a.c.py + m);
        const double* dgp = is00 ? a.c.d0p : a.c.dgp;
        // ---- u*, v* (one matrix, two right-hand sides) and w*, in the type T
        auto helmholtz = [&](auto tag) {
            typedef decltype(tag) T;
            typedef typename V2<T>::T T2;
            const double* dgu = is00 ? a.c.d0u : a.c.dgu;
            const double* dgw = is00 ? a.c.d0w : a.c.dgw;
            // u*, v* (two right-hand sides of one matrix) and w* (its own matrix):
            // two independent systems; in FP32 solved phase by phase side by side,
            // in FP64 one after the other (side by side they would not fit the registers)
            const float rlam = (float)(rk * lam);
            auto cf = [&](int r, T& aa, T& bb, T& cc) {
                if (r < nz) {
                    if constexpr (sizeof(T) == sizeof(float)) {
                        const int t = tpos(r);
                        aa = HT[t]; cc = HT[K * 32 + t]; bb = HT[2 * K * 32 + t] - rlam;
                    } else {
                        aa = (T)(rk * __ldg(a.c.au + r));
                        cc = (T)(rk * __ldg(a.c.cu + r));
                        bb = (T)(1.0 + rk * (-lam + __ldg(dgu + r)));
                    }
                } else { aa = T(0); bb = T(1); cc = T(0); }
            };
            auto cfw = [&](int r, T& aa, T& bb, T& cc) {
                if (r < nz - 1) {
                    if constexpr (sizeof(T) == sizeof(float)) {
                        const int t = tpos(r);
                        aa = HT[3 * K * 32 + t]; cc = HT[4 * K * 32 + t]; bb = HT[5 * K * 32 + t] - rlam;
                    } else {
                        aa = (T)(rk * __ldg(a.c.aw + r));
                        cc = (T)(rk * __ldg(a.c.cw + r));
                        bb = (T)(1.0 + rk * (-lam + __ldg(dgw + r)));
                    }
                } else { aa = T(0); bb = T(1); cc = T(0); }
            };
            auto load_uv = [&](T2 (&d)[2][K]) {
#pragma unroll
                for (int i = 0; i < K; ++i) {
                    const int r = r0 + i;
                    if (r < nz) {
                        const TT xu = SU[i * RP + ln], xv = SV[i * RP + ln];
                        double ux = (double)xu.x;
                        if (is00 && r == 0) ux += a.bcu0;
                        if (is00 && r == nz - 1) ux += a.bcu1;
                        d[0][i] = mk2<T>((T)ux, (T)xu.y);
                        d[1][i] = mk2<T>((T)xv.x, (T)xv.y);
                    } else {
                        d[0][i] = mk2<T>(T(0), T(0));
                        d[1][i] = mk2<T>(T(0), T(0));
                    }
                }
            };
            auto load_w = [&](T2 (&dw)[1][K]) {
#pragma unroll
                for (int i = 0; i < K; ++i) {
                    const TT x = SW[i * RP + ln];
                    dw[0][i] = r0 + i < nz - 1 ? mk2<T>((T)x.x, (T)x.y) : mk2<T>(T(0), T(0));
                }
            };
            auto store_uv = [&](const T2 (&d)[2][K]) {
#pragma unroll
                for (int i = 0; i < K; ++i) {
                    SU[i * RP + ln] = mk2<R>((R)d[0][i].x, (R)d[0][i].y);
                    SV[i * RP + ln] = mk2<R>((R)d[1][i].x, (R)d[1][i].y);
                }
            };
            auto store_w = [&](const T2 (&dw)[1][K]) {
#pragma unroll
                for (int i = 0; i < K; ++i) SW[i * RP + ln] = mk2<R>((R)dw[0][i].x, (R)dw[0][i].y);
            };
            if constexpr (sizeof(T) == sizeof(float)) {
                T2 d[2][K], dw[1][K];
                load_uv(d);
                load_w(dw);
                warp_partition_solve2_t<T, K, 2, 1>(cf, d, cfw, dw, ln);
                store_uv(d);
                store_w(dw);
            } else {
                {
                    T2 d[2][K];
                    load_uv(d);
                    warp_partition_solve_t<T, K, 2>(cf, d, ln);
                    store_uv(d);
                }
                {
                    T2 dw[1][K];
                    load_w(dw);
                    warp_partition_solve_t<T, K, 1>(cfw, dw, ln);
                    store_w(dw);
                }
            }
        };
        if (is00) helmholtz(double(0)); else helmholtz(R(0));
        __syncwarp();
        // ---- phi: source div(u*)/dt, Poisson with the null-space pin on (0,0), FP64
        const double2 DX = kCW ? make_double2(cw[4], cw[5]) : __ldg(a.c.dx + l);
        const double2 DY = kCW ? make_double2(cw[6], cw[7]) : __ldg(a.c.dy + m);
        const double rdt = 1.0 / dt;
        {
            auto ldt = [&](const TT* S, int idx) { const TT x = S[idx]; return make_double2((double)x.x, (double)x.y); };
            const double2 wlast = ldt(SW, (K - 1) * RP + ln);
            double2 wprev0 = shfl_up2(wlast, 1);
            if (ln == 0) wprev0 = make_double2(0, 0);
#pragma unroll
            for (int i = 0; i < K; ++i) {
                const int r = r0 + i;
                if (r < nz) {
                    const double2 us = ldt(SU, i * RP + ln), vs = ldt(SV, i * RP + ln), ws = ldt(SW, i * RP + ln);
                    const double2 wm = i > 0 ? ldt(SW, (i - 1) * RP + ln) : wprev0;
                    const double rdz = dtab(3, r);
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
                    if (sizeof(R) == sizeof(float) && !is00) {
                        aa = dtab(0, r); cc = dtab(1, r); bb = dtab(2, r) + rk * lamp;
                    } else {
                        aa = rk * __ldg(a.c.ap + r);
                        cc = (is00 && r == 0) ? 0.0 : rk * __ldg(a.c.cp + r);
                        bb = rk * (lamp + __ldg(dgp + r));
                    }
                } else { aa = 0.0; bb = 1.0; cc = 0.0; }
            };
            warp_partition_solve<K, 1>(cf, ph, ln);
        }
        // ---- projection of u*, v*, w* in place in the tiles
        {
            const double2 GX = kCW ? make_double2(cw[8], cw[9]) : __ldg(a.c.gx + l);
            const double2 GY = kCW ? make_double2(cw[10], cw[11]) : __ldg(a.c.gy + m);
            const double cpr = rk * dt;
            const double2 nxt0 = shfl_dn2(ph[0][0], 1);
#pragma unroll
            for (int i = 0; i < K; ++i) {
                const int r = r0 + i;
                if (r >= nz) continue;
                const double2 pc = ph[0][i];
                const double2 pu = (r == nz - 1) ? pc : (i < K - 1 ? ph[0][i + 1] : nxt0);
                const TT us = SU[i * RP + ln], vs = SV[i * RP + ln], ws = SW[i * RP + ln];
                const double rdzt = dtab(4, r);
                const double2 gu = zmul(GX, pc), gv = zmul(GY, pc);
                SU[i * RP + ln] = mk2<R>((R)((double)us.x - cpr * gu.x), (R)((double)us.y - cpr * gu.y));
                SV[i * RP + ln] = mk2<R>((R)((double)vs.x - cpr * gv.x), (R)((double)vs.y - cpr * gv.y));
                SW[i * RP + ln] = r <= nz - 2 ? mk2<R>((R)((double)ws.x - cpr * (pu.x - pc.x) * rdzt),
                                                       (R)((double)ws.y - cpr * (pu.y - pc.y) * rdzt))
                                              : mk2<R>(R(0), R(0));
            }
        }
    } else {
#pragma unroll
        for (int i = 0; i < K; ++i) ph[0][i] = make_double2(0, 0);
    }
    __syncthreads();
    store(a.qu, TU, nz);
    store(a.qv, TV, nz);
    store(a.qw, TW, nz);
    __syncthreads();
    // ---- psi = phi - rk_c dt nu/2 lap(phi), staged through the u tile
    {
        const double2 nxt0 = shfl_dn2(ph[0][0], 1);
        const double2 prv0 = shfl_up2(ph[0][K - 1], 1);
        if (active) {
            const double lxy = kCW ? cw[12] + cw[13] : __ldg(a.c.lx + l) + __ldg(a.c.ly + m);
            const double cps = rk * 0.5 * dt * a.nu;
#pragma unroll
            for (int i = 0; i < K; ++i) {
                const int r = r0 + i;
                if (r >= nz) continue;
                const double2 pc = ph[0][i];
                const double2 pu = (r == nz - 1) ? pc : (i < K - 1 ? ph[0][i + 1] : nxt0);
                const double2 pd = (r == 0) ? pc : (i > 0 ? ph[0][i - 1] : prv0);
                const double rdzt = dtab(4, r), rdzb = dtab(5, r), rdz = dtab(3, r);
                double2 lz;
                lz.x = ((pu.x - pc.x) * rdzt - (pc.x - pd.x) * rdzb) * rdz;
                lz.y = ((pu.y - pc.y) * rdzt - (pc.y - pd.y) * rdzb) * rdz;
                SU[i * RP + ln] = mk2<R>((R)(pc.x - cps * (lxy * pc.x + lz.x)), (R)(pc.y - cps * (lxy * pc.y + lz.y)));
            }
        }
    }
    __syncthreads();
    store(a.psi, TU, nz);
}
template <typename R, int K>
__global__ void __launch_bounds__(CT_COLS * 32, 2) k_column_fd_tile_r(ColArgs<R> a) { k_column_fd_tile_r_body<R, K>(a, blockIdx, gridDim); }

// ---------------------------------------------------------------------------
// Temperature Helmholtz solve (tbnd) through one coalescing tile: a block of
// CT_COLS warps loads the rows of CT_COLS adjacent columns of q_t with
// row-contiguous loads, each warp solves one column in FP64 from the tile, and
// the solution (0 on truncated modes) leaves through the tile with
// row-contiguous stores. All of a block's loads come before its stores, so the
// solution may overwrite q_t. (One warp per column reading and writing a row a
// lane: 76 -> 67 us mixed, 91 -> 68 us FP64 a launch at 256 x 256 x 128.)
// ---------------------------------------------------------------------------
// FP32 storage: the tile and, after it, the per-level matrix rows of the sub-step
// in FP32 (rk at, rk ct, 1 + rk dgt) in the [i][lane] order of the solves
template <int K> __host__ size_t column_t_tile_smem(size_t elem)
{
    return (size_t)CT_COLS * ct_stride_e<K>(elem) * elem + (elem == sizeof(float2) ? (size_t)3 * K * 32 * sizeof(float) : 0);
}

template <typename R, int K>
__device__ __forceinline__ void k_column_t_tile_body(const ColTArgs<R>& a, const uint3 blockIdx, const dim3 gridDim)
{
    typedef typename V2<R>::T TT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (a.halt && *a.halt) return;
    const int ln = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const long long ncol = a.g.ncol;
    const long long c0 = (long long)blockIdx.x * CT_COLS;
    const long long c = c0 + wp;
    const int nz = a.g.nz;
    constexpr int STR = CtLayout<TT>::template stride<K>();
    constexpr int RP = CtLayout<TT>::rp;
    TT* TQ = reinterpret_cast<TT*>(smem_raw);
    // FP32 storage: the sub-step's matrix rows in FP32 after the tile
    float* TB = reinterpret_cast<float*>(TQ + CT_COLS * STR);
    if constexpr (sizeof(R) == sizeof(float)) {
        const double rk = a.rk_c;
        for (int r = threadIdx.x; r < nz; r += blockDim.x) {
            const int t = (r % K) * 32 + r / K;
            TB[t] = (float)(rk * __ldg(a.c.at + r));
            TB[K * 32 + t] = (float)(rk * __ldg(a.c.ct + r));
            TB[2 * K * 32 + t] = (float)(1.0 + rk * __ldg(a.c.dgt + r));
        }
    }
    {
        TT v[K];
#pragma unroll
        for (int it = 0; it < K; ++it) {
            const int idx = threadIdx.x + it * CT_COLS * 32;
            const int r = idx / CT_COLS, cb = idx - r * CT_COLS;
            const long long cc = c0 + cb;
            v[it] = (idx < nz * CT_COLS && cc < ncol) ? a.qt[(long long)r * ncol + cc] : mk2<R>(R(0), R(0));
        }
#pragma unroll
        for (int it = 0; it < K; ++it) {
            const int idx = threadIdx.x + it * CT_COLS * 32;
            const int r = idx / CT_COLS, cb = idx - r * CT_COLS;
            if (idx < nz * CT_COLS) TQ[cb * STR + (r % K) * RP + r / K] = v[it];
        }
    }
    __syncthreads();
    TT* SQ = TQ + wp * STR;
    if (c < ncol) {
        const int l = (int)(c % a.g.nxh), m = (int)(c / a.g.nxh);
        const bool is00 = (c == 0);
        const double rk = a.rk_c;
        const double lam = __ldg(a.c.hxt + l) + __ldg(a.c.hyt + m);
        const double* dg = is00 ? a.c.d0t : a.c.dgt;
        const int r0 = ln * K;
        const bool tr = spec_truncated(l, m, a.g.ny, a.ltr, a.mtr);
        if (sizeof(R) == sizeof(float) && !is00) {
            // FP32 storage, every mode but the mean: the diagonally dominant
            // Helmholtz system in FP32, as the momentum ones (the mean mode keeps
            // FP64 with the wall constants)
            const float rlam = (float)(rk * lam);
            float2 df[1][K];
#pragma unroll
            for (int i = 0; i < K; ++i) {
                const TT x = SQ[i * RP + ln];
                df[0][i] = r0 + i < nz ? make_float2((float)x.x, (float)x.y) : make_float2(0.0f, 0.0f);
            }
            auto cf = [&](int r, float& aa, float& bb, float& cc) {
                if (r < nz) {
                    const int t = (r % K) * 32 + r / K;
                    aa = TB[t]; cc = TB[K * 32 + t]; bb = TB[2 * K * 32 + t] - rlam;
                } else { aa = 0.0f; bb = 1.0f; cc = 0.0f; }
            };
            warp_partition_solve_t<float, K, 1>(cf, df, ln);
#pragma unroll
            for (int i = 0; i < K; ++i) SQ[i * RP + ln] = tr ? mk2<R>(R(0), R(0)) : mk2<R>((R)df[0][i].x, (R)df[0][i].y);
        } else {
            double2 d[1][K];
#pragma unroll
            for (int i = 0; i < K; ++i) {
                const int r = r0 + i;
                if (r < nz) {
                    const TT x = SQ[i * RP + ln];
                    d[0][i] = make_double2((double)x.x, (double)x.y);
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
#pragma unroll
            for (int i = 0; i < K; ++i) {
                const double2 v = tr ? make_double2(0, 0) : d[0][i];
                SQ[i * RP + ln] = mk2<R>((R)v.x, (R)v.y);
            }
        }
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < nz * CT_COLS; idx += blockDim.x) {
        const int r = idx / CT_COLS, cb = idx - r * CT_COLS;
        const long long cc = c0 + cb;
        if (cc < ncol) a.out[(long long)r * ncol + cc] = TQ[cb * STR + (r % K) * RP + r / K];
    }
}
template <typename R, int K>
__global__ void __launch_bounds__(CT_COLS * 32, 2) k_column_t_tile(ColTArgs<R> a) { k_column_t_tile_body<R, K>(a, blockIdx, gridDim); }
