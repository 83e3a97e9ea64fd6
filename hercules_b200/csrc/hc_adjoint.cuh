// hc_adjoint.cuh -- discrete adjoint of the FD sub-step (no counterpart in the
// reference). Scope: FP64, cds = 1 or 2, constant forcing (dp_opt = 1 or 3),
// temperature with a constant Richardson number, no damping; RK3 or AB2; body
// force.
//
// One forward sub-step maps (u, v, w, p, f_prev) to (u', v', w', p', f):
//   f   = F(u, v, w) + body force                    (momentum RHS, k_rhs_momentum)
//   q   = u + dt (rk_a f + rk_b f_prev) + c_d L u - rk_c dt G p
//   (u', v', w', psi) = M q,   M = iFFT . C . FFT     (column solves + projection)
//   p'  = p + psi
// Its adjoint, given the adjoints of the outputs:
//   lambda_q  = M^T (lambda_u', lambda_v', lambda_w', lambda_p'),
//               M^T = iFFT . C^H . FFT (the same transforms; C^H per wavenumber)
//   lambda_f  = dt rk_a lambda_q + lambda_f(out);  lambda_f_prev = dt rk_b lambda_q
//   lambda_u  = lambda_q + c_d L^T lambda_q + (dF/du)^T lambda_f, and alike for v, w
//   lambda_p  = lambda_p' - rk_c dt G^T lambda_q;     lambda_bodyforce += lambda_f
// The nonlinear RHS is differentiated by transposed stencils in two gather
// passes, without atomics (so the gradient is bitwise reproducible): first the
// adjoint of every interpolant (uhx ... vhz) at its own point, gathered from the
// equations whose differences read it, then the adjoint of every raw value,
// gathered through the interpolation weights, the identity, the diffusion and
// pressure-gradient stencils and the z ghost relations (the ghost of a wall
// value folds back onto that value).
#pragma once
#include "hc_fd.cuh"
#include "hc_column_warp.cuh"

struct AdjRhsArgs {
    Acc<double> a;                 // the forward state at the sub-step's start
    const double* lq[3];           // lambda_q (physical)
    const double* lf_out[3];       // adjoint of the new histories ff, gg, hh
    double* lf_prev[3];            // out: adjoint of the old histories (not lf_out's buffers)
    double* lbf[3];                // body-force gradient, accumulated
    double* ax[8];                 // adjoints of the interpolants uhx, uhy, vhx, vhy, whx, why, uhz, vhz
    double* out[4];                // lambda_u, v, w (written), lambda_p (accumulated)
    double* out_t;                 // lambda_T (accumulated: the buoyancy of the w equation); null: none
    double got;                    // g/T0 of the buoyancy term
    double rk_a, rk_b, rk_c;
    Phys ph;
};

// staggered first difference of the x/y fluxes: D(h)(i) = sum_q c(q) h(i + off(q)),
// off = 2, 1, 0, -1 (cds=2, c = -1, 27, -27, 1 over 24) or 1, 0 (cds=1, c = 1, -1)
template <int CDS> struct Dif {
    static constexpr int n = CDS == 1 ? 2 : 4;
    __device__ static int off(int q) { return CDS == 1 ? 1 - q : 2 - q; }
    __device__ static double c(int q) { return CDS == 1 ? (q == 0 ? 1.0 : -1.0) : (q == 0 ? -1.0 : q == 1 ? 27.0 : q == 2 ? -27.0 : 1.0) / 24.0; }
};

__device__ __forceinline__ long long adj_at(const Geo& g, int i, int j, int k)
{
    return ((long long)k * g.ny + wrapi(j, g.ny)) * g.nx + wrapi(i, g.nx);
}

// Wrapped neighbour offsets of one point: i-2..i+2 and rows j-2..j+2 of level k.
struct Nbr {
    long long kz;
    int xi[5];
    int yj[5];
    __device__ __forceinline__ Nbr(const Geo& g, int i, int j, int k)
    {
        kz = (long long)k * g.nxy;
#pragma unroll
        for (int d = -2; d <= 2; ++d) {
            xi[d + 2] = wrapi(i + d, g.nx);
            yj[d + 2] = wrapi(j + d, g.ny) * g.nx;
        }
    }
    __device__ __forceinline__ long long at(int di, int dj) const { return kz + yj[dj + 2] + xi[di + 2]; }
};

// Pass 1, per point: the adjoint of every interpolant evaluated at this point,
// gathered from the right-hand sides that read it (lambda_f = dt rk_a lambda_q +
// lambda_f(out) at those points), and this point's history and body-force
// adjoints. The interpolants are the forward ones (same weights and wall rules).
template <int CDS>
__global__ void __launch_bounds__(256) k_rhs_adj_interp(AdjRhsArgs m)
{
    const Geo& g = m.a.g;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= g.nx || j >= g.ny) return;
    const int nz = g.nz;
    const Nbr N(g, i, j, k);
    const long long id = N.at(0, 0), up = g.nxy;
    const bool wrow = k <= nz - 2;           // this level carries a w equation
    const double dta = m.ph.dt * m.rk_a, dtb = m.ph.dt * m.rk_b;
    auto L = [&](int c, long long q) { return dta * __ldg(m.lq[c] + q) + __ldg(m.lf_out[c] + q); };
    for (int c = 0; c < 3; ++c) {
        if (c < 2 || wrow) {
            m.lf_prev[c][id] = dtb * m.lq[c][id];
            m.lbf[c][id] += L(c, id);
        } else {
            m.lf_prev[c][id] = m.lf_out[c][id];       // hh of the top-wall level is carried over
        }
    }
    double sxu = 0, syu = 0, sxv = 0, syv = 0, sxw = 0, syw = 0;
#pragma unroll
    for (int q = 0; q < Dif<CDS>::n; ++q) {
        const int o = Dif<CDS>::off(q);
        const double cx = Dif<CDS>::c(q) / g.dx, cy = Dif<CDS>::c(q) / g.dy;
        sxu += cx * L(0, N.at(-o, 0));          // uux: uhx(i) in the U equations at i - off
        syu += cy * L(0, N.at(0, 1 - o));       // uvy: uhy vhx(j) at j - off + 1
        sxv += cx * L(1, N.at(1 - o, 0));       // vux: vhx uhy(i) at i - off + 1
        syv += cy * L(1, N.at(0, -o));          // vvy: vhy(j) at j - off
        if (wrow) {
            sxw += cx * L(2, N.at(1 - o, 0));   // wux: whx uhz(i)
            syw += cy * L(2, N.at(0, 1 - o));   // wvy: why vhz(j)
        }
    }
    const double* U = m.a.f.u;
    const double* V = m.a.f.v;
    const double* W = m.a.f.w;
    auto ld = [&](const double* f, int di, int dj) { return __ldg(f + N.at(di, dj)); };
    double uhx, uhy, vhx, vhy;
    if (CDS == 1) {
        uhx = 0.5 * (ld(U, 0, 0) + ld(U, -1, 0));
        uhy = 0.5 * (ld(U, 0, 1) + ld(U, 0, 0));
        vhx = 0.5 * (ld(V, 1, 0) + ld(V, 0, 0));
        vhy = 0.5 * (ld(V, 0, 0) + ld(V, 0, -1));
    } else {
        uhx = (-ld(U, 1, 0) + 9.0 * ld(U, 0, 0) + 9.0 * ld(U, -1, 0) - ld(U, -2, 0)) * 0.0625;
        uhy = (-ld(U, 0, 2) + 9.0 * ld(U, 0, 1) + 9.0 * ld(U, 0, 0) - ld(U, 0, -1)) * 0.0625;
        vhx = (-ld(V, 2, 0) + 9.0 * ld(V, 1, 0) + 9.0 * ld(V, 0, 0) - ld(V, -1, 0)) * 0.0625;
        vhy = (-ld(V, 0, 1) + 9.0 * ld(V, 0, 0) + 9.0 * ld(V, 0, -1) - ld(V, 0, -2)) * 0.0625;
    }
    const double um = m.a.um, fc = m.ph.fc;
    const bool cor = m.ph.dp_opt == 3;
    m.ax[0][id] = -(2.0 * uhx + um) * sxu;
    m.ax[1][id] = -vhx * (syu + sxv) - (cor ? 0.5 * fc * (L(1, id) + L(1, N.at(1, 0))) : 0.0);
    m.ax[2][id] = -uhy * syu - (uhy + um) * sxv + (cor ? 0.5 * fc * (L(0, id) + L(0, N.at(0, 1))) : 0.0);
    m.ax[3][id] = -2.0 * vhy * syv;
    if (wrow) {
        // uwz, vwz: the face k between levels k and k+1 enters both with 1/dz
        const double rz0 = 1.0 / ldz(g.z.dz, k), rz1 = 1.0 / ldz(g.z.dz, k + 1);
        const double zu = -L(0, id) * rz0 + L(0, id + up) * rz1;
        const double zv = -L(1, id) * rz0 + L(1, id + up) * rz1;
        const double l = ldz(g.z.l_t, k);
        const double uhz = __ldg(U + id + up) * l + __ldg(U + id) * (1.0 - l);
        const double vhz = __ldg(V + id + up) * l + __ldg(V + id) * (1.0 - l);
        double whx, why;
        if (CDS == 1) {
            whx = 0.5 * (ld(W, 1, 0) + ld(W, 0, 0));
            why = 0.5 * (ld(W, 0, 1) + ld(W, 0, 0));
        } else {
            whx = (-ld(W, 2, 0) + 9.0 * ld(W, 1, 0) + 9.0 * ld(W, 0, 0) - ld(W, -1, 0)) * 0.0625;
            why = (-ld(W, 0, 2) + 9.0 * ld(W, 0, 1) + 9.0 * ld(W, 0, 0) - ld(W, 0, -1)) * 0.0625;
        }
        m.ax[4][id] = uhz * zu - (uhz + um) * sxw;
        m.ax[5][id] = vhz * zv - vhz * syw;
        m.ax[6][id] = whx * zu - whx * sxw;
        m.ax[7][id] = why * zv - why * syw;
    } else {
        m.ax[4][id] = 0.0; m.ax[5][id] = 0.0; m.ax[6][id] = 0.0; m.ax[7][id] = 0.0;
    }
}

// Pass 2, per point: lambda_u, v, w, p by the transposed stencils -- the
// interpolant adjoints through the transposed interpolation weights, lambda_q
// through the identity, the transposed diffusion (horizontal stencils are
// symmetric; the wall ghosts of the z second difference fold back onto the
// first and last levels) and the transposed pressure gradient, plus the w^2
// flux of the w equation. lambda_p keeps its incoming value (p' = p + psi).
template <int CDS>
__global__ void __launch_bounds__(256) k_rhs_adj_gather(AdjRhsArgs m)
{
    const Geo& g = m.a.g;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= g.nx || j >= g.ny) return;
    const int nz = g.nz;
    const Nbr N(g, i, j, k);
    const long long id = N.at(0, 0), up = g.nxy;
    const bool wrow = k <= nz - 2;
    const double dt = m.ph.dt, cdif = m.rk_c * 0.5 * dt * m.ph.nu, crp = m.rk_c * dt, dta = dt * m.rk_a;
    auto X = [&](int f, int di, int dj) { return __ldg(m.ax[f] + N.at(di, dj)); };
    auto Q = [&](int c, int di, int dj) { return __ldg(m.lq[c] + N.at(di, dj)); };
    auto dz = [&](int kk) { return ldz(g.z.dz, kk); };
    auto dzt = [&](int kk) { return ldz(g.z.dz_t, kk); };
    auto dzb = [&](int kk) { return ldz(g.z.dz_b, kk); };
    double lu, lv, lw, lp;
    // ---- transposed interpolation weights
    if (CDS == 1) {
        lu = 0.5 * (X(0, 0, 0) + X(0, 1, 0)) + 0.5 * (X(1, 0, -1) + X(1, 0, 0));
        lv = 0.5 * (X(2, -1, 0) + X(2, 0, 0)) + 0.5 * (X(3, 0, 0) + X(3, 0, 1));
        lw = 0.5 * (X(4, -1, 0) + X(4, 0, 0)) + 0.5 * (X(5, 0, -1) + X(5, 0, 0));
    } else {
        lu = (-X(0, -1, 0) + 9.0 * X(0, 0, 0) + 9.0 * X(0, 1, 0) - X(0, 2, 0)) * 0.0625 +
             (-X(1, 0, -2) + 9.0 * X(1, 0, -1) + 9.0 * X(1, 0, 0) - X(1, 0, 1)) * 0.0625;
        lv = (-X(2, -2, 0) + 9.0 * X(2, -1, 0) + 9.0 * X(2, 0, 0) - X(2, 1, 0)) * 0.0625 +
             (-X(3, 0, -1) + 9.0 * X(3, 0, 0) + 9.0 * X(3, 0, 1) - X(3, 0, 2)) * 0.0625;
        lw = (-X(4, -2, 0) + 9.0 * X(4, -1, 0) + 9.0 * X(4, 0, 0) - X(4, 1, 0)) * 0.0625 +
             (-X(5, 0, -2) + 9.0 * X(5, 0, -1) + 9.0 * X(5, 0, 0) - X(5, 0, 1)) * 0.0625;
    }
    if (k >= 1) {
        const double l = ldz(g.z.l_t, k - 1);
        lu += __ldg(m.ax[6] + id - up) * l;
        lv += __ldg(m.ax[7] + id - up) * l;
    }
    if (wrow) {
        const double l = ldz(g.z.l_t, k);
        lu += __ldg(m.ax[6] + id) * (1.0 - l);
        lv += __ldg(m.ax[7] + id) * (1.0 - l);
    }
    // ---- identity and horizontal diffusion (symmetric stencils)
    double hq[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        if (c == 2 && !wrow) { hq[c] = 0.0; continue; }
        const double q0 = Q(c, 0, 0);
        double h;
        if (CDS == 1) {
            h = (Q(c, 1, 0) - 2.0 * q0 + Q(c, -1, 0)) / g.dx2 + (Q(c, 0, 1) - 2.0 * q0 + Q(c, 0, -1)) / g.dy2;
        } else {
            h = (-Q(c, 2, 0) + 16.0 * Q(c, 1, 0) - 30.0 * q0 + 16.0 * Q(c, -1, 0) - Q(c, -2, 0)) / (12.0 * g.dx2) +
                (-Q(c, 0, 2) + 16.0 * Q(c, 0, 1) - 30.0 * q0 + 16.0 * Q(c, 0, -1) - Q(c, 0, -2)) / (12.0 * g.dy2);
        }
        hq[c] = q0 + cdif * h;
    }
    // lambda_q of the same column at levels k-1, k, k+1 (zero where no equation)
    auto qz = [&](int c, int kk) -> double {
        if (kk < 0 || kk >= nz || (c == 2 && kk > nz - 2)) return 0.0;
        return __ldg(m.lq[c] + id + (long long)(kk - k) * up);
    };
    const bool closed = m.a.closed;
    {   // u, v: second difference over cell centres with the no-slip / free-slip ghosts
        const double qu = qz(0, k), qv = qz(1, k);
        const double e0 = (1.0 / dzt(k) + 1.0 / dzb(k)) / dz(k);
        double zu = -qu * e0, zv = -qv * e0;
        if (k >= 1) { const double e = 1.0 / (dzt(k - 1) * dz(k - 1)); zu += qz(0, k - 1) * e; zv += qz(1, k - 1) * e; }
        if (k <= nz - 2) { const double e = 1.0 / (dzb(k + 1) * dz(k + 1)); zu += qz(0, k + 1) * e; zv += qz(1, k + 1) * e; }
        if (k == 0) { const double e = 1.0 / (dzb(0) * dz(0)); zu -= qu * e; zv -= qv * e; }
        if (k == nz - 1) { const double e = (closed ? -1.0 : 1.0) / (dzt(k) * dz(k)); zu += qu * e; zv += qv * e; }
        lu += hq[0] + cdif * zu;
        lv += hq[1] + cdif * zv;
    }
    const double qwm = qz(2, k - 1), qw0 = qz(2, k), qwp = qz(2, k + 1);
    {   // w: second difference over faces (w = 0 below the first face), rows k <= nz-2
        double zw = wrow ? -qw0 * (1.0 / dz(k + 1) + 1.0 / dz(k)) / dzt(k) : 0.0;
        if (k >= 1) zw += qwm / (dz(k) * dzt(k - 1));
        if (k + 1 <= nz - 2) zw += qwp / (dz(k + 1) * dzt(k + 1));
        lw += hq[2] + cdif * zw;
        // w^2 flux: ((w(k) + w(k+1)) / 2)^2 - ((w(k) + w(k-1)) / 2)^2 over dz_t at rows k' = k-1, k, k+1
        auto Lfw = [&](int kk) -> double {
            if (kk < 0 || kk > nz - 2) return 0.0;
            const long long q = id + (long long)(kk - k) * up;
            return dta * __ldg(m.lq[2] + q) + __ldg(m.lf_out[2] + q);
        };
        const double* W = m.a.f.w;
        const double wm = k >= 1 ? __ldg(W + id - up) : 0.0, wc = __ldg(W + id);
        const double wp = wrow ? __ldg(W + id + up) : 0.0;
        const double l0 = Lfw(k), lm = Lfw(k - 1), lp1 = Lfw(k + 1);
        if (wrow) lw += l0 / dzt(k) * (-0.5 * (wc + wp) + 0.5 * (wc + wm));
        if (k >= 1) lw -= lm / dzt(k - 1) * 0.5 * (wm + wc);
        if (k + 1 <= nz - 2) lw += lp1 / dzt(k + 1) * 0.5 * (wp + wc);
        // buoyancy got ((1 - l_t(k')) T(k') + l_t(k') T(k'+1)) in the w equations k' = k, k-1
        if (m.out_t) {
            double bt = 0.0;
            if (wrow) bt += (1.0 - ldz(g.z.l_t, k)) * l0;
            if (k >= 1) bt += ldz(g.z.l_t, k - 1) * lm;
            m.out_t[id] += m.got * bt;
        }
    }
    // pressure gradients of the three equations
    if (CDS == 1) {
        lp = -crp / g.dx * (Q(0, -1, 0) - Q(0, 0, 0)) - crp / g.dy * (Q(1, 0, -1) - Q(1, 0, 0));
    } else {
        lp = -crp / (24.0 * g.dx) * (-Q(0, -2, 0) + 27.0 * Q(0, -1, 0) - 27.0 * Q(0, 0, 0) + Q(0, 1, 0)) -
             crp / (24.0 * g.dy) * (-Q(1, 0, -2) + 27.0 * Q(1, 0, -1) - 27.0 * Q(1, 0, 0) + Q(1, 0, 1));
    }
    lp += crp * (qw0 / dzt(k) - (k >= 1 ? qwm / dzt(k - 1) : 0.0));
    m.out[0][id] = lu;
    m.out[1][id] = lv;
    m.out[2][id] = lw;
    m.out[3][id] += lp;
}

// ---------------------------------------------------------------------------
// C^H per wavenumber column: the adjoint of k_column_fd_warp's map
//   u* = Hu^-1 qu, v* = Hu^-1 qv, w* = Hw^-1 qw (rows 0..nz-2)
//   s  = (DX u* + DY v* + dz-difference of w*) / dt      (s(0) = 0 for the (0,0) mode)
//   phi = P^-1 s
//   u' = u* - cpr GX phi, v' = v* - cpr GY phi, w'(k) = w*(k) - cpr Gz phi (k <= nz-2), w'(nz-1) = 0
//   psi = phi - cps (lxy phi + Lz phi)                    (Neumann ghosts of phi)
// applied in reverse with every complex symbol conjugated and every matrix
// transposed. In: adjoints of u', v', w', psi (spectra); out: adjoints of qu, qv,
// qw (written over the first three).
// ---------------------------------------------------------------------------
struct ColAdjArgs {
    double2* au; double2* av; double2* aw; const double2* apsi;
    ColCoef c;
    Geo g;
    double rk_c, dt, nu;
};

__device__ __forceinline__ double2 zconj(double2 a) { return make_double2(a.x, -a.y); }

template <int K>
__global__ void __launch_bounds__(CW_WARPS * 32) k_column_fd_adj(ColAdjArgs a)
{
    const int ln = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const long long ncol = a.g.ncol;
    const long long c = (long long)blockIdx.x * CW_WARPS + wp;
    if (c >= ncol) return;
    const int nz = a.g.nz;
    const int l = (int)(c % a.g.nxh), m = (int)(c / a.g.nxh);
    const bool is00 = (c == 0);
    const double rk = a.rk_c, dt = a.dt, rdt = 1.0 / dt;
    const double cpr = rk * dt, cps = rk * 0.5 * dt * a.nu;
    const double lam = __ldg(a.c.hx + l) + __ldg(a.c.hy + m);
    const double lamp = __ldg(a.c.px + l) + __ldg(a.c.py + m);
    const double lxy = __ldg(a.c.lx + l) + __ldg(a.c.ly + m);
    const double* dgu = is00 ? a.c.d0u : a.c.dgu;
    const double* dgw = is00 ? a.c.d0w : a.c.dgw;
    const double* dgp = is00 ? a.c.d0p : a.c.dgp;
    const double2 DX = __ldg(a.c.dx + l), DY = __ldg(a.c.dy + m), GX = __ldg(a.c.gx + l), GY = __ldg(a.c.gy + m);
    const int r0 = ln * K;
    auto ld = [&](const double2* f, int r) { return r < nz ? f[(long long)r * ncol + c] : make_double2(0, 0); };
    double2 Au[K], Av[K], Aw[K], Ap[K];
#pragma unroll
    for (int i = 0; i < K; ++i) {
        Au[i] = ld(a.au, r0 + i); Av[i] = ld(a.av, r0 + i);
        Aw[i] = (r0 + i <= nz - 2) ? ld(a.aw, r0 + i) : make_double2(0, 0);   // w'(nz-1) = 0 for any input
        Ap[i] = ld(a.apsi, r0 + i);
    }
    // neighbours across the lane boundary
    const double2 Ap_prev = shfl_up2(Ap[K - 1], 1), Ap_next = shfl_dn2(Ap[0], 1);
    const double2 Aw_prev = shfl_up2(Aw[K - 1], 1);
    auto rdzt = [&](int r) { return __ldg(a.c.rdzt + r); };
    auto rdzb = [&](int r) { return __ldg(a.c.rdzb + r); };
    auto rdz = [&](int r) { return __ldg(a.c.rdz + r); };
    // ---- lambda_phi = (psi^T + projection^T) of the output adjoints
    double2 lp[1][K];
#pragma unroll
    for (int i = 0; i < K; ++i) {
        const int r = r0 + i;
        if (r >= nz) { lp[0][i] = make_double2(0, 0); continue; }
        const double2 pc = Ap[i];
        const double2 pm = i > 0 ? Ap[i - 1] : Ap_prev;      // Ap(r-1)
        const double2 pn = i < K - 1 ? Ap[i + 1] : Ap_next;  // Ap(r+1)
        // Lz^T Ap (r): diagonal of row r, plus row r-1's super and row r+1's sub entries
        const double diag = -((r < nz - 1 ? rdzt(r) : 0.0) + (r > 0 ? rdzb(r) : 0.0)) * rdz(r);
        double2 lz = make_double2(diag * pc.x, diag * pc.y);
        if (r >= 1) { const double e = rdzt(r - 1) * rdz(r - 1); lz.x += e * pm.x; lz.y += e * pm.y; }
        if (r + 1 <= nz - 1) { const double e = rdzb(r + 1) * rdz(r + 1); lz.x += e * pn.x; lz.y += e * pn.y; }
        double2 v = make_double2(pc.x * (1.0 - cps * lxy) - cps * lz.x, pc.y * (1.0 - cps * lxy) - cps * lz.y);
        // projection: -cpr (conj GX Au + conj GY Av + Gz^T Aw)
        const double2 gx = zmul(zconj(GX), Au[i]), gy = zmul(zconj(GY), Av[i]);
        v.x -= cpr * (gx.x + gy.x); v.y -= cpr * (gx.y + gy.y);
        // Gz phi (k) = (phi(k+1) - phi(k)) rdzt(k), k <= nz-2: Gz^T Aw (r) = -rdzt(r) Aw(r) + rdzt(r-1) Aw(r-1)
        double2 gz = make_double2(0, 0);
        if (r <= nz - 2) { gz.x -= rdzt(r) * Aw[i].x; gz.y -= rdzt(r) * Aw[i].y; }
        if (r >= 1) { const double2 wm = i > 0 ? Aw[i - 1] : Aw_prev; gz.x += rdzt(r - 1) * wm.x; gz.y += rdzt(r - 1) * wm.y; }
        v.x -= cpr * gz.x; v.y -= cpr * gz.y;
        lp[0][i] = v;
    }
    // ---- lambda_s = P^-T lambda_phi (transposed rows: sub = cc(r-1), super = aa(r+1))
    {
        auto aaP = [&](int r) { return rk * __ldg(a.c.ap + r); };
        auto ccP = [&](int r) { return (is00 && r == 0) ? 0.0 : rk * __ldg(a.c.cp + r); };
        auto cf = [&](int r, double& aa, double& bb, double& cc) {
            if (r < nz) {
                aa = r >= 1 ? ccP(r - 1) : 0.0;
                cc = r + 1 <= nz - 1 ? aaP(r + 1) : 0.0;
                bb = rk * (lamp + __ldg(dgp + r));
            } else { aa = 0.0; bb = 1.0; cc = 0.0; }
        };
        warp_partition_solve<K, 1>(cf, lp, ln);
    }
    if (is00 && ln == 0) lp[0][0] = make_double2(0, 0);       // s(0) was overwritten by the pin
    // ---- lambda_u*, lambda_v*, lambda_w* (divergence^T added to the projection's)
    double2 d[2][K], dw[1][K];
    const double2 ls_next = shfl_dn2(lp[0][0], 1);
#pragma unroll
    for (int i = 0; i < K; ++i) {
        const int r = r0 + i;
        const double2 ls = lp[0][i];
        const double2 ux = zmul(zconj(DX), ls), vy = zmul(zconj(DY), ls);
        d[0][i] = r < nz ? make_double2(Au[i].x + ux.x * rdt, Au[i].y + ux.y * rdt) : make_double2(0, 0);
        d[1][i] = r < nz ? make_double2(Av[i].x + vy.x * rdt, Av[i].y + vy.y * rdt) : make_double2(0, 0);
        // s(r) uses +w*(r) rdz(r) and s(r+1) uses -w*(r) rdz(r+1)
        double2 v = Aw[i];
        if (r < nz) { v.x += rdz(r) * rdt * ls.x; v.y += rdz(r) * rdt * ls.y; }
        if (r + 1 < nz) {
            const double2 lsn = i < K - 1 ? lp[0][i + 1] : ls_next;
            v.x -= rdz(r + 1) * rdt * lsn.x; v.y -= rdz(r + 1) * rdt * lsn.y;
        }
        dw[0][i] = r <= nz - 2 ? v : make_double2(0, 0);      // w*(nz-1) = 0 for any qw
    }
    // ---- lambda_q = H^-T lambda_*
    {
        auto aaU = [&](int r) { return rk * __ldg(a.c.au + r); };
        auto ccU = [&](int r) { return rk * __ldg(a.c.cu + r); };
        auto cf = [&](int r, double& aa, double& bb, double& cc) {
            if (r < nz) {
                aa = r >= 1 ? ccU(r - 1) : 0.0;
                cc = r + 1 <= nz - 1 ? aaU(r + 1) : 0.0;
                bb = 1.0 + rk * (-lam + __ldg(dgu + r));
            } else { aa = 0.0; bb = 1.0; cc = 0.0; }
        };
        warp_partition_solve<K, 2>(cf, d, ln);
    }
    {
        auto aaW = [&](int r) { return rk * __ldg(a.c.aw + r); };
        auto ccW = [&](int r) { return rk * __ldg(a.c.cw + r); };
        auto cf = [&](int r, double& aa, double& bb, double& cc) {
            if (r < nz - 1) {
                aa = r >= 1 ? ccW(r - 1) : 0.0;
                cc = r + 1 <= nz - 2 ? aaW(r + 1) : 0.0;
                bb = 1.0 + rk * (-lam + __ldg(dgw + r));
            } else { aa = 0.0; bb = 1.0; cc = 0.0; }
        };
        warp_partition_solve<K, 1>(cf, dw, ln);
    }
#pragma unroll
    for (int i = 0; i < K; ++i) {
        const int r = r0 + i;
        if (r >= nz) continue;
        const long long id = (long long)r * ncol + c;
        a.au[id] = d[0][i];
        a.av[id] = d[1][i];
        a.aw[id] = r <= nz - 2 ? dw[0][i] : make_double2(0, 0);
    }
}

// ---------------------------------------------------------------------------
// Temperature (isscalar = 1). The forward sub-step ends with
//   ss  = -Dx(thx u') - Dy(thy v') - Dz(thz w') - um Dx(thx)     (get_temperature_cnvdiff,
//   qt  = T + dt (rk_a ss + rk_b ss_prev) + c_t L T               src/module_cnvdiff.f90:381-473)
//   T'  = M_T qt,   M_T = iFFT . H_T^-1 . FFT                     (the Dirichlet T Helmholtz solve)
// where u', v', w' are the velocities this sub-step produced and T the
// temperature it started from; the momentum right-hand side of the same
// sub-step read T through the buoyancy term got ((1 - l_t) T(k) + l_t T(k+1)) of
// the w equation. Its adjoint runs first in the reverse sweep:
//   lambda_qt = M_T^T lambda_T',  lambda_ss = dt rk_a lambda_qt + lambda_ss(out),
//   lambda_ss_prev = dt rk_b lambda_qt,
//   lambda_T  = lambda_qt + c_t L^T lambda_qt + (dss/dT)^T lambda_ss,
//   lambda_u' += (dss/du')^T lambda_ss (and v', w'),
// again as two gather passes (interpolant adjoints, then raw values).
// ---------------------------------------------------------------------------
struct AdjTArgs {
    Acc<double> a;                 // T at the sub-step's start; f.u, f.v, f.w = u', v', w'
    const double* lqt;             // lambda_qt (physical)
    const double* lss_out;         // adjoint of the new history ss
    double* lss_prev;              // out: adjoint of the old history
    double* ax[3];                 // adjoints of thx, thy, thz at each point
    double* lvel[3];               // lambda_u', v', w': accumulated
    double* out_t;                 // lambda_T: written
    double rk_a, rk_b, rk_c;
    Phys ph;
};

// Pass 1: the adjoints of thx, thy, thz at this point, its velocity adjoints
// (the fluxes thx u' etc. are products at this point), and the history adjoint.
template <int CDS>
__global__ void __launch_bounds__(256) k_t_adj_interp(AdjTArgs m)
{
    const Geo& g = m.a.g;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= g.nx || j >= g.ny) return;
    const int nz = g.nz;
    const Nbr N(g, i, j, k);
    const long long id = N.at(0, 0), up = g.nxy;
    const double dta = m.ph.dt * m.rk_a;
    auto L = [&](long long q) { return dta * __ldg(m.lqt + q) + __ldg(m.lss_out + q); };
    m.lss_prev[id] = m.ph.dt * m.rk_b * m.lqt[id];
    // the T fluxes sit one point lower than the momentum ones the Dif offsets
    // describe: tux(i) = (-F(i+1) + 27 F(i) - 27 F(i-1) + F(i-2)) / 24 dx, so the
    // difference at i + 1 - off reads the flux of face i
    double sx = 0.0, sy = 0.0;
#pragma unroll
    for (int q = 0; q < Dif<CDS>::n; ++q) {
        const int o = 1 - Dif<CDS>::off(q);
        sx += Dif<CDS>::c(q) / g.dx * L(N.at(o, 0));
        sy += Dif<CDS>::c(q) / g.dy * L(N.at(0, o));
    }
    const Acc<double>& A = m.a;
    const double thx = A.template thx<CDS>(i, j, k), thy = A.template thy<CDS>(i, j, k);
    const double u1 = __ldg(A.f.u + id), v1 = __ldg(A.f.v + id);
    m.ax[0][id] = -(u1 + A.um) * sx;
    m.ax[1][id] = -v1 * sy;
    m.lvel[0][id] += -thx * sx;
    m.lvel[1][id] += -thy * sy;
    // z: Dz(FZ)(k) = (FZ(k) - FZ(k-1)) / dz(k); FZ(k) = thz(k) w'(k), w'(nz-1) = 0
    if (k <= nz - 2) {
        const double lfz = -L(id) / ldz(g.z.dz, k) + L(id + up) / ldz(g.z.dz, k + 1);
        const double l = ldz(g.z.l_t, k);
        const double thz = __ldg(A.f.t + id + up) * l + __ldg(A.f.t + id) * (1.0 - l);
        m.ax[2][id] = __ldg(A.f.w + id) * lfz;
        m.lvel[2][id] += thz * lfz;
    } else {
        m.ax[2][id] = 0.0;
    }
}

// Pass 2: lambda_T by the transposed interpolation weights, the identity, the
// transposed diffusion (the ghosts fold back with weight tbs at the bottom: -1
// for 2 tbot - T(0), +1 for a fixed gradient; -1 for 2 ttop - T(nz-1) at the top)
// and thz's z weights.
template <int CDS>
__global__ void __launch_bounds__(256) k_t_adj_gather(AdjTArgs m)
{
    const Geo& g = m.a.g;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= g.nx || j >= g.ny) return;
    const int nz = g.nz;
    const Nbr N(g, i, j, k);
    const long long id = N.at(0, 0), up = g.nxy;
    auto X = [&](int f, int di, int dj) { return __ldg(m.ax[f] + N.at(di, dj)); };
    auto Q = [&](int di, int dj) { return __ldg(m.lqt + N.at(di, dj)); };
    auto dz = [&](int kk) { return ldz(g.z.dz, kk); };
    auto dzt = [&](int kk) { return ldz(g.z.dz_t, kk); };
    auto dzb = [&](int kk) { return ldz(g.z.dz_b, kk); };
    const double ct = m.rk_c * 0.5 * m.ph.dt * m.ph.alpha;
    double lt;
    // thx(i) = (-T(i+2) + 9 T(i+1) + 9 T(i) - T(i-1)) / 16, thy alike
    if (CDS == 1) {
        lt = 0.5 * (X(0, -1, 0) + X(0, 0, 0)) + 0.5 * (X(1, 0, -1) + X(1, 0, 0));
    } else {
        lt = (-X(0, -2, 0) + 9.0 * X(0, -1, 0) + 9.0 * X(0, 0, 0) - X(0, 1, 0)) * 0.0625 +
             (-X(1, 0, -2) + 9.0 * X(1, 0, -1) + 9.0 * X(1, 0, 0) - X(1, 0, 1)) * 0.0625;
    }
    // thz(k) = l_t(k) T(k+1) + (1 - l_t(k)) T(k) on the faces k <= nz-2
    if (k <= nz - 2) lt += (1.0 - ldz(g.z.l_t, k)) * __ldg(m.ax[2] + id);
    if (k >= 1) lt += ldz(g.z.l_t, k - 1) * __ldg(m.ax[2] + id - up);
    // identity and horizontal diffusion (symmetric stencils)
    const double q0 = Q(0, 0);
    double h;
    if (CDS == 1) {
        h = (Q(1, 0) - 2.0 * q0 + Q(-1, 0)) / g.dx2 + (Q(0, 1) - 2.0 * q0 + Q(0, -1)) / g.dy2;
    } else {
        h = (-Q(2, 0) + 16.0 * Q(1, 0) - 30.0 * q0 + 16.0 * Q(-1, 0) - Q(-2, 0)) / (12.0 * g.dx2) +
            (-Q(0, 2) + 16.0 * Q(0, 1) - 30.0 * q0 + 16.0 * Q(0, -1) - Q(0, -2)) / (12.0 * g.dy2);
    }
    lt += q0 + ct * h;
    // tzz(k) = ((T(k+1) - T(k)) / dz_t(k) - (T(k) - T(k-1)) / dz_b(k)) / dz(k), transposed
    auto qz = [&](int kk) -> double { return (kk < 0 || kk >= nz) ? 0.0 : __ldg(m.lqt + id + (long long)(kk - k) * up); };
    double zt = -q0 * (1.0 / dzt(k) + 1.0 / dzb(k)) / dz(k);
    if (k >= 1) zt += qz(k - 1) / (dzt(k - 1) * dz(k - 1));
    if (k <= nz - 2) zt += qz(k + 1) / (dzb(k + 1) * dz(k + 1));
    if (k == 0) zt += m.a.tbs * q0 / (dzb(0) * dz(0));        // T(-1) = tbs T(0) + tba
    if (k == nz - 1) zt -= q0 / (dzt(k) * dz(k));             // T(nz) = 2 ttop - T(nz-1)
    lt += ct * zt;
    m.out_t[id] = lt;
}

// H_T^-T per wavenumber column (the T Helmholtz matrix is real, so its adjoint is
// its transpose): in place on the spectra of lambda_T', giving those of lambda_qt.
struct ColTAdjArgs {
    double2* at;
    ColCoef c;
    Geo g;
    double rk_c;
};

template <int K>
__global__ void __launch_bounds__(CW_WARPS * 32) k_column_t_adj(ColTAdjArgs a)
{
    const int ln = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const long long ncol = a.g.ncol;
    const long long c = (long long)blockIdx.x * CW_WARPS + wp;
    if (c >= ncol) return;
    const int nz = a.g.nz;
    const int l = (int)(c % a.g.nxh), m = (int)(c / a.g.nxh);
    const double rk = a.rk_c;
    const double lam = __ldg(a.c.hxt + l) + __ldg(a.c.hyt + m);
    const double* dg = c == 0 ? a.c.d0t : a.c.dgt;
    const int r0 = ln * K;
    double2 d[1][K];
#pragma unroll
    for (int i = 0; i < K; ++i) d[0][i] = r0 + i < nz ? a.at[(long long)(r0 + i) * ncol + c] : make_double2(0, 0);
    auto cf = [&](int r, double& aa, double& bb, double& cc) {
        if (r < nz) {
            aa = r >= 1 ? rk * __ldg(a.c.ct + r - 1) : 0.0;
            cc = r + 1 <= nz - 1 ? rk * __ldg(a.c.at + r + 1) : 0.0;
            bb = 1.0 + rk * (-lam + __ldg(dg + r));
        } else { aa = 0.0; bb = 1.0; cc = 0.0; }
    };
    warp_partition_solve<K, 1>(cf, d, ln);
#pragma unroll
    for (int i = 0; i < K; ++i)
        if (r0 + i < nz) a.at[(long long)(r0 + i) * ncol + c] = d[0][i];
}
