// hc_adjoint.cuh -- discrete adjoint of the FD sub-step (no counterpart in the
// reference). Scope: FP64, cds = 1 or 2, constant forcing (dp_opt = 1 or 3),
// no temperature, no damping; RK3 or AB2; body force.
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
// The nonlinear RHS is differentiated point by point in reverse mode: every
// interpolant and difference of the forward expression passes its adjoint back
// to the raw values it read, through the same periodic wrap and z ghost
// relations (the ghost of a wall value folds back onto that value), accumulated
// with FP64 atomics.
#pragma once
#include "hc_fd.cuh"
#include "hc_column_warp.cuh"

struct AdjFields {
    double* u; double* v; double* w; double* p;       // adjoint accumulators (scatter targets)
};

struct AdjRhsArgs {
    Acc<double> a;                 // the forward state at the sub-step's start
    const double* lq[3];           // lambda_q (physical)
    const double* lf_out[3];       // adjoint of the new histories ff, gg, hh
    double* lf_prev[3];            // out: adjoint of the old histories
    double* lbf[3];                // body-force gradient, accumulated
    AdjFields out;                 // lambda_u, v, w, p accumulated
    double rk_a, rk_b, rk_c;
    Phys ph;
};

// ---- scatter helpers: adjoint of a raw read (wrap + ghost relation) ----------
struct AdjScatter {
    const Geo& g;
    int closed;
    AdjFields t;
    __device__ __forceinline__ long long at(int i, int j, int k) const
    {
        return ((long long)k * g.ny + wrapi(j, g.ny)) * g.nx + wrapi(i, g.nx);
    }
    // U(k<0) = -U(0) - 2 u_mrf; U(k>=nz) = closed ? -U(nz-1) - 2 u_mrf : U(nz-1)
    __device__ __forceinline__ void U(int i, int j, int k, double lam) const
    {
        if (lam == 0.0) return;
        if (k < 0) { atomicAdd(t.u + at(i, j, 0), -lam); return; }
        if (k >= g.nz) { atomicAdd(t.u + at(i, j, g.nz - 1), closed ? -lam : lam); return; }
        atomicAdd(t.u + at(i, j, k), lam);
    }
    __device__ __forceinline__ void V(int i, int j, int k, double lam) const
    {
        if (lam == 0.0) return;
        if (k < 0) { atomicAdd(t.v + at(i, j, 0), -lam); return; }
        if (k >= g.nz) { atomicAdd(t.v + at(i, j, g.nz - 1), closed ? -lam : lam); return; }
        atomicAdd(t.v + at(i, j, k), lam);
    }
    // W(k<0) = 0; W(k>=nz) = -W(nz-2)
    __device__ __forceinline__ void W(int i, int j, int k, double lam) const
    {
        if (lam == 0.0 || k < 0) return;
        if (k >= g.nz) { atomicAdd(t.w + at(i, j, g.nz - 2), -lam); return; }
        atomicAdd(t.w + at(i, j, k), lam);
    }
    __device__ __forceinline__ void P(int i, int j, int k, double lam) const
    {
        if (lam == 0.0) return;
        k = k < 0 ? 0 : (k >= g.nz ? g.nz - 1 : k);
        atomicAdd(t.p + at(i, j, k), lam);
    }
    // interpolants (get_interp_fields_uvwhxyz with the ghosts of update_boundary_uvwhxyz)
    template <int CDS> __device__ __forceinline__ void uhx(int i, int j, int k, double lam) const
    {
        if (CDS == 1) { U(i, j, k, 0.5 * lam); U(i - 1, j, k, 0.5 * lam); return; }
        U(i + 1, j, k, -lam / 16); U(i, j, k, 9 * lam / 16); U(i - 1, j, k, 9 * lam / 16); U(i - 2, j, k, -lam / 16);
    }
    template <int CDS> __device__ __forceinline__ void uhy(int i, int j, int k, double lam) const
    {
        if (CDS == 1) { U(i, j + 1, k, 0.5 * lam); U(i, j, k, 0.5 * lam); return; }
        U(i, j + 2, k, -lam / 16); U(i, j + 1, k, 9 * lam / 16); U(i, j, k, 9 * lam / 16); U(i, j - 1, k, -lam / 16);
    }
    template <int CDS> __device__ __forceinline__ void vhx(int i, int j, int k, double lam) const
    {
        if (CDS == 1) { V(i + 1, j, k, 0.5 * lam); V(i, j, k, 0.5 * lam); return; }
        V(i + 2, j, k, -lam / 16); V(i + 1, j, k, 9 * lam / 16); V(i, j, k, 9 * lam / 16); V(i - 1, j, k, -lam / 16);
    }
    template <int CDS> __device__ __forceinline__ void vhy(int i, int j, int k, double lam) const
    {
        if (CDS == 1) { V(i, j, k, 0.5 * lam); V(i, j - 1, k, 0.5 * lam); return; }
        V(i, j + 1, k, -lam / 16); V(i, j, k, 9 * lam / 16); V(i, j - 1, k, 9 * lam / 16); V(i, j - 2, k, -lam / 16);
    }
    template <int CDS> __device__ __forceinline__ void whx(int i, int j, int k, double lam) const
    {
        if (k < 0 || k >= g.nz - 1) return;
        if (CDS == 1) { W(i + 1, j, k, 0.5 * lam); W(i, j, k, 0.5 * lam); return; }
        W(i + 2, j, k, -lam / 16); W(i + 1, j, k, 9 * lam / 16); W(i, j, k, 9 * lam / 16); W(i - 1, j, k, -lam / 16);
    }
    template <int CDS> __device__ __forceinline__ void why(int i, int j, int k, double lam) const
    {
        if (k < 0 || k >= g.nz - 1) return;
        if (CDS == 1) { W(i, j + 1, k, 0.5 * lam); W(i, j, k, 0.5 * lam); return; }
        W(i, j + 2, k, -lam / 16); W(i, j + 1, k, 9 * lam / 16); W(i, j, k, 9 * lam / 16); W(i, j - 1, k, -lam / 16);
    }
    __device__ __forceinline__ void uhz(int i, int j, int k, double lam) const
    {
        if (k < 0) return;
        if (k >= g.nz - 1) { if (!closed) U(i, j, g.nz - 1, lam); return; }
        const double l = ldz(g.z.l_t, k);
        U(i, j, k + 1, lam * l); U(i, j, k, lam * (1.0 - l));
    }
    __device__ __forceinline__ void vhz(int i, int j, int k, double lam) const
    {
        if (k < 0) return;
        if (k >= g.nz - 1) { if (!closed) V(i, j, g.nz - 1, lam); return; }
        const double l = ldz(g.z.l_t, k);
        V(i, j, k + 1, lam * l); V(i, j, k, lam * (1.0 - l));
    }
};

// staggered first difference D(f)(i) over the points i+2, i+1, i, i-1 (cds=2) or
// i+1, i (cds=1) of the *flux position* index: coefficients and offsets
template <int CDS> struct Dif {
    static constexpr int n = CDS == 1 ? 2 : 4;
    __device__ static double c(int q) { return CDS == 1 ? (q == 0 ? 1.0 : -1.0) : (q == 0 ? -1.0 : q == 1 ? 27.0 : q == 2 ? -27.0 : 1.0); }
    __device__ static double den() { return CDS == 1 ? 1.0 : 24.0; }
};

// Reverse mode of k_rhs_momentum at one point (i, j, k).
template <int CDS>
__global__ void __launch_bounds__(256) k_rhs_momentum_adj(AdjRhsArgs m)
{
    const Acc<double>& A = m.a;
    const Geo& g = A.g;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= g.nx || j >= g.ny) return;
    const long long id = ((long long)k * g.ny + j) * g.nx + i;
    const AdjScatter S{g, A.closed, m.out};
    const double dx = g.dx, dy = g.dy, dx2 = g.dx2, dy2 = g.dy2;
    const double dt = m.ph.dt, nu = m.ph.nu, um = A.um, fc = m.ph.fc;
    const double dz = ldz(g.z.dz, k), dzt = ldz(g.z.dz_t, k), dzb = ldz(g.z.dz_b, k);
    const double cdif = m.rk_c * 0.5 * dt * nu;
    const double crp = m.rk_c * dt;
    // offsets of the difference D(.) of the x/y fluxes: flux points i+2, i+1, i, i-1 (cds=2)
    const int o2[4] = {2, 1, 0, -1}, o1[2] = {1, 0};
    // ---------------- U ----------------
    {
        const double Lq = m.lq[0][id];
        const double Lf = dt * m.rk_a * Lq + m.lf_out[0][id];
        m.lf_prev[0][id] = dt * m.rk_b * Lq;
        m.lbf[0][id] += Lf;
        // uux = D_x(uhx^2) over uhx at i+2, i+1, i, i-1 (cds=1: i+1, i); f -= uux + um D_x(uhx)
        for (int q = 0; q < Dif<CDS>::n; ++q) {
            const int ii = i + (CDS == 1 ? o1[q] : o2[q]);
            const double h = A.template uhx<CDS>(ii, j, k);
            const double cq = Dif<CDS>::c(q) / (Dif<CDS>::den() * dx);
            S.template uhx<CDS>(ii, j, k, -Lf * cq * (2.0 * h + um));
        }
        // uvy = D_y(uhy vhx) over j+1, j, j-1, j-2 (cds=1: j, j-1)
        for (int q = 0; q < Dif<CDS>::n; ++q) {
            const int jj = j + (CDS == 1 ? o1[q] - 1 : o2[q] - 1);
            const double cq = Dif<CDS>::c(q) / (Dif<CDS>::den() * dy);
            const double dB = -Lf * cq;
            S.template uhy<CDS>(i, jj, k, dB * A.template vhx<CDS>(i, jj, k));
            S.template vhx<CDS>(i, jj, k, dB * A.template uhy<CDS>(i, jj, k));
        }
        // uwz = (uhz whx(k) - uhz whx(k-1)) / dz
        {
            const double dC = -Lf / dz;
            S.uhz(i, j, k, dC * A.template whx<CDS>(i, j, k));
            S.template whx<CDS>(i, j, k, dC * A.uhz(i, j, k));
            S.uhz(i, j, k - 1, -dC * A.template whx<CDS>(i, j, k - 1));
            S.template whx<CDS>(i, j, k - 1, -dC * A.uhz(i, j, k - 1));
        }
        if (m.ph.dp_opt == 3) {      // fc (0.5 (vhx(j) + vhx(j-1)) - vg)
            S.template vhx<CDS>(i, j, k, 0.5 * fc * Lf);
            S.template vhx<CDS>(i, j - 1, k, 0.5 * fc * Lf);
        }
        // qu = u + ... + c_d (uxx + uyy + uzz) - rk_c dt dpdx
        S.U(i, j, k, Lq);
        if (CDS == 1) {
            S.U(i + 1, j, k, cdif * Lq / dx2); S.U(i, j, k, -2.0 * cdif * Lq / dx2); S.U(i - 1, j, k, cdif * Lq / dx2);
            S.U(i, j + 1, k, cdif * Lq / dy2); S.U(i, j, k, -2.0 * cdif * Lq / dy2); S.U(i, j - 1, k, cdif * Lq / dy2);
            S.P(i + 1, j, k, -crp * Lq / dx); S.P(i, j, k, crp * Lq / dx);
        } else {
            const double e[5] = {-1.0, 16.0, -30.0, 16.0, -1.0};
            for (int q = 0; q < 5; ++q) {
                S.U(i + 2 - q, j, k, cdif * Lq * e[q] / (12.0 * dx2));
                S.U(i, j + 2 - q, k, cdif * Lq * e[q] / (12.0 * dy2));
            }
            const double c4[4] = {-1.0, 27.0, -27.0, 1.0};
            for (int q = 0; q < 4; ++q) S.P(i + 2 - q, j, k, -crp * Lq * c4[q] / (24.0 * dx));
        }
        S.U(i, j, k + 1, cdif * Lq / (dzt * dz));
        S.U(i, j, k, -cdif * Lq * (1.0 / dzt + 1.0 / dzb) / dz);
        S.U(i, j, k - 1, cdif * Lq / (dzb * dz));
    }
    // ---------------- V ----------------
    {
        const double Lq = m.lq[1][id];
        const double Lf = dt * m.rk_a * Lq + m.lf_out[1][id];
        m.lf_prev[1][id] = dt * m.rk_b * Lq;
        m.lbf[1][id] += Lf;
        // vux = D_x(vhx uhy) over i+1, i, i-1, i-2 (cds=1: i, i-1); vx = D_x(vhx) likewise
        for (int q = 0; q < Dif<CDS>::n; ++q) {
            const int ii = i + (CDS == 1 ? o1[q] - 1 : o2[q] - 1);
            const double cq = Dif<CDS>::c(q) / (Dif<CDS>::den() * dx);
            const double dB = -Lf * cq;
            S.template vhx<CDS>(ii, j, k, dB * (A.template uhy<CDS>(ii, j, k) + um));
            S.template uhy<CDS>(ii, j, k, dB * A.template vhx<CDS>(ii, j, k));
        }
        // vvy = D_y(vhy^2) over j+2, j+1, j, j-1 (cds=1: j+1, j)
        for (int q = 0; q < Dif<CDS>::n; ++q) {
            const int jj = j + (CDS == 1 ? o1[q] : o2[q]);
            const double h = A.template vhy<CDS>(i, jj, k);
            const double cq = Dif<CDS>::c(q) / (Dif<CDS>::den() * dy);
            S.template vhy<CDS>(i, jj, k, -Lf * cq * 2.0 * h);
        }
        {
            const double dC = -Lf / dz;
            S.vhz(i, j, k, dC * A.template why<CDS>(i, j, k));
            S.template why<CDS>(i, j, k, dC * A.vhz(i, j, k));
            S.vhz(i, j, k - 1, -dC * A.template why<CDS>(i, j, k - 1));
            S.template why<CDS>(i, j, k - 1, -dC * A.vhz(i, j, k - 1));
        }
        if (m.ph.dp_opt == 3) {      // fc (ug - 0.5 (uhy(i) + uhy(i-1)) - um)
            S.template uhy<CDS>(i, j, k, -0.5 * fc * Lf);
            S.template uhy<CDS>(i - 1, j, k, -0.5 * fc * Lf);
        }
        S.V(i, j, k, Lq);
        if (CDS == 1) {
            S.V(i + 1, j, k, cdif * Lq / dx2); S.V(i, j, k, -2.0 * cdif * Lq / dx2); S.V(i - 1, j, k, cdif * Lq / dx2);
            S.V(i, j + 1, k, cdif * Lq / dy2); S.V(i, j, k, -2.0 * cdif * Lq / dy2); S.V(i, j - 1, k, cdif * Lq / dy2);
            S.P(i, j + 1, k, -crp * Lq / dy); S.P(i, j, k, crp * Lq / dy);
        } else {
            const double e[5] = {-1.0, 16.0, -30.0, 16.0, -1.0};
            for (int q = 0; q < 5; ++q) {
                S.V(i + 2 - q, j, k, cdif * Lq * e[q] / (12.0 * dx2));
                S.V(i, j + 2 - q, k, cdif * Lq * e[q] / (12.0 * dy2));
            }
            const double c4[4] = {-1.0, 27.0, -27.0, 1.0};
            for (int q = 0; q < 4; ++q) S.P(i, j + 2 - q, k, -crp * Lq * c4[q] / (24.0 * dy));
        }
        S.V(i, j, k + 1, cdif * Lq / (dzt * dz));
        S.V(i, j, k, -cdif * Lq * (1.0 / dzt + 1.0 / dzb) / dz);
        S.V(i, j, k - 1, cdif * Lq / (dzb * dz));
    }
    // ---------------- W (k <= nz-2; the top-wall level passes its history through) ----------------
    if (k <= g.nz - 2) {
        const double Lq = m.lq[2][id];
        const double Lf = dt * m.rk_a * Lq + m.lf_out[2][id];
        m.lf_prev[2][id] = dt * m.rk_b * Lq;
        m.lbf[2][id] += Lf;
        // wux = D_x(whx uhz) over i+1, i, i-1, i-2 (cds=1: i, i-1); wx = D_x(whx)
        for (int q = 0; q < Dif<CDS>::n; ++q) {
            const int ii = i + (CDS == 1 ? o1[q] - 1 : o2[q] - 1);
            const double cq = Dif<CDS>::c(q) / (Dif<CDS>::den() * dx);
            const double dB = -Lf * cq;
            S.template whx<CDS>(ii, j, k, dB * (A.uhz(ii, j, k) + um));
            S.uhz(ii, j, k, dB * A.template whx<CDS>(ii, j, k));
        }
        // wvy = D_y(why vhz) over j+1, j, j-1, j-2 (cds=1: j, j-1)
        for (int q = 0; q < Dif<CDS>::n; ++q) {
            const int jj = j + (CDS == 1 ? o1[q] - 1 : o2[q] - 1);
            const double cq = Dif<CDS>::c(q) / (Dif<CDS>::den() * dy);
            const double dB = -Lf * cq;
            S.template why<CDS>(i, jj, k, dB * A.vhz(i, jj, k));
            S.vhz(i, jj, k, dB * A.template why<CDS>(i, jj, k));
        }
        // wwz = ((0.5 (w + w(k+1)))^2 - (0.5 (w + w(k-1)))^2) / dz_t
        {
            const double wc = A.W(i, j, k), wp = A.W(i, j, k + 1), wm = A.W(i, j, k - 1);
            const double d1 = -Lf / dzt * 0.5 * (wc + wp), d2 = Lf / dzt * 0.5 * (wc + wm);
            S.W(i, j, k, d1 + d2); S.W(i, j, k + 1, d1); S.W(i, j, k - 1, d2);
        }
        S.W(i, j, k, Lq);
        if (CDS == 1) {
            S.W(i + 1, j, k, cdif * Lq / dx2); S.W(i, j, k, -2.0 * cdif * Lq / dx2); S.W(i - 1, j, k, cdif * Lq / dx2);
            S.W(i, j + 1, k, cdif * Lq / dy2); S.W(i, j, k, -2.0 * cdif * Lq / dy2); S.W(i, j - 1, k, cdif * Lq / dy2);
        } else {
            const double e[5] = {-1.0, 16.0, -30.0, 16.0, -1.0};
            for (int q = 0; q < 5; ++q) {
                S.W(i + 2 - q, j, k, cdif * Lq * e[q] / (12.0 * dx2));
                S.W(i, j + 2 - q, k, cdif * Lq * e[q] / (12.0 * dy2));
            }
        }
        const double dzp = ldz(g.z.dz, k + 1);
        S.W(i, j, k + 1, cdif * Lq / (dzp * dzt));
        S.W(i, j, k, -cdif * Lq * (1.0 / dzp + 1.0 / dz) / dzt);
        S.W(i, j, k - 1, cdif * Lq / (dz * dzt));
        S.P(i, j, k + 1, -crp * Lq / dzt);
        S.P(i, j, k, crp * Lq / dzt);
    } else {
        m.lf_prev[2][id] = m.lf_out[2][id];
    }
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
