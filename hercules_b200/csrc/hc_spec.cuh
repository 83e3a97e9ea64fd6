// hc_spec.cuh -- kernels of the pseudo-spectral time step (cds = 3).
//
// The reference (time_advancement_sp, src/module_navier_stokes.f90:371-517, with
// the operators of src/module_spectral.f90) keeps u, v, w, p, t and the
// explicit-term histories ff, gg, hh, ss as 2-D spectra per level and takes
// every horizontal derivative by multiplying with i k. This engine keeps the
// same state as half spectra [k][m][l] (l < nx/2) and restructures the work:
//   * every physical-space product of get_momentum_cnvdiff_spec (:35-504) is
//     formed in one pass (k_spec_products) and the eight resulting fields go
//     through one batched forward FFT; the skew-symmetric terms (issk = 1) are
//     added into the same fields, which FFT linearity allows;
//   * the terms the reference forms in physical space from u, v, w, p and phi
//     with linear z-stencils (d2/dz2, dp/dz, dw/dz, dphi/dz) are applied to the
//     spectra directly, with the ghost values of update_boundary_uvw/p/t
//     (src/module_boundary.f90:33-196) carried over to the modes (a constant
//     ghost offset lands on the (0,0) mode only);
//   * Rayleigh damping (rayleigh_damping_spec, src/module_spectral.f90:1345-1391)
//     is applied on the fly from a per-level table (sigma, plane mean), so the
//     undamped spectra stay available for the terms the reference takes from
//     the (undamped) physical fields;
//   * the solves, the divergence source, the projection, the pressure update,
//     the 2/3-rule truncation and the divergence diagnostic are fused into one
//     warp-per-column kernel (k_column_sp_warp).
// All arithmetic of the spectral operators is FP64; spectra are stored in the
// storage precision.
#pragma once
#include "hc_column_warp.cuh"
#include "hc_fd.cuh"

// x / y wavenumber of half-spectrum column (l, m); the y Nyquist row (m = ny/2)
// is zeroed by every dev_fft_* operator and forward transform of the reference.
struct SpecWave {
    double kx, ky;    // 2 pi l / lx, 2 pi m' / ly (0 on the Nyquist row)
    double zp;        // 0 on the Nyquist row, else 1
    bool is00;
};
__device__ __forceinline__ SpecWave spec_wave(long long c, const Geo& g, double tpx, double tpy)
{
    SpecWave s;
    const int l = (int)(c % g.nxh), m = (int)(c / g.nxh);
    const int ms = m < g.ny / 2 ? m : m - g.ny;
    const bool nyq = (m == g.ny / 2);
    s.kx = nyq ? 0.0 : tpx * l;
    s.ky = nyq ? 0.0 : tpy * ms;
    s.zp = nyq ? 0.0 : 1.0;
    s.is00 = (c == 0);
    return s;
}
__device__ __forceinline__ double2 mul_i(double2 a, double k) { return make_double2(-k * a.y, k * a.x); }   // i k a
__device__ __forceinline__ double2 zfma(double2 acc, double2 a, double s) { return make_double2(acc.x + s * a.x, acc.y + s * a.y); }

// damped value of a mode: c - sigma (c - mean), the mean being real
__device__ __forceinline__ double2 damp_mode(double2 c, double sig, double mall)
{
    return make_double2(c.x - sig * (c.x - mall), c.y - sig * c.y);
}

// ---------------------------------------------------------------------------
// plane means of the damped levels (rayleigh_damping_spec :1345-1391): the real
// part of the sum over the full spectrum, i.e. the l = 0 column once and every
// l > 0 mode twice (its conjugate partner is not stored), divided by nx ny.
// grid (levels, fields), 256 threads; fixed reduction order.
// ---------------------------------------------------------------------------
template <typename R> struct DampArgs {
    const typename V2<R>::T* f[5];   // S_u, S_v, S_w, S_p, S_t
    double* mean;                    // [5][nz], written for k >= kd
    Geo g;
    int kd;
    const int* halt;
};

template <typename R>
__global__ void __launch_bounds__(256) k_spec_damp_mean(DampArgs<R> a)
{
    __shared__ double sh[8];
    if (a.halt && *a.halt) return;
    const int k = a.kd + blockIdx.x, f = blockIdx.y;
    const long long ncol = a.g.ncol;
    const typename V2<R>::T* s = a.f[f] + (long long)k * ncol;
    double sm = 0.0;
    for (long long c = threadIdx.x; c < ncol; c += blockDim.x) {
        const double re = (double)s[c].x;
        sm += (c % a.g.nxh == 0) ? re : 2.0 * re;
    }
    sm = warp_sum(sm);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = sm;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
        a.mean[f * a.g.nz + k] = t / (double)a.g.nx / (double)a.g.ny;
    }
}

// per-level damping of field f: (sigma, mean); sigma = 0 below the layer
struct DampTab {
    const double* sig;     // [nz] (null: no damping)
    const double* mean;    // [5][nz]
    __device__ __forceinline__ double2 at(double2 c, int f, int k, int nz) const
    {
        if (!sig) return c;
        const double s = __ldg(sig + k);
        return s == 0.0 ? c : damp_mode(c, s, mean[f * nz + k]);
    }
};

// ---------------------------------------------------------------------------
// spectra of the horizontal derivatives of the damped u, v, w for the skew-
// symmetric terms (issk = 1): i kx D_u, i ky D_u, i kx D_v, i ky D_v, i kx D_w,
// i ky D_w (dev_fft_linear_cmplx :1274-1340, Nyquist row zeroed)
// ---------------------------------------------------------------------------
template <typename R> struct DerivArgs {
    const typename V2<R>::T* s[3];   // S_u, S_v, S_w
    typename V2<R>::T* out[6];
    DampTab dt;
    Geo g;
    double tpx, tpy;
    const int* halt;
};

template <typename R>
__global__ void __launch_bounds__(256) k_spec_deriv(DerivArgs<R> a)
{
    if (a.halt && *a.halt) return;
    const long long ncol = a.g.ncol, n = ncol * a.g.nz;
    for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < n; id += (long long)gridDim.x * blockDim.x) {
        const long long c = id % ncol;
        const int k = (int)(id / ncol);
        const SpecWave w = spec_wave(c, a.g, a.tpx, a.tpy);
#pragma unroll
        for (int f = 0; f < 3; ++f) {
            const double2 d = a.dt.at(ld2<R>(a.s[f], id), f, k, a.g.nz);
            st2<R>(a.out[2 * f], id, mul_i(d, w.kx));
            st2<R>(a.out[2 * f + 1], id, mul_i(d, w.ky));
        }
    }
}

// spectral_truncation (src/module_spectral.f90:1222-1268) of nf spectra
template <typename R> struct TruncArgs {
    typename V2<R>::T* f[5];
    int nf;
    Geo g;
    int ltr, mtr;
};

template <typename R>
__global__ void __launch_bounds__(256) k_spec_truncate(TruncArgs<R> a)
{
    const long long ncol = a.g.ncol, n = ncol * a.g.nz;
    for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < n; id += (long long)gridDim.x * blockDim.x) {
        const long long c = id % ncol;
        if (!spec_truncated((int)(c % a.g.nxh), (int)(c / a.g.nxh), a.g.ny, a.ltr, a.mtr)) continue;
        for (int f = 0; f < a.nf; ++f) st2<R>(a.f[f], id, make_double2(0, 0));
    }
}

// ---------------------------------------------------------------------------
// physical-space products of get_momentum_cnvdiff_spec (:35-504), one thread per
// (i, j), marching over a chunk of levels with the z neighbours in registers:
//   P0 = u u, P1 = u v, P2 = v v                       (dev_fft_nonlinear_cmplx)
//   P3 = u_t w, P4 = v_t w    (u_t = l_t u(k+1) + (1 - l_t) u(k), the w equation)
//   P5..P7 = the per-equation physical terms that are transformed without a
//   derivative: pressure drive / Coriolis / buoyancy divided by coe_sk, minus
//   the vertical flux divergence, minus (issk = 1) the three skew-symmetric
//   products, whose spectra the reference subtracts with the same factor coe_sk.
// Ghost values follow update_boundary_uvw / update_boundary_t.
// ---------------------------------------------------------------------------
template <typename R> struct ProdArgs {
    const R* u; const R* v; const R* w; const R* t;
    const R* d[6];          // issk: du/dx, du/dy, dv/dx, dv/dy, dw/dx, dw/dy (physical), else null
    const R* bf[3];         // body force (null: none); enters the histories with factor 1
    R* out[8];
    Geo g;
    const double* rdz; const double* rdzt;   // [nz] 1/dz, 1/dz_t
    const DevScalars* sc;
    double um, fc, ug, vg, t_ref, tbs, tba, ttop, inv_coe;   // T(-1) = tbs T(0) + tba
    int closed, dp3, scalar, skew, kchunk;
    const int* halt;
};

// Products and assemble load each level one level ahead (below). Registers:
// products at three resident blocks (at 256 x 256 x 128: FP32 storage 186 ->
// 114 us, FP64 152 -> 143 us a launch); assemble at two blocks with FP32
// storage (243 -> 98 us) and the compiler's own budget with FP64 (354 -> 161
// us; bounded to two blocks it spilled and took 211 us)
template <typename R> struct AsmMinBlocks { static constexpr int v = sizeof(R) == sizeof(float) ? 2 : 1; };

// The eight products of one point (the arithmetic both product kernels share):
// z neighbours of u, v, w (m: level below, k, p: above) and t (k, p) with their
// ghost values, the six skew derivatives at level k (skew), the body force (bf,
// null: none) and the z factors l_t, l_b, 1/dz, 1/dz_t of level k.
template <typename R>
__device__ __forceinline__ void spec_point_products(const ProdArgs<R>& a, double dpx, double got, double ic,
                                                    double um_, double uk, double up, double vm, double vk, double vp,
                                                    double wm, double wk, double wp, double tk, double tp,
                                                    const R* dd, const double* bf, double lt, double lb, double rdz,
                                                    double rdzt, double o[8])
{
    const double um = a.um;
    const double a1u = up * lt + uk * (1.0 - lt), a2u = um_ * lb + uk * (1.0 - lb);
    const double a1v = vp * lt + vk * (1.0 - lt), a2v = vm * lb + vk * (1.0 - lb);
    double cu = ic * (a.dp3 ? a.fc * (vk - a.vg) : dpx) - (a1u * wk - a2u * wm) * rdz;
    double cv = ic * (a.dp3 ? a.fc * (a.ug - uk - um) : 0.0) - (a1v * wk - a2v * wm) * rdz;
    const double hp = 0.5 * (wk + wp), hm = 0.5 * (wk + wm);
    const double tmpw = (hp * hp - hm * hm) * rdzt;
    double cw = a.scalar ? ic * (got * ((1.0 - lt) * tk + lt * tp - a.t_ref)) - tmpw : -tmpw;
    if (a.skew) {
        const double wc = 0.5 * (wk + wm);
        cu -= uk * (double)dd[0] + vk * (double)dd[1] + (a1u - a2u) * rdz * wc;
        cv -= uk * (double)dd[2] + vk * (double)dd[3] + (a1v - a2v) * rdz * wc;
        cw -= a1u * (double)dd[4] + a1v * (double)dd[5] + wk * ((hp - hm) * rdzt);
    }
    if (bf) {
        cu += ic * bf[0];
        cv += ic * bf[1];
        cw += ic * bf[2];
    }
    o[0] = uk * uk; o[1] = uk * vk; o[2] = vk * vk; o[3] = a1u * wk; o[4] = a1v * wk;
    o[5] = cu; o[6] = cv; o[7] = cw;
}

// k_spec_products stages what a level reads (u, v, w, t one level up and the six
// skew derivatives) in shared memory with per-thread cp.async copies, D levels
// ahead of use: three with FP32 storage, one with FP64. Each thread copies and
// reads only its own words, so the ring needs no block barrier; a slot is
// refilled one level after it was read. Held in registers one level ahead, the
// FP32 loads carried half the bytes of the FP64 ones and the kernel held 0.58 of
// the HBM bandwidth at 256 x 256 x 128. The z factors of the chunk sit in shared
// memory too (a chunk has at most SPEC_KCHUNK_MAX levels).
#define SPEC_KCHUNK_MAX 32
template <typename R> struct ProdAhead { static constexpr int v = sizeof(R) == sizeof(float) ? 3 : 1; };
constexpr int PROD_NT = 256, PROD_NW = 10;   // threads a block, words a level

template <int B> __device__ __forceinline__ void sp_cp(void* dst, const void* src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(src), "n"(B) : "memory");
}
__device__ __forceinline__ void sp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void sp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <typename R>
__global__ void __launch_bounds__(PROD_NT, 3) k_spec_products(ProdArgs<R> a)
{
    if (a.halt && *a.halt) return;
    const Geo& g = a.g;
    const int nz = g.nz;
    const int k0 = blockIdx.y * a.kchunk, k1 = min(nz, k0 + a.kchunk);
    constexpr int D = ProdAhead<R>::v, NS = D + 1;
    // l_t, l_b, 1/dz, 1/dz_t of the chunk's levels; the ring [slot][word][thread]
    __shared__ double zs[4][SPEC_KCHUNK_MAX];
    __shared__ R ring[NS][PROD_NW][PROD_NT];
    for (int i = threadIdx.x; i < 4 * (k1 - k0); i += blockDim.x) {
        const int f = i / (k1 - k0), k = k0 + i % (k1 - k0);
        zs[f][k - k0] = f == 0 ? ldz(g.z.l_t, k) : f == 1 ? ldz(g.z.l_b, k) : f == 2 ? a.rdz[k] : a.rdzt[k];
    }
    __syncthreads();
    const int tid = threadIdx.x;
    const long long ij = (long long)blockIdx.x * PROD_NT + tid;
    if (ij >= g.nxy) return;
    const long long nxy = g.nxy;
    const double um = a.um;
    // stored value of the level a vertical neighbour reads (clamped; w reads
    // nz-2 above the top) and the ghost rules of update_boundary_uvw / _t on it
    const int nz1 = nz - 1;
    auto iC = [&](int k) { return k < 0 ? 0 : (k > nz1 ? nz1 : k); };
    auto iW = [&](int k) { return k < 0 ? 0 : (k > nz1 ? nz - 2 : k); };
    auto raw = [&](const R* f, int kk) -> R { return f[(long long)kk * nxy + ij]; };
    auto gU = [&](R r, int k) -> double {
        return (k < 0 || (k >= nz && a.closed)) ? -(double)r - 2.0 * um : (double)r;
    };
    auto gV = [&](R r, int k) -> double { return (k < 0 || (k >= nz && a.closed)) ? -(double)r : (double)r; };
    auto gW = [&](R r, int k) -> double { return k < 0 ? 0.0 : (k >= nz ? -(double)r : (double)r); };
    auto gT = [&](R r, int k) -> double {
        if (!a.scalar) return 0.0;
        return k < 0 ? a.tbs * (double)r + a.tba : (k >= nz ? 2.0 * a.ttop - (double)r : (double)r);
    };
    // the copies of level k (u, v, w, t at level k+1; derivatives at level k) into
    // a slot, as one commit group (empty past the chunk, so that the group count
    // stays one a level)
    auto issue = [&](int k, int slot) {
        if (k < k1) {
            const int L = k + 1;
            sp_cp<sizeof(R)>(&ring[slot][0][tid], a.u + (long long)iC(L) * nxy + ij);
            sp_cp<sizeof(R)>(&ring[slot][1][tid], a.v + (long long)iC(L) * nxy + ij);
            sp_cp<sizeof(R)>(&ring[slot][2][tid], a.w + (long long)iW(L) * nxy + ij);
            if (a.scalar) sp_cp<sizeof(R)>(&ring[slot][3][tid], a.t + (long long)iC(L) * nxy + ij);
            if (a.skew) {
#pragma unroll
                for (int f = 0; f < 6; ++f) sp_cp<sizeof(R)>(&ring[slot][4 + f][tid], a.d[f] + (long long)k * nxy + ij);
            }
        }
        sp_commit();
    };
#pragma unroll
    for (int s = 0; s < D; ++s) issue(k0 + s, s);
    const double dpx = a.sc->dpx_drive, got = a.sc->got, ic = a.inv_coe;
    double um_, uk, vm, vk, wm, wk, tk;
    {
        const R u0 = raw(a.u, iC(k0 - 1)), v0 = raw(a.v, iC(k0 - 1)), w0 = raw(a.w, iW(k0 - 1));
        const R u1 = raw(a.u, iC(k0)), v1 = raw(a.v, iC(k0)), w1 = raw(a.w, iW(k0));
        const R t1 = a.scalar ? raw(a.t, iC(k0)) : R(0);
        um_ = gU(u0, k0 - 1); uk = gU(u1, k0); vm = gV(v0, k0 - 1); vk = gV(v1, k0);
        wm = gW(w0, k0 - 1); wk = gW(w1, k0); tk = gT(t1, k0);
    }
    // slot s of the unrolled inner loop holds level kb + s
    for (int kb = k0; kb < k1; kb += NS) {
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const int k = kb + s;
            if (k >= k1) break;
            sp_wait<D - 1>();      // level k's group (D - 1 newer ones may still run)
            R cur[PROD_NW];
#pragma unroll
            for (int f = 0; f < PROD_NW; ++f) cur[f] = ring[s][f][tid];
            issue(k + D, (s + D) % NS);   // refills the slot of level k - 1
            const double up = gU(cur[0], k + 1), vp = gV(cur[1], k + 1), wp = gW(cur[2], k + 1), tp = gT(cur[3], k + 1);
            const long long q = (long long)k * nxy + ij;
            double bfv[3], o[8];
            if (a.bf[0]) { bfv[0] = (double)a.bf[0][q]; bfv[1] = (double)a.bf[1][q]; bfv[2] = (double)a.bf[2][q]; }
            spec_point_products<R>(a, dpx, got, ic, um_, uk, up, vm, vk, vp, wm, wk, wp, tk, tp, cur + 4,
                                   a.bf[0] ? bfv : nullptr, zs[0][k - k0], zs[1][k - k0], zs[2][k - k0], zs[3][k - k0], o);
#pragma unroll
            for (int f = 0; f < 8; ++f) a.out[f][q] = (R)o[f];
            um_ = uk; uk = up; vm = vk; vk = vp; wm = wk; wk = wp; tk = tp;
        }
    }
    sp_wait<0>();
}

// ---------------------------------------------------------------------------
// k_spec_products_fx: the products of k_spec_products and their forward x
// transform (the x half of dev_fft_nonlinear_cmplx / real_2_cmplx) in one pass.
// A block of 128 threads takes one y row j and a chunk of levels. Per level each
// thread forms the eight products at its x pairs (2e, 2e+1), rounded to the
// storage type as the separate kernel stores them; the eight rows then go
// through the shared-memory passes of k_fft_x_r2c_t (same plan, same arithmetic)
// and leave as x half spectra, row k ny + j of nx/2 modes, which the y transform
// takes in place. The physical products never reach HBM: a point moves 10 words
// in and 8 out, against 10 + 8 for the products and 8 + 8 for the transform.
// What level k+1 reads is copied (cp.async, each thread its own pairs) into the
// other of two shared slots while level k is formed and transformed; a slot is
// refilled one level after it was read, two block barriers later.
// ---------------------------------------------------------------------------
template <typename R> struct ProdFxArgs {
    ProdArgs<R> p;                     // p.out[f]: the x half spectra (complex rows)
    const typename V2<R>::T* tw;       // exp(-2 pi i e / (nx/2)), e < nx/2
    const typename V2<R>::T* wp;       // exp(-2 pi i l / nx), l < nx/2
    R scale;                           // 1/nx
};
template <typename R, int N, int RMAX> struct SpxCfg {
    static constexpr int NT = 128, L = 8, EPT = (N + NT - 1) / NT;
    static constexpr int G = FPad<R>::G, LS = FLine<N, G>::stride;
    // the passes' two buffers (the product rows share the second when there are
    // two passes or more: the first pass has read them before it is written;
    // the last pass of an even count lands there too, and the next level's
    // products wait for a barrier after the unpacking), two slots of 10 rows of pairs
    static constexpr int np = FPlan<N, RMAX>::npass;
    static constexpr size_t smem = ((size_t)(np >= 2 ? 2 : 3) * L * LS + (size_t)2 * PROD_NW * N) *
                                   sizeof(typename V2<R>::T);
    // FP32 up to nx/2 = 128: four blocks an SM (128 registers a thread; bounded
    // to five, with the column values carried in the storage type, it took 11 %
    // more instructions and 184 against 165 us at 256 x 256 x 128)
    static constexpr int minb = sizeof(R) == sizeof(float) && N <= 128 ? 4 : 1;
};

template <typename R, int N, int RMAX>
__global__ void __launch_bounds__(128, (SpxCfg<R, N, RMAX>::minb)) k_spec_products_fx(ProdFxArgs<R> A)
{
    typedef typename V2<R>::T T2;
    typedef SpxCfg<R, N, RMAX> CF;
    constexpr int NT = CF::NT, L = CF::L, EPT = CF::EPT, G = CF::G, LS = CF::LS;
    const ProdArgs<R>& a = A.p;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (a.halt && *a.halt) return;
    const Geo& g = a.g;
    const int nz = g.nz, j = blockIdx.x;
    const int k0 = blockIdx.y * a.kchunk, k1 = min(nz, k0 + a.kchunk);
    // C: the product rows; A, B: the passes' buffers (the last pass lands in Z);
    // slot [2][word][pair]: u, v, w, t of level k+1 and the derivatives of level k
    constexpr int np = FPlan<N, RMAX>::npass;
    static_assert(np == CF::np, "plan of the shared-memory layout");
    T2* Ab = reinterpret_cast<T2*>(smem_raw);
    T2* Bb = Ab + L * LS;
    T2* Cb = np >= 2 ? Bb : Bb + L * LS;
    T2* slot = Bb + (np >= 2 ? 1 : 2) * L * LS;
    T2* Z = (np % 2 == 1) ? Ab : Bb;
    __shared__ double zs[4][SPEC_KCHUNK_MAX];
    for (int i = threadIdx.x; i < 4 * (k1 - k0); i += blockDim.x) {
        const int f = i / (k1 - k0), k = k0 + i % (k1 - k0);
        zs[f][k - k0] = f == 0 ? ldz(g.z.l_t, k) : f == 1 ? ldz(g.z.l_b, k) : f == 2 ? a.rdz[k] : a.rdzt[k];
    }
    const int tid = threadIdx.x;
    const long long nxy = g.nxy, row = (long long)j * g.nx;
    const double um = a.um;
    const int nz1 = nz - 1;
    auto iC = [&](int k) { return k < 0 ? 0 : (k > nz1 ? nz1 : k); };
    auto iW = [&](int k) { return k < 0 ? 0 : (k > nz1 ? nz - 2 : k); };
    auto gU = [&](R r, int k) -> double {
        return (k < 0 || (k >= nz && a.closed)) ? -(double)r - 2.0 * um : (double)r;
    };
    auto gV = [&](R r, int k) -> double { return (k < 0 || (k >= nz && a.closed)) ? -(double)r : (double)r; };
    auto gW = [&](R r, int k) -> double { return k < 0 ? 0.0 : (k >= nz ? -(double)r : (double)r); };
    auto gT = [&](R r, int k) -> double {
        if (!a.scalar) return 0.0;
        return k < 0 ? a.tbs * (double)r + a.tba : (k >= nz ? 2.0 * a.ttop - (double)r : (double)r);
    };
    // the pair (2e, 2e+1) of a field at a stored level
    auto gp = [&](const R* f, int kk, int e) { return f + (long long)kk * nxy + row + 2 * e; };
    auto ld2 = [&](const R* f, int kk, int e) -> T2 { return *reinterpret_cast<const T2*>(gp(f, kk, e)); };
    // copies of what level k reads into slot sl, one commit group
    auto issue = [&](int k, int sl) {
        T2* S = slot + sl * PROD_NW * N;
        const int Lk = k + 1;
#pragma unroll
        for (int i = 0; i < EPT; ++i) {
            const int e = tid + i * NT;
            if (e >= N) continue;
            sp_cp<sizeof(T2)>(S + 0 * N + e, gp(a.u, iC(Lk), e));
            sp_cp<sizeof(T2)>(S + 1 * N + e, gp(a.v, iC(Lk), e));
            sp_cp<sizeof(T2)>(S + 2 * N + e, gp(a.w, iW(Lk), e));
            if (a.scalar) sp_cp<sizeof(T2)>(S + 3 * N + e, gp(a.t, iC(Lk), e));
            if (a.skew) {
#pragma unroll
                for (int f = 0; f < 6; ++f) sp_cp<sizeof(T2)>(S + (4 + f) * N + e, gp(a.d[f], k, e));
            }
        }
        sp_commit();
    };
    issue(k0, 0);
    __syncthreads();                 // zs
    auto cx = [](T2 v, int c) -> R { return c == 0 ? v.x : v.y; };
    const double dpx = a.sc->dpx_drive, got = a.sc->got, ic = a.inv_coe;
    // the columns' carried values: [element][x of the pair]
    double um_[EPT][2], uk[EPT][2], vm[EPT][2], vk[EPT][2], wm[EPT][2], wk[EPT][2], tk[EPT][2];
#pragma unroll
    for (int i = 0; i < EPT; ++i) {
        const int e = tid + i * NT;
        if (e >= N) continue;
        const T2 u0 = ld2(a.u, iC(k0 - 1), e), v0 = ld2(a.v, iC(k0 - 1), e), w0 = ld2(a.w, iW(k0 - 1), e);
        const T2 u1 = ld2(a.u, iC(k0), e), v1 = ld2(a.v, iC(k0), e), w1 = ld2(a.w, iW(k0), e);
        const T2 t1 = a.scalar ? ld2(a.t, iC(k0), e) : mk2<R>(R(0), R(0));
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            um_[i][c] = gU(cx(u0, c), k0 - 1); uk[i][c] = gU(cx(u1, c), k0);
            vm[i][c] = gV(cx(v0, c), k0 - 1); vk[i][c] = gV(cx(v1, c), k0);
            wm[i][c] = gW(cx(w0, c), k0 - 1); wk[i][c] = gW(cx(w1, c), k0); tk[i][c] = gT(cx(t1, c), k0);
        }
    }
    const SmemIO<T2, LS, G> cin{Cb}, zout{Z};
    const R zero = R(0);
    for (int k = k0; k < k1; ++k) {
        const int sl = (k - k0) & 1;
        sp_wait<0>();
        const T2* S = slot + sl * PROD_NW * N;
        // the thread's own pairs of level k, then level k+1's copies into the other slot
        T2 cur[EPT][PROD_NW];
#pragma unroll
        for (int i = 0; i < EPT; ++i) {
            const int e = tid + i * NT;
#pragma unroll
            for (int f = 0; f < PROD_NW; ++f) cur[i][f] = e < N ? S[f * N + e] : mk2<R>(zero, zero);
        }
        if (k + 1 < k1) issue(k + 1, sl ^ 1);
        const double lt = zs[0][k - k0], lb = zs[1][k - k0], rdz = zs[2][k - k0], rdzt = zs[3][k - k0];
#pragma unroll
        for (int i = 0; i < EPT; ++i) {
            const int e = tid + i * NT;
            if (e >= N) continue;
            R pr[8][2];
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const double up = gU(cx(cur[i][0], c), k + 1), vp = gV(cx(cur[i][1], c), k + 1);
                const double wp = gW(cx(cur[i][2], c), k + 1), tp = gT(cx(cur[i][3], c), k + 1);
                R dd[6];
#pragma unroll
                for (int f = 0; f < 6; ++f) dd[f] = cx(cur[i][4 + f], c);
                double bfv[3], o[8];
                if (a.bf[0]) {
                    const long long q = (long long)k * nxy + row + 2 * e + c;
                    bfv[0] = (double)a.bf[0][q]; bfv[1] = (double)a.bf[1][q]; bfv[2] = (double)a.bf[2][q];
                }
                spec_point_products<R>(a, dpx, got, ic, um_[i][c], uk[i][c], up, vm[i][c], vk[i][c], vp,
                                       wm[i][c], wk[i][c], wp, tk[i][c], tp, dd, a.bf[0] ? bfv : nullptr,
                                       lt, lb, rdz, rdzt, o);
#pragma unroll
                for (int f = 0; f < 8; ++f) pr[f][c] = (R)o[f];
                um_[i][c] = uk[i][c]; uk[i][c] = up; vm[i][c] = vk[i][c]; vk[i][c] = vp;
                wm[i][c] = wk[i][c]; wk[i][c] = wp; tk[i][c] = tp;
            }
#pragma unroll
            for (int f = 0; f < 8; ++f) cin.st(f, e, mk2<R>(pr[f][0], pr[f][1]));
        }
        __syncthreads();
        run_passes<R, N, -1, RMAX, L, NT, false, 0>(cin, zout, Ab, Bb, A.tw);
        __syncthreads();
        // unpack the half-length transform into the nx/2 modes, as k_fft_x_r2c_t
        // (a thread keeps its modes l and their twiddle over the eight rows)
        const long long orow = ((long long)k * g.ny + j) * N;
        const R sc = A.scale;
        for (int l = tid; l < N; l += NT) {
            const T2 w = __ldg(A.wp + l);
            const int i0 = fpi<G>(l), i1 = fpi<G>(l == 0 ? 0 : N - l);
#pragma unroll
            for (int line = 0; line < L; ++line) {
                const T2 z = Z[line * LS + i0];
                T2 zc = Z[line * LS + i1];
                zc.y = -zc.y;
                const T2 ev = mk2<R>(R(0.5) * (z.x + zc.x), R(0.5) * (z.y + zc.y));
                const T2 dv = mk2<R>(R(0.5) * (z.x - zc.x), R(0.5) * (z.y - zc.y));
                const T2 wd = cmulc(w, dv);
                reinterpret_cast<T2*>(a.out[line])[orow + l] = mk2<R>((ev.x + wd.y) * sc, (ev.y - wd.x) * sc);
            }
        }
        // with an even number of passes the last one lands in B, where the next
        // level's products go: every thread must be done unpacking first
        if constexpr (np >= 2 && np % 2 == 0) __syncthreads();
    }
    sp_wait<0>();
}

// ---------------------------------------------------------------------------
// Right-hand sides and new explicit-term histories of the momentum equations,
// mode by mode (get_momentum_cnvdiff_spec :35-504). One thread per column
// (l, m), marching over a chunk of levels with the z neighbours in registers.
// With D_x the damped and S_x the undamped spectrum, ad = rk_c dt nu / 2:
//   q_u = D_u - ad (kx^2 + ky^2) D_u + ad Lz S_u - rk_c dt i kx D_p + rk_b dt ff
//   ff' = -u_mrf i kx D_u - coe (i kx F[uu] + i ky F[uv]) + coe F[P5]
//   q_u += rk_a dt ff'
// and alike for v (gg) and w (hh, with -rk_c dt d/dz S_p and the staggered
// operator Lzw). Lz / Lzw / d/dz act on the modes with the ghost values the
// reference's boundary routines give the physical fields.
// ---------------------------------------------------------------------------
template <typename R> struct AsmArgs {
    const typename V2<R>::T* su; const typename V2<R>::T* sv; const typename V2<R>::T* sw; const typename V2<R>::T* sp;
    const typename V2<R>::T* F[8];    // spectra of P0..P7
    typename V2<R>::T* ff; typename V2<R>::T* gg; typename V2<R>::T* hh;   // in: old, out: new
    typename V2<R>::T* qu; typename V2<R>::T* qv; typename V2<R>::T* qw;
    DampTab dt;
    Geo g;
    const double* rdz; const double* rdzt; const double* rdzb;   // [nz] 1/dz, 1/dz_t, 1/dz_b
    double tpx, tpy;
    double rk_a, rk_b, rk_c, dtime, nu, um, coe;
    int closed, kchunk;
    const int* halt;
};

template <typename R>
__global__ void __launch_bounds__(256, AsmMinBlocks<R>::v) k_spec_assemble(AsmArgs<R> a)
{
    typedef typename V2<R>::T T2;
    if (a.halt && *a.halt) return;
    const Geo& g = a.g;
    const long long ncol = g.ncol;
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncol) return;
    const int nz = g.nz;
    const int k0 = blockIdx.y * a.kchunk, k1 = min(nz, k0 + a.kchunk);
    const SpecWave wv = spec_wave(c, g, a.tpx, a.tpy);
    const double o00 = wv.is00 ? -2.0 * a.um : 0.0;     // u ghost offset, (0,0) mode only
    auto ldr = [&](const T2* f, int k) -> T2 { return f[(long long)k * ncol + c]; };
    auto dbl = [](T2 v) { return make_double2((double)v.x, (double)v.y); };
    const int nz1 = nz - 1;
    // ghost rules of the vertical neighbours, applied to the stored value of the
    // level they read (raw index: clamp for u, v, p; w reads nz-2 above the top)
    auto gU = [&](T2 r, int k) -> double2 {
        const double2 s = dbl(r);
        return (k < 0 || (k >= nz && a.closed)) ? make_double2(-s.x + o00, -s.y) : s;
    };
    auto gV = [&](T2 r, int k) -> double2 {
        const double2 s = dbl(r);
        return (k < 0 || (k >= nz && a.closed)) ? make_double2(-s.x, -s.y) : s;
    };
    // w as the physical field sees it: 0 below the bottom wall and on the top wall
    auto gW = [&](T2 r, int k) -> double2 {
        if (k < 0 || k == nz1) return make_double2(0, 0);
        const double2 s = dbl(r);
        return k >= nz ? make_double2(-s.x, -s.y) : s;
    };
    auto iU = [&](int k) { return k < 0 ? 0 : (k > nz1 ? nz1 : k); };
    auto iW = [&](int k) { return k < 0 ? 0 : (k > nz1 ? nz - 2 : k); };
    const double ad = a.rk_c * 0.5 * a.dtime * a.nu, cdt = a.rk_c * a.dtime;
    const double bdt = a.rk_b * a.dtime, adt = a.rk_a * a.dtime, coe = a.coe;
    const double k2 = wv.kx * wv.kx + wv.ky * wv.ky;
    double2 um_ = gU(ldr(a.su, iU(k0 - 1)), k0 - 1), uk = gU(ldr(a.su, iU(k0)), k0);
    double2 vm = gV(ldr(a.sv, iU(k0 - 1)), k0 - 1), vk = gV(ldr(a.sv, iU(k0)), k0);
    double2 wm = gW(ldr(a.sw, iW(k0 - 1)), k0 - 1), wk = gW(ldr(a.sw, iW(k0)), k0);
    double2 pk = dbl(ldr(a.sp, iU(k0)));
    // everything a level reads from global memory (level k+1 of u, v, w, p, level
    // k of the raw w spectrum, the eight product spectra and the histories) is
    // loaded one level ahead in the storage type, so that its latency overlaps
    // the previous level's arithmetic and stores
    struct Lv { T2 up, vp, wp, pp, w0, F[8], h[3]; };
    auto fetch = [&](int k, Lv& L) {
        L.up = ldr(a.su, iU(k + 1)); L.vp = ldr(a.sv, iU(k + 1));
        L.wp = ldr(a.sw, iW(k + 1)); L.pp = ldr(a.sp, iU(k + 1));
        L.w0 = ldr(a.sw, k);
#pragma unroll
        for (int f = 0; f < 8; ++f) L.F[f] = ldr(a.F[f], k);
        L.h[0] = ldr(a.ff, k); L.h[1] = ldr(a.gg, k); L.h[2] = ldr(a.hh, k);
    };
    auto zfac = [&](int k, double* z) {
        z[0] = a.rdz[k]; z[1] = a.rdzt[k]; z[2] = a.rdzb[k];
        z[3] = k + 1 < nz ? a.rdz[k + 1] : 1.0 / ldz(g.z.dz, k + 1);
    };
    Lv cur;
    double zc[4];
    fetch(k0, cur);
    zfac(k0, zc);
    for (int k = k0; k < k1; ++k) {
        Lv nxt;
        double zn[4] = {0, 0, 0, 0};
        if (k + 1 < k1) { fetch(k + 1, nxt); zfac(k + 1, zn); }
        const double2 up = gU(cur.up, k + 1), vp = gV(cur.vp, k + 1), wp = gW(cur.wp, k + 1), pp = dbl(cur.pp);
        const long long id = (long long)k * ncol + c;
        const double rdz = zc[0], rdzt = zc[1], rdzb = zc[2], rdz1 = zc[3];
        const double2 Du = a.dt.at(uk, 0, k, nz);
        const double2 Dv = a.dt.at(vk, 1, k, nz);
        const double2 Dw = a.dt.at(dbl(cur.w0), 2, k, nz);
        const double2 Dp = a.dt.at(pk, 3, k, nz);
        const double2 Fuu = dbl(cur.F[0]), Fuv = dbl(cur.F[1]), Fvv = dbl(cur.F[2]), Futw = dbl(cur.F[3]);
        const double2 Fvtw = dbl(cur.F[4]), Fcu = dbl(cur.F[5]), Fcv = dbl(cur.F[6]), Fcw = dbl(cur.F[7]);
        // vertical operators (zero on the Nyquist row, as the forward FFT leaves them)
        const double zs = wv.zp;
        const double2 lzu = make_double2(zs * (((up.x - uk.x) * rdzt - (uk.x - um_.x) * rdzb) * rdz),
                                         zs * (((up.y - uk.y) * rdzt - (uk.y - um_.y) * rdzb) * rdz));
        const double2 lzv = make_double2(zs * (((vp.x - vk.x) * rdzt - (vk.x - vm.x) * rdzb) * rdz),
                                         zs * (((vp.y - vk.y) * rdzt - (vk.y - vm.y) * rdzb) * rdz));
        const double2 lzw = make_double2(zs * (((wp.x - wk.x) * rdz1 - (wk.x - wm.x) * rdz) * rdzt),
                                         zs * (((wp.y - wk.y) * rdz1 - (wk.y - wm.y) * rdz) * rdzt));
        const double2 dpz = make_double2(zs * (pp.x - pk.x) * rdzt, zs * (pp.y - pk.y) * rdzt);
        // u
        double2 q = zfma(zfma(Du, Du, -ad * k2), lzu, ad);
        q = zfma(q, mul_i(Dp, wv.kx), -cdt);
        q = zfma(q, dbl(cur.h[0]), bdt);
        double2 h = make_double2(0, 0);
        h = zfma(h, mul_i(Du, wv.kx), -a.um);
        h = zfma(h, mul_i(Fuu, wv.kx), -coe);
        h = zfma(h, mul_i(Fuv, wv.ky), -coe);
        h = zfma(h, Fcu, coe);
        st2<R>(a.ff, id, h);
        st2<R>(a.qu, id, zfma(q, h, adt));
        // v
        q = zfma(zfma(Dv, Dv, -ad * k2), lzv, ad);
        q = zfma(q, mul_i(Dp, wv.ky), -cdt);
        q = zfma(q, dbl(cur.h[1]), bdt);
        h = make_double2(0, 0);
        h = zfma(h, mul_i(Dv, wv.kx), -a.um);
        h = zfma(h, mul_i(Fuv, wv.kx), -coe);
        h = zfma(h, mul_i(Fvv, wv.ky), -coe);
        h = zfma(h, Fcv, coe);
        st2<R>(a.gg, id, h);
        st2<R>(a.qv, id, zfma(q, h, adt));
        // w
        q = zfma(zfma(Dw, Dw, -ad * k2), lzw, ad);
        q = zfma(q, dpz, -cdt);
        q = zfma(q, dbl(cur.h[2]), bdt);
        h = make_double2(0, 0);
        h = zfma(h, mul_i(Dw, wv.kx), -a.um);
        h = zfma(h, mul_i(Futw, wv.kx), -coe);
        h = zfma(h, mul_i(Fvtw, wv.ky), -coe);
        h = zfma(h, Fcw, coe);
        st2<R>(a.hh, id, h);
        st2<R>(a.qw, id, zfma(q, h, adt));
        um_ = uk; uk = up; vm = vk; vk = vp; wm = wk; wk = wp; pk = pp;
        cur = nxt;
#pragma unroll
        for (int f = 0; f < 4; ++f) zc[f] = zn[f];
    }
}

// ---------------------------------------------------------------------------
// temperature (get_temperature_cnvdiff_spec :509-595): products u t, t v and the
// vertical flux divergence d(t w)/dz with the new u, v, w and the old t
// ---------------------------------------------------------------------------
template <typename R> struct ProdTArgs {
    const R* u; const R* v; const R* w; const R* t;
    R* out[3];
    Geo g;
    double tbs, tba, ttop;   // T(-1) = tbs T(0) + tba
    int kchunk;
    const int* halt;
};

template <typename R>
__global__ void __launch_bounds__(PROD_NT) k_spec_products_t(ProdTArgs<R> a)
{
    if (a.halt && *a.halt) return;
    const Geo& g = a.g;
    const int nz = g.nz;
    const int k0 = blockIdx.y * a.kchunk, k1 = min(nz, k0 + a.kchunk);
    // t one level up and u, v, w of a level staged D levels ahead in a
    // per-thread cp.async ring, the z factors of the chunk in shared memory
    // (see k_spec_products)
    constexpr int D = ProdAhead<R>::v, NS = D + 1, NW = 4;
    __shared__ double zs[3][SPEC_KCHUNK_MAX];
    __shared__ R ring[NS][NW][PROD_NT];
    for (int i = threadIdx.x; i < 3 * (k1 - k0); i += blockDim.x) {
        const int f = i / (k1 - k0), k = k0 + i % (k1 - k0);
        zs[f][k - k0] = ldz(f == 0 ? g.z.l_t : f == 1 ? g.z.l_b : g.z.dz, k);
    }
    __syncthreads();
    const int tid = threadIdx.x;
    const long long ij = (long long)blockIdx.x * PROD_NT + tid;
    if (ij >= g.nxy) return;
    const long long nxy = g.nxy;
    // stored t of the level a neighbour reads (clamped) and the ghost rule of
    // update_boundary_t on it
    const int nz1 = nz - 1;
    auto tq = [&](int k) { return (long long)(k < 0 ? 0 : (k > nz1 ? nz1 : k)) * nxy + ij; };
    auto gT = [&](R r, int k) -> double {
        return k < 0 ? a.tbs * (double)r + a.tba : (k >= nz ? 2.0 * a.ttop - (double)r : (double)r);
    };
    auto issue = [&](int k, int slot) {
        if (k < k1) {
            const long long q = (long long)k * nxy + ij;
            sp_cp<sizeof(R)>(&ring[slot][0][tid], a.t + tq(k + 1));
            sp_cp<sizeof(R)>(&ring[slot][1][tid], a.u + q);
            sp_cp<sizeof(R)>(&ring[slot][2][tid], a.v + q);
            sp_cp<sizeof(R)>(&ring[slot][3][tid], a.w + q);
        }
        sp_commit();
    };
#pragma unroll
    for (int s = 0; s < D; ++s) issue(k0 + s, s);
    double tm = gT(a.t[tq(k0 - 1)], k0 - 1), tk = gT(a.t[tq(k0)], k0);
    double wm = k0 > 0 ? (double)a.w[(long long)(k0 - 1) * nxy + ij] : 0.0;
    for (int kb = k0; kb < k1; kb += NS) {
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const int k = kb + s;
            if (k >= k1) break;
            sp_wait<D - 1>();
            R cur[NW];
#pragma unroll
            for (int f = 0; f < NW; ++f) cur[f] = ring[s][f][tid];
            issue(k + D, (s + D) % NS);
            const double tp = gT(cur[0], k + 1);
            const long long q = (long long)k * nxy + ij;
            const double uk = (double)cur[1], vk = (double)cur[2], wk = (double)cur[3];
            const double lt = zs[0][k - k0], lb = zs[1][k - k0];
            const double a1 = tp * lt + tk * (1.0 - lt), a2 = tm * lb + tk * (1.0 - lb);
            a.out[0][q] = (R)(uk * tk);
            a.out[1][q] = (R)(tk * vk);
            a.out[2][q] = (R)((a1 * wk - a2 * wm) / zs[2][k - k0]);
            tm = tk; tk = tp; wm = wk;
        }
    }
    sp_wait<0>();
}

// k_spec_products_t_fx: the three temperature products of k_spec_products_t and
// their forward x transform in one pass, as k_spec_products_fx (three rows a
// level; t one level up and u, v, w of the level arrive by cp.async one level
// ahead; the products are rounded to the storage type before the passes).
template <typename R> struct ProdTFxArgs {
    ProdTArgs<R> p;                    // p.out[f]: the x half spectra (complex rows)
    const typename V2<R>::T* tw;       // exp(-2 pi i e / (nx/2)), e < nx/2
    const typename V2<R>::T* wp;       // exp(-2 pi i l / nx), l < nx/2
    R scale;                           // 1/nx
};
template <typename R, int N, int RMAX> struct SpxTCfg {
    static constexpr int NT = 128, L = 3, NW = 4;
    static constexpr int G = FPad<R>::G, LS = FLine<N, G>::stride;
    static constexpr int np = FPlan<N, RMAX>::npass;
    static constexpr size_t smem = ((size_t)(np >= 2 ? 2 : 3) * L * LS + (size_t)2 * NW * N) *
                                   sizeof(typename V2<R>::T);
};

template <typename R, int N, int RMAX>
__global__ void __launch_bounds__(128) k_spec_products_t_fx(ProdTFxArgs<R> A)
{
    typedef typename V2<R>::T T2;
    typedef SpxTCfg<R, N, RMAX> CF;
    constexpr int NT = CF::NT, L = CF::L, NW = CF::NW, G = CF::G, LS = CF::LS, EPT = (N + NT - 1) / NT;
    const ProdTArgs<R>& a = A.p;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (a.halt && *a.halt) return;
    const Geo& g = a.g;
    const int nz = g.nz, j = blockIdx.x;
    const int k0 = blockIdx.y * a.kchunk, k1 = min(nz, k0 + a.kchunk);
    constexpr int np = CF::np;
    T2* Ab = reinterpret_cast<T2*>(smem_raw);
    T2* Bb = Ab + L * LS;
    T2* Cb = np >= 2 ? Bb : Bb + L * LS;
    T2* slot = Bb + (np >= 2 ? 1 : 2) * L * LS;
    T2* Z = (np % 2 == 1) ? Ab : Bb;
    __shared__ double zs[3][SPEC_KCHUNK_MAX];
    for (int i = threadIdx.x; i < 3 * (k1 - k0); i += blockDim.x) {
        const int f = i / (k1 - k0), k = k0 + i % (k1 - k0);
        zs[f][k - k0] = ldz(f == 0 ? g.z.l_t : f == 1 ? g.z.l_b : g.z.dz, k);
    }
    const int tid = threadIdx.x;
    const long long nxy = g.nxy, row = (long long)j * g.nx;
    const int nz1 = nz - 1;
    auto tq = [&](int k) { return (long long)(k < 0 ? 0 : (k > nz1 ? nz1 : k)) * nxy + row; };
    auto gT = [&](R r, int k) -> double {
        return k < 0 ? a.tbs * (double)r + a.tba : (k >= nz ? 2.0 * a.ttop - (double)r : (double)r);
    };
    auto issue = [&](int k, int sl) {
        T2* S = slot + sl * NW * N;
        const long long q = (long long)k * nxy + row;
#pragma unroll
        for (int i = 0; i < EPT; ++i) {
            const int e = tid + i * NT;
            if (e >= N) continue;
            sp_cp<sizeof(T2)>(S + 0 * N + e, a.t + tq(k + 1) + 2 * e);
            sp_cp<sizeof(T2)>(S + 1 * N + e, a.u + q + 2 * e);
            sp_cp<sizeof(T2)>(S + 2 * N + e, a.v + q + 2 * e);
            sp_cp<sizeof(T2)>(S + 3 * N + e, a.w + q + 2 * e);
        }
        sp_commit();
    };
    issue(k0, 0);
    __syncthreads();                 // zs
    auto cx = [](T2 v, int c) -> R { return c == 0 ? v.x : v.y; };
    double tm[EPT][2], tk[EPT][2], wm[EPT][2];
#pragma unroll
    for (int i = 0; i < EPT; ++i) {
        const int e = tid + i * NT;
        if (e >= N) continue;
        const T2 t0 = *reinterpret_cast<const T2*>(a.t + tq(k0 - 1) + 2 * e);
        const T2 t1 = *reinterpret_cast<const T2*>(a.t + tq(k0) + 2 * e);
        const T2 w0 = k0 > 0 ? *reinterpret_cast<const T2*>(a.w + (long long)(k0 - 1) * nxy + row + 2 * e)
                             : mk2<R>(R(0), R(0));
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            tm[i][c] = gT(cx(t0, c), k0 - 1); tk[i][c] = gT(cx(t1, c), k0);
            wm[i][c] = k0 > 0 ? (double)cx(w0, c) : 0.0;
        }
    }
    const SmemIO<T2, LS, G> cin{Cb}, zout{Z};
    const R zero = R(0);
    for (int k = k0; k < k1; ++k) {
        const int sl = (k - k0) & 1;
        sp_wait<0>();
        const T2* S = slot + sl * NW * N;
        T2 cur[EPT][NW];
#pragma unroll
        for (int i = 0; i < EPT; ++i) {
            const int e = tid + i * NT;
#pragma unroll
            for (int f = 0; f < NW; ++f) cur[i][f] = e < N ? S[f * N + e] : mk2<R>(zero, zero);
        }
        if (k + 1 < k1) issue(k + 1, sl ^ 1);
        const double lt = zs[0][k - k0], lb = zs[1][k - k0], dz = zs[2][k - k0];
#pragma unroll
        for (int i = 0; i < EPT; ++i) {
            const int e = tid + i * NT;
            if (e >= N) continue;
            R pr[3][2];
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const double tp = gT(cx(cur[i][0], c), k + 1);
                const double uk = (double)cx(cur[i][1], c), vk = (double)cx(cur[i][2], c), wk = (double)cx(cur[i][3], c);
                const double a1 = tp * lt + tk[i][c] * (1.0 - lt), a2 = tm[i][c] * lb + tk[i][c] * (1.0 - lb);
                pr[0][c] = (R)(uk * tk[i][c]);
                pr[1][c] = (R)(tk[i][c] * vk);
                pr[2][c] = (R)((a1 * wk - a2 * wm[i][c]) / dz);
                tm[i][c] = tk[i][c]; tk[i][c] = tp; wm[i][c] = wk;
            }
#pragma unroll
            for (int f = 0; f < 3; ++f) cin.st(f, e, mk2<R>(pr[f][0], pr[f][1]));
        }
        __syncthreads();
        run_passes<R, N, -1, RMAX, L, NT, false, 0>(cin, zout, Ab, Bb, A.tw);
        __syncthreads();
        const long long orow = ((long long)k * g.ny + j) * N;
        const R sc = A.scale;
        for (int l = tid; l < N; l += NT) {
            const T2 w = __ldg(A.wp + l);
            const int i0 = fpi<G>(l), i1 = fpi<G>(l == 0 ? 0 : N - l);
#pragma unroll
            for (int line = 0; line < L; ++line) {
                const T2 z = Z[line * LS + i0];
                T2 zc = Z[line * LS + i1];
                zc.y = -zc.y;
                const T2 ev = mk2<R>(R(0.5) * (z.x + zc.x), R(0.5) * (z.y + zc.y));
                const T2 dv = mk2<R>(R(0.5) * (z.x - zc.x), R(0.5) * (z.y - zc.y));
                const T2 wd = cmulc(w, dv);
                reinterpret_cast<T2*>(a.out[line])[orow + l] = mk2<R>((ev.x + wd.y) * sc, (ev.y - wd.x) * sc);
            }
        }
        if constexpr (np >= 2 && np % 2 == 0) __syncthreads();   // C shares Z (see k_spec_products_fx)
    }
    sp_wait<0>();
}

template <typename R> struct AsmTArgs {
    const typename V2<R>::T* st;
    const typename V2<R>::T* F[3];
    typename V2<R>::T* ss;     // in: old, out: new
    typename V2<R>::T* qt;
    DampTab dt;
    Geo g;
    const double* rdz; const double* rdzt; const double* rdzb;   // [nz] 1/dz, 1/dz_t, 1/dz_b
    double tpx, tpy;
    double rk_a, rk_b, rk_c, dtime, alpha, um, tbs, tba, ttop;   // T(-1) = tbs T(0) + tba
    int kchunk;
    const int* halt;
};

template <typename R>
__global__ void __launch_bounds__(256) k_spec_assemble_t(AsmTArgs<R> a)
{
    typedef typename V2<R>::T T2;
    if (a.halt && *a.halt) return;
    const Geo& g = a.g;
    const long long ncol = g.ncol;
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncol) return;
    const int nz = g.nz;
    const int k0 = blockIdx.y * a.kchunk, k1 = min(nz, k0 + a.kchunk);
    const SpecWave wv = spec_wave(c, g, a.tpx, a.tpy);
    auto ldr = [&](const T2* f, int k) -> T2 { return f[(long long)k * ncol + c]; };
    auto dbl = [](T2 v) { return make_double2((double)v.x, (double)v.y); };
    const int nz1 = nz - 1;
    // stored spectrum of the level a neighbour reads (clamped) and the ghost rule
    // of update_boundary_t on it (a constant offset lands on the (0,0) mode only)
    auto gT = [&](T2 r, int k) -> double2 {
        const double2 s = dbl(r);
        if (k < 0) return make_double2(a.tbs * s.x + (wv.is00 ? a.tba : 0.0), a.tbs * s.y);
        if (k >= nz) return make_double2(-s.x + (wv.is00 ? 2.0 * a.ttop : 0.0), -s.y);
        return s;
    };
    auto iC = [&](int k) { return k < 0 ? 0 : (k > nz1 ? nz1 : k); };
    const double at = a.rk_c * 0.5 * a.dtime * a.alpha;
    const double bdt = a.rk_b * a.dtime, adt = a.rk_a * a.dtime;
    const double k2 = wv.kx * wv.kx + wv.ky * wv.ky;
    double2 tm = gT(ldr(a.st, iC(k0 - 1)), k0 - 1), tk = gT(ldr(a.st, iC(k0)), k0);
    // everything a level reads is loaded one level ahead in the storage type
    // (see k_spec_assemble)
    struct Lv { T2 tp, ss, F[3]; double rdz, rdzt, rdzb; };
    auto fetch = [&](int k, Lv& L) {
        L.tp = ldr(a.st, iC(k + 1)); L.ss = ldr(a.ss, k);
#pragma unroll
        for (int f = 0; f < 3; ++f) L.F[f] = ldr(a.F[f], k);
        L.rdz = a.rdz[k]; L.rdzt = a.rdzt[k]; L.rdzb = a.rdzb[k];
    };
    Lv cur;
    fetch(k0, cur);
    for (int k = k0; k < k1; ++k) {
        Lv nxt;
        if (k + 1 < k1) fetch(k + 1, nxt);
        const double2 tp = gT(cur.tp, k + 1);
        const long long id = (long long)k * ncol + c;
        const double rdz = cur.rdz, rdzt = cur.rdzt, rdzb = cur.rdzb;
        const double2 Dt = a.dt.at(tk, 4, k, nz);
        const double zs = wv.zp;
        const double2 lzt = make_double2(zs * (((tp.x - tk.x) * rdzt - (tk.x - tm.x) * rdzb) * rdz),
                                         zs * (((tp.y - tk.y) * rdzt - (tk.y - tm.y) * rdzb) * rdz));
        double2 q = zfma(zfma(Dt, Dt, -at * k2), lzt, at);
        q = zfma(q, dbl(cur.ss), bdt);
        double2 h = make_double2(0, 0);
        h = zfma(h, mul_i(Dt, wv.kx), -a.um);
        h = zfma(h, mul_i(dbl(cur.F[0]), wv.kx), -1.0);
        h = zfma(h, mul_i(dbl(cur.F[1]), wv.ky), -1.0);
        h = zfma(h, dbl(cur.F[2]), -1.0);
        st2<R>(a.ss, id, h);
        st2<R>(a.qt, id, zfma(q, h, adt));
        tm = tk; tk = tp;
        cur = nxt;
    }
}

// screen_div_error_spec (src/module_spectral.f90:899-1007) on the physical image
// of the divergence spectrum: per block sum |div|, the div of largest magnitude
// and a NaN flag over u, v, w (same partial layout as k_div_check). V points a
// thread and load (16-byte loads when the host finds the fields aligned; the
// n % V points past the last full vector are taken one a thread).
template <typename R, int V> struct alignas(sizeof(R) * V) DivVec { R x[V]; };

template <typename R, int V>
__global__ void __launch_bounds__(256) k_spec_div_reduce(const R* div, FieldsIn<R> f, long long n, double* part)
{
    __shared__ double s_sum[8], s_max[8];
    __shared__ int s_nan;
    const int tid = threadIdx.x;
    if (tid == 0) s_nan = 0;
    __syncthreads();
    double sm = 0.0, mx = 0.0;
    int nan = 0;
    auto point = [&](R dr, R ur, R vr, R wr) {
        const double d = (double)dr, uc = (double)ur, vc = (double)vr, wc = (double)wr;
        if (uc != uc || vc != vc || wc != wc || d != d) { nan = 1; return; }
        sm += fabs(d);
        mx = absmax_pick(mx, d);
    };
    typedef DivVec<R, V> Vt;
    const long long nv = n / V, stride = (long long)gridDim.x * blockDim.x;
    const long long i0 = (long long)blockIdx.x * blockDim.x + tid;
#pragma unroll 2
    for (long long i = i0; i < nv; i += stride) {
        const Vt d = reinterpret_cast<const Vt*>(div)[i], u = reinterpret_cast<const Vt*>(f.u)[i];
        const Vt v = reinterpret_cast<const Vt*>(f.v)[i], w = reinterpret_cast<const Vt*>(f.w)[i];
#pragma unroll
        for (int e = 0; e < V; ++e) point(d.x[e], u.x[e], v.x[e], w.x[e]);
    }
    for (long long q = nv * V + i0; q < n; q += stride) point(div[q], f.u[q], f.v[q], f.w[q]);
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

// ---------------------------------------------------------------------------
// Fused wall-normal part of one spectral sub-step, one warp per column (l, m)
// (rows per lane K = ceil(nz/32)), in the order of time_advancement_sp
// (src/module_navier_stokes.f90:371-517):
//   u*, v*, w* Helmholtz solves (poisson_solver_fft_spec :602-746, ubnd and
//   zstagger as the finite-difference path); the phi source get_div_spec/dt
//   (:752-795) with the delnull pin; the phi Poisson solve; the pressure update
//   p = D_p + phi - rk_c dt nu/2 lap(phi) (calculate_new_p_spec :854-894); the
//   projection (calculate_uvw_spec :801-849); the 2/3-rule truncation of u, v,
//   w, p; and the divergence spectrum of the final fields for the diagnostic.
// phi is stored untruncated (the reference's physical phi is its image).
// ---------------------------------------------------------------------------
template <typename R> struct SpColArgs {
    ColArgs<R> b;                    // qu, qv, qw: assembled right-hand sides (read only)
    typename V2<R>::T* su; typename V2<R>::T* sv; typename V2<R>::T* sw; typename V2<R>::T* sp;
    typename V2<R>::T* phi; typename V2<R>::T* div;
    DampTab dt;
    int ltr, mtr;
};

template <typename R> __device__ __forceinline__ double2 round_to(double2 v)
{
    return make_double2((double)(R)v.x, (double)(R)v.y);
}

template <typename R, int K>
__global__ void __launch_bounds__(CW_WARPS * 32, 4) k_column_sp_warp(SpColArgs<R> A)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const ColArgs<R>& a = A.b;
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
    const bool is00 = (c == 0), nyq = (m == a.g.ny / 2);
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
    // ---- phi: source (i kx u* + i ky v* + dw*/dz) / dt, zero on the Nyquist row
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
            if (r < nz && !nyq) {
                const double2 us = SU[i * 32 + ln], vs = SV[i * 32 + ln], ws = SW[i * 32 + ln];
                const double2 wm = i > 0 ? SW[(i - 1) * 32 + ln] : wprev0;
                const double rdz = __ldg(a.c.rdz + r);
                double2 dv = zadd(zmul(DX, us), zmul(DY, vs));
                dv = zadd(dv, make_double2((ws.x - wm.x) * rdz, (ws.y - wm.y) * rdz));
                ph[0][i] = make_double2(dv.x * rdt, dv.y * rdt);
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
    // ---- pressure update, projection, truncation
    const bool tr = spec_truncated(l, m, a.g.ny, A.ltr, A.mtr);
    {
        // the old pressure spectrum of the lane's rows, all loaded before the
        // first row's stores (read in the row loop, every row waited on its own load)
        typename V2<R>::T spv[K];
#pragma unroll
        for (int i = 0; i < K; ++i) {
            const int r = r0 + i;
            if (r < nz) spv[i] = A.sp[(long long)r * ncol + c];
            else { spv[i].x = R(0); spv[i].y = R(0); }
        }
        const double2 GX = __ldg(a.c.gx + l), GY = __ldg(a.c.gy + m);
        const double lxy = __ldg(a.c.lx + l) + __ldg(a.c.ly + m);
        const double cpr = rk * dt, cps = rk * 0.5 * dt * a.nu;
        double2 nxt0 = shfl_dn2(ph[0][0], 1);
        double2 prv0 = shfl_up2(ph[0][K - 1], 1);
#pragma unroll
        for (int i = 0; i < K; ++i) {
            const int r = r0 + i;
            if (r >= nz) continue;
            const long long id = (long long)r * ncol + c;
            const double2 pc = ph[0][i];
            const double2 pu = (r == nz - 1) ? pc : (i < K - 1 ? ph[0][i + 1] : nxt0);
            const double2 pd = (r == 0) ? pc : (i > 0 ? ph[0][i - 1] : prv0);
            const double2 us = SU[i * 32 + ln], vs = SV[i * 32 + ln], ws = SW[i * 32 + ln];
            const double rdzt = __ldg(a.c.rdzt + r), rdzb = __ldg(a.c.rdzb + r), rdz = __ldg(a.c.rdz + r);
            double2 fu = zsub(us, zscale(zmul(GX, pc), cpr));
            double2 fv = zsub(vs, zscale(zmul(GY, pc), cpr));
            double2 fw = r <= nz - 2 ? make_double2(ws.x - cpr * (pu.x - pc.x) * rdzt, ws.y - cpr * (pu.y - pc.y) * rdzt)
                                     : make_double2(0, 0);
            double2 lz;
            lz.x = ((pu.x - pc.x) * rdzt - (pc.x - pd.x) * rdzb) * rdz;
            lz.y = ((pu.y - pc.y) * rdzt - (pc.y - pd.y) * rdzb) * rdz;
            const double2 psi = make_double2(pc.x - cps * (lxy * pc.x + lz.x), pc.y - cps * (lxy * pc.y + lz.y));
            double2 fp = zadd(A.dt.at(make_double2((double)spv[i].x, (double)spv[i].y), 3, r, nz), psi);
            if (tr) { fu = make_double2(0, 0); fv = fu; fw = fu; fp = fu; }
            st2<R>(A.phi, id, pc);
            st2<R>(A.su, id, fu);
            st2<R>(A.sv, id, fv);
            st2<R>(A.sw, id, fw);
            st2<R>(A.sp, id, fp);
            SU[i * 32 + ln] = round_to<R>(fu);
            SV[i * 32 + ln] = round_to<R>(fv);
            SW[i * 32 + ln] = round_to<R>(fw);
        }
    }
    __syncwarp();
    // ---- divergence spectrum of the stored fields (the physical w is 0 below
    //      the bottom wall and on the top wall)
#pragma unroll
    for (int i = 0; i < K; ++i) {
        const int r = r0 + i;
        if (r >= nz) continue;
        const long long id = (long long)r * ncol + c;
        double2 dv = make_double2(0, 0);
        if (!nyq) {
            const double2 fu = SU[i * 32 + ln], fv = SV[i * 32 + ln], fw = SW[i * 32 + ln];
            const double2 fwm = r == 0 ? make_double2(0, 0) : (i > 0 ? SW[(i - 1) * 32 + ln] : SW[(K - 1) * 32 + ln - 1]);
            const double rdz = __ldg(a.c.rdz + r);
            dv = zadd(zmul(DX, fu), zmul(DY, fv));
            dv = zadd(dv, make_double2((fw.x - fwm.x) * rdz, (fw.y - fwm.y) * rdz));
        }
        st2<R>(A.div, id, dv);
    }
}

// The same column work as k_column_sp_warp with the coalescing tiles of
// k_column_fd_tile_r: a block of SP_COLS warps stages the rows of SP_COLS
// adjacent columns (q_u, q_v, q_w and the old pressure spectrum) in shared
// memory with row-contiguous loads, each warp solves one column from the tiles,
// and the results (u, v, w, p, phi, the divergence spectrum) leave through the
// tiles with row-contiguous stores; the warp kernel read and wrote every row of
// its column with one access per lane (32 rows of one column per instruction).
// columns a block (8 warps); 4 columns of 4 warps, at 4 resident blocks, took
// 216 against 212 us a launch mixed and 294 against 275 us FP64 at 256 x 256 x 128
#define SP_COLS 8
template <int K> __host__ size_t column_sp_tile_smem(size_t elem)
{
    return (size_t)4 * SP_COLS * ct_stride_e<K>(elem) * elem;
}

template <typename R, int K>
__global__ void __launch_bounds__(SP_COLS * 32, 16 / SP_COLS) k_column_sp_tile(SpColArgs<R> A)
{
    typedef typename V2<R>::T TT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const ColArgs<R>& a = A.b;
    if (a.halt && *a.halt) return;
    const int ln = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const long long ncol = a.g.ncol;
    const long long c0 = (long long)blockIdx.x * SP_COLS;
    const long long c = c0 + wp;
    const bool active = c < ncol;
    const int nz = a.g.nz;
    constexpr int STR = CtLayout<TT>::template stride<K>();
    constexpr int RP = CtLayout<TT>::rp;
    TT* TU = reinterpret_cast<TT*>(smem_raw);
    TT* TV = TU + SP_COLS * STR;
    TT* TW = TV + SP_COLS * STR;
    TT* TP = TW + SP_COLS * STR;
    // element (column cb, row r) at cb * STR + (r % K) * RP + r / K: lane ln of
    // a warp holds rows ln K .. ln K + K - 1 of its column
    auto load = [&](const TT* __restrict__ q, TT* T, int nrows) {
        TT v[K];
#pragma unroll
        for (int it = 0; it < K; ++it) {
            const int idx = threadIdx.x + it * SP_COLS * 32;
            const int r = idx / SP_COLS, cb = idx - r * SP_COLS;
            const long long cc = c0 + cb;
            v[it] = (idx < nrows * SP_COLS && cc < ncol) ? q[(long long)r * ncol + cc] : mk2<R>(R(0), R(0));
        }
#pragma unroll
        for (int it = 0; it < K; ++it) {
            const int idx = threadIdx.x + it * SP_COLS * 32;
            const int r = idx / SP_COLS, cb = idx - r * SP_COLS;
            if (idx < nrows * SP_COLS) T[cb * STR + (r % K) * RP + r / K] = v[it];
        }
    };
    auto store = [&](TT* __restrict__ q, const TT* T) {
        for (int idx = threadIdx.x; idx < nz * SP_COLS; idx += blockDim.x) {
            const int r = idx / SP_COLS, cb = idx - r * SP_COLS;
            const long long cc = c0 + cb;
            if (cc < ncol) q[(long long)r * ncol + cc] = T[cb * STR + (r % K) * RP + r / K];
        }
    };
    load(a.qu, TU, nz);
    load(a.qv, TV, nz);
    load(a.qw, TW, nz - 1);
    load(A.sp, TP, nz);
    __syncthreads();
    TT* SU = TU + wp * STR;
    TT* SV = TV + wp * STR;
    TT* SW = TW + wp * STR;
    TT* SP = TP + wp * STR;
    auto dbl = [](TT v) { return make_double2((double)v.x, (double)v.y); };
    auto put = [](TT* S, int q, double2 v) { S[q] = mk2<R>((R)v.x, (R)v.y); };
    const int r0 = ln * K;
    double2 ph[1][K];
    double2 dvr[K];      // the divergence spectrum of the lane's rows
    if (active) {
        const int l = (int)(c % a.g.nxh), m = (int)(c / a.g.nxh);
        const bool is00 = (c == 0), nyq = (m == a.g.ny / 2);
        const double rk = a.rk_c, dt = a.dt;
        const double lam = __ldg(a.c.hx + l) + __ldg(a.c.hy + m);
        const double lamp = __ldg(a.c.px + l) + __ldg(a.c.py + m);
        const double* dgu = is00 ? a.c.d0u : a.c.dgu;
        const double* dgw = is00 ? a.c.d0w : a.c.dgw;
        const double* dgp = is00 ? a.c.d0p : a.c.dgp;
        // ---- u*, v*: one matrix, two right-hand sides. u*, v*, w* stay in FP64
        //      registers until the projection, as the warp kernel keeps them in
        //      FP64 shared memory (the tiles hold the storage type)
        double2 us_[K], vs_[K], ws_[K];
        if (sizeof(R) == sizeof(float) && !is00) {
            // FP32 storage, every mode but the mean: the two diagonally dominant
            // Helmholtz systems in FP32, side by side (as the FD column kernel);
            // the results join the FP64 projection
            float2 d[2][K], dw[1][K];
#pragma unroll
            for (int i = 0; i < K; ++i) {
                const int r = r0 + i;
                const TT xu = SU[i * RP + ln], xv = SV[i * RP + ln], xw = SW[i * RP + ln];
                d[0][i] = r < nz ? make_float2((float)xu.x, (float)xu.y) : make_float2(0.0f, 0.0f);
                d[1][i] = r < nz ? make_float2((float)xv.x, (float)xv.y) : make_float2(0.0f, 0.0f);
                dw[0][i] = r < nz - 1 ? make_float2((float)xw.x, (float)xw.y) : make_float2(0.0f, 0.0f);
            }
            auto cfu = [&](int r, float& aa, float& bb, float& cc) {
                if (r < nz) {
                    aa = (float)(rk * __ldg(a.c.au + r));
                    cc = (float)(rk * __ldg(a.c.cu + r));
                    bb = (float)(1.0 + rk * (-lam + __ldg(dgu + r)));
                } else { aa = 0.0f; bb = 1.0f; cc = 0.0f; }
            };
            auto cfw = [&](int r, float& aa, float& bb, float& cc) {
                if (r < nz - 1) {
                    aa = (float)(rk * __ldg(a.c.aw + r));
                    cc = (float)(rk * __ldg(a.c.cw + r));
                    bb = (float)(1.0 + rk * (-lam + __ldg(dgw + r)));
                } else { aa = 0.0f; bb = 1.0f; cc = 0.0f; }
            };
            warp_partition_solve2_t<float, K, 2, 1>(cfu, d, cfw, dw, ln);
#pragma unroll
            for (int i = 0; i < K; ++i) {
                us_[i] = make_double2((double)d[0][i].x, (double)d[0][i].y);
                vs_[i] = make_double2((double)d[1][i].x, (double)d[1][i].y);
                ws_[i] = make_double2((double)dw[0][i].x, (double)dw[0][i].y);
            }
        } else {
        {
            double2 d[2][K];
#pragma unroll
            for (int i = 0; i < K; ++i) {
                const int r = r0 + i;
                if (r < nz) {
                    d[0][i] = dbl(SU[i * RP + ln]);
                    d[1][i] = dbl(SV[i * RP + ln]);
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
            for (int i = 0; i < K; ++i) { us_[i] = d[0][i]; vs_[i] = d[1][i]; }
        }
        {
            double2 dw[1][K];
#pragma unroll
            for (int i = 0; i < K; ++i) {
                const int r = r0 + i;
                dw[0][i] = r < nz - 1 ? dbl(SW[i * RP + ln]) : make_double2(0, 0);
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
            for (int i = 0; i < K; ++i) ws_[i] = dw[0][i];
        }
        }
        // ---- phi: source (i kx u* + i ky v* + dw*/dz) / dt, zero on the Nyquist row
        const double2 DX = __ldg(a.c.dx + l), DY = __ldg(a.c.dy + m);
        const double rdt = 1.0 / dt;
        {
            double2 wprev0 = shfl_up2(ws_[K - 1], 1);
            if (ln == 0) wprev0 = make_double2(0, 0);
#pragma unroll
            for (int i = 0; i < K; ++i) {
                const int r = r0 + i;
                if (r < nz && !nyq) {
                    const double2 wm = i > 0 ? ws_[i - 1] : wprev0;
                    const double rdz = __ldg(a.c.rdz + r);
                    double2 dv = zadd(zmul(DX, us_[i]), zmul(DY, vs_[i]));
                    dv = zadd(dv, make_double2((ws_[i].x - wm.x) * rdz, (ws_[i].y - wm.y) * rdz));
                    ph[0][i] = make_double2(dv.x * rdt, dv.y * rdt);
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
        // ---- pressure update, projection, truncation: results into the tiles
        const bool tr = spec_truncated(l, m, a.g.ny, A.ltr, A.mtr);
        {
            const double2 GX = __ldg(a.c.gx + l), GY = __ldg(a.c.gy + m);
            const double lxy = __ldg(a.c.lx + l) + __ldg(a.c.ly + m);
            const double cpr = rk * dt, cps = rk * 0.5 * dt * a.nu;
            const double2 nxt0 = shfl_dn2(ph[0][0], 1);
            const double2 prv0 = shfl_up2(ph[0][K - 1], 1);
#pragma unroll
            for (int i = 0; i < K; ++i) {
                const int r = r0 + i;
                if (r >= nz) continue;
                const double2 pc = ph[0][i];
                const double2 pu = (r == nz - 1) ? pc : (i < K - 1 ? ph[0][i + 1] : nxt0);
                const double2 pd = (r == 0) ? pc : (i > 0 ? ph[0][i - 1] : prv0);
                const double rdzt = __ldg(a.c.rdzt + r), rdzb = __ldg(a.c.rdzb + r), rdz = __ldg(a.c.rdz + r);
                double2 fu = zsub(us_[i], zscale(zmul(GX, pc), cpr));
                double2 fv = zsub(vs_[i], zscale(zmul(GY, pc), cpr));
                double2 fw = r <= nz - 2 ? make_double2(ws_[i].x - cpr * (pu.x - pc.x) * rdzt, ws_[i].y - cpr * (pu.y - pc.y) * rdzt)
                                         : make_double2(0, 0);
                double2 lz;
                lz.x = ((pu.x - pc.x) * rdzt - (pc.x - pd.x) * rdzb) * rdz;
                lz.y = ((pu.y - pc.y) * rdzt - (pc.y - pd.y) * rdzb) * rdz;
                const double2 psi = make_double2(pc.x - cps * (lxy * pc.x + lz.x), pc.y - cps * (lxy * pc.y + lz.y));
                double2 fp = zadd(A.dt.at(dbl(SP[i * RP + ln]), 3, r, nz), psi);
                if (tr) { fu = make_double2(0, 0); fv = fu; fw = fu; fp = fu; }
                put(SU, i * RP + ln, fu);
                put(SV, i * RP + ln, fv);
                put(SW, i * RP + ln, fw);
                put(SP, i * RP + ln, fp);
            }
        }
        __syncwarp();
        // ---- divergence spectrum of the stored fields (the physical w is 0 below
        //      the bottom wall and on the top wall)
        const double2 wlast = dbl(SW[(K - 1) * RP + ln]);
        double2 wbelow0 = shfl_up2(wlast, 1);
#pragma unroll
        for (int i = 0; i < K; ++i) {
            const int r = r0 + i;
            double2 dv = make_double2(0, 0);
            if (r < nz && !nyq) {
                const double2 fu = dbl(SU[i * RP + ln]), fv = dbl(SV[i * RP + ln]), fw = dbl(SW[i * RP + ln]);
                const double2 fwm = r == 0 ? make_double2(0, 0) : (i > 0 ? dbl(SW[(i - 1) * RP + ln]) : wbelow0);
                const double rdz = __ldg(a.c.rdz + r);
                dv = zadd(zmul(DX, fu), zmul(DY, fv));
                dv = zadd(dv, make_double2((fw.x - fwm.x) * rdz, (fw.y - fwm.y) * rdz));
            }
            dvr[i] = dv;
        }
    }
    __syncthreads();
    store(A.su, TU);
    store(A.sv, TV);
    store(A.sw, TW);
    store(A.sp, TP);
    __syncthreads();
    // phi and the divergence spectrum through the first two tiles
    if (active) {
#pragma unroll
        for (int i = 0; i < K; ++i) {
            put(SU, i * RP + ln, ph[0][i]);
            put(SV, i * RP + ln, dvr[i]);
        }
    }
    __syncthreads();
    store(A.phi, TU);
    store(A.div, TV);
}
