// hc_rhs_strip.cuh -- FP32 momentum right-hand side (get_momentum_cnvdiff,
// src/module_cnvdiff.f90:35-374) that evaluates every interpolant product only
// where a flux difference reads it.
//
// In the reference's flux form, per equation and direction, a difference reads a
// product on one axis only:
//   U: d/dx uhx^2 (x),  d/dy uhy*vhx (y),  d/dz uhz*whx (own point)
//   V: d/dx uhy*vhx (x), d/dy vhy^2 (y),   d/dz vhz*why (own point)
//   W: d/dx uhz*whx (x), d/dy vhz*why (y),  w^2 in z (own point)
// so uhx and uhz*whx are needed on an x strip of the tile (its rows, two extra
// columns either side), vhy and vhz*why on a y strip (its columns, two extra rows
// either side) and uhy*vhx on both strips -- never on the corners of the halo.
// A block owns a 64 x 16 tile (a thread: two adjacent x points in two adjacent
// rows with FP32 storage, 256 threads; in one row with FP64 storage, 512 threads)
// and marches up a run of k levels. Per level it
//   1. computes the five products on their strips from the raw planes of level k
//      (u, v, w, p with a 4-point x / 3-point y halo) and k+1 (shared memory);
//   2. evaluates the three equations at its points from the raw planes and the
//      product strips, with the level-(k-1) values a thread needs (u, v, w,
//      uhz*whx, vhz*why at its own points) carried in registers;
// while the planes of level k+2 arrive in a third slot of each field's ring by
// cp.async (16-byte copies, no registers). Ghost levels are never staged: below
// the first level the no-slip / impermeable values follow from the first level
// (update_boundary_uvw, src/module_boundary.f90:33-112) and above the last one
// only the own-point values enter, also by formula. Built without a moving frame
// (u_mrf = 0) and without the Ekman forcing (dp_opt 1 or 2), for nx >= 64 (rows of
// whole 16-byte chunks) and ny >= 32; other cases run the tiled kernels.
#pragma once
#include "hc_rhs_tiled2.cuh"

#define RS_TX 64                      // tile points in x
#define RS_TY 16                      // tile rows
#define RS_HX 4                       // raw-window halo in x (keeps rows 16-byte aligned)
#define RS_HY 3                       // raw-window halo in y
#define RS_W (RS_TX + 2 * RS_HX)      // 72
#define RS_H (RS_TY + 2 * RS_HY)      // 22
#define RS_P (RS_W * RS_H)            // 1584 floats a plane
#define RS_NC4 (RS_W / 4)             // 18 16-byte chunks a row
#define RS_NPOS (RS_NC4 * RS_H)       // 396 chunks a plane
// product strips (floats)
#define RS_AW (RS_TX + 4)             // x strip width: x from -2 to 65
#define RS_BH (RS_TY + 4)             // y strip height: y from -2 to 17
#define RS_F_UHX 0                                  // [16][68]  uhx on the x strip
#define RS_F_CZ (RS_F_UHX + RS_TY * RS_AW)          // [16][68]  uhz*whx on the x strip
#define RS_F_B (RS_F_CZ + RS_TY * RS_AW)            // [20][68]  uhy*vhx on both strips
#define RS_F_VHY (RS_F_B + RS_BH * RS_AW)           // [20][64]  vhy on the y strip
#define RS_F_EZ (RS_F_VHY + RS_BH * RS_TX)          // [20][64]  vhz*why on the y strip
#define RS_NF (RS_F_EZ + RS_BH * RS_TX)

// launch shape per storage type: FP32 256 threads (two rows a thread), two blocks
// an SM; FP64 512 threads (one row a thread), one block an SM (196 KB of planes)
template <typename R> struct RsCfg {
    static constexpr int RQ = sizeof(R) == sizeof(float) ? 2 : 1;     // rows a thread
    static constexpr int NT = 32 * RS_TY / RQ;                          // threads a block
    static constexpr int NW = NT / 32;                                  // warps a block
    static constexpr int MINB = sizeof(R) == sizeof(float) ? 2 : 1;     // blocks an SM
    static constexpr int EPC = 16 / (int)sizeof(R);                     // elements a 16-byte chunk
    static constexpr int NCH = RS_W / EPC;                              // chunks a row
    static constexpr int NPOS = NCH * RS_H;                             // chunks a plane
    static_assert(NPOS <= 2 * NT, "two chunk positions a thread");
};

template <typename R> __host__ inline size_t rhs_strip_smem() { return sizeof(R) * ((size_t)12 * RS_P + RS_NF); }

// the strip kernel covers this case (the host falls back to the tiled kernels otherwise):
// rows of 16-byte chunks need nx to be a multiple of 16 / sizeof(R)
__host__ inline bool rhs_strip_ok(int nx, int ny, double u_mrf, int dp_opt, size_t elem)
{
    return nx % (int)(16 / elem) == 0 && nx >= 64 && ny >= 32 && u_mrf == 0.0 && dp_opt != 3;
}

__device__ __forceinline__ void rs_cp16(void* dst, const void* src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void rs_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void rs_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// fourth-order mid-point interpolant (-a + 9 b + 9 c - d) / 16 and its
// second-order form (b + c) / 2 (get_interp_fields_uvwhxyz, src/module_tools.f90:410-468)
template <typename R, int CDS> __device__ __forceinline__ R rs_mid(R a, R b, R c, R d)
{
    if (CDS == 1) return R(0.5) * (b + c);
    return (R(9) * (b + c) - (a + d)) * R(0.0625);
}
// staggered first difference (-a2 + 27 a1 - 27 a0 + am) (the 1/(24 h) applied by the caller);
// second order: a1 - a0 (the 1/h applied by the caller)
template <typename R, int CDS> __device__ __forceinline__ R rs_d1(R a2, R a1, R a0, R am)
{
    if (CDS == 1) return a1 - a0;
    return R(27) * (a1 - a0) - (a2 - am);
}
// centred second difference (-a2 + 16 a1 - 30 a0 + 16 am - am2) or a1 - 2 a0 + am
template <typename R, int CDS> __device__ __forceinline__ R rs_d2(R a2, R a1, R a0, R am, R am2)
{
    if (CDS == 1) return (a1 + am) - R(2) * a0;
    return R(16) * (a1 + am) - R(30) * a0 - (a2 + am2);
}
// pairs of adjacent x points as one 8-byte (FP32) or 16-byte (FP64) shared-memory access
template <typename R> __device__ __forceinline__ typename V2<R>::T ld2r(const R* p, int i)
{
    return *reinterpret_cast<const typename V2<R>::T*>(p + i);
}
template <typename R> __device__ __forceinline__ void st2r(R* p, int i, R a, R b)
{
    *reinterpret_cast<typename V2<R>::T*>(p + i) = mk2<R>(a, b);
}
// six consecutive values p[i-2 .. i+3] (i even) as v[0..5]
template <typename R> __device__ __forceinline__ void ld6r(const R* p, int i, R* v)
{
    const typename V2<R>::T a = ld2r(p, i - 2), b = ld2r(p, i), c = ld2r(p, i + 2);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y; v[4] = c.x; v[5] = c.y;
}

template <typename R, int CDS>
__device__ __forceinline__ void k_rhs_momentum_strip_body(const RhsTArgs<R>& a, const uint3 blockIdx, const dim3 gridDim)
{
    typedef typename V2<R>::T R2;
    constexpr int RQ = RsCfg<R>::RQ, NT = RsCfg<R>::NT, NW = RsCfg<R>::NW;
    constexpr int EPC = RsCfg<R>::EPC, NCH = RsCfg<R>::NCH, NPOS = RsCfg<R>::NPOS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* SR = reinterpret_cast<R*>(smem_raw);              // [4 fields][3 slots][RS_P]
    R* FL = SR + 12 * RS_P;                                   // product strips
    R* F_UHX = FL + RS_F_UHX;
    R* F_CZ = FL + RS_F_CZ;
    R* F_B = FL + RS_F_B;
    R* F_VHY = FL + RS_F_VHY;
    R* F_EZ = FL + RS_F_EZ;

    const Geo& g = a.g;
    const int nz = g.nz, nx = g.nx, ny = g.ny;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int closed = a.ph.ochannel == 0;
    const int tiles_x = (nx + RS_TX - 1) / RS_TX;
    const long long ntiles = (long long)tiles_x * ((ny + RS_TY - 1) / RS_TY);
    // the (tile, level) work of this block: with a level chunk (a.kchunk > 0) block b
    // takes chunk b / ntiles of tile b % ntiles, so that the blocks in flight cover
    // neighbouring tiles at the same levels and share their halo rows in L2; with
    // a.kchunk = 0 the blocks split the work, tiles in order and levels ascending,
    // into equal runs (one wave, no tail)
    long long wcur, wend;
    if (a.kchunk > 0) {
        const long long t = blockIdx.x % ntiles, c = blockIdx.x / ntiles;
        wcur = t * nz + c * a.kchunk;
        wend = t * nz + min((long long)nz, (c + 1) * a.kchunk);
    } else {
        const long long work = ntiles * nz;
        wcur = work * blockIdx.x / gridDim.x;
        wend = work * (blockIdx.x + 1) / gridDim.x;
    }
    const R* zrdz = (const R*)a.zm;
    const R* zrdzt = (const R*)a.zm + nz;
    const R* zrdzb = (const R*)a.zm + 2 * nz;
    const R* zlt = (const R*)a.zm + 3 * nz;
    const R* zrdzp = (const R*)a.zm + 4 * nz;
    auto plane = [&](int f, int lvl) { return SR + (f * 3 + lvl % 3) * RS_P; };

    const R rdx = R(1) / (R)g.dx, rdy = R(1) / (R)g.dy;
    const R r24dx = R(1) / (R(24) * (R)g.dx), r24dy = R(1) / (R(24) * (R)g.dy);
    const R r12dx2 = R(1) / (R(12) * (R)g.dx2), r12dy2 = R(1) / (R(12) * (R)g.dy2);
    const R rdx2 = R(1) / (R)g.dx2, rdy2 = R(1) / (R)g.dy2;
    const R sx1 = CDS == 1 ? rdx : r24dx, sy1 = CDS == 1 ? rdy : r24dy;     // first differences
    const R sx2 = CDS == 1 ? rdx2 : r12dx2, sy2 = CDS == 1 ? rdy2 : r12dy2; // second differences
    const R dt = (R)a.ph.dt, nu = (R)a.ph.nu;
    const R rka = (R)a.rk_a, rkb = (R)a.rk_b, rkc = (R)a.rk_c;
    const R cdif = rkc * R(0.5) * dt * nu, cgp = rkc * dt;
    const R dpx = (R)a.sc->dpx_drive;
    const R got = (R)a.sc->got, tref = (R)a.ph.t_ref;
    const bool scalar = a.ph.isscalar == 1;

    double dv_sum = 0.0, dv_max = 0.0;
    int dv_nan = 0;
    // the thread's points in a tile: x = x0 + 2 lane + s, rows y0 + 2 wid + q (s, q in {0, 1})
    const int xl = 2 * lane, rl0 = RQ * wid;
    int rc[2];
#pragma unroll
    for (int q = 0; q < RQ; ++q) rc[q] = (rl0 + q + RS_HY) * RS_W + xl + RS_HX;    // own raw index (even)
    // this thread's two 16-byte chunk positions of a plane
    const bool has1 = threadIdx.x + NT < NPOS;
    const int row0 = threadIdx.x / NCH, c40 = threadIdx.x - row0 * NCH;
    const int row1 = (threadIdx.x + NT) / NCH, c41 = threadIdx.x + NT - row1 * NCH;
    const int dst0 = row0 * RS_W + EPC * c40, dst1 = row1 * RS_W + EPC * c41;

    while (wcur < wend) {
    // ---- one segment: levels kb .. ke-1 of one tile
    const long long tile = wcur / nz;
    const int kb = (int)(wcur - tile * nz);
    const int ke = (int)min((long long)nz, (long long)kb + (wend - wcur));
    wcur += ke - kb;
    const int x0 = (int)(tile % tiles_x) * RS_TX, y0 = (int)(tile / tiles_x) * RS_TY;
    // wrapped source offsets of the chunk positions (the periodic comm_bound halo)
    const int src0 = (((y0 - RS_HY + row0) % ny + ny) % ny) * nx + ((x0 - RS_HX + EPC * c40) % nx + nx) % nx;
    const int src1 = has1 ? (((y0 - RS_HY + row1) % ny + ny) % ny) * nx + ((x0 - RS_HX + EPC * c41) % nx + nx) % nx : 0;
    auto stage = [&](int lvl) {       // cp.async of the four planes of an interior level
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            const R* src = f == 0 ? a.f.u : (f == 1 ? a.f.v : (f == 2 ? a.f.w : a.f.p));
            const R* base = src + (long long)lvl * g.nxy;
            R* d = plane(f, lvl);
            rs_cp16(d + dst0, base + src0);
            if (has1) rs_cp16(d + dst1, base + src1);
        }
    };
    if (kb > 0) stage(kb - 1);
    stage(kb);
    if (kb + 1 < nz) stage(kb + 1);
    rs_commit();
    rs_wait_all();
    __syncthreads();

    const int xi = x0 + xl;
    const bool xin = xi < nx;
    bool act[2];
    int gid[2];
#pragma unroll
    for (int q = 0; q < RQ; ++q) {
        act[q] = xin && (y0 + rl0 + q) < ny;
        gid[q] = (y0 + rl0 + q) * nx + xi;                             // + k nxy
    }

    // values of level k-1 at the own points: u, v, w, uhz*whx, vhz*why
    R um1[2][2], vm1[2][2], wm1[2][2], czp[2][2], ezp[2][2];
    if (kb == 0) {
        // no-slip, impermeable bottom wall: u(-1) = -u(0), v(-1) = -v(0), w(-1) = 0;
        // w vanishes below, so both level-(-1) products are 0
        const R* u0 = plane(0, 0); const R* v0 = plane(1, 0);
#pragma unroll
        for (int q = 0; q < RQ; ++q) {
            const R2 uc = ld2r(u0, rc[q]), vc = ld2r(v0, rc[q]);
            um1[q][0] = -uc.x; um1[q][1] = -uc.y; vm1[q][0] = -vc.x; vm1[q][1] = -vc.y;
            wm1[q][0] = wm1[q][1] = R(0);
            czp[q][0] = czp[q][1] = ezp[q][0] = ezp[q][1] = R(0);
        }
    } else {
        const int L = kb - 1;
        const R* u0 = plane(0, L); const R* v0 = plane(1, L); const R* w0 = plane(2, L);
        const R* u1 = plane(0, L + 1); const R* v1 = plane(1, L + 1);
        const R l = zlt[L];
#pragma unroll
        for (int q = 0; q < RQ; ++q) {
            const int r = rc[q];
            R wx[6];
            ld6r(w0, r, wx);
            const R2 wy1 = ld2r(w0, r + RS_W), wy2 = ld2r(w0, r + 2 * RS_W), wym = ld2r(w0, r - RS_W);
            const R2 uc = ld2r(u0, r), vc = ld2r(v0, r), wc = ld2r(w0, r);
            const R2 uu = ld2r(u1, r), vv = ld2r(v1, r);
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                const R ucs = s ? uc.y : uc.x, vcs = s ? vc.y : vc.x;
                const R whx = rs_mid<R, CDS>(wx[4 + s], wx[3 + s], wx[2 + s], wx[1 + s]);
                const R why = rs_mid<R, CDS>(s ? wy2.y : wy2.x, s ? wy1.y : wy1.x, s ? wc.y : wc.x, s ? wym.y : wym.x);
                const R uhz = (s ? uu.y : uu.x) * l + ucs * (R(1) - l);
                const R vhz = (s ? vv.y : vv.x) * l + vcs * (R(1) - l);
                czp[q][s] = uhz * whx;
                ezp[q][s] = vhz * why;
                um1[q][s] = ucs; vm1[q][s] = vcs; wm1[q][s] = s ? wc.y : wc.x;
            }
        }
    }
    __syncthreads();      // level kb-1's slot is refilled with level kb+2 below

    for (int k = kb; k < ke; ++k) {
        const bool next_in = k + 1 < nz;          // level k+1 is interior (staged)
        if (k + 2 < nz && k + 1 < ke) { stage(k + 2); rs_commit(); }
        const bool wface = k < nz - 1;
        const R lt = __ldg(zlt + k);
        const R* u0 = plane(0, k); const R* v0 = plane(1, k);
        const R* w0 = plane(2, k); const R* p0 = plane(3, k);
        const R* u1 = plane(0, k + 1); const R* v1 = plane(1, k + 1);
        const R* w1 = plane(2, k + 1); const R* p1 = plane(3, k + 1);
        const long long kofs = (long long)k * g.nxy;

        // the thread's history values of this level, issued before the products so
        // that their latency overlaps them
        R2 hf[2], hg[2], hh[2];
#pragma unroll
        for (int q = 0; q < RQ; ++q) {
            hf[q] = hg[q] = hh[q] = mk2<R>(R(0), R(0));
            if (act[q]) {
                const long long id = kofs + gid[q];
                hf[q] = *reinterpret_cast<const R2*>(a.ff + id);
                hg[q] = *reinterpret_cast<const R2*>(a.gg + id);
                if (wface) hh[q] = *reinterpret_cast<const R2*>(a.hh + id);
            }
        }
        // optional own-point inputs (body force, temperature), read where they are used
        auto ld_own = [&](const R* base, int q, long long extra) {
            return act[q] ? *reinterpret_cast<const R2*>(base + kofs + gid[q] + extra) : mk2<R>(R(0), R(0));
        };

        // ---- 1. the products on their strips (37 warp jobs of one row each)
        for (int job = wid; job < 37; job += NW) {
            if (job <= 16) {
                // x strip: rows 0..15; job 16 is the two 2-column side pieces
                int fx, fy;
                if (job < 16) { fx = 2 * lane; fy = job; }
                else { fy = lane & 15; fx = (lane >> 4) ? RS_TX : -2; }
                const int r = (fy + RS_HY) * RS_W + fx + RS_HX;
                R ux[6], vx[6], wx[6];
                ld6r(u0, r, ux); ld6r(v0, r, vx);
                const R2 uym = ld2r(u0, r - RS_W), uy1 = ld2r(u0, r + RS_W), uy2 = ld2r(u0, r + 2 * RS_W);
                R2 up = mk2<R>(R(0), R(0));
                if (wface) { ld6r(w0, r, wx); up = ld2r(u1, r); }
                R o_uhx[2], o_cz[2], o_b[2];
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    o_uhx[s] = rs_mid<R, CDS>(ux[3 + s], ux[2 + s], ux[1 + s], ux[s]);
                    const R uhy = rs_mid<R, CDS>(s ? uy2.y : uy2.x, s ? uy1.y : uy1.x, ux[2 + s], s ? uym.y : uym.x);
                    const R vhx = rs_mid<R, CDS>(vx[4 + s], vx[3 + s], vx[2 + s], vx[1 + s]);
                    o_b[s] = uhy * vhx;
                    if (wface) {
                        const R whx = rs_mid<R, CDS>(wx[4 + s], wx[3 + s], wx[2 + s], wx[1 + s]);
                        const R uhz = (s ? up.y : up.x) * lt + ux[2 + s] * (R(1) - lt);
                        o_cz[s] = uhz * whx;
                    } else {
                        o_cz[s] = R(0);       // w = 0 on the top face: whx = 0
                    }
                }
                const int ea = fy * RS_AW + fx + 2;
                st2r(F_UHX, ea, o_uhx[0], o_uhx[1]);
                st2r(F_CZ, ea, o_cz[0], o_cz[1]);
                st2r(F_B, (fy + 2) * RS_AW + fx + 2, o_b[0], o_b[1]);
            } else {
                // y strip: own columns, rows -2..17
                const int fx = 2 * lane, fy = job - 17 - 2;
                const int r = (fy + RS_HY) * RS_W + fx + RS_HX;
                const R2 vc = ld2r(v0, r);
                if (fy >= -1) {       // vhy at rows -1..17 (reads rows fy-2..fy+1)
                    const R2 vm = ld2r(v0, r - RS_W), vm2 = ld2r(v0, r - 2 * RS_W), v1y = ld2r(v0, r + RS_W);
                    st2r(F_VHY, (fy + 2) * RS_TX + fx, rs_mid<R, CDS>(v1y.x, vc.x, vm.x, vm2.x),
                         rs_mid<R, CDS>(v1y.y, vc.y, vm.y, vm2.y));
                }
                if (fy <= 16) {       // vhz*why at rows -2..16 (reads w rows fy-1..fy+2)
                    R e0 = R(0), e1 = R(0);
                    if (wface) {
                        const R2 wc = ld2r(w0, r), wym = ld2r(w0, r - RS_W), wy1 = ld2r(w0, r + RS_W),
                                     wy2 = ld2r(w0, r + 2 * RS_W);
                        const R2 vp = ld2r(v1, r);
                        e0 = (vp.x * lt + vc.x * (R(1) - lt)) * rs_mid<R, CDS>(wy2.x, wy1.x, wc.x, wym.x);
                        e1 = (vp.y * lt + vc.y * (R(1) - lt)) * rs_mid<R, CDS>(wy2.y, wy1.y, wc.y, wym.y);
                    }
                    st2r(F_EZ, (fy + 2) * RS_TX + fx, e0, e1);
                }
                if (fy < 0 || fy == 16) {     // uhy*vhx on the rows beyond the x strip
                    R vx[6];
                    ld6r(v0, r, vx);
                    const R2 uc = ld2r(u0, r), uym = ld2r(u0, r - RS_W), uy1 = ld2r(u0, r + RS_W),
                                 uy2 = ld2r(u0, r + 2 * RS_W);
                    const R b0 = rs_mid<R, CDS>(uy2.x, uy1.x, uc.x, uym.x) * rs_mid<R, CDS>(vx[4], vx[3], vx[2], vx[1]);
                    const R b1 = rs_mid<R, CDS>(uy2.y, uy1.y, uc.y, uym.y) * rs_mid<R, CDS>(vx[5], vx[4], vx[3], vx[2]);
                    st2r(F_B, (fy + 2) * RS_AW + fx + 2, b0, b1);
                }
            }
        }
        __syncthreads();

        // ---- 2. the three equations at the thread's four points
        const R rdz = __ldg(zrdz + k), rdzt = __ldg(zrdzt + k), rdzb = __ldg(zrdzb + k);
        const R rdzp = __ldg(zrdzp + k);
        const double dxd = g.dx, dyd = g.dy, dzd = ldz(g.z.dz, k);
        const int fa0 = rl0 * RS_AW + xl + 2;                  // own index in the x strip
        const int fb0 = (rl0 + 2) * RS_AW + xl + 2;            // own index in the uhy*vhx plane
        const int fv0 = (rl0 + 2) * RS_TX + xl;                // own index in the y strip
#pragma unroll
        for (int q = 0; q < RQ; ++q) {
            const int r = rc[q];
            // divergence of the incoming fields (FP64, the previous sub-step's check)
            R ux[6];
            ld6r(u0, r, ux);
            const R2 vc = ld2r(v0, r), vym = ld2r(v0, r - RS_W), vym2 = ld2r(v0, r - 2 * RS_W),
                         vy1 = ld2r(v0, r + RS_W);
            const R2 wc = ld2r(w0, r);
            if (a.part_div && act[q]) {
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const int c = 2 + s;
                    const double uc = ux[c], vcs = s ? vc.y : vc.x, wcs = s ? wc.y : wc.x;
                    double dux[4] = {(double)ux[c + 1], uc, (double)ux[c - 1], (double)ux[c - 2]};
                    double dvy[4] = {(double)(s ? vy1.y : vy1.x), vcs, (double)(s ? vym.y : vym.x),
                                     (double)(s ? vym2.y : vym2.x)};
                    const double d = fd_div_point<CDS>(dux, dvy, wcs, k > 0 ? (double)wm1[q][s] : 0.0, dxd, dyd, dzd);
                    if (uc != uc || vcs != vcs || wcs != wcs || d != d) dv_nan = 1;
                    else { dv_sum += fabs(d); dv_max = absmax_pick(dv_max, d); }
                }
            }
            R out_f[3][2], out_q[3][2];
            // ---------------- U ----------------
            {
                R px[6], fh[6];
                ld6r(p0, r, px);
                ld6r(F_UHX, fa0 + q * RS_AW, fh);
                const R2 uy2 = ld2r(u0, r + 2 * RS_W), uy1 = ld2r(u0, r + RS_W);
                const R2 uym = ld2r(u0, r - RS_W), uym2 = ld2r(u0, r - 2 * RS_W);
                const int fb = fb0 + q * RS_AW;
                const R2 b1 = ld2r(F_B, fb + RS_AW), b0 = ld2r(F_B, fb), bm = ld2r(F_B, fb - RS_AW),
                             bm2 = ld2r(F_B, fb - 2 * RS_AW);
                const R2 cz = ld2r(F_CZ, fa0 + q * RS_AW);
                const R2 uz1 = next_in ? ld2r(u1, r) : mk2<R>(R(0), R(0));
                const R2 bxq = a.bfx ? ld_own(a.bfx, q, 0) : mk2<R>(R(0), R(0));
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const int c = 2 + s;
                    const R uc = ux[c];
                    const R h2 = fh[c + 2], h1 = fh[c + 1], h0 = fh[c], hm = fh[c - 1];
                    const R uux = rs_d1<R, CDS>(h2 * h2, h1 * h1, h0 * h0, hm * hm) * sx1;
                    const R uvy = rs_d1<R, CDS>(s ? b1.y : b1.x, s ? b0.y : b0.x, s ? bm.y : bm.x, s ? bm2.y : bm2.x) * sy1;
                    const R uxx = rs_d2<R, CDS>(ux[c + 2], ux[c + 1], uc, ux[c - 1], ux[c - 2]) * sx2;
                    const R uyy = rs_d2<R, CDS>(s ? uy2.y : uy2.x, s ? uy1.y : uy1.x, uc, s ? uym.y : uym.x,
                                                 s ? uym2.y : uym2.x) * sy2;
                    const R dpdx = rs_d1<R, CDS>(px[c + 2], px[c + 1], px[c], px[c - 1]) * sx1;
                    const R czs = s ? cz.y : cz.x;
                    const R uwz = (czs - czp[q][s]) * rdz;
                    czp[q][s] = czs;
                    // above the last level: no-slip (closed) or free-slip (open) top
                    const R up = next_in ? (s ? uz1.y : uz1.x) : (closed ? -uc : uc);
                    const R uzz = ((up - uc) * rdzt - (uc - um1[q][s]) * rdzb) * rdz;
                    um1[q][s] = uc;
                    const R fu = -uux - uvy - uwz + dpx + (s ? bxq.y : bxq.x);
                    out_f[0][s] = fu;
                    out_q[0][s] = uc + dt * (rka * fu + rkb * (s ? hf[q].y : hf[q].x)) + cdif * (uxx + uyy + uzz) -
                                  cgp * dpdx;
                }
                if (act[q] && a.uhx_s)
                    *reinterpret_cast<R2*>(a.uhx_s + kofs + gid[q]) = mk2<R>(fh[2], fh[3]);
            }
            // ---------------- V ----------------
            {
                R vx[6], fbx[6];
                ld6r(v0, r, vx);
                ld6r(F_B, fb0 + q * RS_AW, fbx);
                const R2 vy2 = ld2r(v0, r + 2 * RS_W);
                const int fv = fv0 + q * RS_TX;
                const R2 hy2 = ld2r(F_VHY, fv + 2 * RS_TX), hy1 = ld2r(F_VHY, fv + RS_TX), hy0 = ld2r(F_VHY, fv),
                             hym = ld2r(F_VHY, fv - RS_TX);
                const R2 ez = ld2r(F_EZ, fv);
                const R2 pc = ld2r(p0, r), py2 = ld2r(p0, r + 2 * RS_W), py1 = ld2r(p0, r + RS_W),
                             pym = ld2r(p0, r - RS_W);
                const R2 vz1 = next_in ? ld2r(v1, r) : mk2<R>(R(0), R(0));
                const R2 byq = a.bfx ? ld_own(a.bfy, q, 0) : mk2<R>(R(0), R(0));
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const int c = 2 + s;
                    const R vcs = vx[c];
                    const R vux = rs_d1<R, CDS>(fbx[c + 1], fbx[c], fbx[c - 1], fbx[c - 2]) * sx1;
                    const R y2 = s ? hy2.y : hy2.x, y1 = s ? hy1.y : hy1.x, y0v = s ? hy0.y : hy0.x,
                                ym = s ? hym.y : hym.x;
                    const R vvy = rs_d1<R, CDS>(y2 * y2, y1 * y1, y0v * y0v, ym * ym) * sy1;
                    const R vxx = rs_d2<R, CDS>(vx[c + 2], vx[c + 1], vcs, vx[c - 1], vx[c - 2]) * sx2;
                    const R vyy = rs_d2<R, CDS>(s ? vy2.y : vy2.x, s ? vy1.y : vy1.x, vcs, s ? vym.y : vym.x,
                                                 s ? vym2.y : vym2.x) * sy2;
                    const R dpdy = rs_d1<R, CDS>(s ? py2.y : py2.x, s ? py1.y : py1.x, s ? pc.y : pc.x,
                                                  s ? pym.y : pym.x) * sy1;
                    const R ezs = s ? ez.y : ez.x;
                    const R vwz = (ezs - ezp[q][s]) * rdz;
                    ezp[q][s] = ezs;
                    const R vp = next_in ? (s ? vz1.y : vz1.x) : (closed ? -vcs : vcs);
                    const R vzz = ((vp - vcs) * rdzt - (vcs - vm1[q][s]) * rdzb) * rdz;
                    vm1[q][s] = vcs;
                    const R fv_ = -vux - vvy - vwz + (s ? byq.y : byq.x);
                    out_f[1][s] = fv_;
                    out_q[1][s] = vcs + dt * (rka * fv_ + rkb * (s ? hg[q].y : hg[q].x)) + cdif * (vxx + vyy + vzz) -
                                  cgp * dpdy;
                }
                if (act[q] && a.vhy_s)
                    *reinterpret_cast<R2*>(a.vhy_s + kofs + gid[q]) = hy0;
            }
            // ---------------- W (k <= nz-2) ----------------
            if (wface) {
                R wx[6], fcz[6];
                ld6r(w0, r, wx);
                ld6r(F_CZ, fa0 + q * RS_AW, fcz);
                const R2 wy2 = ld2r(w0, r + 2 * RS_W), wy1 = ld2r(w0, r + RS_W);
                const R2 wym = ld2r(w0, r - RS_W), wym2 = ld2r(w0, r - 2 * RS_W);
                const int fv = fv0 + q * RS_TX;
                const R2 e1 = ld2r(F_EZ, fv + RS_TX), e0 = ld2r(F_EZ, fv), em = ld2r(F_EZ, fv - RS_TX),
                             em2 = ld2r(F_EZ, fv - 2 * RS_TX);
                const R2 wz1 = ld2r(w1, r), pz1 = ld2r(p1, r), pc = ld2r(p0, r);
                const R2 bzq = a.bfx ? ld_own(a.bfz, q, 0) : mk2<R>(R(0), R(0));
                R2 tk = mk2<R>(R(0), R(0)), tk1 = tk;
                if (scalar) { tk = ld_own(a.f.t, q, 0); tk1 = ld_own(a.f.t, q, g.nxy); }
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const int c = 2 + s;
                    const R wcs = wx[c], wp = s ? wz1.y : wz1.x, wm = wm1[q][s];
                    const R wux = rs_d1<R, CDS>(fcz[c + 1], fcz[c], fcz[c - 1], fcz[c - 2]) * sx1;
                    const R wvy = rs_d1<R, CDS>(s ? e1.y : e1.x, s ? e0.y : e0.x, s ? em.y : em.x, s ? em2.y : em2.x) * sy1;
                    const R wxx = rs_d2<R, CDS>(wx[c + 2], wx[c + 1], wcs, wx[c - 1], wx[c - 2]) * sx2;
                    const R wyy = rs_d2<R, CDS>(s ? wy2.y : wy2.x, s ? wy1.y : wy1.x, wcs, s ? wym.y : wym.x,
                                                 s ? wym2.y : wym2.x) * sy2;
                    R a1 = R(0.5) * (wcs + wp); a1 = a1 * a1;
                    R a2 = R(0.5) * (wcs + wm); a2 = a2 * a2;
                    const R wwz = (a1 - a2) * rdzt;
                    const R wzz = ((wp - wcs) * rdzp - (wcs - wm) * rdz) * rdzt;
                    R fw = -wux - wvy - wwz;
                    if (scalar) fw = fw + got * ((R(1) - lt) * (s ? tk.y : tk.x) + lt * (s ? tk1.y : tk1.x) - tref);
                    fw += s ? bzq.y : bzq.x;
                    const R dpdz = ((s ? pz1.y : pz1.x) - (s ? pc.y : pc.x)) * rdzt;
                    out_f[2][s] = fw;
                    out_q[2][s] = wcs + dt * (rka * fw + rkb * (s ? hh[q].y : hh[q].x)) + cdif * (wxx + wyy + wzz) -
                                  cgp * dpdz;
                }
            }
#pragma unroll
            for (int s = 0; s < 2; ++s) wm1[q][s] = s ? wc.y : wc.x;
            if (act[q]) {
                const long long id = kofs + gid[q];
                *reinterpret_cast<R2*>(a.ff + id) = mk2<R>(out_f[0][0], out_f[0][1]);
                *reinterpret_cast<R2*>(a.qu + id) = mk2<R>(out_q[0][0], out_q[0][1]);
                *reinterpret_cast<R2*>(a.gg + id) = mk2<R>(out_f[1][0], out_f[1][1]);
                *reinterpret_cast<R2*>(a.qv + id) = mk2<R>(out_q[1][0], out_q[1][1]);
                if (wface) {
                    *reinterpret_cast<R2*>(a.hh + id) = mk2<R>(out_f[2][0], out_f[2][1]);
                    *reinterpret_cast<R2*>(a.qw + id) = mk2<R>(out_q[2][0], out_q[2][1]);
                }
            }
        }
        rs_wait_all();
        __syncthreads();
    }
    }   // segments

    if (a.part_div) {
        __shared__ double s_sum[NW], s_max[NW];
        __shared__ int s_nan;
        if (threadIdx.x == 0) s_nan = 0;
        __syncthreads();
        if (dv_nan) s_nan = 1;
        dv_sum = warp_sum(dv_sum);
        dv_max = warp_absmax(dv_max);
        if (lane == 0) { s_sum[wid] = dv_sum; s_max[wid] = dv_max; }
        __syncthreads();
        if (wid == 0) {
            dv_sum = lane < NW ? s_sum[lane] : 0.0;
            dv_max = lane < NW ? s_max[lane] : 0.0;
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
__global__ void __launch_bounds__(RsCfg<R>::NT, RsCfg<R>::MINB) k_rhs_momentum_strip(RhsTArgs<R> a) { k_rhs_momentum_strip_body<R, CDS>(a, blockIdx, gridDim); }

// ---------------------------------------------------------------------------
// Temperature right-hand side on strips (get_temperature_cnvdiff,
// src/module_cnvdiff.f90:381-473): the fluxes thx*u (x strip) and thy*v (y
// strip) are formed once per face from the staged planes of T, u and v of the
// level (a two-slot cp.async ring: level k+1 arrives while k is computed), and
// thz*w of the level below is carried in registers. T ghosts by formula: 2 tbot -
// T(0) below, 2 ttop - T(nz-1) above (update_boundary_t, src/module_boundary.f90:
// 176-183), thz = tbot / ttop at the walls where w = 0. Same tiles, threads and
// grid as the momentum strip kernel; no damping.
// ---------------------------------------------------------------------------
#define RT_F_THX 0                                   // [16][68] thx on the x strip
#define RT_F_FX (RT_F_THX + RS_TY * RS_AW)           // [16][68] thx*u on the x strip
#define RT_F_FY (RT_F_FX + RS_TY * RS_AW)            // [20][64] thy*v on the y strip
#define RT_NF (RT_F_FY + RS_BH * RS_TX)

template <typename R> __host__ inline size_t rhs_t_strip_smem() { return sizeof(R) * ((size_t)6 * RS_P + RT_NF); }

template <typename R, int CDS>
__device__ __forceinline__ void k_rhs_t_strip_body(const TempArgs<R>& m, const uint3 blockIdx, const dim3 gridDim)
{
    typedef typename V2<R>::T R2;
    constexpr int RQ = RsCfg<R>::RQ, NT = RsCfg<R>::NT, NW = RsCfg<R>::NW;
    constexpr int EPC = RsCfg<R>::EPC, NCH = RsCfg<R>::NCH, NPOS = RsCfg<R>::NPOS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* SR = reinterpret_cast<R*>(smem_raw);              // [3 fields: T, u, v][2 slots][RS_P]
    R* FL = SR + 6 * RS_P;
    R* F_THX = FL + RT_F_THX;
    R* F_FX = FL + RT_F_FX;
    R* F_FY = FL + RT_F_FY;
    const Acc<R>& A = m.a;
    const Geo& g = A.g;
    const int nz = g.nz, nx = g.nx, ny = g.ny;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int tiles_x = (nx + RS_TX - 1) / RS_TX;
    const long long ntiles = (long long)tiles_x * ((ny + RS_TY - 1) / RS_TY);
    const int kch = m.kchunk;
    const long long t = blockIdx.x % ntiles, c = blockIdx.x / ntiles;
    const int kb = (int)(c * kch), ke = min(nz, (int)((c + 1) * kch));
    const int x0 = (int)(t % tiles_x) * RS_TX, y0 = (int)(t / tiles_x) * RS_TY;
    const R* zrdz = (const R*)m.zm;
    const R* zrdzt = (const R*)m.zm + nz;
    const R* zrdzb = (const R*)m.zm + 2 * nz;
    const R* zlt = (const R*)m.zm + 3 * nz;
    auto plane = [&](int f, int lvl) { return SR + (f * 2 + (lvl & 1)) * RS_P; };

    const bool has1 = threadIdx.x + NT < NPOS;
    const int row0 = threadIdx.x / NCH, c40 = threadIdx.x - row0 * NCH;
    const int row1 = (threadIdx.x + NT) / NCH, c41 = threadIdx.x + NT - row1 * NCH;
    const int dst0 = row0 * RS_W + EPC * c40, dst1 = row1 * RS_W + EPC * c41;
    const int src0 = (((y0 - RS_HY + row0) % ny + ny) % ny) * nx + ((x0 - RS_HX + EPC * c40) % nx + nx) % nx;
    const int src1 = has1 ? (((y0 - RS_HY + row1) % ny + ny) % ny) * nx + ((x0 - RS_HX + EPC * c41) % nx + nx) % nx : 0;
    auto stage = [&](int lvl) {
#pragma unroll
        for (int f = 0; f < 3; ++f) {
            const R* src = f == 0 ? A.f.t : (f == 1 ? A.f.u : A.f.v);
            const R* base = src + (long long)lvl * g.nxy;
            R* d = plane(f, lvl);
            rs_cp16(d + dst0, base + src0);
            if (has1) rs_cp16(d + dst1, base + src1);
        }
    };
    stage(kb);
    rs_commit();
    rs_wait_all();
    __syncthreads();

    const R rdx = R(1) / (R)g.dx, rdy = R(1) / (R)g.dy;
    const R sx1 = CDS == 1 ? rdx : R(1) / (R(24) * (R)g.dx), sy1 = CDS == 1 ? rdy : R(1) / (R(24) * (R)g.dy);
    const R sx2 = CDS == 1 ? R(1) / (R)g.dx2 : R(1) / (R(12) * (R)g.dx2);
    const R sy2 = CDS == 1 ? R(1) / (R)g.dy2 : R(1) / (R(12) * (R)g.dy2);
    const R dt = (R)m.ph.dt, al = (R)m.ph.alpha, um = A.um;
    const R rka = (R)m.rk_a, rkb = (R)m.rk_b, cdif = (R)m.rk_c * R(0.5) * dt * al;
    const R tbs = A.tbs, tba = A.tba, ttop = A.ttop;
    const int xl = 2 * lane, rl0 = RQ * wid;
    const int xi = x0 + xl;
    bool act[2];
    int gid[2], rc[2];
#pragma unroll
    for (int q = 0; q < RQ; ++q) {
        act[q] = xi < nx && (y0 + rl0 + q) < ny;
        gid[q] = (y0 + rl0 + q) * nx + xi;
        rc[q] = (rl0 + q + RS_HY) * RS_W + xl + RS_HX;
    }
    auto ld_own = [&](const R* base, int q, long long ofs) {
        return act[q] ? *reinterpret_cast<const R2*>(base + ofs + gid[q]) : mk2<R>(R(0), R(0));
    };
    // level k-1 at the own points: T and thz*w (0 below the bottom wall, where w = 0)
    R tm1[2][2], fzp[2][2];
#pragma unroll
    for (int q = 0; q < RQ; ++q) {
        if (kb == 0) {
            const R2 tc = ld2r(plane(0, 0), rc[q]);
            tm1[q][0] = tbs * tc.x + tba; tm1[q][1] = tbs * tc.y + tba;
            fzp[q][0] = fzp[q][1] = R(0);
        } else {
            const long long o = (long long)(kb - 1) * g.nxy;
            const R2 ta = ld_own(A.f.t, q, o), tb = ld2r(plane(0, kb), rc[q]), wa = ld_own(A.f.w, q, o);
            const R l = zlt[kb - 1];
            tm1[q][0] = ta.x; tm1[q][1] = ta.y;
            fzp[q][0] = (tb.x * l + ta.x * (R(1) - l)) * wa.x;
            fzp[q][1] = (tb.y * l + ta.y * (R(1) - l)) * wa.y;
        }
    }

    for (int k = kb; k < ke; ++k) {
        if (k + 1 < ke) { stage(k + 1); rs_commit(); }
        const R* T0 = plane(0, k); const R* U0 = plane(1, k); const R* V0 = plane(2, k);
        const long long kofs = (long long)k * g.nxy;
        // own-point inputs: w(k), T(k+1), the history
        R2 wk[2], tp[2], s0[2];
#pragma unroll
        for (int q = 0; q < RQ; ++q) {
            wk[q] = ld_own(A.f.w, q, kofs);
            tp[q] = k + 1 < nz ? ld_own(A.f.t, q, kofs + g.nxy) : mk2<R>(R(0), R(0));
            s0[q] = ld_own(m.ss, q, kofs);
        }
        // ---- fluxes on their strips: 17 x-strip jobs (rows 0..15, then the side
        // pieces), 19 y-strip jobs (rows -2..16)
        for (int job = wid; job < 36; job += NW) {
            if (job <= 16) {
                int fx, fy;
                if (job < 16) { fx = 2 * lane; fy = job; }
                else { fy = lane & 15; fx = (lane >> 4) ? RS_TX : -2; }
                const int r = (fy + RS_HY) * RS_W + fx + RS_HX;
                R tx[6];
                ld6r(T0, r, tx);
                const R2 uc = ld2r(U0, r);
                const R h0 = rs_mid<R, CDS>(tx[4], tx[3], tx[2], tx[1]);
                const R h1 = rs_mid<R, CDS>(tx[5], tx[4], tx[3], tx[2]);
                const int ea = fy * RS_AW + fx + 2;
                st2r(F_THX, ea, h0, h1);
                st2r(F_FX, ea, h0 * uc.x, h1 * uc.y);
            } else {
                const int fx = 2 * lane, fy = job - 17 - 2;
                const int r = (fy + RS_HY) * RS_W + fx + RS_HX;
                const R2 tc = ld2r(T0, r), tym = ld2r(T0, r - RS_W), ty1 = ld2r(T0, r + RS_W), ty2 = ld2r(T0, r + 2 * RS_W);
                const R2 vc = ld2r(V0, r);
                st2r(F_FY, (fy + 2) * RS_TX + fx, rs_mid<R, CDS>(ty2.x, ty1.x, tc.x, tym.x) * vc.x,
                     rs_mid<R, CDS>(ty2.y, ty1.y, tc.y, tym.y) * vc.y);
            }
        }
        __syncthreads();
        const R rdz = zrdz[k], rdzt = zrdzt[k], rdzb = zrdzb[k], lt = zlt[k];
        const int fa0 = rl0 * RS_AW + xl + 2, fv0 = (rl0 + 2) * RS_TX + xl;
#pragma unroll
        for (int q = 0; q < RQ; ++q) {
            const int r = rc[q];
            R tx[6], fx6[6], hx6[6];
            ld6r(T0, r, tx);
            ld6r(F_FX, fa0 + q * RS_AW, fx6);
            if (um != R(0)) ld6r(F_THX, fa0 + q * RS_AW, hx6);
            const R2 ty2 = ld2r(T0, r + 2 * RS_W), ty1 = ld2r(T0, r + RS_W), tym = ld2r(T0, r - RS_W),
                     tym2 = ld2r(T0, r - 2 * RS_W);
            const int fv = fv0 + q * RS_TX;
            const R2 y1 = ld2r(F_FY, fv + RS_TX), y0v = ld2r(F_FY, fv), ym = ld2r(F_FY, fv - RS_TX),
                     ym2 = ld2r(F_FY, fv - 2 * RS_TX);
            R out_s[2], out_q[2];
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                const int c = 2 + s;
                const R tc = tx[c];
                const R tux = rs_d1<R, CDS>(fx6[c + 1], fx6[c], fx6[c - 1], fx6[c - 2]) * sx1;
                const R tvy = rs_d1<R, CDS>(s ? y1.y : y1.x, s ? y0v.y : y0v.x, s ? ym.y : ym.x, s ? ym2.y : ym2.x) * sy1;
                const R txx = rs_d2<R, CDS>(tx[c + 2], tx[c + 1], tc, tx[c - 1], tx[c - 2]) * sx2;
                const R tyy = rs_d2<R, CDS>(s ? ty2.y : ty2.x, s ? ty1.y : ty1.x, tc, s ? tym.y : tym.x,
                                            s ? tym2.y : tym2.x) * sy2;
                // thz*w at the top face of the level; 0 on the top wall (w = 0 there)
                const R tpv = k + 1 < nz ? (s ? tp[q].y : tp[q].x) : R(2) * ttop - tc;
                const R fz = k < nz - 1 ? (tpv * lt + tc * (R(1) - lt)) * (s ? wk[q].y : wk[q].x) : R(0);
                const R twz = (fz - fzp[q][s]) * rdz;
                fzp[q][s] = fz;
                const R tzz = ((tpv - tc) * rdzt - (tc - tm1[q][s]) * rdzb) * rdz;
                tm1[q][s] = tc;
                R sv = -tux - tvy - twz;
                if (um != R(0)) sv -= um * (rs_d1<R, CDS>(hx6[c + 1], hx6[c], hx6[c - 1], hx6[c - 2]) * sx1);
                out_s[s] = sv;
                out_q[s] = tc + dt * (rka * sv + rkb * (s ? s0[q].y : s0[q].x)) + cdif * (txx + tyy + tzz);
            }
            if (act[q]) {
                const long long id = kofs + gid[q];
                *reinterpret_cast<R2*>(m.ss + id) = mk2<R>(out_s[0], out_s[1]);
                *reinterpret_cast<R2*>(m.qt + id) = mk2<R>(out_q[0], out_q[1]);
            }
        }
        rs_wait_all();
        __syncthreads();
    }
}
template <typename R, int CDS>
__global__ void __launch_bounds__(RsCfg<R>::NT, RsCfg<R>::MINB) k_rhs_t_strip(TempArgs<R> m)
{
    k_rhs_t_strip_body<R, CDS>(m, blockIdx, gridDim);
}
