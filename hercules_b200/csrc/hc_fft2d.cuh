// hc_fft2d.cuh -- both halves of mpi_2d_fft (src/module_tools.f90:518-700) in one
// kernel per (field, plane): the x and y transforms meet in distributed shared
// memory instead of in HBM.
//
// The separate x and y kernels (hc_fft_t.cuh) write the half-transformed plane to
// HBM and read it back: per point and field a forward transform moves 4 words
// where the data itself needs 2 (a real value in, a half-spectrum value out), an
// inverse one 4 (5 with p += psi) where it needs 2 (3). Here a thread-block
// cluster of C CTAs holds one plane in its shared memory:
//   forward: CTA c transforms rows m in [c LX, (c+1) LX) along x (LX = ny / C) and
//            splits them into the nx/2 stored modes (scaled by 1/nx); after a
//            cluster barrier it transforms columns l in [c LY, (c+1) LY)
//            (LY = nx/2 / C) along y, its first pass reading every row from the
//            CTA that owns it (DSMEM loads), and writes the spectrum (scaled by
//            1/ny, Nyquist row zeroed);
//   inverse: CTA c transforms its columns along y (Nyquist row zeroed before);
//            after a barrier it gathers its rows from the other CTAs, applying the
//            c2r pre-split on the way, and after a second barrier (the columns it
//            read may be reused) transforms the rows along x and stores them (or
//            adds them, p += psi).
// The clusters are persistent: each takes the planes cl, cl + ncl, ... and, as it
// starts one plane, asks for the 128-byte lines of its next plane's HBM input
// (prefetch.global.L2), so those loads overlap the current plane's work (one
// plane a cluster in flight without it left the HBM idle between the phases: 30 %
// of the warps active, the cluster barriers dominating). A shared-memory staging
// buffer instead would need 152 KB a CTA at 512 x 384, and 16-CTA clusters of one
// CTA an SM do not fit a GPC. Both lengths must take exactly
// two Stockham passes of the compile-time plan. Same arithmetic as the separate
// kernels: the same passes, twiddle tables and split steps. Every CTA of a
// cluster takes the same planes and the same path through the barriers (the halt
// flag is read before the first one and is not written during the kernel).
#pragma once
#include <cooperative_groups.h>
#include "hc_fft_t.cuh"

template <typename R> struct F2Args {
    const void* in[HC_FFT_TMAXF];    // forward: physical fields; inverse: half spectra
    void* out[HC_FFT_TMAXF];         // forward: half spectra; inverse: physical fields
    int add[HC_FFT_TMAXF];           // inverse: 1 = out += result
    int nz, nplanes;                 // planes of a field; fields x nz
    const typename V2<R>::T* twx;    // exp(-2 pi i e / (nx/2))
    const typename V2<R>::T* wp;     // exp(-2 pi i l / nx)
    const typename V2<R>::T* twy;    // exp(-2 pi i e / ny)
    R scale_x, scale_y;              // forward: 1/nx, 1/ny
    const int* halt;
};

// Shape of a fused transform: NXH = nx/2 complex values a row, NY rows, C CTAs a
// cluster, NT threads a CTA, MINB resident CTAs an SM.
template <typename R, int NXH, int NY, int C, int NT, int MINB> struct F2Shape {
    typedef typename V2<R>::T T2;
    static constexpr int RMAX = 16;
    static constexpr int G = FPad<R>::G;
    static constexpr int LSX = FLine<NXH, G>::stride;
    static constexpr int LX = NY / C, LY = NXH / C;           // rows, columns a CTA
    // x buffers: row-major with padded rows; y buffers: element-major ([m][column]),
    // so that the lanes of a warp, which take consecutive columns, touch
    // consecutive words (column-major rows of 384 padded elements put 16 columns
    // on two bank offsets)
    static constexpr int BUF = LX * LSX > LY * NY ? LX * LSX : LY * NY;
    static constexpr size_t smem = (size_t)2 * BUF * sizeof(T2);
    typedef FPlan<NXH, RMAX> PX;
    typedef FPlan<NY, RMAX> PY;
    static_assert(NXH % C == 0 && NY % C == 0, "the cluster divides the plane");
    static_assert(PX::valid && PY::valid && PX::npass == 2 && PY::npass == 2, "two passes a direction");
    static_assert((LY * sizeof(T2)) % 128 == 0, "a CTA's column piece of a row is whole 128-byte lines");
};

// y buffer of a CTA: element e of its column `line` at b[e * LD + line]
template <typename T2, int LD> struct F2Cols {
    T2* b;
    __device__ __forceinline__ T2 ld(int line, int e) const { return b[e * LD + line]; }
    __device__ __forceinline__ void st(int line, int e, T2 v) const { b[e * LD + line] = v; }
};
// element m of column l0 + line, read from the CTA of the cluster that holds row m
// (its buffer in the x layout [row][padded l])
template <typename T2, int LX, int LSX, int G, int C> struct F2RemoteRows {
    T2* local; int l0;
    __device__ __forceinline__ T2 ld(int line, int e) const
    {
        const int own = e / LX;
        const T2* b = C > 1 ? cooperative_groups::this_cluster().map_shared_rank(local, own) : local;
        return b[(e - own * LX) * LSX + fpi<G>(l0 + line)];
    }
};

template <int C> __device__ __forceinline__ void f2_cluster_sync()
{
    if constexpr (C > 1) cooperative_groups::this_cluster().sync();
    else __syncthreads();
}

__device__ __forceinline__ void f2_prefetch_l2(const void* p)
{
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// forward: physical planes -> half spectra; ncl persistent clusters of C CTAs
template <typename R, int NXH, int NY, int C, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_fft2d_fwd(const __grid_constant__ F2Args<R> a)
{
    typedef F2Shape<R, NXH, NY, C, NT, MINB> S;
    typedef typename V2<R>::T T2;
    constexpr int G = S::G, LSX = S::LSX, LX = S::LX, LY = S::LY;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (a.halt && *a.halt) return;
    T2* P0 = reinterpret_cast<T2*>(smem_raw);
    T2* P1 = P0 + S::BUF;
    const int c = C > 1 ? (int)cooperative_groups::this_cluster().block_rank() : 0;
    const int cl = blockIdx.x / C, ncl = gridDim.x / C;
    const int m0 = c * LX, l0 = c * LY;
    for (int q = cl; q < a.nplanes; q += ncl) {
        const int f = q / a.nz, k = q - f * a.nz;
        if (q + ncl < a.nplanes) {
            // the CTA's LX rows of its next plane, contiguous in HBM
            const int fn = (q + ncl) / a.nz, kn = q + ncl - fn * a.nz;
            const char* nb = reinterpret_cast<const char*>(reinterpret_cast<const T2*>(a.in[fn]) + ((long long)kn * NY + m0) * NXH);
            for (int o = threadIdx.x * 128; o < LX * NXH * (int)sizeof(T2); o += NT * 128) f2_prefetch_l2(nb + o);
        }
        __syncthreads();
        // ---- x: rows m0.. of plane k, nx reals packed as NXH complex values
        const XRowsIn<T2, NXH> rows{reinterpret_cast<const T2*>(a.in[f]) + ((long long)k * NY + m0) * NXH, LX};
        const SmemIO<T2, LSX, G> x0{P0}, x1{P1};
        stock_pass<R, NXH, -1, S::PX::rad(0), S::PX::span(0), LX, NT, false>(rows, x0, a.twx);
        __syncthreads();
        stock_pass<R, NXH, -1, S::PX::rad(1), S::PX::span(1), LX, NT, false>(x0, x1, a.twx);
        __syncthreads();
        // split into the stored modes X(l) = E(l) - i W_l D(l), scaled by 1/nx, into P0
        const R sx = a.scale_x;
        for (int idx = threadIdx.x; idx < LX * NXH; idx += NT) {
            const int line = idx / NXH, l = idx - line * NXH;
            const T2 z = P1[line * LSX + fpi<G>(l)];
            T2 zc = P1[line * LSX + fpi<G>(l == 0 ? 0 : NXH - l)];
            zc.y = -zc.y;
            const T2 e = mk2<R>(R(0.5) * (z.x + zc.x), R(0.5) * (z.y + zc.y));
            const T2 dd = mk2<R>(R(0.5) * (z.x - zc.x), R(0.5) * (z.y - zc.y));
            const T2 wd = cmulc(__ldg(a.wp + l), dd);
            P0[line * LSX + fpi<G>(l)] = mk2<R>((e.x + wd.y) * sx, (e.y - wd.x) * sx);
        }
        // every CTA's modes are in place (P1 free: the split read it)
        f2_cluster_sync<C>();
        // ---- y: columns l0.. ; the first pass reads row m from the CTA that holds it
        const F2RemoteRows<T2, LX, LSX, G, C> cols{P0, l0};
        const F2Cols<T2, LY> y1{P1};
        stock_pass<R, NY, -1, S::PY::rad(0), S::PY::span(0), LY, NT, true>(cols, y1, a.twy);
        // no CTA reads another's P0 after this barrier (it also orders P1)
        f2_cluster_sync<C>();
        const YColsOut<R, NY, -1> dst{reinterpret_cast<T2*>(a.out[f]) + (long long)k * NY * NXH, l0, NXH, a.scale_y};
        stock_pass<R, NY, -1, S::PY::rad(1), S::PY::span(1), LY, NT, true>(y1, dst, a.twy);
    }
}

// inverse: half spectra -> physical planes (stored, or added with add[f])
template <typename R, int NXH, int NY, int C, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_fft2d_inv(const __grid_constant__ F2Args<R> a)
{
    typedef F2Shape<R, NXH, NY, C, NT, MINB> S;
    typedef typename V2<R>::T T2;
    constexpr int G = S::G, LSX = S::LSX, LX = S::LX, LY = S::LY;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (a.halt && *a.halt) return;
    T2* P0 = reinterpret_cast<T2*>(smem_raw);
    T2* P1 = P0 + S::BUF;
    const int c = C > 1 ? (int)cooperative_groups::this_cluster().block_rank() : 0;
    const int cl = blockIdx.x / C, ncl = gridDim.x / C;
    const int m0 = c * LX, l0 = c * LY;
    for (int q = cl; q < a.nplanes; q += ncl) {
        const int f = q / a.nz, k = q - f * a.nz;
        if (q + ncl < a.nplanes) {
            // the CTA's column piece of every row of its next plane (whole lines)
            const int fn = (q + ncl) / a.nz, kn = q + ncl - fn * a.nz;
            const T2* nb = reinterpret_cast<const T2*>(a.in[fn]) + (long long)kn * NY * NXH + l0;
            constexpr int LPR = LY * (int)sizeof(T2) / 128;         // lines a row piece
            for (int o = threadIdx.x; o < NY * LPR; o += NT) {
                const int e = o / LPR, ln = o - e * LPR;
                f2_prefetch_l2(reinterpret_cast<const char*>(nb + (long long)e * NXH) + 128 * ln);
            }
        }
        if (a.add[f]) {
            // the rows this CTA adds to (p += psi) are read only in the last pass:
            // bring their 128-byte lines into L2 now
            const char* pb = reinterpret_cast<const char*>(reinterpret_cast<const T2*>(a.out[f]) + ((long long)k * NY + m0) * NXH);
            for (int o = threadIdx.x * 128; o < LX * NXH * (int)sizeof(T2); o += NT * 128)
                asm volatile("prefetch.global.L2 [%0];" ::"l"(pb + o));
        }
        __syncthreads();
        // ---- y: columns l0.. of plane k (Nyquist row zeroed before), P0 -> P1
        const YColsIn<T2, NY, 1> src{reinterpret_cast<const T2*>(a.in[f]) + (long long)k * NY * NXH, l0, NXH};
        const F2Cols<T2, LY> y0{P0}, y1{P1};
        stock_pass<R, NY, 1, S::PY::rad(0), S::PY::span(0), LY, NT, true>(src, y0, a.twy);
        __syncthreads();
        stock_pass<R, NY, 1, S::PY::rad(1), S::PY::span(1), LY, NT, true>(y0, y1, a.twy);
        // every CTA's columns are in place
        f2_cluster_sync<C>();
        // ---- gather rows m0.. with the c2r pre-split
        //   Z(l) = (X(l) + conj X(N-l)) + i conj(W_l) (X(l) - conj X(N-l)),
        // the partner of l = 0 being the x Nyquist mode (zero, not stored); one item
        // per pair (l, N-l), all of a thread's loads issued before they are used
        auto ldx = [&](int line, int l) -> T2 {     // X(l) of row m0 + line
            const int own = l / LY;
            const T2* b = C > 1 ? cooperative_groups::this_cluster().map_shared_rank(P1, own) : P1;
            return b[(m0 + line) * LY + (l - own * LY)];
        };
        auto zsplit = [&](T2 a0, T2 b0, int ll) {
            T2 bc = b0; bc.y = -bc.y;
            T2 wc = __ldg(a.wp + ll);
            wc.y = -wc.y;
            const T2 s = cadd2(a0, bc);
            const T2 d = cmulc(wc, csub2(a0, bc));
            return mk2<R>(s.x - d.y, s.y + d.x);
        };
        constexpr int NP = NXH / 2 + 1;
        constexpr int ROUNDS = (LX * NP + NT - 1) / NT;
        {
            T2 xs[ROUNDS], ys[ROUNDS];
#pragma unroll
            for (int r = 0; r < ROUNDS; ++r) {
                const int idx = threadIdx.x + r * NT;
                const int line = idx / NP, l = idx - line * NP;
                xs[r] = mk2<R>(R(0), R(0));
                ys[r] = xs[r];
                if (idx < LX * NP) {
                    xs[r] = ldx(line, l);
                    if (l != 0) ys[r] = ldx(line, NXH - l);
                }
            }
#pragma unroll
            for (int r = 0; r < ROUNDS; ++r) {
                const int idx = threadIdx.x + r * NT;
                if (idx >= LX * NP) break;
                const int line = idx / NP, l = idx - line * NP;
                P0[line * LSX + fpi<G>(l)] = zsplit(xs[r], ys[r], l);
                if (l != 0 && 2 * l != NXH) P0[line * LSX + fpi<G>(NXH - l)] = zsplit(ys[r], xs[r], NXH - l);
            }
        }
        // no CTA reads another's P1 after this barrier (it also orders P0)
        f2_cluster_sync<C>();
        // ---- x: rows m0.., P0 -> P1 -> HBM
        const SmemIO<T2, LSX, G> x0{P0}, x1{P1};
        stock_pass<R, NXH, 1, S::PX::rad(0), S::PX::span(0), LX, NT, false>(x0, x1, a.twx);
        __syncthreads();
        const XRowsOut<T2, NXH> dst{reinterpret_cast<T2*>(a.out[f]) + ((long long)k * NY + m0) * NXH, LX, a.add[f]};
        stock_pass<R, NXH, 1, S::PX::rad(1), S::PX::span(1), LX, NT, false>(x1, dst, a.twx);
    }
}
