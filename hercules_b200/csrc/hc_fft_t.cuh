// hc_fft_t.cuh -- FFT kernels specialised at compile time on the transform length.
//
// Same transforms and conventions as hc_fft.cuh (mpi_2d_fft,
// src/module_tools.f90:518-700: forward e^{-i}, each direction divided by its
// length, y Nyquist zeroed, x Nyquist not stored), but for the common lengths the
// length N, the radix of every Stockham pass, the lines per block and all index
// arithmetic are template constants:
//   * radix-16 / 8 / 4 / 2 butterflies for the power-of-two part of N (split into
//     passes of at most RMAX points, as evenly as possible), then radix 3 and 5;
//     a radix-8 or radix-16 butterfly is itself a 2x4 / 4x4 Cooley-Tukey split
//     with constant inner twiddles, so a 256-point line needs two passes;
//   * every shared-memory index is padded by one slot per PADG elements, which
//     removes the bank conflicts of the strided stores of the first passes;
//   * twiddles come from a table in the storage precision (no FP64->FP32
//     conversions in the mixed-precision build).
#pragma once
#include "hc_fft.cuh"

#define HC_FFT_TMAXF 16

// ----------------------------------------------------------------------------
// compile-time plan
// ----------------------------------------------------------------------------
__host__ __device__ constexpr int fft_pow2_exp(int n) { return (n % 2 == 0) ? 1 + fft_pow2_exp(n / 2) : 0; }
__host__ __device__ constexpr int fft_exp_of(int n, int q) { return (n % q == 0) ? 1 + fft_exp_of(n / q, q) : 0; }
__host__ __device__ constexpr int fft_log2(int r) { return r <= 1 ? 0 : 1 + fft_log2(r / 2); }

// Passes: the power-of-two part in passes of at most RMAX points, as evenly as
// possible; one factor 3 folded with 8 or 4 of them into a radix-24 / radix-12
// pass (so 384 = 16 x 24 and 192 = 8 x 24 take two passes); remaining factors
// 3 and 5 as radix-3 / radix-5 passes. FF puts the folded pass first (any order
// of the radices is a valid Stockham plan; the spans follow the order).
template <int N, int RMAX, bool FF = false> struct FPlan {
    static constexpr int e2all = fft_pow2_exp(N);
    static constexpr int e3 = fft_exp_of(N, 3);
    static constexpr int e5 = fft_exp_of(N, 5);
    static constexpr int fold = e3 >= 1 ? (e2all >= 3 ? 3 : (e2all >= 2 ? 2 : 0)) : 0;   // 2^fold folded with a 3
    static constexpr int e2 = e2all - fold;
    static constexpr int bits = fft_log2(RMAX);
    static constexpr int q2 = (e2 + bits - 1) / bits;            // power-of-two passes
    static constexpr int qd = q2 > 0 ? q2 : 1;                   // divisor guard when there is no 2^k pass
    static constexpr int nfold = fold ? 1 : 0;
    static constexpr int npass = q2 + nfold + (e3 - nfold) + e5;
    static constexpr bool valid = (N == (1 << e2all) * (e3 == 0 ? 1 : (e3 == 1 ? 3 : (e3 == 2 ? 9 : 27))) *
                                           (e5 == 0 ? 1 : (e5 == 1 ? 5 : 25)));
    // radix of the p-th of the passes other than the folded one
    __host__ __device__ static constexpr int rest(int p)
    {
        return p < q2 ? (1 << (e2 / qd + (p < e2 % qd ? 1 : 0))) : (p < q2 + e3 - nfold ? 3 : 5);
    }
    __host__ __device__ static constexpr int rad(int p)
    {
        return FF && nfold ? (p == 0 ? (3 << fold) : rest(p - 1))
                           : (p < q2 ? rest(p) : (p < q2 + nfold ? (3 << fold) : rest(p - nfold)));
    }
    // product of the radices of passes 0..p-1 (the Stockham span Ns of pass p)
    __host__ __device__ static constexpr int span(int p) { return p == 0 ? 1 : span(p - 1) * rad(p - 1); }
    __host__ __device__ static constexpr int maxrad(int p = 0) { return p >= npass ? 1 : (rad(p) > maxrad(p + 1) ? rad(p) : maxrad(p + 1)); }
};

// padded shared-memory slot of element e of a line: one spare slot per G elements
template <int G> __device__ __forceinline__ int fpi(int e) { return e + e / G; }
template <int N, int G> struct FLine { static constexpr int stride = N + (N - 1) / G + 1; };
// 16-byte complex (double2): 8 per 128-byte wavefront; 8-byte (float2): 16
template <typename R> struct FPad { static constexpr int G = sizeof(R) == 8 ? 8 : 16; };

// ----------------------------------------------------------------------------
// butterflies with compile-time radix
// ----------------------------------------------------------------------------
// cos(2 pi e / 48) on the quarter wave e in [0, 12] (angles k x 7.5 degrees),
// exact values from sqrt(2), sqrt(3), sqrt(6) and half-angle identities
__host__ __device__ constexpr double cosq48(int e)
{
    return e == 0 ? 1.0 : e == 1 ? 0.991444861373810411145 : e == 2 ? 0.965925826289068286750
         : e == 3 ? 0.923879532511286756128 : e == 4 ? 0.866025403784438646764 : e == 5 ? 0.793353340291235164580
         : e == 6 ? 0.707106781186547524401 : e == 7 ? 0.608761429008720639416 : e == 8 ? 0.5
         : e == 9 ? 0.382683432365089771728 : e == 10 ? 0.258819045102520762349 : e == 11 ? 0.130526192220051591548
         : 0.0;
}
// cos and sin of 2 pi e / 48 for any e (reduced by quarter-wave symmetry)
__host__ __device__ constexpr double cos48(int e)
{
    return ((e % 48) + 48) % 48 <= 12 ? cosq48(((e % 48) + 48) % 48)
         : ((e % 48) + 48) % 48 <= 24 ? -cosq48(24 - ((e % 48) + 48) % 48)
         : ((e % 48) + 48) % 48 <= 36 ? -cosq48(((e % 48) + 48) % 48 - 24)
         : cosq48(48 - ((e % 48) + 48) % 48);
}
__host__ __device__ constexpr double sin48(int e) { return cos48(e - 12); }

// v * exp(S 2 pi i E / M) for M dividing 48 (4, 8, 12, 16, 24); E compile-time
template <int M, int E, int S, typename T2> __device__ __forceinline__ T2 twc(T2 v)
{
    static_assert(48 % M == 0, "constant twiddles cover divisors of 48");
    constexpr int e = (E * (48 / M)) % 48;
    typedef decltype(v.x) R;
    if (e == 0) return v;
    if (e == 24) { T2 r; r.x = -v.x; r.y = -v.y; return r; }
    if (e == 12) return mul_si<S>(v);                // exp(S i pi/2) = S i
    if (e == 36) return mul_si<-S>(v);
    const R c = (R)cos48(e), s = (R)(S * sin48(e));
    T2 r; r.x = v.x * c - v.y * s; r.y = v.x * s + v.y * c; return r;
}

template <int RAD, int S, typename T2> struct Dft;

template <int S, typename T2> struct Dft<2, S, T2> {
    static __device__ __forceinline__ void run(T2* v) { T2 a = v[0], b = v[1]; v[0] = cadd2(a, b); v[1] = csub2(a, b); }
};
template <int S, typename T2> struct Dft<4, S, T2> {
    static __device__ __forceinline__ void run(T2* v)
    {
        T2 s02 = cadd2(v[0], v[2]), d02 = csub2(v[0], v[2]);
        T2 s13 = cadd2(v[1], v[3]), d13 = mul_si<S>(csub2(v[1], v[3]));
        v[0] = cadd2(s02, s13); v[1] = cadd2(d02, d13); v[2] = csub2(s02, s13); v[3] = csub2(d02, d13);
    }
};
template <int S, typename T2> struct Dft<3, S, T2> {
    static __device__ __forceinline__ void run(T2* v) { dft_small<decltype(v[0].x), S>(v, 3); }
};
template <int S, typename T2> struct Dft<5, S, T2> {
    static __device__ __forceinline__ void run(T2* v) { dft_small<decltype(v[0].x), S>(v, 5); }
};

// y[n2 N1 + k1] *= w_M^{n2 k1}, unrolled so that every exponent is a constant
template <int N1, int M, int S, int I, typename T2> __device__ __forceinline__ void tw_split(T2* y)
{
    if constexpr (I < M) {
        y[I] = twc<M, (I / N1) * (I % N1), S>(y[I]);
        tw_split<N1, M, S, I + 1>(y);
    }
}

// DFT of size N1*N2 by one Cooley-Tukey split (n = N2 n1 + n2, k = k1 + N1 k2):
// N2 inner DFTs of size N1, the twiddles w^{n2 k1}, N1 outer DFTs of size N2.
template <int N1, int N2, int S, typename T2> __device__ __forceinline__ void dft_split(T2* v)
{
    constexpr int M = N1 * N2;
    T2 y[M];
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) {
        T2 t[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) t[n1] = v[N2 * n1 + n2];
        Dft<N1, S, T2>::run(t);
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) y[n2 * N1 + k1] = t[k1];
    }
    tw_split<N1, M, S, 0>(y);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) {
        T2 t[N2];
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) t[n2] = y[n2 * N1 + k1];
        Dft<N2, S, T2>::run(t);
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) v[k1 + N1 * k2] = t[k2];
    }
}
template <int S, typename T2> struct Dft<8, S, T2> {
    static __device__ __forceinline__ void run(T2* v) { dft_split<2, 4, S>(v); }
};
template <int S, typename T2> struct Dft<16, S, T2> {
    static __device__ __forceinline__ void run(T2* v) { dft_split<4, 4, S>(v); }
};
template <int S, typename T2> struct Dft<12, S, T2> {
    static __device__ __forceinline__ void run(T2* v) { dft_split<4, 3, S>(v); }
};
template <int S, typename T2> struct Dft<24, S, T2> {
    static __device__ __forceinline__ void run(T2* v) { dft_split<8, 3, S>(v); }
};

// ----------------------------------------------------------------------------
// Stockham passes over LINES lines of length N
// ----------------------------------------------------------------------------
// One pass of radix RAD with span NS: item j of a line reads element j + r N/RAD
// (r < RAD), multiplies by w^{r k N/(NS RAD)} (k = j mod NS), transforms, and
// writes element (j/NS) NS RAD + k + r NS. The first pass's reads and the last
// pass's writes walk consecutive elements with consecutive items, so those two
// passes read and write global memory directly; only the passes in between go
// through shared memory. SRC::ld(line, e) and DST::st(line, e, v) are the
// element accessors; LMINOR maps consecutive threads to consecutive lines
// (y direction, whose lines are the strided columns) instead of consecutive
// elements of one line (x direction).
template <typename T2, int LS, int G> struct SmemIO {
    T2* b;
    __device__ __forceinline__ T2 ld(int line, int e) const { return b[line * LS + fpi<G>(e)]; }
    __device__ __forceinline__ void st(int line, int e, T2 v) const { b[line * LS + fpi<G>(e)] = v; }
};

template <typename R, int N, int S, int RAD, int NS, int LINES, int NT, bool LMINOR, class SRC, class DST>
__device__ __forceinline__ void stock_pass(const SRC& src, const DST& dst, const typename V2<R>::T* __restrict__ tw)
{
    typedef typename V2<R>::T T2;
    constexpr int NR = N / RAD;
    constexpr int TS = N / (NS * RAD);
    for (int it = threadIdx.x; it < LINES * NR; it += NT) {
        int line, j;
        if (LMINOR) { j = it / LINES; line = it - j * LINES; }
        else { line = it / NR; j = it - line * NR; }
        const int k = NS == 1 ? 0 : j % NS;
        T2 v[RAD];
#pragma unroll
        for (int r = 0; r < RAD; ++r) {
            T2 x = src.ld(line, j + r * NR);
            if (NS > 1 && r > 0) {
                T2 w = __ldg(tw + r * k * TS);
                if (S > 0) w.y = -w.y;
                x = cmulc(x, w);
            }
            v[r] = x;
        }
        Dft<RAD, S, T2>::run(v);
        const int base = (j / NS) * NS * RAD + k;
#pragma unroll
        for (int r = 0; r < RAD; ++r) dst.st(line, base + r * NS, v[r]);
    }
}

// Passes P..npass-1. Pass P reads SRC; passes after the first read shared
// buffer A (ping-pong with B); the last pass writes DST. Every pass but the last
// ends with a barrier.
// LSO: the shared lines' stride (0: FLine's).
template <typename R, int N, int S, int RMAX, int LINES, int NT, bool LMINOR, int P, bool FF = false, int LSO = 0,
          class SRC, class DST>
__device__ __forceinline__ void run_passes(const SRC& src, const DST& dst, typename V2<R>::T* A, typename V2<R>::T* B,
                                           const typename V2<R>::T* tw)
{
    typedef FPlan<N, RMAX, FF> PL;
    typedef typename V2<R>::T T2;
    constexpr int G = FPad<R>::G, LS = LSO ? LSO : FLine<N, G>::stride;
    if constexpr (P == PL::npass - 1) {
        stock_pass<R, N, S, PL::rad(P), PL::span(P), LINES, NT, LMINOR>(src, dst, tw);
    } else {
        const SmemIO<T2, LS, G> out{A};
        stock_pass<R, N, S, PL::rad(P), PL::span(P), LINES, NT, LMINOR>(src, out, tw);
        __syncthreads();
        const SmemIO<T2, LS, G> in{A};
        run_passes<R, N, S, RMAX, LINES, NT, LMINOR, P + 1, FF, LSO>(in, dst, B, A, tw);
    }
}

// Shared line buffers per kernel. y: one between two passes, two (ping-pong)
// from three passes on, one staging buffer for an in-place single pass. x: the
// split step's buffer plus at most one more, reused in turn by the passes.
template <int N, int RMAX> struct FBufs {
    static constexpr int np = FPlan<N, RMAX>::npass;
    static constexpr int y = np >= 3 ? 2 : 1;
    static constexpr int x = np >= 2 ? 2 : 1;
};

// ----------------------------------------------------------------------------
// kernel arguments
// ----------------------------------------------------------------------------
template <typename R> struct FxArgs {
    const void* in[HC_FFT_TMAXF];
    void* out[HC_FFT_TMAXF];
    int add[HC_FFT_TMAXF];           // inverse only: 1 = out += result
    long long nrows;                 // ny*nz rows of nx reals
    const typename V2<R>::T* tw;     // exp(-2 pi i e / N), e < N = nx/2
    const typename V2<R>::T* wp;     // exp(-2 pi i l / nx), l < nx/2
    R scale;                         // forward: 1/nx
    const int* halt;
};

template <typename R> struct FyArgs {
    const typename V2<R>::T* src[HC_FFT_TMAXF];   // null: transform dst in place
    typename V2<R>::T* dst[HC_FFT_TMAXF];
    int nxh;
    const typename V2<R>::T* tw;     // exp(-2 pi i e / ny), e < ny
    R scale;                         // forward: 1/ny
    const int* halt;
};

// x: 1024 complex values (at least one line) per block of 128 threads (against
// 2048 values with 256 threads: FP32 c2r 488 -> 463 us at 512 x 384 x 256, 4
// fields; FP64 r2c 179 -> 164 us and c2r 116 -> 106 us at 256 x 256 x 128;
// 2048 values with 128 threads, or 1024 with 64, were slower)
template <typename R, int N> struct FxLines { static constexpr int v = N >= 1024 ? 1 : 1024 / N; };
template <typename R, int N> struct FxThreads { static constexpr int v = 128; };
#define HC_FFT_NT 256
// y: tiles of 8 columns with 16 threads a column (64-byte row segments in FP32,
// 128 in FP64), 4 columns for 256-point columns; below 64 points 8 columns with
// 256 threads. Narrower tiles keep more, smaller blocks resident: against 16
// columns with 256 threads, at 512 x 384 x 256 (3 and 4 fields) FP32 forward
// 359 -> 322 us and inverse 480 -> 423 us, FP64 inverse 1034 -> 987 us;
// 256-point columns (256 x 256 x 128 spectral, 4 columns) FP32 194 -> 105 and
// 132 -> 75 us, FP64 244 -> 177 and 169 -> 122 us. 32 columns with 512 threads
// were slower (404 and 525 us), and 4 columns of 384 points too (417 and 553 us).
template <typename R, int N> struct FyLines {
    static constexpr int v = N >= 64 ? (N == 256 ? 4 : 8) : 8;
};
template <typename R, int N> struct FyThreads { static constexpr int v = N >= 64 ? FyLines<R, N>::v * 16 : HC_FFT_NT; };

template <typename R, int N, int RMAX> __host__ __device__ constexpr size_t fft_x_smem()
{
    return (size_t)FBufs<N, RMAX>::x * FxLines<R, N>::v * FLine<N, FPad<R>::G>::stride * sizeof(typename V2<R>::T);
}
// y tiles in FP32 put the folded pass first where the other order would start
// with a pass of fewer than 16 points: 192 = 24 x 8 then reads 24 elements a
// thread in one round instead of 8 elements in 1.5 rounds (forward 85 -> 70 us,
// inverse 107 -> 97 us at 256 x 192 x 256, 3 and 4 fields). 384 = 16 x 24 keeps
// radix 16 first: radix 24 first gained nothing forward and spilled inverse
// there, and in FP64 it was slower in both directions.
template <typename R, int N, int RMAX> struct FyFoldFirst {
    typedef FPlan<N, RMAX> PL;
    static constexpr bool v = sizeof(R) == sizeof(float) && PL::nfold == 1 && PL::rad(0) < 16;
};

// Shared-memory wavefronts of one warp's access to elements at a[0..31] (-1: lane
// idle) of W per 128 bytes: the most distinct elements that fall on one of the W
// bank groups (8-byte elements: 16 groups of two banks; 16-byte: 8 of four).
template <int W> __host__ __device__ constexpr int f_wavefronts(const int (&a)[32])
{
    int cnt[W] = {};
    for (int l = 0; l < 32; ++l) {
        if (a[l] < 0) continue;
        bool first = true;
        for (int t = 0; t < l; ++t)
            if (a[t] == a[l]) first = false;
        if (first) ++cnt[a[l] % W];
    }
    int m = 0;
    for (int q = 0; q < W; ++q) m = cnt[q] > m ? cnt[q] : m;
    return m;
}
// Wavefronts of the first warp's shared-memory reads and writes over the plan's
// passes (radix slots r = 0, 1; the others repeat them shifted) for y lines of
// stride LS: consecutive lanes take consecutive lines, then the next item
// (stock_pass with LMINOR); padded index e + e / G.
template <int N, int RMAX, bool FF, int LINES, int G, int W> __host__ __device__ constexpr int f_ycost(int LS)
{
    typedef FPlan<N, RMAX, FF> PL;
    int cost = 0;
    for (int p = 0; p < PL::npass; ++p) {
        const int RAD = PL::rad(p), NS = PL::span(p), NR = N / RAD;
        for (int r = 0; r < 2 && r < RAD; ++r) {
            int rd[32] = {}, wr[32] = {};
            for (int it = 0; it < 32; ++it) {
                const int j = it / LINES, line = it % LINES;
                if (j >= NR) { rd[it] = -1; wr[it] = -1; continue; }
                const int er = j + r * NR;
                const int ew = (j / NS) * NS * RAD + (NS == 1 ? 0 : j % NS) + r * NS;
                rd[it] = line * LS + er + er / G;
                wr[it] = line * LS + ew + ew / G;
            }
            if (p > 0) cost += f_wavefronts<W>(rd);
            if (p < PL::npass - 1) cost += f_wavefronts<W>(wr);
        }
    }
    return cost;
}
// y line stride: FLine's stride plus the pad in [0, W) with the fewest
// wavefronts. With FLine's own stride (408 for 384 FP32 points) the 8 lines a warp
// touches sit on two bank offsets and every access of the passes is 4-way
// conflicted (8-way in FP64).
template <typename R, int N, int RMAX> struct FyStride {
    static constexpr int G = FPad<R>::G, W = 128 / (2 * (int)sizeof(R)), base = FLine<N, G>::stride;
    static constexpr int LINES = FyLines<R, N>::v;
    static constexpr bool FF = FyFoldFirst<R, N, RMAX>::v;
    static constexpr int pick()
    {
        int best = 0, bc = 1 << 30;
        for (int q = 0; q < W; ++q) {
            const int c = f_ycost<N, RMAX, FF, LINES, G, W>(base + q);
            if (c < bc) { bc = c; best = q; }
        }
        return base + best;
    }
    static constexpr int v = pick();
};

template <typename R, int N, int RMAX> __host__ __device__ constexpr size_t fft_y_smem()
{
    return (size_t)FBufs<N, RMAX>::y * FyLines<R, N>::v * FyStride<R, N, RMAX>::v * sizeof(typename V2<R>::T);
}
// y kernels in FP32: registers sized for as many resident blocks as the shared
// memory allows, at 64 registers a thread at least (1024 threads an SM)
template <typename R, int N, int RMAX> struct FyMinBlocks {
    static constexpr int bysmem = (int)((227 * 1024) / (fft_y_smem<R, N, RMAX>() + 1024));
    static constexpr int byreg = 4 * HC_FFT_NT / FyThreads<R, N>::v;
    static constexpr int v = bysmem < 1 ? 1 : (bysmem > byreg ? byreg : bysmem);
};

// ---- global accessors -------------------------------------------------------
template <typename T2, int N> struct XRowsIn {       // rows row0.., zero past the last
    const T2* in; int nr;
    __device__ __forceinline__ T2 ld(int line, int e) const
    {
        if (line < nr) return in[(long long)line * N + e];
        T2 z; z.x = 0; z.y = 0; return z;
    }
};
template <typename T2, int N> struct XRowsOut {      // c2r result, stored or added
    T2* out; int nr; int add;
    __device__ __forceinline__ void st(int line, int e, T2 v) const
    {
        if (line >= nr) return;
        T2* p = out + (long long)line * N + e;
        if (add) { const T2 o = *p; v.x += o.x; v.y += o.y; }
        *p = v;
    }
};
template <typename T2, int N, int S> struct YColsIn {   // column l0+line of one plane
    const T2* s; int l0, nxh;
    __device__ __forceinline__ T2 ld(int line, int e) const
    {
        const int l = l0 + line;
        T2 z; z.x = 0; z.y = 0;
        if (l >= nxh || (S > 0 && e == N / 2)) return z;   // inverse: Nyquist zeroed before
        return s[(long long)e * nxh + l];
    }
};
template <typename R, int N, int S> struct YColsOut {
    typedef typename V2<R>::T T2;
    T2* d; int l0, nxh; R sc;
    __device__ __forceinline__ void st(int line, int e, T2 v) const
    {
        const int l = l0 + line;
        if (l >= nxh) return;
        if (S < 0) {                                       // forward: 1/ny, Nyquist zeroed after
            v.x *= sc; v.y *= sc;
            if (e == N / 2) { v.x = 0; v.y = 0; }
        }
        d[(long long)e * nxh + l] = v;
    }
};

// ----------------------------------------------------------------------------
// x direction, forward: real rows -> nx/2 modes, divided by nx
// ----------------------------------------------------------------------------
template <typename R, int N, int RMAX>
__device__ __forceinline__ void k_fft_x_r2c_t_body(const FxArgs<R>& a, const uint3 blockIdx, const dim3 gridDim)
{
    constexpr int NTX = FxThreads<R, N>::v;
    typedef typename V2<R>::T T2;
    constexpr int G = FPad<R>::G, LS = FLine<N, G>::stride, L = FxLines<R, N>::v;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (a.halt && *a.halt) return;
    // pass q (not the last) writes A for even q, B for odd q; the last pass lands
    // in the buffer it does not read, where the split step finds it
    T2* A = reinterpret_cast<T2*>(smem_raw);
    T2* B = A + (FBufs<N, RMAX>::x >= 2 ? L * LS : 0);
    const int f = blockIdx.y;
    const long long row0 = (long long)blockIdx.x * L;
    const int nr = (int)min((long long)L, a.nrows - row0);
    const XRowsIn<T2, N> src{reinterpret_cast<const T2*>(a.in[f]) + row0 * N, nr};
    // the last pass lands in the shared buffer the split step reads
    constexpr int np = FPlan<N, RMAX>::npass;
    T2* Z = (np % 2 == 1) ? A : B;
    const SmemIO<T2, LS, G> zout{Z};
    run_passes<R, N, -1, RMAX, L, NTX, false, 0>(src, zout, A, B, a.tw);
    __syncthreads();
    T2* out = reinterpret_cast<T2*>(a.out[f]) + row0 * N;
    const R sc = a.scale;
    for (int idx = threadIdx.x; idx < nr * N; idx += NTX) {
        const int line = idx / N, l = idx - line * N;
        const T2 z = Z[line * LS + fpi<G>(l)];
        T2 zc = Z[line * LS + fpi<G>(l == 0 ? 0 : N - l)];
        zc.y = -zc.y;
        const T2 e = mk2<R>(R(0.5) * (z.x + zc.x), R(0.5) * (z.y + zc.y));
        const T2 dd = mk2<R>(R(0.5) * (z.x - zc.x), R(0.5) * (z.y - zc.y));
        const T2 wd = cmulc(__ldg(a.wp + l), dd);          // X = E - i W D
        out[idx] = mk2<R>((e.x + wd.y) * sc, (e.y - wd.x) * sc);
    }
}
template <typename R, int N, int RMAX>
__global__ void __launch_bounds__(FxThreads<R, N>::v) k_fft_x_r2c_t(FxArgs<R> a) { k_fft_x_r2c_t_body<R, N, RMAX>(a, blockIdx, gridDim); }

// ----------------------------------------------------------------------------
// x direction, inverse: nx/2 modes -> real rows (unnormalised), stored or added
// ----------------------------------------------------------------------------
template <typename R, int N, int RMAX>
__device__ __forceinline__ void k_fft_x_c2r_t_body(const FxArgs<R>& a, const uint3 blockIdx, const dim3 gridDim)
{
    constexpr int NTX = FxThreads<R, N>::v;
    typedef typename V2<R>::T T2;
    constexpr int G = FPad<R>::G, LS = FLine<N, G>::stride, L = FxLines<R, N>::v;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (a.halt && *a.halt) return;
    // the pre-split lines Zs feed pass 0; later passes alternate A and Zs
    T2* Zs = reinterpret_cast<T2*>(smem_raw);
    T2* A = Zs + (FBufs<N, RMAX>::x >= 2 ? L * LS : 0);
    T2* B = Zs;
    const int f = blockIdx.y;
    const long long row0 = (long long)blockIdx.x * L;
    const int nr = (int)min((long long)L, a.nrows - row0);
    const T2* in = reinterpret_cast<const T2*>(a.in[f]) + row0 * N;
    if (a.add[f]) {
        // the rows this block adds to (p += psi) are read only in the last pass:
        // bring their 128-byte lines into L2 now, so that read does not wait on HBM
        const char* pb = reinterpret_cast<const char*>(reinterpret_cast<const T2*>(a.out[f]) + row0 * N);
        const int nbytes = nr * N * (int)sizeof(T2);
        for (int o = threadIdx.x * 128; o < nbytes; o += NTX * 128)
            asm volatile("prefetch.global.L2 [%0];" ::"l"(pb + o));
    }
    // pre-split straight from global: Z(l) = (X(l) + conj X(N-l)) + i conj(W_l) (X(l) - conj X(N-l));
    // the partner of l = 0 is the x Nyquist mode (zero, not stored). FP32: one
    // thread per pair (l, N-l), so every mode is read once.
    auto zsplit = [&](T2 a0, T2 b0, int ll) {               // a0 = X(ll), b0 = X(N-ll)
        T2 bc = b0; bc.y = -bc.y;
        T2 wc = __ldg(a.wp + ll);
        wc.y = -wc.y;
        const T2 s = cadd2(a0, bc);
        const T2 d = cmulc(wc, csub2(a0, bc));
        return mk2<R>(s.x - d.y, s.y + d.x);                   // s + i d
    };
    if constexpr (sizeof(R) == 8) {
        // FP64: one thread per mode, the partner read again; the loads of four
        // modes are issued before any of them is split
        constexpr int IT = (L * N + NTX - 1) / NTX;
#pragma unroll
        for (int q0 = 0; q0 < IT; q0 += 4) {
            T2 xs[4], ys[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int idx = threadIdx.x + (q0 + q) * NTX;
                const int line = idx / N, l = idx - line * N;
                xs[q] = mk2<R>(R(0), R(0));
                ys[q] = xs[q];
                if (q0 + q < IT && idx < L * N && line < nr) {
                    xs[q] = in[(long long)line * N + l];
                    if (l != 0) ys[q] = in[(long long)line * N + N - l];
                }
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int idx = threadIdx.x + (q0 + q) * NTX;
                if (q0 + q >= IT || idx >= L * N) break;
                const int line = idx / N, l = idx - line * N;
                Zs[line * LS + fpi<G>(l)] = zsplit(xs[q], ys[q], l);
            }
        }
        __syncthreads();
        const SmemIO<T2, LS, G> src64{Zs};
        const XRowsOut<T2, N> dst64{reinterpret_cast<T2*>(a.out[f]) + row0 * N, nr, a.add[f]};
        run_passes<R, N, 1, RMAX, L, NTX, false, 0>(src64, dst64, A, B, a.tw);
        return;
    }
    // all of a thread's pairs are loaded before any is used, so the loads overlap
    constexpr int NP = N / 2 + 1;
    constexpr int ROUNDS = (L * NP + NTX - 1) / NTX;
    T2 xs[ROUNDS], ys[ROUNDS];
#pragma unroll
    for (int q = 0; q < ROUNDS; ++q) {
        const int idx = threadIdx.x + q * NTX;
        const int line = idx / NP, l = idx - line * NP;
        xs[q] = mk2<R>(R(0), R(0));
        ys[q] = xs[q];
        if (idx < L * NP && line < nr) {
            xs[q] = in[(long long)line * N + l];
            if (l != 0) ys[q] = in[(long long)line * N + N - l];
        }
    }
#pragma unroll
    for (int q = 0; q < ROUNDS; ++q) {
        const int idx = threadIdx.x + q * NTX;
        if (idx >= L * NP) break;
        const int line = idx / NP, l = idx - line * NP;
        Zs[line * LS + fpi<G>(l)] = zsplit(xs[q], ys[q], l);
        if (l != 0 && 2 * l != N) Zs[line * LS + fpi<G>(N - l)] = zsplit(ys[q], xs[q], N - l);
    }
    __syncthreads();
    const SmemIO<T2, LS, G> src{Zs};
    const XRowsOut<T2, N> dst{reinterpret_cast<T2*>(a.out[f]) + row0 * N, nr, a.add[f]};
    run_passes<R, N, 1, RMAX, L, NTX, false, 0>(src, dst, A, B, a.tw);
}
template <typename R, int N, int RMAX>
__global__ void __launch_bounds__(FxThreads<R, N>::v) k_fft_x_c2r_t(FxArgs<R> a) { k_fft_x_c2r_t_body<R, N, RMAX>(a, blockIdx, gridDim); }

// ----------------------------------------------------------------------------
// y direction on the half spectrum [k][m][l]: tiles of FyLines<R, N> columns l of
// one plane k; grid (ceil(nxh/TL), nz, fields)
// ----------------------------------------------------------------------------
template <typename R, int N, int S, int RMAX>
__device__ __forceinline__ void fft_y_tile(const FyArgs<R>& a, const uint3 blockIdx)
{
    typedef typename V2<R>::T T2;
    constexpr int G = FPad<R>::G, LS = FyStride<R, N, RMAX>::v, TL = FyLines<R, N>::v, NT = FyThreads<R, N>::v;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (a.halt && *a.halt) return;
    T2* A = reinterpret_cast<T2*>(smem_raw);
    T2* B = A + (FBufs<N, RMAX>::y >= 2 ? TL * LS : 0);
    const int l0 = blockIdx.x * TL;
    const long long plane = (long long)blockIdx.y * N * a.nxh;
    T2* d = a.dst[blockIdx.z] + plane;
    const T2* s = a.src[blockIdx.z] ? a.src[blockIdx.z] + plane : d;
    const YColsIn<T2, N, S> src{s, l0, a.nxh};
    const YColsOut<R, N, S> dst{d, l0, a.nxh, a.scale};
    if constexpr (FPlan<N, RMAX>::npass == 1) {
        // one pass: in place is safe only through a barrier between reads and writes
        if (s == d) {
            const SmemIO<T2, LS, G> stage{A};
            for (int idx = threadIdx.x; idx < TL * N; idx += NT) {
                const int m = idx / TL, lt = idx - m * TL;
                stage.st(lt, m, src.ld(lt, m));
            }
            __syncthreads();
            stock_pass<R, N, S, FPlan<N, RMAX>::rad(0), 1, TL, NT, true>(stage, dst, a.tw);
            return;
        }
    }
    // in place (s == d) with two or more passes: the first pass reads every
    // element of the tile before its barrier, and only the last pass writes it
    run_passes<R, N, S, RMAX, TL, NT, true, 0, FyFoldFirst<R, N, RMAX>::v, LS>(src, dst, A, B, a.tw);
}

template <typename R, int N, int S, int RMAX>
__device__ __forceinline__ void k_fft_y_t_body(const FyArgs<R>& a, const uint3 blockIdx, const dim3 gridDim)
{
    fft_y_tile<R, N, S, RMAX>(a, blockIdx);
}
// FP64: the compiler's own register budget
template <typename R, int N, int S, int RMAX>
__global__ void __launch_bounds__(FyThreads<R, N>::v) k_fft_y_t(FyArgs<R> a) { k_fft_y_t_body<R, N, S, RMAX>(a, blockIdx, gridDim); }
// FP32: registers sized for FyMinBlocks resident blocks
template <int N, int S, int RMAX>
__global__ void __launch_bounds__(FyThreads<float, N>::v, FyMinBlocks<float, N, RMAX>::v) k_fft_y_t32(FyArgs<float> a)
{
    k_fft_y_t_body<float, N, S, RMAX>(a, blockIdx, gridDim);
}
// the y kernel of a length and its launch bounds (threads, resident blocks)
template <typename R, int N, int S, int RMAX> struct FyKernel {
    static constexpr void (*f)(FyArgs<R>) = k_fft_y_t<R, N, S, RMAX>;
    static constexpr int minb = 1;
};
template <int N, int S, int RMAX> struct FyKernel<float, N, S, RMAX> {
    static constexpr void (*f)(FyArgs<float>) = k_fft_y_t32<N, S, RMAX>;
    static constexpr int minb = FyMinBlocks<float, N, RMAX>::v;
};
