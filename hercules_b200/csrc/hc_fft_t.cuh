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

template <int N, int RMAX> struct FPlan {
    static constexpr int e2 = fft_pow2_exp(N);
    static constexpr int e3 = fft_exp_of(N, 3);
    static constexpr int e5 = fft_exp_of(N, 5);
    static constexpr int bits = fft_log2(RMAX);
    static constexpr int q2 = (e2 + bits - 1) / bits;            // power-of-two passes
    static constexpr int npass = q2 + e3 + e5;
    static constexpr bool valid = (N == (1 << e2) * (e3 == 0 ? 1 : (e3 == 1 ? 3 : (e3 == 2 ? 9 : 27))) *
                                           (e5 == 0 ? 1 : (e5 == 1 ? 5 : 25)));
    __host__ __device__ static constexpr int rad(int p)
    {
        return p < q2 ? (1 << (e2 / q2 + (p < e2 % q2 ? 1 : 0))) : (p < q2 + e3 ? 3 : 5);
    }
    // product of the radices of passes 0..p-1 (the Stockham span Ns of pass p)
    __host__ __device__ static constexpr int span(int p) { return p == 0 ? 1 : span(p - 1) * rad(p - 1); }
};

// padded shared-memory slot of element e of a line: one spare slot per G elements
template <int G> __device__ __forceinline__ int fpi(int e) { return e + e / G; }
template <int N, int G> struct FLine { static constexpr int stride = N + (N - 1) / G + 1; };
// 16-byte complex (double2): 8 per 128-byte wavefront; 8-byte (float2): 16
template <typename R> struct FPad { static constexpr int G = sizeof(R) == 8 ? 8 : 16; };

// ----------------------------------------------------------------------------
// butterflies with compile-time radix
// ----------------------------------------------------------------------------
// cos(2 pi e / 16) and sin(2 pi e / 16), e taken mod 16
__host__ __device__ constexpr double cos16(int e)
{
    return (e & 15) == 0 ? 1.0 : (e & 15) == 1 ? 0.92387953251128675613 : (e & 15) == 2 ? 0.70710678118654752440
         : (e & 15) == 3 ? 0.38268343236508977173 : (e & 15) == 4 ? 0.0 : (e & 15) == 5 ? -0.38268343236508977173
         : (e & 15) == 6 ? -0.70710678118654752440 : (e & 15) == 7 ? -0.92387953251128675613 : (e & 15) == 8 ? -1.0
         : (e & 15) == 9 ? -0.92387953251128675613 : (e & 15) == 10 ? -0.70710678118654752440
         : (e & 15) == 11 ? -0.38268343236508977173 : (e & 15) == 12 ? 0.0 : (e & 15) == 13 ? 0.38268343236508977173
         : (e & 15) == 14 ? 0.70710678118654752440 : 0.92387953251128675613;
}
__host__ __device__ constexpr double sin16(int e) { return cos16(e - 4); }

// v * exp(S 2 pi i E / M) for M in {4, 8, 16}; E compile-time
template <int M, int E, int S, typename T2> __device__ __forceinline__ T2 twc(T2 v)
{
    constexpr int e = (E * (16 / M)) & 15;
    typedef decltype(v.x) R;
    if (e == 0) return v;
    if (e == 8) { T2 r; r.x = -v.x; r.y = -v.y; return r; }
    if (e == 4) return mul_si<S>(v);                 // exp(S i pi/2) = S i
    if (e == 12) return mul_si<-S>(v);
    const R c = (R)cos16(e), s = (R)(S * sin16(e));
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

// ----------------------------------------------------------------------------
// Stockham passes over LINES lines of length N held in shared memory
// ----------------------------------------------------------------------------
// One pass of radix RAD with span NS: item j of a line reads s[j + r N/RAD],
// r < RAD, multiplies by w^{r k N/(NS RAD)} (k = j mod NS), transforms, and
// writes d[(j/NS) NS RAD + k + r NS].
template <typename R, int N, int S, int RAD, int NS, int LINES, int NT>
__device__ __forceinline__ void stock_pass(const typename V2<R>::T* __restrict__ src, typename V2<R>::T* __restrict__ dst,
                                           const typename V2<R>::T* __restrict__ tw)
{
    typedef typename V2<R>::T T2;
    constexpr int G = FPad<R>::G;
    constexpr int LS = FLine<N, G>::stride;
    constexpr int NR = N / RAD;
    constexpr int TS = N / (NS * RAD);
    for (int it = threadIdx.x; it < LINES * NR; it += NT) {
        const int line = it / NR;
        const int j = it - line * NR;
        const int k = NS == 1 ? 0 : j % NS;
        const T2* s = src + line * LS;
        T2* d = dst + line * LS;
        T2 v[RAD];
#pragma unroll
        for (int r = 0; r < RAD; ++r) {
            T2 x = s[fpi<G>(j + r * NR)];
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
        for (int r = 0; r < RAD; ++r) d[fpi<G>(base + r * NS)] = v[r];
    }
}

// Runs passes P..npass-1 and returns the buffer holding the transform.
template <typename R, int N, int S, int RMAX, int LINES, int NT, int P>
__device__ __forceinline__ typename V2<R>::T* run_passes(typename V2<R>::T* src, typename V2<R>::T* dst,
                                                         const typename V2<R>::T* tw)
{
    typedef FPlan<N, RMAX> PL;
    if constexpr (P >= PL::npass) {
        return src;
    } else {
        stock_pass<R, N, S, PL::rad(P), PL::span(P), LINES, NT>(src, dst, tw);
        __syncthreads();
        return run_passes<R, N, S, RMAX, LINES, NT, P + 1>(dst, src, tw);
    }
}

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

// lines per block: about 2048 complex values per block, at least one line
template <int N> struct FxLines { static constexpr int v = N >= 2048 ? 1 : 2048 / N; };
// y tiles: 8 columns (128-byte runs of FP64, 64-byte runs of FP32)
#define HC_FFT_TL 8
#define HC_FFT_NT 256

template <typename R, int N, int LINES> __host__ __device__ constexpr size_t fft_t_smem()
{
    return 2 * (size_t)LINES * FLine<N, FPad<R>::G>::stride * sizeof(typename V2<R>::T);
}

// ----------------------------------------------------------------------------
// x direction, forward: real rows -> nx/2 modes, divided by nx
// ----------------------------------------------------------------------------
template <typename R, int N, int RMAX>
__global__ void __launch_bounds__(HC_FFT_NT) k_fft_x_r2c_t(FxArgs<R> a)
{
    typedef typename V2<R>::T T2;
    constexpr int G = FPad<R>::G, LS = FLine<N, G>::stride, L = FxLines<N>::v;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (a.halt && *a.halt) return;
    T2* A = reinterpret_cast<T2*>(smem_raw);
    T2* B = A + L * LS;
    const int f = blockIdx.y;
    const long long row0 = (long long)blockIdx.x * L;
    const int nr = (int)min((long long)L, a.nrows - row0);
    const T2* in = reinterpret_cast<const T2*>(a.in[f]) + row0 * N;
    for (int idx = threadIdx.x; idx < L * N; idx += HC_FFT_NT) {
        const int line = idx / N, l = idx - line * N;
        A[line * LS + fpi<G>(l)] = idx < nr * N ? in[idx] : mk2<R>(R(0), R(0));
    }
    __syncthreads();
    T2* Z = run_passes<R, N, -1, RMAX, L, HC_FFT_NT, 0>(A, B, a.tw);
    T2* out = reinterpret_cast<T2*>(a.out[f]) + row0 * N;
    const R sc = a.scale;
    for (int idx = threadIdx.x; idx < nr * N; idx += HC_FFT_NT) {
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

// ----------------------------------------------------------------------------
// x direction, inverse: nx/2 modes -> real rows (unnormalised), stored or added
// ----------------------------------------------------------------------------
template <typename R, int N, int RMAX>
__global__ void __launch_bounds__(HC_FFT_NT) k_fft_x_c2r_t(FxArgs<R> a)
{
    typedef typename V2<R>::T T2;
    constexpr int G = FPad<R>::G, LS = FLine<N, G>::stride, L = FxLines<N>::v;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (a.halt && *a.halt) return;
    T2* A = reinterpret_cast<T2*>(smem_raw);
    T2* B = A + L * LS;
    const int f = blockIdx.y;
    const long long row0 = (long long)blockIdx.x * L;
    const int nr = (int)min((long long)L, a.nrows - row0);
    const T2* in = reinterpret_cast<const T2*>(a.in[f]) + row0 * N;
    for (int idx = threadIdx.x; idx < L * N; idx += HC_FFT_NT) {
        const int line = idx / N, l = idx - line * N;
        A[line * LS + fpi<G>(l)] = idx < nr * N ? in[idx] : mk2<R>(R(0), R(0));
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < L * N; idx += HC_FFT_NT) {
        const int line = idx / N, l = idx - line * N;
        const T2 x = A[line * LS + fpi<G>(l)];
        T2 xn = mk2<R>(R(0), R(0));
        if (l != 0) { xn = A[line * LS + fpi<G>(N - l)]; xn.y = -xn.y; }
        T2 wc = __ldg(a.wp + l);
        wc.y = -wc.y;
        const T2 s = cadd2(x, xn);
        const T2 d = cmulc(wc, csub2(x, xn));
        B[line * LS + fpi<G>(l)] = mk2<R>(s.x - d.y, s.y + d.x);     // s + i d
    }
    __syncthreads();
    T2* Z = run_passes<R, N, 1, RMAX, L, HC_FFT_NT, 0>(B, A, a.tw);
    T2* out = reinterpret_cast<T2*>(a.out[f]) + row0 * N;
    const int add = a.add[f];
    for (int idx = threadIdx.x; idx < nr * N; idx += HC_FFT_NT) {
        const int line = idx / N, l = idx - line * N;
        T2 v = Z[line * LS + fpi<G>(l)];
        if (add) { const T2 o = out[idx]; v.x += o.x; v.y += o.y; }
        out[idx] = v;
    }
}

// ----------------------------------------------------------------------------
// y direction on the half spectrum [k][m][l]: tiles of HC_FFT_TL columns l of one
// plane k; grid (ceil(nxh/TL), nz, fields)
// ----------------------------------------------------------------------------
template <typename R, int N, int S, int RMAX>
__global__ void __launch_bounds__(HC_FFT_NT) k_fft_y_t(FyArgs<R> a)
{
    typedef typename V2<R>::T T2;
    constexpr int G = FPad<R>::G, LS = FLine<N, G>::stride, TL = HC_FFT_TL, NYQ = N / 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (a.halt && *a.halt) return;
    T2* A = reinterpret_cast<T2*>(smem_raw);
    T2* B = A + TL * LS;
    const int nxh = a.nxh;
    const int l0 = blockIdx.x * TL;
    const long long plane = (long long)blockIdx.y * N * nxh;
    T2* d = a.dst[blockIdx.z] + plane;
    const T2* s = a.src[blockIdx.z] ? a.src[blockIdx.z] + plane : d;
    for (int idx = threadIdx.x; idx < TL * N; idx += HC_FFT_NT) {
        const int lt = idx % TL, m = idx / TL;
        const int l = l0 + lt;
        T2 v = mk2<R>(R(0), R(0));
        if (l < nxh && !(S > 0 && m == NYQ)) v = s[(long long)m * nxh + l];
        A[lt * LS + fpi<G>(m)] = v;
    }
    __syncthreads();
    T2* Z = run_passes<R, N, S, RMAX, TL, HC_FFT_NT, 0>(A, B, a.tw);
    const R sc = a.scale;
    for (int idx = threadIdx.x; idx < TL * N; idx += HC_FFT_NT) {
        const int lt = idx % TL, m = idx / TL;
        const int l = l0 + lt;
        if (l >= nxh) continue;
        T2 v = Z[lt * LS + fpi<G>(m)];
        if (S < 0) {
            v.x *= sc; v.y *= sc;
            if (m == NYQ) v = mk2<R>(R(0), R(0));
        }
        d[(long long)m * nxh + l] = v;
    }
}
