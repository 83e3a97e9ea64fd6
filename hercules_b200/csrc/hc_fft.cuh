// hc_fft.cuh -- batched shared-memory FFTs replacing mpi_2d_fft
// (src/module_tools.f90:518-700), FFTW sign conventions: forward e^{-i}, each
// direction divided by its length, inverse unnormalised; the y Nyquist mode is
// zeroed after the forward and before the inverse transform, and the x Nyquist
// mode is not stored at all (a real row of nx values maps to nx/2 complex modes).
//
// x direction: real rows of nx values are packed as nx/2 complex numbers and
// transformed with one complex FFT of length nx/2 plus a split step (r2c / c2r).
// y direction: c2c over m for every (k, l), tiles of TL columns staged in SMEM.
// Each transform is a Stockham autosort FFT with radix-2/3/4/5 passes, ping-pong
// between two SMEM buffers, twiddles read from a per-length table.
#pragma once
#include "hc_common.cuh"

#define HC_MAX_PASS 16

struct FftPlan {
    int n;
    int npass;
    int rad[HC_MAX_PASS];
    const double2* tw;     // tw[e] = exp(-2 pi i e / n), e in [0, n)
};

template <typename T2> __device__ __forceinline__ T2 cmulc(T2 a, T2 b)
{
    T2 r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
template <typename T2> __device__ __forceinline__ T2 cadd2(T2 a, T2 b) { T2 r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename T2> __device__ __forceinline__ T2 csub2(T2 a, T2 b) { T2 r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
// multiply by (S i): S = -1 -> -i, S = +1 -> +i
template <int S, typename T2> __device__ __forceinline__ T2 mul_si(T2 a)
{
    T2 r;
    if (S > 0) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; }
    return r;
}

template <typename R, int S>
__device__ __forceinline__ void dft_small(typename V2<R>::T* v, int rr)
{
    typedef typename V2<R>::T T2;
    if (rr == 2) {
        T2 a = v[0], b = v[1];
        v[0] = cadd2(a, b); v[1] = csub2(a, b);
    } else if (rr == 4) {
        T2 s02 = cadd2(v[0], v[2]), d02 = csub2(v[0], v[2]);
        T2 s13 = cadd2(v[1], v[3]), d13 = mul_si<S>(csub2(v[1], v[3]));
        v[0] = cadd2(s02, s13);
        v[1] = cadd2(d02, d13);
        v[2] = csub2(s02, s13);
        v[3] = csub2(d02, d13);
    } else if (rr == 3) {
        const R h = R(0.86602540378443864676);
        T2 a = v[0], b = v[1], c = v[2];
        T2 t1 = cadd2(b, c);
        T2 t2; t2.x = a.x - R(0.5) * t1.x; t2.y = a.y - R(0.5) * t1.y;
        T2 d = mul_si<S>(csub2(b, c)); d.x *= h; d.y *= h;
        v[0] = cadd2(a, t1);
        v[1] = cadd2(t2, d);
        v[2] = csub2(t2, d);
    } else {   // 5
        const R c1 = R(0.30901699437494742410), c2 = R(-0.80901699437494742410);
        const R s1 = R(0.95105651629515357212), s2 = R(0.58778525229247312917);
        T2 a = v[0];
        T2 b1 = cadd2(v[1], v[4]), b2 = cadd2(v[2], v[3]);
        T2 d1 = csub2(v[1], v[4]), d2 = csub2(v[2], v[3]);
        T2 r1, r2, q1, q2;
        r1.x = a.x + c1 * b1.x + c2 * b2.x; r1.y = a.y + c1 * b1.y + c2 * b2.y;
        r2.x = a.x + c2 * b1.x + c1 * b2.x; r2.y = a.y + c2 * b1.y + c1 * b2.y;
        T2 e1; e1.x = s1 * d1.x + s2 * d2.x; e1.y = s1 * d1.y + s2 * d2.y;
        T2 e2; e2.x = s2 * d1.x - s1 * d2.x; e2.y = s2 * d1.y - s1 * d2.y;
        q1 = mul_si<S>(e1); q2 = mul_si<S>(e2);
        v[0] = cadd2(a, cadd2(b1, b2));
        v[1] = cadd2(r1, q1);
        v[4] = csub2(r1, q1);
        v[2] = cadd2(r2, q2);
        v[3] = csub2(r2, q2);
    }
}

// Stockham passes over nlines lines of length pl.n stored with stride lstride.
// Returns the buffer holding the result (A or B). Ends with __syncthreads().
template <typename R, int S>
__device__ typename V2<R>::T* stockham(typename V2<R>::T* A, typename V2<R>::T* B,
                                       int nlines, int lstride, const FftPlan& pl)
{
    typedef typename V2<R>::T T2;
    const int N = pl.n;
    T2* src = A;
    T2* dst = B;
    int Ns = 1;
    for (int p = 0; p < pl.npass; ++p) {
        const int rr = pl.rad[p];
        const int NR = N / rr;
        const int ts = N / (Ns * rr);
        const int items = nlines * NR;
        for (int it = threadIdx.x; it < items; it += blockDim.x) {
            const int line = it / NR;
            const int j = it - line * NR;
            const int k = j % Ns;
            const T2* s = src + line * lstride;
            T2* d = dst + line * lstride;
            T2 v[5];
#pragma unroll
            for (int r = 0; r < 5; ++r) {
                if (r < rr) {
                    T2 x = s[j + r * NR];
                    if (r > 0 && k > 0) {
                        double2 w = __ldg(pl.tw + r * k * ts);
                        T2 tw; tw.x = (R)w.x; tw.y = (R)(S < 0 ? w.y : -w.y);
                        x = cmulc(x, tw);
                    }
                    v[r] = x;
                }
            }
            dft_small<R, S>(v, rr);
            const int idxD = (j / Ns) * Ns * rr + k;
#pragma unroll
            for (int r = 0; r < 5; ++r)
                if (r < rr) d[idxD + r * Ns] = v[r];
        }
        __syncthreads();
        T2* t = src; src = dst; dst = t;
        Ns *= rr;
    }
    return src;
}

#define HC_FFT_MAXF 16

// ---------------------------------------------------------------------------
// x direction, forward: real rows -> nx/2 modes, divided by nx
// ---------------------------------------------------------------------------
template <typename R> struct FftXArgs {
    const R* in[HC_FFT_MAXF];
    typename V2<R>::T* out[HC_FFT_MAXF];
    long long nrows;        // ny*nz
    int rows;               // rows per block
    FftPlan pl;             // length nx/2
    const double2* wpack;   // exp(-2 pi i l / nx), l in [0, nx/2)
    double scale;           // 1/nx
    const int* halt;        // skip all work when nonzero (NaN seen)
};

template <typename R>
__device__ __forceinline__ void k_fft_x_r2c_body(const FftXArgs<R>& a, const uint3 blockIdx, const dim3 gridDim)
{
    typedef typename V2<R>::T T2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (a.halt && *a.halt) return;
    const int N = a.pl.n;
    T2* A = reinterpret_cast<T2*>(smem_raw);
    T2* B = A + a.rows * N;
    const int f = blockIdx.y;
    const long long row0 = (long long)blockIdx.x * a.rows;
    const int nr = (int)min((long long)a.rows, a.nrows - row0);
    const T2* in = reinterpret_cast<const T2*>(a.in[f]) + row0 * N;
    for (int idx = threadIdx.x; idx < nr * N; idx += blockDim.x) A[idx] = in[idx];
    __syncthreads();
    T2* Z = stockham<R, -1>(A, B, nr, N, a.pl);
    T2* out = a.out[f] + row0 * N;
    const R sc = (R)a.scale;
    for (int idx = threadIdx.x; idx < nr * N; idx += blockDim.x) {
        const int line = idx / N;
        const int l = idx - line * N;
        T2 z = Z[line * N + l];
        T2 zc = Z[line * N + (l == 0 ? 0 : N - l)];
        zc.y = -zc.y;
        T2 e; e.x = R(0.5) * (z.x + zc.x); e.y = R(0.5) * (z.y + zc.y);
        T2 dd; dd.x = R(0.5) * (z.x - zc.x); dd.y = R(0.5) * (z.y - zc.y);
        double2 w = __ldg(a.wpack + l);
        T2 wr; wr.x = (R)w.x; wr.y = (R)w.y;
        // X = E - i W D
        T2 wd = cmulc(wr, dd);
        T2 X; X.x = e.x + wd.y; X.y = e.y - wd.x;
        X.x *= sc; X.y *= sc;
        out[idx] = X;
    }
}
template <typename R>
__global__ void __launch_bounds__(256) k_fft_x_r2c(FftXArgs<R> a) { k_fft_x_r2c_body<R>(a, blockIdx, gridDim); }

// ---------------------------------------------------------------------------
// x direction, inverse: nx/2 modes -> real rows (unnormalised), stored or added
// ---------------------------------------------------------------------------
template <typename R> struct FftXInvArgs {
    const typename V2<R>::T* in[HC_FFT_MAXF];
    R* out[HC_FFT_MAXF];
    int add[HC_FFT_MAXF];   // 1: out += result (pressure update), 0: out = result
    long long nrows;
    int rows;
    FftPlan pl;
    const double2* wpack;
    const int* halt;
};

template <typename R>
__device__ __forceinline__ void k_fft_x_c2r_body(const FftXInvArgs<R>& a, const uint3 blockIdx, const dim3 gridDim)
{
    typedef typename V2<R>::T T2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (a.halt && *a.halt) return;
    const int N = a.pl.n;
    T2* A = reinterpret_cast<T2*>(smem_raw);
    T2* B = A + a.rows * N;
    const int f = blockIdx.y;
    const long long row0 = (long long)blockIdx.x * a.rows;
    const int nr = (int)min((long long)a.rows, a.nrows - row0);
    const T2* in = a.in[f] + row0 * N;
    for (int idx = threadIdx.x; idx < nr * N; idx += blockDim.x) A[idx] = in[idx];
    __syncthreads();
    for (int idx = threadIdx.x; idx < nr * N; idx += blockDim.x) {
        const int line = idx / N;
        const int l = idx - line * N;
        T2 x = A[line * N + l];
        T2 xn;
        if (l == 0) { xn.x = R(0); xn.y = R(0); } else { xn = A[line * N + N - l]; xn.y = -xn.y; }
        double2 w = __ldg(a.wpack + l);
        T2 wc; wc.x = (R)w.x; wc.y = (R)(-w.y);
        T2 s = cadd2(x, xn);
        T2 d = cmulc(wc, csub2(x, xn));
        T2 zp; zp.x = s.x - d.y; zp.y = s.y + d.x;     // s + i d
        B[idx] = zp;
    }
    __syncthreads();
    T2* z = stockham<R, 1>(B, A, nr, N, a.pl);
    T2* out = reinterpret_cast<T2*>(a.out[f]) + row0 * N;
    const int add = a.add[f];
    for (int idx = threadIdx.x; idx < nr * N; idx += blockDim.x) {
        T2 v = z[idx];
        if (add) { T2 o = out[idx]; v.x += o.x; v.y += o.y; }
        out[idx] = v;
    }
}
template <typename R>
__global__ void __launch_bounds__(256) k_fft_x_c2r(FftXInvArgs<R> a) { k_fft_x_c2r_body<R>(a, blockIdx, gridDim); }

// ---------------------------------------------------------------------------
// y direction, in place on the half spectrum [k][m][l]
// ---------------------------------------------------------------------------
template <typename R> struct FftYArgs {
    const typename V2<R>::T* src[HC_FFT_MAXF];   // null: transform data in place
    typename V2<R>::T* data[HC_FFT_MAXF];
    int nxh, ny, tl;
    FftPlan pl;             // length ny
    double scale;           // forward: 1/ny
    const int* halt;
};

template <typename R, int S>
__device__ __forceinline__ void k_fft_y_body(const FftYArgs<R>& a, const uint3 blockIdx, const dim3 gridDim)
{
    typedef typename V2<R>::T T2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (a.halt && *a.halt) return;
    const int ny = a.ny, tl = a.tl, ls = ny + 1;
    T2* A = reinterpret_cast<T2*>(smem_raw);
    T2* B = A + tl * ls;
    const int l0 = blockIdx.x * tl;
    const long long k = blockIdx.y;
    T2* d = a.data[blockIdx.z] + k * (long long)ny * a.nxh;
    const T2* sd = a.src[blockIdx.z] ? a.src[blockIdx.z] + k * (long long)ny * a.nxh : d;
    const int nyq = ny / 2;
    for (int idx = threadIdx.x; idx < tl * ny; idx += blockDim.x) {
        const int lt = idx % tl, m = idx / tl;
        const int l = l0 + lt;
        T2 v; v.x = R(0); v.y = R(0);
        if (l < a.nxh && !(S > 0 && m == nyq)) v = sd[(long long)m * a.nxh + l];
        A[lt * ls + m] = v;
    }
    __syncthreads();
    T2* z = stockham<R, S>(A, B, tl, ls, a.pl);
    const R sc = (R)a.scale;
    for (int idx = threadIdx.x; idx < tl * ny; idx += blockDim.x) {
        const int lt = idx % tl, m = idx / tl;
        const int l = l0 + lt;
        if (l >= a.nxh) continue;
        T2 v = z[lt * ls + m];
        if (S < 0) {
            v.x *= sc; v.y *= sc;
            if (m == nyq) { v.x = R(0); v.y = R(0); }
        }
        d[(long long)m * a.nxh + l] = v;
    }
}
template <typename R, int S>
__global__ void __launch_bounds__(256) k_fft_y(FftYArgs<R> a) { k_fft_y_body<R, S>(a, blockIdx, gridDim); }
