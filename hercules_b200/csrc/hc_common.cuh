// hc_common.cuh -- shared device-side definitions of the B200 time-step engine.
//
// Layout in HBM (all fields interior-only, no stored ghost cells):
//   physical field  f[(k*ny + j)*nx + i], i fastest (the Fortran interior order)
//   half spectrum   s[(k*ny + m)*nxh + l], l in [0,nx/2) (the x Nyquist mode, zeroed
//                   by the reference in every transform, is not stored), m in [0,ny)
//                   in FFT order, complex (R2 = double2 / float2)
// Horizontal ghost cells of the reference (comm_bound, src/module_boundary.f90:361-487)
// become a periodic index wrap; the z ghost cells (update_boundary_*) are applied
// when a value is loaded.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define HC_PI 3.1415926535897932

template <typename R> struct V2;
template <> struct V2<double> { typedef double2 T; };
template <> struct V2<float>  { typedef float2 T; };

template <typename R> __host__ __device__ __forceinline__ typename V2<R>::T mk2(R x, R y)
{
    typename V2<R>::T r; r.x = x; r.y = y; return r;
}

// per-k vertical metrics, indexed by Fortran k-1 (length nz+4);
// interior level kk (0-based) sits at Fortran k = kk+3, i.e. array index kk+2.
struct ZGrid {
    const double* dz;
    const double* dz_t;
    const double* dz_b;
    const double* l_t;
    const double* l_b;
};

struct Geo {
    int nx, ny, nz, nxh;
    long long nxy;       // nx*ny
    long long n;         // nx*ny*nz
    long long ncol;      // nxh*ny spectral columns
    double dx, dy, dx2, dy2;
    ZGrid z;
};

// physics constants of the step (src/module_parameters.f90:85-117)
struct Phys {
    double dt, nu, alpha, um, fc, ug, vg, t_ref, tbot, ttop;
    int cds, dp_opt, isscalar, ochannel, dts;
};

// device-resident scalar state (the reference's module scalars)
struct DevScalars {
    double dpx_drive;
    double ubar;
    double got;
    double time_sim;
    double cfl;          // CFL of the current fields
    double div_hist;     // signed value at the largest |div| seen so far
    double div_avg[3];
    double div_max[3];
    int step;            // completed steps
    int nan_flag;
    int tstat_n;         // statistics steps whose temperature terms are deferred (no temperature equation)
};

__device__ __forceinline__ int wrapi(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

__device__ __forceinline__ double ldz(const double* a, int kk) { return __ldg(a + kk + 2); }
