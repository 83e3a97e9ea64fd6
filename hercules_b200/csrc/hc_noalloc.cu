// hc_noalloc.cu -- divergence check of caller-owned fields that allocates no
// device memory.
//
// Who needs this: a host that keeps every device buffer under its own control
// and lets no library call cudaMalloc -- for example a Fortran code whose device
// memory is laid out once by its own arena or OpenACC data regions, or a solver
// that must not add allocations (and the implicit synchronisation they bring)
// inside its time loop. Such a caller passes its own u, v, w and an output slot;
// the per-block partial sums this check needs live in a fixed array that is part
// of the library image instead of in memory obtained at run time.
#include <cuda_runtime.h>
#include <mutex>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "../../include/hercules_b200.h"
#include "hc_fd.cuh"

// Largest nz accepted (the array holds the nz+4 vertical spacings).
#define NOALLOC_NZ_MAX 4096
#define NOALLOC_DZ_SLOTS (NOALLOC_NZ_MAX + 4)
// Scratch: vertical spacings, then 3 partial results per reduction block.
#define NOALLOC_DOUBLES (NOALLOC_DZ_SLOTS + 3 * RED_BLOCKS)

// One copy per device that loads the library, kept until the process exits
// (about 61 KB). Every call on a device reuses it.
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_DOUBLES];

// Host code may not use g_noalloc_scratch as an address: on the host that name is
// only a stand-in. The device address is looked up once per device, on the first
// call made with that device current, and kept for the life of the process: after
// cudaDeviceReset on that device the cached address is stale, so a process that
// resets a device must not call this entry point on it again.
#define NOALLOC_MAX_DEVICES 64
static double* g_scratch_addr[NOALLOC_MAX_DEVICES];
static std::mutex g_scratch_mu;

static int scratch_address(double** out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) return HC_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        double* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void**)&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr) {
            fprintf(stderr, "hercules_b200: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
            return HC_ERR_CUDA;
        }
        g_scratch_addr[dev] = ptr;
    }
    *out = g_scratch_addr[dev];
    return HC_OK;
}

// Combine the per-block partials of k_div_check in the same fixed order as the
// time step's finaliser: out = {sum|div| / (nx ny nz), signed div at max |div|, nan}.
__global__ void __launch_bounds__(256) k_noalloc_div_final(const double* part, long long nb, double nx, double ny,
                                                           double nz, double* out)
{
    __shared__ double sh[256];
    const int tid = threadIdx.x;
    double sm = 0.0, mx = 0.0, nn = 0.0;
    for (long long b = tid; b < nb; b += blockDim.x) {
        sm += part[3 * b];
        mx = absmax_pick(mx, part[3 * b + 1]);
        nn = fmax(nn, part[3 * b + 2]);
    }
    sh[tid] = sm;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) { if (tid < o) sh[tid] = sh[tid] + sh[tid + o]; __syncthreads(); }
    sm = sh[0];
    __syncthreads();
    sh[tid] = mx;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) { if (tid < o) sh[tid] = absmax_pick(sh[tid], sh[tid + o]); __syncthreads(); }
    mx = sh[0];
    __syncthreads();
    sh[tid] = nn;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) { if (tid < o) sh[tid] = fmax(sh[tid], sh[tid + o]); __syncthreads(); }
    nn = sh[0];
    if (tid == 0) {
        out[0] = sm / nx / ny / nz;
        out[1] = mx;
        out[2] = nn;
    }
}

template <typename R, int CDS>
static int run_div(const Geo& g, const void* u, const void* v, const void* w, double* part, long long nb,
                   double* out, cudaStream_t st)
{
    FieldsIn<R> f;
    f.u = (const R*)u; f.v = (const R*)v; f.w = (const R*)w; f.p = nullptr; f.t = nullptr;
    DivArgs<R> da;
    da.f = f; da.g = g; da.part = part;
    k_div_check<R, CDS><<<(unsigned)nb, 256, 0, st>>>(da);
    if (cudaGetLastError() != cudaSuccess) return HC_ERR_CUDA;
    k_noalloc_div_final<<<1, 256, 0, st>>>(part, nb, (double)g.nx, (double)g.ny, (double)g.nz, out);
    if (cudaGetLastError() != cudaSuccess) return HC_ERR_CUDA;
    return HC_OK;
}

extern "C" int hc_divergence_noalloc(const hc_params* p, const double* dz, const void* u, const void* v,
                                     const void* w, double* out_dev, void* stream)
{
    if (!p || !dz || !u || !v || !w || !out_dev) return HC_ERR_ARG;
    if (p->cds != 1 && p->cds != 2) return HC_ERR_ARG;
    if (p->precision != HC_PREC_FP64 && p->precision != HC_PREC_MIXED) return HC_ERR_ARG;
    // the same grid rules as hc_create (even nx and ny, src/module_parameters.f90:266-270):
    // with FP32 fields the kernel reads two adjacent x points as one 8-byte value, so an
    // odd nx would put those reads at odd offsets
    if (p->nx < 8 || p->ny < 4 || p->nz < 3 || (p->nx & 1) || (p->ny & 1)) return HC_ERR_PARAM;
    // every load is 8 bytes wide (one double, or a pair of floats) and so is the result
    if ((((uintptr_t)u) | ((uintptr_t)v) | ((uintptr_t)w) | ((uintptr_t)out_dev)) & 7u) return HC_ERR_ARG;
    const long long n = (long long)p->nx * p->ny * p->nz;
    if (p->nz > NOALLOC_NZ_MAX || n > 2147483647LL) {
        fprintf(stderr, "hercules_b200: hc_divergence_noalloc supports nz <= %d and nx*ny*nz < 2^31 "
                        "(got %d x %d x %d)\n", NOALLOC_NZ_MAX, p->nx, p->ny, p->nz);
        return HC_ERR_SIZE;
    }
    double* base = nullptr;
    int rc = scratch_address(&base);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    // the vertical spacings go into the first slots of the shared array
    if (cudaMemcpyToSymbolAsync(g_noalloc_scratch, dz, (size_t)(p->nz + 4) * sizeof(double), 0,
                                cudaMemcpyHostToDevice, st) != cudaSuccess)
        return HC_ERR_CUDA;
    Geo g;
    memset(&g, 0, sizeof(g));
    g.nx = p->nx; g.ny = p->ny; g.nz = p->nz; g.nxh = p->nx / 2;
    g.nxy = (long long)p->nx * p->ny; g.n = n; g.ncol = (long long)g.nxh * p->ny;
    g.dx = p->lx / p->nx; g.dy = p->ly / p->ny; g.dx2 = g.dx * g.dx; g.dy2 = g.dy * g.dy;
    g.z.dz = base;
    double* part = base + NOALLOC_DZ_SLOTS;
    long long nb = (n + 255) / 256;
    if (nb > RED_BLOCKS) nb = RED_BLOCKS;
    // every block writes all three of its partial slots, so nothing needs clearing
    if (p->precision == HC_PREC_MIXED)
        return p->cds == 1 ? run_div<float, 1>(g, u, v, w, part, nb, out_dev, st) : run_div<float, 2>(g, u, v, w, part, nb, out_dev, st);
    return p->cds == 1 ? run_div<double, 1>(g, u, v, w, part, nb, out_dev, st) : run_div<double, 2>(g, u, v, w, part, nb, out_dev, st);
}
