// hc_api.cu -- C-ABI of the B200 time-step engine (declared in include/hercules_b200.h).
//
// One handle owns one channel: its device state, one CUDA stream and the host
// set-up that the reference's `drive` performs before the time loop
// (src/module_navier_stokes.f90:53-129). hc_step issues, per RK sub-step,
//   substep_begin -> momentum RHS -> forward 2-D FFT -> column solve (3 Helmholtz +
//   phi Poisson + projection) -> inverse 2-D FFT (+ p update)
//   [-> temperature RHS -> FFT -> T column solve -> iFFT] -> divergence check
// and per step the statistics/bulk-velocity/CFL pass and a one-block finaliser
// that writes the step's diagnostics and the next step's scalars on the device.
//
// This file holds the device scalar kernels, the handle, the launch recorder,
// the grid and coefficient tables and the C-ABI; the host code of the transforms
// (hc_host_fft.cuh), the FD step (hc_host_step.cuh), the spectral step
// (hc_host_spec.cuh), the adjoint (hc_host_adjoint.cuh) and the ensemble
// (hc_host_ensemble.cuh) is included at its place, so the library stays one
// translation unit and every kernel template is instantiated once.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include <vector>

#include "../../include/hercules_b200.h"
#include "hc_common.cuh"
#include "hc_fd.cuh"
#include "hc_fft_t.cuh"
#include "hc_fft2d.cuh"
#include "hc_column.cuh"
#include "hc_rhs_tiled.cuh"
#include "hc_rhs_tiled2.cuh"
#include "hc_rhs_strip.cuh"
#include "hc_column_warp.cuh"
#include "hc_spec.cuh"
#include "hc_adjoint.cuh"
#include "hc_group.cuh"

// ---------------------------------------------------------------------------
// small device kernels for the scalar state
// ---------------------------------------------------------------------------
struct ScalarArgs {
    DevScalars* sc;
    int sub;               // 0-based sub-step
    double dt;
    int dp_opt;
    double dpx_coef, um;
    int is_ri_var;
    double ri_str, ri_end;
    int imax;
};

// screen_cpu_time's time_sim += dt (src/module_io.f90:68), update_ri
// (src/module_parameters.f90:580-590) and update_dpx_drive (:594-613), which the
// reference calls at the start of every sub-step's RHS.
__device__ __forceinline__ void k_substep_begin_body(const ScalarArgs& a, const uint3 blockIdx, const dim3 gridDim)
{
    DevScalars* s = a.sc;
    if (s->nan_flag) return;
    if (a.sub == 0) {
        s->step += 1;
        s->time_sim = s->time_sim + a.dt;
        if (a.is_ri_var == 1) s->got = a.ri_str + (a.ri_end - a.ri_str) * 1.0 / a.imax * s->step;
    }
    if (a.dp_opt == 1) s->dpx_drive = 1.0;
    else if (a.dp_opt == 2) s->dpx_drive = s->dpx_drive - (s->ubar + a.um - 1.0) * a.dpx_coef;
}
__global__ void k_substep_begin(ScalarArgs a) { k_substep_begin_body(a, blockIdx, gridDim); }

struct FinalArgs {
    DevScalars* sc;
    const double* part_div;   // [3][stride][3]
    long long stride;
    long long nbq[3];         // partial blocks written for each sub-step
    int nsub;
    const double* part_st;    // [nbs][2]
    long long nbs;
    double inv_n;             // 1/(nx ny nz) as the reference's sequential division
    double nx, ny, nz, lz;
    int dp_opt;
    hc_diag* diag;            // ring of diag_cap records, slot (step - 1) % diag_cap
    int diag_cap;
    int write_diag;
    int cds;
    int set_ubar;             // 0: keep the bulk velocity (spectral set-up)
};

__device__ double block_sum_fixed(double v, double* sh)
{
    const int tid = threadIdx.x;
    sh[tid] = v;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (tid < o) sh[tid] = sh[tid] + sh[tid + o];
        __syncthreads();
    }
    double r = sh[0];
    __syncthreads();
    return r;
}
__device__ double block_max_fixed(double v, double* sh)
{
    const int tid = threadIdx.x;
    sh[tid] = v;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (tid < o) sh[tid] = fmax(sh[tid], sh[tid + o]);
        __syncthreads();
    }
    double r = sh[0];
    __syncthreads();
    return r;
}
__device__ double block_absmax_fixed(double v, double* sh)
{
    const int tid = threadIdx.x;
    sh[tid] = v;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (tid < o) sh[tid] = absmax_pick(sh[tid], sh[tid + o]);
        __syncthreads();
    }
    double r = sh[0];
    __syncthreads();
    return r;
}

// End-of-step finaliser (one block of 256 threads, fixed reduction order).
__device__ __forceinline__ void k_finalize_body(const FinalArgs& a, const uint3 blockIdx, const dim3 gridDim)
{
    __shared__ double sh[256];
    DevScalars* s = a.sc;
    const int tid = threadIdx.x;
    const bool halted_before = s->nan_flag != 0;
    const double cfl_start = s->cfl;
    double davg[3] = {0, 0, 0}, dmax[3] = {0, 0, 0};
    int nan = 0;
    for (int q = 0; q < a.nsub; ++q) {
        const double* p = a.part_div + (long long)q * a.stride * 3;
        double sm = 0.0, mx = 0.0, nn = 0.0;
        for (long long b = tid; b < a.nbq[q]; b += blockDim.x) {
            sm += p[3 * b];
            mx = absmax_pick(mx, p[3 * b + 1]);
            nn = fmax(nn, p[3 * b + 2]);
        }
        sm = block_sum_fixed(sm, sh);
        mx = block_absmax_fixed(mx, sh);
        nn = block_max_fixed(nn, sh);
        davg[q] = sm / a.nx / a.ny / a.nz;
        dmax[q] = a.cds == 3 ? fabs(mx) : mx;
        if (nn != 0.0) nan = 1;
    }
    double ub = 0.0, cf = 0.0;
    for (long long b = tid; b < a.nbs; b += blockDim.x) {
        ub += a.part_st[2 * b];
        cf = fmax(cf, a.part_st[2 * b + 1]);
    }
    ub = block_sum_fixed(ub, sh);
    cf = block_max_fixed(cf, sh);
    if (tid != 0) return;
    if (halted_before) return;
    for (int q = 0; q < a.nsub; ++q) {
        s->div_avg[q] = davg[q];
        s->div_max[q] = dmax[q];
        if (fabs(dmax[q]) > fabs(s->div_hist)) s->div_hist = dmax[q];
    }
    if (a.dp_opt == 2 && a.set_ubar) s->ubar = ub / a.lz / a.nx / a.ny;
    s->cfl = cf;
    if (nan) s->nan_flag = 1;
    if (a.write_diag) {
        hc_diag* d = a.diag + (s->step - 1) % a.diag_cap;
        d->time_sim = s->time_sim;
        d->cfl = cfl_start;
        d->div_avg = davg[a.nsub - 1];
        d->div_max = dmax[a.nsub - 1];
        d->div_hist_max = s->div_hist;
        d->ubar = a.dp_opt == 2 ? s->ubar : 0.0;
        d->dpx_drive = s->dpx_drive;
        d->got = s->got;
        for (int q = 0; q < 3; ++q) {
            d->div_avg_sub[q] = q < a.nsub ? davg[q] : 0.0;
            d->div_max_sub[q] = q < a.nsub ? dmax[q] : 0.0;
        }
        d->nan_flag = nan;
        d->step = s->step;
    }
}
__global__ void __launch_bounds__(256) k_finalize(FinalArgs a) { k_finalize_body(a, blockIdx, gridDim); }

template <typename R>
__global__ void k_convert_in(const double* src, R* dst, long long n)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = (R)src[i];
}

// ---------------------------------------------------------------------------
// handle
// ---------------------------------------------------------------------------
enum { F_U, F_V, F_W, F_P, F_T, F_FF, F_GG, F_HH, F_SS, F_QU, F_QV, F_QW, F_UHX, F_VHY, NFLD };

// kernel categories for the optional per-launch CUDA-event profile
enum { K_BEGIN, K_RHS_MOM, K_FFT_X_FWD, K_FFT_Y_FWD, K_COLUMN, K_FFT_Y_INV, K_FFT_X_INV,
       K_RHS_T, K_COLUMN_T, K_DIV, K_STATS, K_FINAL, K_SPEC_PROD, K_SPEC_ASM, K_SPEC_AUX, K_ADJ_COLUMN,
       K_ADJ_RHS, K_FFT2D_FWD, K_FFT2D_INV, K_SPEC_PRODFX, K_NCAT };
static const char* K_NAMES[K_NCAT] = {"substep_begin", "rhs_momentum", "fft_x_r2c", "fft_y_fwd", "column_fd",
                                      "fft_y_inv", "fft_x_c2r", "rhs_temperature", "column_t", "div_check",
                                      "stats", "finalize", "spec_products", "spec_assemble", "aux", "adj_column",
                                      "adj_rhs", "fft2d_fwd", "fft2d_inv", "spec_products_fx"};

// spectral-path buffers (cds = 3), each n values of the storage type: the half
// spectra of the state and histories, phi, the divergence, the assembled
// right-hand sides and work fields (physical products / their spectra)
enum { SP_U, SP_V, SP_W, SP_P, SP_T, SP_FF, SP_GG, SP_HH, SP_SS, SP_PHI, SP_DIV, SP_QU, SP_QV, SP_QW, SP_W0,
       NSP = SP_W0 + 14 };

#define ADJ_GRAPHS 4
// FP32 storage: mean accumulators sum each window of this many steps in FP32
// before it is folded into their FP64 sums
#define STATS_WINDOW 16

struct hc_handle {
    hc_params p;
    int dev;
    cudaStream_t st;
    Geo g;
    Phys ph;
    size_t rsz;              // bytes of the storage type
    void* fld[NFLD];
    void* spec[4];
    void* sp[NSP];           // cds = 3 only
    double* dsig;            // cds = 3, isdamp = 1: sigma per level (0 below the layer)
    double* dmean;           // [5][nz] plane means of the damped levels
    void* dstale;            // FD, isdamp = 1: undamped copies of u, v, w, p, t on the damped levels
    int div_in_rhs;          // FD without damping: sub-step checks ride in the next RHS
    void* bf[3];             // body force (storage type), allocated by hc_set_body_force
    int has_bf;
    // discrete adjoint (hc_adjoint): one allocation for checkpoints, tape and adjoint fields
    double* adj_buf;
    size_t adj_bytes;
    DevScalars* adj_sc;      // scalar state at each checkpoint and at the end
    int adj_nsc;
    double adj_ms[2];        // forward pass, reverse sweep (recomputation included)
    int adj_nsteps, adj_ckpt, adj_nseg, adj_seglen;
    int adj_ready;           // 1: checkpoints of the last hc_adjoint_forward are valid
    int adj_tape_seg;        // segment whose sub-step start states the tape holds (-1: none)
    cudaGraphExec_t adj_gexec[ADJ_GRAPHS];   // reverse segments, keyed by adj_gkey
    int adj_gkey[ADJ_GRAPHS];
    long long adj_glaunch[ADJ_GRAPHS];
    int adj_gnext;
    long long adj_launches[2];
    // CUDA graph of one step (hc_set_graph): captured on first use, replayed per step
    int use_graph;
    cudaGraphExec_t gexec;
    long long graph_launches;
    double* mean[11];
    float* win[11];          // FP32 storage: the FP32 window sums of the mean accumulators
    double* mtmp;            // FP32 storage: FP64 sums + window, assembled for a download
    // no temperature equation and no damping: T never changes, so the statistics
    // kernel leaves out mean_t, mean_tt, mean_tw and tstat_flush adds them on request
    int tdefer;
    double* mw0;             // mean_w sums at the last flush
    double* zbuf;            // 5*(nz+4) doubles, then zm5d (5*nz doubles) and zm5 (5*nz floats)
    double* zm5d;            // FP64 per-level metrics of the strip RHS
    float* zm5;              // FP32 per-level metrics of the strip RHS
    double* coef;
    ColCoef cc;
    double* scratch;
    ColScratch cs;
    double* part_div;
    double* part_st;
    long long nbd, nbs, stx, sty;
    long long pd_stride;     // partial slots per sub-step (max over the writers)
    dim3 rhs_grid;           // FD momentum RHS grid and its level chunk
    int rhs_kc;
    int rhs_strip;           // the strip kernel (k_rhs_momentum_strip) runs the RHS
    std::vector<GroupRec>* rec;   // non-null: launches are recorded (ensemble plans), not run
    DevScalars* sc;
    hc_diag* diag_dev;
    int diag_cap;
    double2* twbuf;
    void* twt;               // the same tables in the storage precision (FP64: twbuf)
    int fft_tx, fft_ty;      // 1: the compile-time-length kernels serve x / y
    int fft2d;               // 1: the fused 2-D transform kernels (hc_fft2d.cuh) serve both
    int f2_ncl[2];           // their persistent clusters resident at once: forward, inverse
    int spx;                 // 1: the spectral products and their x transform in one kernel (k_spec_products_fx)
    int spx_minb;            // its blocks resident an SM
    int spx_t;               // 1: the temperature products too (k_spec_products_t_fx)
    FftPlan px, py;
    double2* wpack;
    int rows_x, tl_y, col_threads, col_warp;
    size_t smem_x, smem_y;
    double dpx_coef;
    cudaEvent_t e0, e1;
    double last_ms;
    long long launches;
    int initialized;
    std::vector<double> zhost[5];
    // profiling: an event pair per launch, summed per category at the end of hc_step
    int prof;
    int cur_cat;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<int> ev_cat;
    size_t ev_used;
    double cat_ms[K_NCAT];
    long long cat_n[K_NCAT];
};

#define CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { fprintf(stderr, "hercules_b200: %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); return HC_ERR_CUDA; } } while (0)
#define CKL() do { cudaError_t e_ = cudaGetLastError(); if (e_ != cudaSuccess) { fprintf(stderr, "hercules_b200: launch %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); return HC_ERR_CUDA; } ++h->launches; prof_end(h); } while (0)

// Start-of-launch marker (no-op unless profiling): records an event on the
// handle's stream and remembers the category; CKL() records the matching end.
static int prof_begin(hc_handle* h, int cat)
{
    if (!h->prof) return HC_OK;
    if (h->ev_used + 2 > h->ev_pool.size()) {
        for (int q = 0; q < 256; ++q) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) return HC_ERR_CUDA;
            h->ev_pool.push_back(e);
        }
        h->ev_cat.resize(h->ev_pool.size() / 2 + 1);
    }
    h->cur_cat = cat;
    cudaEventRecord(h->ev_pool[h->ev_used], h->st);
    return HC_OK;
}
static void prof_end(hc_handle* h)
{
    if (!h->prof) return;
    cudaEventRecord(h->ev_pool[h->ev_used + 1], h->st);
    h->ev_cat[h->ev_used / 2] = h->cur_cat;
    h->ev_used += 2;
}
static int prof_collect(hc_handle* h)
{
    if (!h->prof || h->ev_used == 0) return HC_OK;
    CK(cudaStreamSynchronize(h->st));
    for (size_t q = 0; q < h->ev_used; q += 2) {
        float ms = 0.0f;
        CK(cudaEventElapsedTime(&ms, h->ev_pool[q], h->ev_pool[q + 1]));
        h->cat_ms[h->ev_cat[q / 2]] += ms;
        h->cat_n[h->ev_cat[q / 2]] += 1;
    }
    h->ev_used = 0;
    return HC_OK;
}

// Launch KFN (whose body is BODY, launched with at most NT threads and MINB
// resident blocks) on the handle's stream, or, while the handle records, keep the
// launch for a grouped ensemble launch of the same body. (Running a channel's own
// launches through k_group too would make them the same compiled code as in an
// ensemble, but reading the arguments through the member table cost 5-6 % of the
// 512 x 384 x 256 step, so a channel alone runs its named kernels.)
template <typename A, void (*KFN)(A), void (*BODY)(const A&, const uint3, const dim3), int NT, int MINB>
static int hc_launch(hc_handle* h, dim3 grid, dim3 block, size_t smem, const A& args)
{
    if (h->rec) {
        GroupRec r;
        r.key = (const void*)&k_group<A, BODY, NT, MINB, GroupCap<A>::v>;
        r.cap = GroupCap<A>::v;
        r.build = &group_build<A, BODY, NT, MINB>;
        r.args.assign(reinterpret_cast<const unsigned char*>(&args), reinterpret_cast<const unsigned char*>(&args) + sizeof(A));
        r.grid = grid; r.block = block; r.smem = smem;
        h->rec->push_back(std::move(r));
        return HC_OK;
    }
    KFN<<<grid, block, smem, h->st>>>(args);
    return HC_OK;
}

static int factor_plan(int n, FftPlan* pl)
{
    pl->n = n;
    pl->npass = 0;
    int m = n;
    const int rads[4] = {4, 2, 3, 5};
    for (int q = 0; q < 4; ++q)
        while (m % rads[q] == 0) {
            if (pl->npass >= HC_MAX_PASS) return HC_ERR_UNSUPPORTED;
            pl->rad[pl->npass++] = rads[q];
            m /= rads[q];
        }
    return m == 1 ? HC_OK : HC_ERR_UNSUPPORTED;
}

// get_mesh_param (src/module_parameters.f90:432-508), Fortran k at [k-1]
static void mesh_host(const hc_params* p, std::vector<double>* z)
{
    const int nz = p->nz, nka = nz + 4, kstr3 = 3, kend3 = nz + 2;
    std::vector<double> zz(nka + 3, 0.0), dz(nka + 3, 0.0), lt(nka + 3, 0.0), lb(nka + 3, 0.0), dzt(nka + 3, 0.0), dzb(nka + 3, 0.0);
    double zmin = 0.0, zmax = p->lz, zmean, coeff_a;
    if (p->ochannel == 0) { zmean = 0.5 * (zmin + zmax); coeff_a = (2.0 + nz) * 0.5; }
    else { zmean = zmin + zmax; coeff_a = (1.0 + nz) * 1.0; }
    for (int k = 1; k <= nz + 1; ++k)
        zz[k + 2] = zmean + (zmin - zmean) / tanh(2.0 * p->zstretch) * tanh(2.0 * p->zstretch * (k - coeff_a) / (1.0 - coeff_a));
    for (int k = kstr3; k <= kend3; ++k) dz[k] = zz[k + 1] - zz[k];
    dz[kstr3 - 1] = dz[kstr3]; dz[kend3 + 1] = dz[kend3];
    dz[kstr3 - 2] = dz[kstr3]; dz[kend3 + 2] = dz[kend3];
    for (int k = kstr3 - 1; k <= kend3 + 1; ++k) {
        lt[k] = dz[k] / (dz[k] + dz[k + 1]);
        lb[k] = dz[k] / (dz[k] + dz[k - 1]);
        dzt[k] = 0.5 * (dz[k] + dz[k + 1]);
        dzb[k] = 0.5 * (dz[k] + dz[k - 1]);
    }
    const std::vector<double>* src[5] = {&dz, &dzt, &dzb, &lt, &lb};
    for (int q = 0; q < 5; ++q) {
        z[q].assign(nka, 0.0);
        for (int k = 1; k <= nka; ++k) z[q][k - 1] = (*src[q])[k];
    }
}

// modified wavenumbers of the coefficient builders (src/module_poisson_solver.f90:71-102, 220-247)
static double helm_sym(int cds, int l, int n, double h2, double dt, double dif, double L)
{
    const double th = 2.0 * HC_PI * l / n;
    if (cds == 1) return 0.5 * dt * (2.0 * cos(th) - 2.0) * dif / h2;
    if (cds == 2) return dt * (-2.0 * cos(2.0 * th) + 32.0 * cos(th) - 30.0) / 24.0 * dif / h2;
    return 0.5 * dt * dif * (-(2.0 * HC_PI / L * l) * (2.0 * HC_PI / L * l));
}
static double pois_sym(int cds, int l, int n, double h2, double L)
{
    const double th = 2.0 * HC_PI * l / n;
    if (cds == 1) return (2.0 * cos(th) - 2.0) / h2;
    if (cds == 2) return (2.0 * cos(3.0 * th) - 108.0 * cos(2.0 * th) + 1566.0 * cos(th) - 1460.0) / 576.0 / h2;
    return -(2.0 * HC_PI / L * l) * (2.0 * HC_PI / L * l);
}

static int build_tables(hc_handle* h)
{
    const hc_params& p = h->p;
    const int nx = p.nx, ny = p.ny, nz = p.nz, nxh = nx / 2, cds = p.cds;
    const double dx = h->g.dx, dy = h->g.dy, dx2 = h->g.dx2, dy2 = h->g.dy2, dt = p.dt, nu = p.nu, al = p.alpha;
    // layout of the coefficient buffer
    std::vector<double> buf;
    auto put = [&](size_t n) { size_t o = buf.size(); buf.resize(o + n, 0.0); return o; };
    size_t o_hx = put(nxh), o_hy = put(ny), o_hxt = put(nxh), o_hyt = put(ny), o_px = put(nxh), o_py = put(ny);
    size_t o_dx = put(2 * nxh), o_dy = put(2 * ny), o_gx = put(2 * nxh), o_gy = put(2 * ny);
    size_t o_lx = put(nxh), o_ly = put(ny);
    size_t o_k[19];
    for (int q = 0; q < 19; ++q) o_k[q] = put(nz);
    auto lsig = [](int idx, int n) { return idx < n / 2 ? idx : idx - n; };
    for (int l = 0; l < nxh; ++l) {
        buf[o_hx + l] = helm_sym(cds, l, nx, dx2, dt, nu, p.lx);
        buf[o_hxt + l] = helm_sym(cds, l, nx, dx2, dt, al, p.lx);
        buf[o_px + l] = pois_sym(cds, l, nx, dx2, p.lx);
    }
    for (int mm = 0; mm < ny; ++mm) {
        const int m = lsig(mm, ny);
        buf[o_hy + mm] = helm_sym(cds, m, ny, dy2, dt, nu, p.ly);
        buf[o_hyt + mm] = helm_sym(cds, m, ny, dy2, dt, al, p.ly);
        buf[o_py + mm] = pois_sym(cds, m, ny, dy2, p.ly);
    }
    // divergence / gradient / second-derivative symbols of the staggered FD operators
    auto fill_ops = [&](int idx, int n, double hh, double L, size_t od, size_t og, size_t ol, int sgn_idx) {
        const int l = sgn_idx;
        const double th = 2.0 * HC_PI * l / n;
        const double c1 = cos(th), s1 = sin(th), c2 = cos(2.0 * th), s2 = sin(2.0 * th);
        double dre, dim, gre, gim, lap;
        if (cds == 3) {
            // dev_fft_linear_cmplx (src/module_spectral.f90:1274-1340): i 2 pi l / L and
            // -(2 pi l / L)^2, zero on the Nyquist mode
            const double kk = (2 * l == -n) ? 0.0 : 2.0 * HC_PI / L * l;
            dre = 0.0; dim = kk; gre = 0.0; gim = kk; lap = -kk * kk;
        } else if (cds == 1) {
            dre = (1.0 - c1) / hh; dim = s1 / hh;
            gre = (c1 - 1.0) / hh; gim = s1 / hh;
            lap = (2.0 * c1 - 2.0) / (hh * hh);
        } else {
            dre = (27.0 - 28.0 * c1 + c2) / (24.0 * hh); dim = (26.0 * s1 - s2) / (24.0 * hh);
            gre = (-c2 + 28.0 * c1 - 27.0) / (24.0 * hh); gim = (26.0 * s1 - s2) / (24.0 * hh);
            lap = (-2.0 * c2 + 32.0 * c1 - 30.0) / (12.0 * hh * hh);
        }
        buf[od + 2 * idx] = dre; buf[od + 2 * idx + 1] = dim;
        buf[og + 2 * idx] = gre; buf[og + 2 * idx + 1] = gim;
        buf[ol + idx] = lap;
    };
    for (int l = 0; l < nxh; ++l) fill_ops(l, nx, dx, p.lx, o_dx, o_gx, o_lx, l);
    for (int mm = 0; mm < ny; ++mm) fill_ops(mm, ny, dy, p.ly, o_dy, o_gy, o_ly, lsig(mm, ny));
    // per-k Thomas coefficients (interior level kk = Fortran k-3)
    const std::vector<double>& DZ = h->zhost[0];
    const std::vector<double>& DZT = h->zhost[1];
    const std::vector<double>& DZB = h->zhost[2];
    auto dz = [&](int kk) { return DZ[kk + 2]; };
    auto dzt = [&](int kk) { return DZT[kk + 2]; };
    auto dzb = [&](int kk) { return DZB[kk + 2]; };
    double* au = &buf[o_k[0]]; double* cu = &buf[o_k[1]]; double* dgu = &buf[o_k[2]]; double* d0u = &buf[o_k[3]];
    double* aw = &buf[o_k[4]]; double* cw = &buf[o_k[5]]; double* dgw = &buf[o_k[6]]; double* d0w = &buf[o_k[7]];
    double* ap = &buf[o_k[8]]; double* cp = &buf[o_k[9]]; double* dgp = &buf[o_k[10]]; double* d0p = &buf[o_k[11]];
    double* at = &buf[o_k[12]]; double* ct = &buf[o_k[13]]; double* dgt = &buf[o_k[14]]; double* d0t = &buf[o_k[15]];
    for (int k = 0; k < nz; ++k) {
        buf[o_k[16] + k] = 1.0 / dz(k);
        buf[o_k[17] + k] = 1.0 / dzt(k);
        buf[o_k[18] + k] = 1.0 / dzb(k);
        // u, v (get_u_eqn_coeff :198-278)
        double a0 = -0.5 * dt * nu / dz(k) / dzb(k), c0 = -0.5 * dt * nu / dz(k) / dzt(k);
        au[k] = k == 0 ? 0.0 : a0;
        cu[k] = k == nz - 1 ? 0.0 : c0;
        dgu[k] = -(k == 0 ? 0.0 : a0) - (k == nz - 1 ? 0.0 : c0);
        d0u[k] = -a0 - c0;
        if (k == 0) d0u[k] = d0u[k] - a0;
        if (k == nz - 1) d0u[k] = p.ochannel == 0 ? d0u[k] - c0 : d0u[k] + c0;
        // t (get_t_eqn_coeff :396-473)
        double a0t = -0.5 * dt * al / dz(k) / dzb(k), c0t = -0.5 * dt * al / dz(k) / dzt(k);
        at[k] = k == 0 ? 0.0 : a0t;
        ct[k] = k == nz - 1 ? 0.0 : c0t;
        dgt[k] = -(k == 0 ? 0.0 : a0t) - (k == nz - 1 ? 0.0 : c0t);
        d0t[k] = -a0t - c0t;
        // the bottom ghost folds with -1 (fixed T) or +1 (fixed gradient)
        if (k == 0) d0t[k] = p.tbc_bot ? d0t[k] + a0t : d0t[k] - a0t;
        if (k == nz - 1) d0t[k] = d0t[k] - c0t;
        // p (get_p_eqn_coeff :49-118)
        double a0p = 1.0 / dz(k) / dzb(k), c0p = 1.0 / dz(k) / dzt(k);
        ap[k] = k == 0 ? 0.0 : a0p;
        cp[k] = k == nz - 1 ? 0.0 : c0p;
        dgp[k] = -(k == 0 ? 0.0 : a0p) - (k == nz - 1 ? 0.0 : c0p);
        d0p[k] = -a0p - c0p;
        if (k == 0) d0p[k] = d0p[k] + a0p;
        if (k == nz - 1) d0p[k] = d0p[k] + c0p;
        // w (get_w_eqn_coeff :304-370), rows 0..nz-2
        if (k <= nz - 2) {
            double a0w = -0.5 * dt * nu / dz(k) / dzt(k), c0w = -0.5 * dt * nu / dz(k + 1) / dzt(k);
            aw[k] = k == 0 ? 0.0 : a0w;
            cw[k] = k == nz - 2 ? 0.0 : c0w;
            dgw[k] = -(k == 0 ? 0.0 : a0w) - (k == nz - 2 ? 0.0 : c0w);
            d0w[k] = -a0w - c0w;
        }
    }
    CK(cudaMalloc(&h->coef, buf.size() * sizeof(double)));
    CK(cudaMemcpy(h->coef, buf.data(), buf.size() * sizeof(double), cudaMemcpyHostToDevice));
    double* b = h->coef;
    ColCoef& c = h->cc;
    c.hx = b + o_hx; c.hy = b + o_hy; c.hxt = b + o_hxt; c.hyt = b + o_hyt; c.px = b + o_px; c.py = b + o_py;
    c.dx = (const double2*)(b + o_dx); c.dy = (const double2*)(b + o_dy);
    c.gx = (const double2*)(b + o_gx); c.gy = (const double2*)(b + o_gy);
    c.lx = b + o_lx; c.ly = b + o_ly;
    c.au = b + o_k[0]; c.cu = b + o_k[1]; c.dgu = b + o_k[2]; c.d0u = b + o_k[3];
    c.aw = b + o_k[4]; c.cw = b + o_k[5]; c.dgw = b + o_k[6]; c.d0w = b + o_k[7];
    c.ap = b + o_k[8]; c.cp = b + o_k[9]; c.dgp = b + o_k[10]; c.d0p = b + o_k[11];
    c.at = b + o_k[12]; c.ct = b + o_k[13]; c.dgt = b + o_k[14]; c.d0t = b + o_k[15];
    c.rdz = b + o_k[16]; c.rdzt = b + o_k[17]; c.rdzb = b + o_k[18];
    return HC_OK;
}

static int upload_zgrid(hc_handle* h)
{
    const int nka = h->p.nz + 4, nz = h->p.nz;
    for (int q = 0; q < 5; ++q)
        CK(cudaMemcpy(h->zbuf + q * nka, h->zhost[q].data(), nka * sizeof(double), cudaMemcpyHostToDevice));
    h->g.z.dz = h->zbuf; h->g.z.dz_t = h->zbuf + nka; h->g.z.dz_b = h->zbuf + 2 * nka;
    h->g.z.l_t = h->zbuf + 3 * nka; h->g.z.l_b = h->zbuf + 4 * nka;
    // per-level metrics of the strip RHS, [5][nz]: 1/dz, 1/dz_t, 1/dz_b, l_t, 1/dz(k+1)
    // (interior level k at Fortran index k+2 of the host arrays), in FP64 and in FP32
    std::vector<double> zd(5 * (size_t)nz);
    std::vector<float> zm(5 * (size_t)nz);
    for (int k = 0; k < nz; ++k) {
        zd[k] = 1.0 / h->zhost[0][k + 2];
        zd[nz + k] = 1.0 / h->zhost[1][k + 2];
        zd[2 * nz + k] = 1.0 / h->zhost[2][k + 2];
        zd[3 * nz + k] = h->zhost[3][k + 2];
        zd[4 * nz + k] = 1.0 / h->zhost[0][k + 3];
        zm[k] = 1.0f / (float)h->zhost[0][k + 2];
        zm[nz + k] = 1.0f / (float)h->zhost[1][k + 2];
        zm[2 * nz + k] = 1.0f / (float)h->zhost[2][k + 2];
        zm[3 * nz + k] = (float)h->zhost[3][k + 2];
        zm[4 * nz + k] = 1.0f / (float)h->zhost[0][k + 3];
    }
    h->zm5d = h->zbuf + 5 * nka;
    h->zm5 = reinterpret_cast<float*>(h->zm5d + 5 * nz);
    CK(cudaMemcpy(h->zm5d, zd.data(), zd.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->zm5, zm.data(), zm.size() * sizeof(float), cudaMemcpyHostToDevice));
    return HC_OK;
}

#include "hc_host_fft.cuh"

#include "hc_host_step.cuh"

#include "hc_host_spec.cuh"

#include "hc_host_adjoint.cuh"

// ---------------------------------------------------------------------------
// C-ABI
// ---------------------------------------------------------------------------
extern "C" {

const char* hc_error_string(int code)
{
    switch (code) {
    case HC_OK: return "ok";
    case HC_ERR_ARG: return "bad argument";
    case HC_ERR_PARAM: return "parameter check failed";
    case HC_ERR_CUDA: return "CUDA error";
    case HC_ERR_NOMEM: return "device allocation failed";
    case HC_ERR_NAN: return "NaN error";
    case HC_ERR_STATE: return "call out of order";
    case HC_ERR_UNSUPPORTED: return "option not supported";
    case HC_ERR_SIZE: return "size beyond the documented maximum";
    }
    return "unknown error";
}

static void graph_drop(hc_handle* h)
{
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    h->gexec = nullptr;
    adj_graph_drop(h);
}

// Capture one full step (all sub-steps, statistics, finaliser) of this handle
// into an executable graph. Every kernel argument of a step is the same from
// step to step (the step counter and the diagnostics slot live on the device),
// so the graph stays valid until a buffer it refers to changes.
static int graph_build(hc_handle* h)
{
    if (h->gexec) return HC_OK;
    const long long l0 = h->launches;
    CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
    int rc = h->rsz == sizeof(float) ? step_dispatch<float>(h) : step_dispatch<double>(h);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(h->st, &g);
    if (rc || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        h->launches = l0;
        return rc ? rc : HC_ERR_CUDA;
    }
    h->graph_launches = h->launches - l0;
    h->launches = l0;
    e = cudaGraphInstantiate(&h->gexec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { h->gexec = nullptr; return HC_ERR_CUDA; }
    return HC_OK;
}

static void free_all(hc_handle* h)
{
    graph_drop(h);
    for (int q = 0; q < NFLD; ++q) if (h->fld[q]) cudaFree(h->fld[q]);
    for (int q = 0; q < 4; ++q) if (h->spec[q]) cudaFree(h->spec[q]);
    for (int q = 0; q < NSP; ++q) if (h->sp[q]) cudaFree(h->sp[q]);
    if (h->dsig) cudaFree(h->dsig);
    if (h->dstale) cudaFree(h->dstale);
    for (int q = 0; q < 3; ++q) if (h->bf[q]) cudaFree(h->bf[q]);
    if (h->adj_buf) cudaFree(h->adj_buf);
    if (h->adj_sc) cudaFree(h->adj_sc);
    if (h->dmean) cudaFree(h->dmean);
    for (int q = 0; q < 11; ++q) if (h->mean[q]) cudaFree(h->mean[q]);
    for (int q = 0; q < 11; ++q) if (h->win[q]) cudaFree(h->win[q]);
    if (h->mtmp) cudaFree(h->mtmp);
    if (h->mw0) cudaFree(h->mw0);
    if (h->zbuf) cudaFree(h->zbuf);
    if (h->coef) cudaFree(h->coef);
    if (h->scratch) cudaFree(h->scratch);
    if (h->part_div) cudaFree(h->part_div);
    if (h->part_st) cudaFree(h->part_st);
    if (h->sc) cudaFree(h->sc);
    if (h->diag_dev) cudaFree(h->diag_dev);
    if (h->twt && h->twt != (void*)h->twbuf) cudaFree(h->twt);
    if (h->twbuf) cudaFree(h->twbuf);
    for (size_t q = 0; q < h->ev_pool.size(); ++q) cudaEventDestroy(h->ev_pool[q]);
    if (h->e0) cudaEventDestroy(h->e0);
    if (h->e1) cudaEventDestroy(h->e1);
    if (h->st) cudaStreamDestroy(h->st);
}

int hc_create(const hc_params* p, hc_handle** out)
{
    if (!p || !out) return HC_ERR_ARG;
    *out = nullptr;
    // initiate_parameters checks (src/module_parameters.f90:266-270) and this engine's limits
    if (p->nx % 2 != 0 || p->ny % 2 != 0) return HC_ERR_PARAM;
    if (p->nx < 8 || p->ny < 4 || p->nz < 3) return HC_ERR_PARAM;
    if (p->cds < 1 || p->cds > 3 || (p->dts != 1 && p->dts != 2) || p->dt <= 0.0) return HC_ERR_PARAM;
    if (p->isscalar != 0 && p->isscalar != 1) return HC_ERR_PARAM;
    if (p->tbc_bot != 0 && p->tbc_bot != 1) return HC_ERR_PARAM;
    if (p->dp_opt < 1 || p->dp_opt > 3) return HC_ERR_PARAM;
    if (p->precision != HC_PREC_FP64 && p->precision != HC_PREC_MIXED) return HC_ERR_PARAM;
    if (p->isdamp == 1 && (p->nzdamp < 1 || p->nzdamp > p->nz - 1)) return HC_ERR_PARAM;
    // the spectral column kernel keeps a whole column in one warp (nz <= 256)
    if (p->cds == 3 && p->nz > 256) return HC_ERR_UNSUPPORTED;

    hc_handle* h = new hc_handle();
    memset((void*)&h->p, 0, sizeof(h->p));
    h->p = *p;
    for (int q = 0; q < NFLD; ++q) h->fld[q] = nullptr;
    for (int q = 0; q < 4; ++q) h->spec[q] = nullptr;
    for (int q = 0; q < NSP; ++q) h->sp[q] = nullptr;
    h->dsig = nullptr; h->dmean = nullptr; h->dstale = nullptr; h->div_in_rhs = 0;
    h->bf[0] = h->bf[1] = h->bf[2] = nullptr; h->has_bf = 0;
    h->adj_buf = nullptr; h->adj_bytes = 0; h->adj_sc = nullptr; h->adj_nsc = 0;
    h->adj_tape_seg = -1; h->adj_gnext = 0;
    for (int q = 0; q < ADJ_GRAPHS; ++q) { h->adj_gexec[q] = nullptr; h->adj_gkey[q] = -1; }
    h->use_graph = 0; h->gexec = nullptr; h->graph_launches = 0; h->rec = nullptr; h->rhs_strip = 0;
    for (int q = 0; q < 11; ++q) { h->mean[q] = nullptr; h->win[q] = nullptr; }
    h->mtmp = nullptr;
    h->mw0 = nullptr;
    h->tdefer = 0;
    h->zbuf = nullptr; h->zm5 = nullptr; h->zm5d = nullptr; h->coef = nullptr; h->scratch = nullptr; h->part_div = nullptr; h->part_st = nullptr;
    h->sc = nullptr; h->diag_dev = nullptr; h->twbuf = nullptr; h->twt = nullptr; h->e0 = nullptr; h->e1 = nullptr; h->st = nullptr;
    h->diag_cap = 0; h->last_ms = 0.0; h->launches = 0; h->initialized = 0;
    h->prof = 0; h->cur_cat = 0; h->ev_used = 0;
    for (int q = 0; q < K_NCAT; ++q) { h->cat_ms[q] = 0.0; h->cat_n[q] = 0; }
    int rc = HC_OK;
#define FAIL(code) do { rc = (code); goto fail; } while (0)
    {
        if (cudaGetDevice(&h->dev) != cudaSuccess) FAIL(HC_ERR_CUDA);
        if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) FAIL(HC_ERR_CUDA);
        if (cudaEventCreate(&h->e0) != cudaSuccess || cudaEventCreate(&h->e1) != cudaSuccess) FAIL(HC_ERR_CUDA);
        h->rsz = p->precision == HC_PREC_MIXED ? sizeof(float) : sizeof(double);
        Geo& g = h->g;
        g.nx = p->nx; g.ny = p->ny; g.nz = p->nz; g.nxh = p->nx / 2;
        g.nxy = (long long)p->nx * p->ny; g.n = g.nxy * p->nz; g.ncol = (long long)g.nxh * p->ny;
        g.dx = p->lx / p->nx; g.dy = p->ly / p->ny; g.dx2 = g.dx * g.dx; g.dy2 = g.dy * g.dy;
        Phys& ph = h->ph;
        ph.dt = p->dt; ph.nu = p->nu; ph.alpha = p->alpha; ph.um = p->u_mrf; ph.fc = p->fc; ph.ug = p->ug;
        ph.vg = p->vg; ph.t_ref = p->t_ref; ph.tbot = p->tbot; ph.ttop = p->ttop;
        ph.cds = p->cds; ph.dp_opt = p->dp_opt; ph.isscalar = p->isscalar; ph.ochannel = p->ochannel; ph.dts = p->dts;
        h->dpx_coef = p->nu * 1.0;
        mesh_host(p, h->zhost);
        const long long n = g.n;
        for (int q = 0; q < NFLD; ++q) {
            if (cudaMalloc(&h->fld[q], n * h->rsz) != cudaSuccess) FAIL(HC_ERR_NOMEM);
            if (cudaMemset(h->fld[q], 0, n * h->rsz) != cudaSuccess) FAIL(HC_ERR_CUDA);
        }
        for (int q = 0; q < 4; ++q) {
            if (cudaMalloc(&h->spec[q], g.ncol * g.nz * 2 * h->rsz) != cudaSuccess) FAIL(HC_ERR_NOMEM);
            if (cudaMemset(h->spec[q], 0, g.ncol * g.nz * 2 * h->rsz) != cudaSuccess) FAIL(HC_ERR_CUDA);
        }
        for (int q = 0; q < 11; ++q) {
            if (cudaMalloc(&h->mean[q], n * sizeof(double)) != cudaSuccess) FAIL(HC_ERR_NOMEM);
            if (cudaMemset(h->mean[q], 0, n * sizeof(double)) != cudaSuccess) FAIL(HC_ERR_CUDA);
            if (h->rsz == sizeof(float)) {
                if (cudaMalloc(&h->win[q], n * sizeof(float)) != cudaSuccess) FAIL(HC_ERR_NOMEM);
                if (cudaMemset(h->win[q], 0, n * sizeof(float)) != cudaSuccess) FAIL(HC_ERR_CUDA);
            }
        }
        if (p->isscalar == 0 && p->isdamp == 0) {
            if (cudaMalloc(&h->mw0, n * sizeof(double)) != cudaSuccess) FAIL(HC_ERR_NOMEM);
            if (cudaMemset(h->mw0, 0, n * sizeof(double)) != cudaSuccess) FAIL(HC_ERR_CUDA);
            h->tdefer = 1;
        }
        if (p->cds == 3) {
            const int nsp = SP_W0 + (p->issk == 1 ? 14 : 8);
            for (int q = 0; q < nsp; ++q) {
                if (cudaMalloc(&h->sp[q], n * h->rsz) != cudaSuccess) FAIL(HC_ERR_NOMEM);
                if (cudaMemset(h->sp[q], 0, n * h->rsz) != cudaSuccess) FAIL(HC_ERR_CUDA);
            }
        }
        if (p->cds == 3 || p->isdamp == 1) {
            if (cudaMalloc(&h->dmean, 5 * p->nz * sizeof(double)) != cudaSuccess) FAIL(HC_ERR_NOMEM);
            if (cudaMemset(h->dmean, 0, 5 * p->nz * sizeof(double)) != cudaSuccess) FAIL(HC_ERR_CUDA);
        }
        if (p->isdamp == 1) {
            // sigma of rayleigh_damping / rayleigh_damping_spec (src/module_tools.f90:705-749,
            // src/module_spectral.f90:1345-1391) per level
            std::vector<double> sig(p->nz, 0.0);
            const int nzd = p->nzdamp;
            for (int kk = p->nz - 1 - nzd; kk < p->nz; ++kk) {
                const double zd = (kk - (p->nz - 1) + nzd) * 1.0 / nzd;
                sig[kk] = p->cdamp * 0.5 * (1.0 - cos(HC_PI * zd));
            }
            if (cudaMalloc(&h->dsig, p->nz * sizeof(double)) != cudaSuccess) FAIL(HC_ERR_NOMEM);
            if (cudaMemcpy(h->dsig, sig.data(), p->nz * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) FAIL(HC_ERR_CUDA);
            if (p->cds != 3) {
                const size_t sb = (size_t)5 * (nzd + 1) * g.nxy * h->rsz;
                if (cudaMalloc(&h->dstale, sb) != cudaSuccess) FAIL(HC_ERR_NOMEM);
            }
        }
        h->div_in_rhs = p->cds != 3 && p->isdamp != 1;
        const long long cz = g.ncol * g.nz;
        if (cudaMalloc(&h->scratch, cz * (3 * sizeof(double) + 4 * sizeof(double2))) != cudaSuccess) FAIL(HC_ERR_NOMEM);
        h->cs.bu = h->scratch; h->cs.bw = h->scratch + cz; h->cs.bp = h->scratch + 2 * cz;
        h->cs.su = (double2*)(h->scratch + 3 * cz); h->cs.sv = h->cs.su + cz; h->cs.sw = h->cs.sv + cz; h->cs.sp = h->cs.sw + cz;
        if (cudaMalloc(&h->zbuf, 5 * (p->nz + 4) * sizeof(double) + 5 * (size_t)p->nz * (sizeof(double) + sizeof(float))) !=
            cudaSuccess)
            FAIL(HC_ERR_NOMEM);
        if ((rc = upload_zgrid(h)) != HC_OK) goto fail;
        if ((rc = build_tables(h)) != HC_OK) goto fail;
        if ((rc = build_fft(h)) != HC_OK) goto fail;
        rc = h->rsz == sizeof(float) ? set_smem_attrs<float>() : set_smem_attrs<double>();
        if (rc != HC_OK) goto fail;
        h->nbd = (g.n + 255) / 256;
        if (h->nbd > RED_BLOCKS) h->nbd = RED_BLOCKS;
        {
            // momentum RHS tiles: enough blocks for ~4 per SM, chunks of 4..32 levels
            h->rhs_strip = rhs_strip_ok(p->nx, p->ny, p->u_mrf, p->dp_opt, h->rsz);
            const int tx_pts = h->rhs_strip ? RS_TX : (h->rsz == sizeof(float) ? R2_TX : RT_TX);
            const int ty_pts = h->rhs_strip ? RS_TY : RT_TY;
            const int bx = (g.nx + tx_pts - 1) / tx_pts, by = (g.ny + ty_pts - 1) / ty_pts;
            int kc = p->tile[2] > 0 ? p->tile[2] : (int)((long long)bx * by * p->nz / (4LL * 148));
            if (p->tile[2] <= 0) { if (kc < 4) kc = 4; if (kc > 32) kc = 32; }
            if (kc < 1) kc = 1;
            if (kc > RT_KMAX) kc = RT_KMAX;
            if (kc > p->nz) kc = p->nz;
            h->rhs_kc = kc;
            h->rhs_grid = dim3(bx, by, (p->nz + kc - 1) / kc);
            if (h->rhs_strip) {
                // one block per (tile, level chunk), RsCfg::MINB resident an SM. Unless tile[2]
                // sets it (a negative value: one wave of equal runs, no chunks), the
                // chunk height in [8, 40] that wastes the least of the last wave of
                // blocks, counting two staged levels of start-up per chunk
                int dev_sm = 148;
                cudaDeviceGetAttribute(&dev_sm, cudaDevAttrMultiProcessorCount, h->dev);
                const long long slots = (long long)(h->rsz == sizeof(float) ? RsCfg<float>::MINB : RsCfg<double>::MINB) * dev_sm;
                const long long ntl = (long long)bx * by;
                int best = p->nz < 8 ? p->nz : 8;
                double best_eff = -1.0;
                for (int c = 8; c <= 40 && c <= p->nz; ++c) {
                    const long long nb = ntl * ((p->nz + c - 1) / c);
                    const double waves = (double)((nb + slots - 1) / slots);
                    const double eff = (double)nb / (waves * slots) * c / (c + 2.0) *
                                       (double)p->nz / (double)(c * ((p->nz + c - 1) / c));
                    if (eff > best_eff + 1e-9) { best_eff = eff; best = c; }
                }
                int kcs = p->tile[2] > 0 ? p->tile[2] : best;
                if (kcs > p->nz) kcs = p->nz;
                long long nb = ntl * ((p->nz + kcs - 1) / kcs);
                if (p->tile[2] < 0) { kcs = 0; nb = slots < ntl * p->nz ? slots : ntl * p->nz; }
                h->rhs_kc = kcs;
                h->rhs_grid = dim3((unsigned)nb, 1, 1);
            }
        }
        h->stx = h->rsz == sizeof(float) ? (g.nxy + 511) / 512 : (g.nxy + 255) / 256;   // k_stats: FP32 pairs
        h->sty = (2 * RED_BLOCKS) / h->stx;
        if (h->sty < 1) h->sty = 1;
        if (h->sty > p->nz) h->sty = p->nz;
        h->nbs = h->stx * h->sty;
        h->pd_stride = h->nbd;
        if (h->nbs > h->pd_stride) h->pd_stride = h->nbs;
        if ((long long)h->rhs_grid.x * h->rhs_grid.y * h->rhs_grid.z > h->pd_stride)
            h->pd_stride = (long long)h->rhs_grid.x * h->rhs_grid.y * h->rhs_grid.z;
        if (cudaMalloc(&h->part_div, 3 * h->pd_stride * 3 * sizeof(double)) != cudaSuccess) FAIL(HC_ERR_NOMEM);
        if (cudaMemset(h->part_div, 0, 3 * h->pd_stride * 3 * sizeof(double)) != cudaSuccess) FAIL(HC_ERR_CUDA);
        if (cudaMalloc(&h->part_st, 2 * h->nbs * sizeof(double)) != cudaSuccess) FAIL(HC_ERR_NOMEM);
        if (cudaMalloc(&h->sc, sizeof(DevScalars)) != cudaSuccess) FAIL(HC_ERR_NOMEM);
        DevScalars s0;
        memset(&s0, 0, sizeof(s0));
        s0.dpx_drive = p->dp_opt == 1 ? 1.0 : 0.0;
        s0.got = p->got;
        if (cudaMemcpy(h->sc, &s0, sizeof(s0), cudaMemcpyHostToDevice) != cudaSuccess) FAIL(HC_ERR_CUDA);
        h->diag_cap = 256;
        if (cudaMalloc(&h->diag_dev, h->diag_cap * sizeof(hc_diag)) != cudaSuccess) FAIL(HC_ERR_NOMEM);
    }
    *out = h;
    return HC_OK;
fail:
    free_all(h);
    delete h;
    return rc;
#undef FAIL
}

int hc_destroy(hc_handle* h)
{
    if (!h) return HC_ERR_ARG;
    cudaStreamSynchronize(h->st);
    free_all(h);
    delete h;
    return HC_OK;
}

int hc_set_grid(hc_handle* h, const double* dz, const double* l_t, const double* l_b, const double* dz_t, const double* dz_b)
{
    if (h) h->adj_ready = 0;     // the adjoint checkpoints no longer describe the state
    if (!h || !dz || !l_t || !l_b || !dz_t || !dz_b) return HC_ERR_ARG;
    if (h->initialized) return HC_ERR_STATE;
    const int nka = h->p.nz + 4;
    const double* src[5] = {dz, dz_t, dz_b, l_t, l_b};
    for (int q = 0; q < 5; ++q) h->zhost[q].assign(src[q], src[q] + nka);
    int rc = upload_zgrid(h);
    if (rc) return rc;
    graph_drop(h);
    cudaFree(h->coef);
    h->coef = nullptr;
    return build_tables(h);
}

int hc_get_grid(hc_handle* h, double* dz, double* l_t, double* l_b, double* dz_t, double* dz_b)
{
    if (!h) return HC_ERR_ARG;
    double* dst[5] = {dz, dz_t, dz_b, l_t, l_b};
    for (int q = 0; q < 5; ++q)
        if (dst[q]) memcpy(dst[q], h->zhost[q].data(), (h->p.nz + 4) * sizeof(double));
    return HC_OK;
}

static void* field_dev(hc_handle* h, int id, int* is_mean)
{
    *is_mean = 0;
    switch (id) {
    case HC_FIELD_U: return h->fld[F_U];
    case HC_FIELD_V: return h->fld[F_V];
    case HC_FIELD_W: return h->fld[F_W];
    case HC_FIELD_P: return h->fld[F_P];
    case HC_FIELD_T: return h->fld[F_T];
    case HC_FIELD_FF: return h->fld[F_FF];
    case HC_FIELD_GG: return h->fld[F_GG];
    case HC_FIELD_HH: return h->fld[F_HH];
    case HC_FIELD_SS: return h->fld[F_SS];
    default: break;
    }
    if (id >= HC_FIELD_MEAN_U && id <= HC_FIELD_MEAN_TW) { *is_mean = 1; return h->mean[id - HC_FIELD_MEAN_U]; }
    return nullptr;
}

// Device staging buffer of n doubles (shared with the mean-field download)
static double* staging(hc_handle* h)
{
    if (!h->mtmp && cudaMalloc((void**)&h->mtmp, h->g.n * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return h->mtmp;
}

static __global__ void k_double_to_float(float* __restrict__ dst, const double* __restrict__ src, long long n)
{
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        dst[q] = (float)src[q];
}
static __global__ void k_float_to_double(double* __restrict__ dst, const float* __restrict__ src, long long n)
{
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        dst[q] = (double)src[q];
}

// An interior-only host array (ghost 0, leading dimensions nx, ny) is copied as
// it is -- straight from the caller's memory, pinned or not -- and converted to
// the storage type on the device; ghosted arrays are packed on the host first.
// Adds the deferred temperature terms of the statistics (no temperature
// equation) to mean_t, mean_tt, mean_tw and restarts the deferral from the
// current mean_w sums.
static int tstat_flush(hc_handle* h)
{
    if (!h->tdefer) return HC_OK;
    const long long n = h->g.n;
    const float* ww = h->win[2];
    if (h->rsz == sizeof(float))
        k_tstat_flush<float><<<RED_BLOCKS, 256, 0, h->st>>>((const float*)h->fld[F_T], h->mean[3], h->mean[9], h->mean[10],
                                                           h->mean[2], ww, h->mw0, &h->sc->tstat_n, h->g.nxy, n);
    else
        k_tstat_flush<double><<<RED_BLOCKS, 256, 0, h->st>>>((const double*)h->fld[F_T], h->mean[3], h->mean[9], h->mean[10],
                                                            h->mean[2], ww, h->mw0, &h->sc->tstat_n, h->g.nxy, n);
    CK(cudaGetLastError());
    k_tstat_snap<<<RED_BLOCKS, 256, 0, h->st>>>(h->mw0, h->mean[2], ww, &h->sc->tstat_n, n);
    CK(cudaGetLastError());
    return HC_OK;
}

int hc_upload(hc_handle* h, int field_id, const double* host, int ld1, int ld2, int ghost)
{
    if (h) h->adj_ready = 0;     // the adjoint checkpoints no longer describe the state
    if (!h || !host || ghost < 0 || ld1 < h->p.nx + 2 * ghost || ld2 < h->p.ny + 2 * ghost) return HC_ERR_ARG;
    if (h->p.cds == 3 && h->initialized) return HC_ERR_STATE;
    int is_mean;
    void* d = field_dev(h, field_id, &is_mean);
    if (!d) return HC_ERR_ARG;
    // deferred temperature statistics are added with the T they were taken with
    if (field_id == HC_FIELD_T || is_mean) { const int frc = tstat_flush(h); if (frc) return frc; }
    const int nx = h->p.nx, ny = h->p.ny, nz = h->p.nz;
    const long long n = (long long)nx * ny * nz;
    const bool contiguous = ghost == 0 && ld1 == nx && ld2 == ny;
    std::vector<double> tmp;
    const double* src = host;
    if (!contiguous) {
        tmp.resize(n);
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                memcpy(&tmp[((long long)k * ny + j) * nx], host + (size_t)ghost + (size_t)ld1 * ((size_t)(j + ghost) + (size_t)ld2 * (size_t)(k + ghost)), nx * sizeof(double));
        src = tmp.data();
    }
    CK(cudaStreamSynchronize(h->st));
    // every copy and conversion on the handle's stream: a synchronous copy from
    // pageable memory may return before its transfer has landed
    if (is_mean || h->rsz == sizeof(double)) {
        CK(cudaMemcpyAsync(d, src, n * sizeof(double), cudaMemcpyHostToDevice, h->st));
        if (is_mean && h->win[0]) CK(cudaMemsetAsync(h->win[field_id - HC_FIELD_MEAN_U], 0, n * sizeof(float), h->st));
    } else {
        double* st = staging(h);
        if (!st) return HC_ERR_NOMEM;
        CK(cudaMemcpyAsync(st, src, n * sizeof(double), cudaMemcpyHostToDevice, h->st));
        k_double_to_float<<<RED_BLOCKS, 256, 0, h->st>>>((float*)d, st, n);
        CK(cudaGetLastError());
    }
    if (field_id == HC_FIELD_MEAN_W && h->tdefer) {
        k_tstat_snap<<<RED_BLOCKS, 256, 0, h->st>>>(h->mw0, h->mean[2], h->win[2], &h->sc->tstat_n, n);
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(h->st));
    return HC_OK;
}

// On the spectral path p, phi and the histories live as spectra only (after
// hc_initialize); their physical images are produced on request.
static int spec_source(hc_handle* h, int field_id)
{
    if (h->p.cds != 3) return -1;
    if (field_id == HC_FIELD_PHI) return SP_PHI;
    if (!h->initialized) return -1;
    switch (field_id) {
    case HC_FIELD_P: return SP_P;
    case HC_FIELD_FF: return SP_FF;
    case HC_FIELD_GG: return SP_GG;
    case HC_FIELD_HH: return SP_HH;
    case HC_FIELD_SS: return SP_SS;
    default: break;
    }
    return -1;
}

static void* download_source(hc_handle* h, int field_id, int* is_mean, int* rc)
{
    *rc = HC_OK;
    if (field_id == HC_FIELD_MEAN_T || field_id == HC_FIELD_MEAN_TT || field_id == HC_FIELD_MEAN_TW) {
        if ((*rc = tstat_flush(h)) != HC_OK) return nullptr;
    }
    const int sid = spec_source(h, field_id);
    if (sid >= 0) {
        *is_mean = 0;
        void* d = nullptr;
        *rc = h->rsz == sizeof(float) ? spec_image<float>(h, sid, &d) : spec_image<double>(h, sid, &d);
        return *rc ? nullptr : d;
    }
    if (field_id == HC_FIELD_PHI) { *rc = HC_ERR_UNSUPPORTED; return nullptr; }
    void* d = field_dev(h, field_id, is_mean);
    if (!d) { *rc = HC_ERR_ARG; return nullptr; }
    if (*is_mean && h->win[0]) {
        // the FP64 sums plus the FP32 window not folded in yet
        if (!h->mtmp && cudaMalloc((void**)&h->mtmp, h->g.n * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            *rc = HC_ERR_NOMEM;
            return nullptr;
        }
        const int q = field_id - HC_FIELD_MEAN_U;
        k_mean_combine<<<RED_BLOCKS, 256, 0, h->st>>>(h->mtmp, h->mean[q], h->win[q], h->g.n);
        if (cudaGetLastError() != cudaSuccess) { *rc = HC_ERR_CUDA; return nullptr; }
        return h->mtmp;
    }
    return d;
}

int hc_download(hc_handle* h, int field_id, double* host, int ld1, int ld2, int ghost)
{
    if (!h || !host || ghost < 0 || ld1 < h->p.nx + 2 * ghost || ld2 < h->p.ny + 2 * ghost) return HC_ERR_ARG;
    int is_mean, rc;
    void* d = download_source(h, field_id, &is_mean, &rc);
    if (!d) return rc;
    const int nx = h->p.nx, ny = h->p.ny, nz = h->p.nz;
    const long long n = (long long)nx * ny * nz;
    const double* src = (const double*)d;
    if (!is_mean && h->rsz == sizeof(float)) {
        double* st = staging(h);
        if (!st) return HC_ERR_NOMEM;
        k_float_to_double<<<RED_BLOCKS, 256, 0, h->st>>>(st, (const float*)d, n);
        CK(cudaGetLastError());
        src = st;
    }
    if (ghost == 0 && ld1 == nx && ld2 == ny) {
        CK(cudaMemcpyAsync(host, src, n * sizeof(double), cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
        return HC_OK;
    }
    std::vector<double> tmp(n);
    CK(cudaMemcpyAsync(tmp.data(), src, n * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            memcpy(host + (size_t)ghost + (size_t)ld1 * ((size_t)(j + ghost) + (size_t)ld2 * (size_t)(k + ghost)), &tmp[((long long)k * ny + j) * nx], nx * sizeof(double));
    return HC_OK;
}

int hc_set_body_force(hc_handle* h, const double* fx, const double* fy, const double* fz)
{
    if (h) h->adj_ready = 0;     // the adjoint checkpoints no longer describe the state
    if (!h) return HC_ERR_ARG;
    graph_drop(h);
    if (!fx && !fy && !fz) { h->has_bf = 0; return HC_OK; }
    const long long n = h->g.n;
    const double* src[3] = {fx, fy, fz};
    for (int q = 0; q < 3; ++q) {
        if (!h->bf[q]) CK(cudaMalloc(&h->bf[q], n * h->rsz));
        CK(cudaStreamSynchronize(h->st));
        if (!src[q]) { CK(cudaMemset(h->bf[q], 0, n * h->rsz)); continue; }
        if (h->rsz == sizeof(double)) {
            CK(cudaMemcpy(h->bf[q], src[q], n * sizeof(double), cudaMemcpyHostToDevice));
        } else {
            std::vector<float> tf(n);
            for (long long i = 0; i < n; ++i) tf[i] = (float)src[q][i];
            CK(cudaMemcpy(h->bf[q], tf.data(), n * sizeof(float), cudaMemcpyHostToDevice));
        }
    }
    h->has_bf = 1;
    return HC_OK;
}

int hc_upload_dev(hc_handle* h, int field_id, const void* dev)
{
    if (h) h->adj_ready = 0;     // the adjoint checkpoints no longer describe the state
    if (!h || !dev) return HC_ERR_ARG;
    if (h->p.cds == 3 && h->initialized) return HC_ERR_STATE;
    int is_mean;
    void* d = field_dev(h, field_id, &is_mean);
    if (!d) return HC_ERR_ARG;
    if (field_id == HC_FIELD_T || is_mean) { const int frc = tstat_flush(h); if (frc) return frc; }
    const size_t bytes = h->g.n * (is_mean ? sizeof(double) : h->rsz);
    CK(cudaMemcpyAsync(d, dev, bytes, cudaMemcpyDeviceToDevice, h->st));
    if (is_mean && h->win[0]) CK(cudaMemsetAsync(h->win[field_id - HC_FIELD_MEAN_U], 0, h->g.n * sizeof(float), h->st));
    if (field_id == HC_FIELD_MEAN_W && h->tdefer) {
        k_tstat_snap<<<RED_BLOCKS, 256, 0, h->st>>>(h->mw0, h->mean[2], h->win[2], &h->sc->tstat_n, h->g.n);
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(h->st));
    return HC_OK;
}

int hc_download_dev(hc_handle* h, int field_id, void* dev)
{
    if (!h || !dev) return HC_ERR_ARG;
    int is_mean, rc;
    void* d = download_source(h, field_id, &is_mean, &rc);
    if (!d) return rc;
    const size_t bytes = h->g.n * (is_mean ? sizeof(double) : h->rsz);
    CK(cudaMemcpyAsync(dev, d, bytes, cudaMemcpyDeviceToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));
    return HC_OK;
}

int hc_initialize(hc_handle* h)
{
    if (h) h->adj_ready = 0;     // the adjoint checkpoints no longer describe the state
    if (!h) return HC_ERR_ARG;
    const hc_params& p = h->p;
    // update_boundary_uvw sets w = 0 on the top wall before the loop (src/module_navier_stokes.f90:127)
    CK(cudaMemsetAsync((char*)h->fld[F_W] + (size_t)(p.nz - 1) * h->g.nxy * h->rsz, 0, h->g.nxy * h->rsz, h->st));
    DevScalars s0;
    memset(&s0, 0, sizeof(s0));
    s0.dpx_drive = p.dp_opt == 1 ? 1.0 : 0.0;
    s0.got = p.is_ri_var == 1 ? p.ri_str + (p.ri_end - p.ri_str) * 1.0 / p.imax * 0 : p.got;
    CK(cudaMemcpyAsync(h->sc, &s0, sizeof(s0), cudaMemcpyHostToDevice, h->st));
    // calculate_ubar (dp_opt=2) and the CFL of the initial fields
    int rc = h->rsz == sizeof(float) ? launch_stats<float>(h, 0) : launch_stats<double>(h, 0);
    if (rc) return rc;
    rc = launch_finalize(h, 0, 0, 1);   // sets ubar of the fields as given
    if (rc) return rc;
    if (p.cds == 3) {
        // the bulk velocity above is that of the fields as given; the spectral
        // set-up then truncates them, and the first step's CFL sees the truncated ones
        rc = h->rsz == sizeof(float) ? init_sp<float>(h) : init_sp<double>(h);
        if (rc) return rc;
        CK(cudaMemsetAsync((char*)h->fld[F_W] + (size_t)(p.nz - 1) * h->g.nxy * h->rsz, 0, h->g.nxy * h->rsz, h->st));
        rc = h->rsz == sizeof(float) ? launch_stats<float>(h, 0) : launch_stats<double>(h, 0);
        if (rc) return rc;
        rc = launch_finalize(h, 0, 0, 0);   // CFL only, keeps that ubar
        if (rc) return rc;
    }
    CK(cudaStreamSynchronize(h->st));
    h->initialized = 1;
    return HC_OK;
}

int hc_step(hc_handle* h, int nsteps, hc_diag* out)
{
    if (h) h->adj_ready = 0;     // the adjoint checkpoints no longer describe the state
    if (!h || nsteps < 0) return HC_ERR_ARG;
    if (!h->initialized) return HC_ERR_STATE;
    DevScalars s;
    CK(cudaMemcpy(&s, h->sc, sizeof(s), cudaMemcpyDeviceToHost));
    if (s.nan_flag) return HC_ERR_NAN;
    h->launches = 0;
    CK(cudaEventRecord(h->e0, h->st));
    int done = 0;
    int rc = HC_OK;
    float total_ms = 0.0f;
    while (done < nsteps) {
        const int chunk = (nsteps - done) < h->diag_cap ? (nsteps - done) : h->diag_cap;
        const int base = s.step + done + 1;
        const bool graph = h->use_graph && !h->prof;
        if (graph && (rc = graph_build(h))) return rc;
        for (int q = 0; q < chunk; ++q) {
            if (graph) {
                CK(cudaGraphLaunch(h->gexec, h->st));
                h->launches += h->graph_launches;
                continue;
            }
            rc = h->rsz == sizeof(float) ? step_dispatch<float>(h) : step_dispatch<double>(h);
            if (rc) return rc;
            if (h->prof && h->ev_used > 4096) { rc = prof_collect(h); if (rc) return rc; }
        }
        if (out) {
            // the finaliser writes step n into slot (n - 1) % diag_cap
            const int s0 = (base - 1) % h->diag_cap;
            const int n1 = chunk < h->diag_cap - s0 ? chunk : h->diag_cap - s0;
            CK(cudaMemcpyAsync(out + done, h->diag_dev + s0, n1 * sizeof(hc_diag), cudaMemcpyDeviceToHost, h->st));
            if (chunk > n1)
                CK(cudaMemcpyAsync(out + done + n1, h->diag_dev, (chunk - n1) * sizeof(hc_diag), cudaMemcpyDeviceToHost, h->st));
        }
        done += chunk;
    }
    CK(cudaEventRecord(h->e1, h->st));
    CK(cudaEventSynchronize(h->e1));
    CK(cudaEventElapsedTime(&total_ms, h->e0, h->e1));
    h->last_ms = total_ms;
    rc = prof_collect(h);
    if (rc) return rc;
    DevScalars s1;
    CK(cudaMemcpy(&s1, h->sc, sizeof(s1), cudaMemcpyDeviceToHost));
    if (s1.nan_flag) return HC_ERR_NAN;
    return rc;
}

int hc_get_scalars(hc_handle* h, double* time_sim, double* dpx_drive, double* ubar, double* got, double* div_hist_max, int* step)
{
    if (!h) return HC_ERR_ARG;
    DevScalars s;
    CK(cudaStreamSynchronize(h->st));
    CK(cudaMemcpy(&s, h->sc, sizeof(s), cudaMemcpyDeviceToHost));
    if (time_sim) *time_sim = s.time_sim;
    if (dpx_drive) *dpx_drive = s.dpx_drive;
    if (ubar) *ubar = s.ubar;
    if (got) *got = s.got;
    if (div_hist_max) *div_hist_max = s.div_hist;
    if (step) *step = s.step;
    return HC_OK;
}

int hc_last_step_ms(hc_handle* h, double* ms)
{
    if (!h || !ms) return HC_ERR_ARG;
    *ms = h->last_ms;
    return HC_OK;
}

int hc_last_launch_count(hc_handle* h, long long* n)
{
    if (!h || !n) return HC_ERR_ARG;
    *n = h->launches;
    return HC_OK;
}

int hc_set_profiling(hc_handle* h, int enable)
{
    if (!h) return HC_ERR_ARG;
    h->prof = enable ? 1 : 0;
    for (int q = 0; q < K_NCAT; ++q) { h->cat_ms[q] = 0.0; h->cat_n[q] = 0; }
    h->ev_used = 0;
    return HC_OK;
}

int hc_set_graph(hc_handle* h, int enable)
{
    if (!h) return HC_ERR_ARG;
    h->use_graph = enable ? 1 : 0;
    if (!enable) graph_drop(h);
    return HC_OK;
}

#include "hc_host_ensemble.cuh"

int hc_adjoint_forward(hc_handle* h, int nsteps, int ckpt)
{
    if (!h || nsteps < 1 || ckpt < 1) return HC_ERR_ARG;
    if (!h->initialized) return HC_ERR_STATE;
    const hc_params& p = h->p;
    if (h->rsz != sizeof(double) || (p.cds != 1 && p.cds != 2) || (p.dp_opt != 1 && p.dp_opt != 3) ||
        (p.isscalar == 1 && p.is_ri_var != 0) || p.isdamp != 0 || p.nz > 256)
        return HC_ERR_UNSUPPORTED;
    h->adj_ready = 0;
    DevScalars s0;
    CK(cudaMemcpy(&s0, h->sc, sizeof(s0), cudaMemcpyDeviceToHost));
    if (s0.nan_flag) return HC_ERR_NAN;
    const long long n = h->g.n;
    const int nsub = p.dts == 2 ? 3 : 1;
    const int nseg = (nsteps + ckpt - 1) / ckpt;
    const int seglen = ckpt < nsteps ? ckpt : nsteps;
    // 30 adjoint fields, nst per checkpoint, ntp per taped sub-step, nst for the final state
    const size_t nst = p.isscalar == 1 ? 9 : 7, ntp = p.isscalar == 1 ? 5 : 4;
    const size_t nfield = 30 + nst * nseg + ntp * seglen * nsub + nst;
    const size_t bytes = nfield * (size_t)n * sizeof(double);
    if (bytes > h->adj_bytes) {
        adj_graph_drop(h);
        if (h->adj_buf) cudaFree(h->adj_buf);
        h->adj_buf = nullptr; h->adj_bytes = 0;
        if (cudaMalloc((void**)&h->adj_buf, bytes) != cudaSuccess) { cudaGetLastError(); return HC_ERR_NOMEM; }
        h->adj_bytes = bytes;
    }
    if (nseg + 1 > h->adj_nsc) {
        if (h->adj_sc) cudaFree(h->adj_sc);
        h->adj_sc = nullptr; h->adj_nsc = 0;
        if (cudaMalloc((void**)&h->adj_sc, (nseg + 1) * sizeof(DevScalars)) != cudaSuccess) { cudaGetLastError(); return HC_ERR_NOMEM; }
        h->adj_nsc = nseg + 1;
    }
    if (nseg != h->adj_nseg || seglen != h->adj_seglen) adj_graph_drop(h);   // the tape moved
    h->adj_nsteps = nsteps; h->adj_ckpt = ckpt; h->adj_nseg = nseg; h->adj_seglen = seglen;
    AdjBufs b = adj_bufs(h);
    int rc = p.cds == 1 ? adjoint_forward<1>(h, b) : adjoint_forward<2>(h, b);
    if (rc) return rc;
    rc = prof_collect(h);
    if (rc) return rc;
    DevScalars s1;
    CK(cudaMemcpy(&s1, h->sc, sizeof(s1), cudaMemcpyDeviceToHost));
    if (s1.nan_flag) return HC_ERR_NAN;
    h->adj_ready = 1;
    return HC_OK;
}

int hc_adjoint_reverse(hc_handle* h, const double* lu, const double* lv, const double* lw, const double* lp,
                       double* gu, double* gv, double* gw, double* gp, double* gbf)
{
    return hc_adjoint_reverse_t(h, lu, lv, lw, lp, nullptr, gu, gv, gw, gp, nullptr, gbf);
}

int hc_adjoint_reverse_t(hc_handle* h, const double* lu, const double* lv, const double* lw, const double* lp,
                         const double* lt, double* gu, double* gv, double* gw, double* gp, double* gt, double* gbf)
{
    if (!h) return HC_ERR_ARG;
    if (!h->adj_ready) return HC_ERR_STATE;
    if ((lt || gt) && h->p.isscalar != 1) return HC_ERR_ARG;
    AdjBufs b = adj_bufs(h);
    const long long n = h->g.n;
    const size_t fb = (size_t)n * sizeof(double);
    const double* seed[4] = {lu, lv, lw, lp};
    for (int f = 0; f < 4; ++f) {
        if (seed[f]) CK(cudaMemcpyAsync(b.lam[f], seed[f], fb, cudaMemcpyHostToDevice, h->st));
        else CK(cudaMemsetAsync(b.lam[f], 0, fb, h->st));
    }
    for (int f = 0; f < 3; ++f) {
        CK(cudaMemsetAsync(b.lh[f], 0, fb, h->st));
        CK(cudaMemsetAsync(b.lbf[f], 0, fb, h->st));
    }
    if (lt) CK(cudaMemcpyAsync(b.lt, lt, fb, cudaMemcpyHostToDevice, h->st));
    else CK(cudaMemsetAsync(b.lt, 0, fb, h->st));
    CK(cudaMemsetAsync(b.ls, 0, fb, h->st));
    int rc = h->p.cds == 1 ? adjoint_reverse<1>(h, b) : adjoint_reverse<2>(h, b);
    if (rc) { h->adj_ready = 0; return rc; }
    rc = prof_collect(h);
    if (rc) return rc;
    double* out[4] = {gu, gv, gw, gp};
    for (int f = 0; f < 4; ++f)
        if (out[f]) CK(cudaMemcpyAsync(out[f], b.lam[f], fb, cudaMemcpyDeviceToHost, h->st));
    if (gbf)
        for (int f = 0; f < 3; ++f) CK(cudaMemcpyAsync(gbf + (size_t)f * n, b.lbf[f], fb, cudaMemcpyDeviceToHost, h->st));
    if (gt) CK(cudaMemcpyAsync(gt, b.lt, fb, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    DevScalars s1;
    CK(cudaMemcpy(&s1, h->sc, sizeof(s1), cudaMemcpyDeviceToHost));
    if (s1.nan_flag) return HC_ERR_NAN;
    return HC_OK;
}

int hc_adjoint(hc_handle* h, int nsteps, int ckpt, const double* lu, const double* lv, const double* lw, const double* lp,
               double* gu, double* gv, double* gw, double* gp, double* gbf)
{
    int rc = hc_adjoint_forward(h, nsteps, ckpt);
    if (rc) return rc;
    return hc_adjoint_reverse(h, lu, lv, lw, lp, gu, gv, gw, gp, gbf);
}

int hc_adjoint_last_ms(hc_handle* h, double* forward_ms, double* reverse_ms, long long* forward_launches,
                       long long* reverse_launches)
{
    if (!h) return HC_ERR_ARG;
    if (forward_ms) *forward_ms = h->adj_ms[0];
    if (reverse_ms) *reverse_ms = h->adj_ms[1];
    if (forward_launches) *forward_launches = h->adj_launches[0];
    if (reverse_launches) *reverse_launches = h->adj_launches[1];
    return HC_OK;
}

int hc_kernel_profile(hc_handle* h, int max, char* names, double* total_ms, long long* launches, int* count)
{
    if (!h || !count) return HC_ERR_ARG;
    int n = 0;
    for (int q = 0; q < K_NCAT && n < max; ++q) {
        if (h->cat_n[q] == 0) continue;
        if (names) { strncpy(names + 32 * n, K_NAMES[q], 31); names[32 * n + 31] = 0; }
        if (total_ms) total_ms[n] = h->cat_ms[q];
        if (launches) launches[n] = h->cat_n[q];
        ++n;
    }
    *count = n;
    return HC_OK;
}

}  // extern "C"
