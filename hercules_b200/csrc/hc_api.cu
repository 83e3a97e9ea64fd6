// hc_api.cu -- C-ABI of the B200 time-step engine (declared in include/hercules_b200.h).
//
// One handle owns one channel: its device state, one CUDA stream and the host
// set-up that the reference's `drive` performs before the time loop
// (src/module_navier_stokes.f90:53-129). hc_step issues, per RK sub-step,
//   substep_begin -> momentum RHS -> r2c x -> c2c y -> column solve (3 Helmholtz +
//   phi Poisson + projection) -> c2c y^-1 -> c2r x^-1 (+ p update)
//   [-> temperature RHS -> FFT -> T column solve -> iFFT] -> divergence check
// and per step the statistics/bulk-velocity/CFL pass and a one-block finaliser
// that writes the step's diagnostics and the next step's scalars on the device.
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
       K_ADJ_RHS, K_FFT2D_FWD, K_FFT2D_INV, K_NCAT };
static const char* K_NAMES[K_NCAT] = {"substep_begin", "rhs_momentum", "fft_x_r2c", "fft_y_fwd", "column_fd",
                                      "fft_y_inv", "fft_x_c2r", "rhs_temperature", "column_t", "div_check",
                                      "stats", "finalize", "spec_products", "spec_assemble", "aux", "adj_column",
                                      "adj_rhs", "fft2d_fwd", "fft2d_inv"};

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

// ---------------------------------------------------------------------------
// compile-time-length FFT kernels (hc_fft_t.cuh): lengths with a specialisation
// ---------------------------------------------------------------------------
#define HC_FFT_T_RMAX 16
#define HC_FFT_T_LENGTHS(X) X(8) X(12) X(16) X(24) X(32) X(40) X(48) X(64) X(80) X(96) X(128) X(160) \
    X(192) X(256) X(320) X(384) X(512)

static bool fft_t_length_ok(int n)
{
    switch (n) {
#define HC_LEN_CASE(N) case N: return true;
    HC_FFT_T_LENGTHS(HC_LEN_CASE)
#undef HC_LEN_CASE
    }
    return false;
}

// op 0: raise the shared-memory limit of the kernels this handle uses;
// op 1: x forward, 2: x inverse, 3: y forward, 4: y inverse
template <typename R, int N> static int fft_t_op(hc_handle* h, int op, const void* args, dim3 grid)
{
    constexpr int RM = HC_FFT_T_RMAX;
    constexpr size_t sx = fft_x_smem<R, N, RM>();
    constexpr size_t sy = fft_y_smem<R, N, RM>();
    static_assert(FPlan<N, RM>::valid, "length must be 2^a 3^b 5^c");
    if (op == 0) {
        if (N == h->g.nxh && h->fft_tx) {
            CK(cudaFuncSetAttribute(k_fft_x_r2c_t<R, N, RM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sx));
            CK(cudaFuncSetAttribute(k_fft_x_c2r_t<R, N, RM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sx));
        }
        if (N == h->g.ny && h->fft_ty) {
            CK(cudaFuncSetAttribute(FyKernel<R, N, -1, RM>::f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sy));
            CK(cudaFuncSetAttribute(FyKernel<R, N, 1, RM>::f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sy));
        }
        return HC_OK;
    }
    constexpr int TX = FxThreads<R, N>::v, TY = FyThreads<R, N>::v;
    if (op == 1)
        return hc_launch<FxArgs<R>, k_fft_x_r2c_t<R, N, RM>, k_fft_x_r2c_t_body<R, N, RM>, TX, 1>(
            h, grid, dim3(TX), sx, *(const FxArgs<R>*)args);
    if (op == 2)
        return hc_launch<FxArgs<R>, k_fft_x_c2r_t<R, N, RM>, k_fft_x_c2r_t_body<R, N, RM>, TX, 1>(
            h, grid, dim3(TX), sx, *(const FxArgs<R>*)args);
    if (op == 3)
        return hc_launch<FyArgs<R>, FyKernel<R, N, -1, RM>::f, k_fft_y_t_body<R, N, -1, RM>, TY, FyKernel<R, N, -1, RM>::minb>(
            h, grid, dim3(TY), sy, *(const FyArgs<R>*)args);
    return hc_launch<FyArgs<R>, FyKernel<R, N, 1, RM>::f, k_fft_y_t_body<R, N, 1, RM>, TY, FyKernel<R, N, 1, RM>::minb>(
        h, grid, dim3(TY), sy, *(const FyArgs<R>*)args);
}

template <typename R> static int fft_t_dispatch(hc_handle* h, int n, int op, const void* args, dim3 grid)
{
    switch (n) {
#define HC_LEN_CASE(N) case N: return fft_t_op<R, N>(h, op, args, grid);
    HC_FFT_T_LENGTHS(HC_LEN_CASE)
#undef HC_LEN_CASE
    }
    return HC_ERR_UNSUPPORTED;
}

// ---------------------------------------------------------------------------
// fused 2-D transforms (hc_fft2d.cuh): one cluster of C CTAs a (field, plane).
// Shapes: nx/2, ny, C, threads a CTA, resident CTAs an SM with FP32 / FP64 storage
// ---------------------------------------------------------------------------
#define HC_FFT2D_SHAPES(X) X(256, 384, 16, 384, 2, 1) X(128, 256, 8, 256, 3, 1) X(128, 192, 8, 256, 3, 1)

template <typename R, int NXH, int NY, int C, int NT, int MINB>
static int fft2d_op(hc_handle* h, int op, const F2Args<R>* a, int nf)
{
    typedef F2Shape<R, NXH, NY, C, NT, MINB> S;
    void (*fwd)(F2Args<R>) = k_fft2d_fwd<R, NXH, NY, C, NT, MINB>;
    void (*inv)(F2Args<R>) = k_fft2d_inv<R, NXH, NY, C, NT, MINB>;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = C; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(NT);
    cfg.dynamicSmemBytes = S::smem;
    cfg.stream = h->st;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    if (op == 0) {
        // shared-memory limit and cluster size; usable only if a cluster fits the device
        for (int q = 0; q < 2; ++q) {
            const void* k = (const void*)(q == 0 ? fwd : inv);
            if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::smem) != cudaSuccess) return HC_ERR_UNSUPPORTED;
            if (C > 8 && cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) return HC_ERR_UNSUPPORTED;
            int ncl = 0;
            cfg.gridDim = dim3(C);
            if (cudaOccupancyMaxActiveClusters(&ncl, k, &cfg) != cudaSuccess || ncl < 1) {
                cudaGetLastError();
                return HC_ERR_UNSUPPORTED;
            }
        }
        return HC_OK;
    }
    cfg.gridDim = dim3((unsigned)((long long)nf * h->g.nz * C));
    CK(cudaLaunchKernelEx(&cfg, op == 1 ? fwd : inv, *a));
    return HC_OK;
}

// op 0: set up (HC_ERR_UNSUPPORTED: no fused shape for this grid); 1 forward; 2 inverse
template <typename R> static int fft2d_dispatch(hc_handle* h, int op, const F2Args<R>* a, int nf)
{
    const int nxh = h->g.nxh, ny = h->g.ny;
#define HC_F2_CASE(NXH, NY, C, NT, M32, M64) \
    if (nxh == NXH && ny == NY) return fft2d_op<R, NXH, NY, C, NT, sizeof(R) == sizeof(float) ? M32 : M64>(h, op, a, nf);
    HC_FFT2D_SHAPES(HC_F2_CASE)
#undef HC_F2_CASE
    return HC_ERR_UNSUPPORTED;
}

template <typename R> static int fft_t_setup(hc_handle* h)
{
    int rc = HC_OK;
    if (h->fft_tx) rc = fft_t_dispatch<R>(h, h->g.nxh, 0, nullptr, dim3());
    if (rc == HC_OK && h->fft_ty && !(h->fft_tx && h->g.ny == h->g.nxh))
        rc = fft_t_dispatch<R>(h, h->g.ny, 0, nullptr, dim3());
    return rc;
}

// y tile width (columns l per block) of the length-n kernel
template <typename R> static int fft_t_ytl(int n)
{
    switch (n) {
#define HC_LEN_CASE(N) case N: return FyLines<R, N>::v;
    HC_FFT_T_LENGTHS(HC_LEN_CASE)
#undef HC_LEN_CASE
    }
    return 1;
}

template <typename R> static long long fft_t_xblocks(int n, long long nrows)
{
    long long lines = 1;
    switch (n) {
#define HC_LEN_CASE(N) case N: lines = FxLines<R, N>::v; break;
    HC_FFT_T_LENGTHS(HC_LEN_CASE)
#undef HC_LEN_CASE
    }
    return (nrows + lines - 1) / lines;
}

static int build_fft(hc_handle* h)
{
    const int nx = h->p.nx, ny = h->p.ny, nxh = nx / 2;
    if (factor_plan(nxh, &h->px) != HC_OK || factor_plan(ny, &h->py) != HC_OK) return HC_ERR_UNSUPPORTED;
    std::vector<double2> tw(nxh + ny + nxh);
    for (int e = 0; e < nxh; ++e) tw[e] = make_double2(cos(2.0 * HC_PI * e / nxh), -sin(2.0 * HC_PI * e / nxh));
    for (int e = 0; e < ny; ++e) tw[nxh + e] = make_double2(cos(2.0 * HC_PI * e / ny), -sin(2.0 * HC_PI * e / ny));
    for (int e = 0; e < nxh; ++e) tw[nxh + ny + e] = make_double2(cos(2.0 * HC_PI * e / nx), -sin(2.0 * HC_PI * e / nx));
    CK(cudaMalloc(&h->twbuf, tw.size() * sizeof(double2)));
    CK(cudaMemcpy(h->twbuf, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice));
    h->px.tw = h->twbuf;
    h->py.tw = h->twbuf + nxh;
    h->wpack = h->twbuf + nxh + ny;
    if (h->rsz == sizeof(double)) {
        h->twt = h->twbuf;
    } else {
        std::vector<float2> tf(tw.size());
        for (size_t e = 0; e < tw.size(); ++e) tf[e] = make_float2((float)tw[e].x, (float)tw[e].y);
        CK(cudaMalloc(&h->twt, tf.size() * sizeof(float2)));
        CK(cudaMemcpy(h->twt, tf.data(), tf.size() * sizeof(float2), cudaMemcpyHostToDevice));
    }
    // explicit tile sizes (tile[0], tile[1]) select the runtime-length kernels
    h->fft_tx = h->p.tile[0] == 0 && fft_t_length_ok(nxh);
    h->fft_ty = h->p.tile[1] == 0 && fft_t_length_ok(ny);
    if (h->fft_tx || h->fft_ty) {
        int rc = h->rsz == sizeof(double) ? fft_t_setup<double>(h) : fft_t_setup<float>(h);
        if (rc != HC_OK) return rc;
    }
    // the fused transforms where a shape exists (and no explicit tile asks for the others)
    h->fft2d = 0;
    if (h->fft_tx && h->fft_ty) {
        const int rc = h->rsz == sizeof(double) ? fft2d_dispatch<double>(h, 0, nullptr, 0) : fft2d_dispatch<float>(h, 0, nullptr, 0);
        h->fft2d = rc == HC_OK;
    }
    const size_t c2 = 2 * h->rsz;     // bytes of one complex
    h->rows_x = h->p.tile[0] > 0 ? h->p.tile[0] : (h->rsz == sizeof(double) ? 1024 : 2048) / nxh;
    if (h->rows_x < 1) h->rows_x = 1; if (h->rows_x > 64) h->rows_x = 64;
    h->smem_x = 2 * (size_t)h->rows_x * nxh * c2;
    // tile[3]: 0 the coalescing-tile column kernels, 1 one thread per column (128 a
    // block), 2 one warp per column without tiles, >= 32 one thread per column with
    // that many threads a block
    h->col_threads = h->p.tile[3] >= 32 ? h->p.tile[3] : 128;
    h->col_warp = (h->p.tile[3] == 0 || h->p.tile[3] == 2) && h->p.nz <= 32 * 8;
    if (h->col_threads < 32 || h->col_threads > 256 || (h->col_threads & 31)) return HC_ERR_PARAM;
    h->tl_y = h->p.tile[1] > 0 ? h->p.tile[1] : 1536 / ny;
    if (h->tl_y < 1) h->tl_y = 1; if (h->tl_y > 32) h->tl_y = 32; if (h->tl_y > nxh) h->tl_y = nxh;
    h->smem_y = 2 * (size_t)h->tl_y * (ny + 1) * c2;
    if (h->smem_x > 200 * 1024 || h->smem_y > 200 * 1024) return HC_ERR_UNSUPPORTED;
    return HC_OK;
}

template <typename R> static int set_smem_attrs()
{
    CK(cudaFuncSetAttribute(k_fft_x_r2c<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    CK(cudaFuncSetAttribute(k_fft_x_c2r<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    CK(cudaFuncSetAttribute(k_fft_y<R, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    CK(cudaFuncSetAttribute(k_fft_y<R, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    {
        // the largest tile (K = 8) bounds every instantiation
        const int sm = (int)column_tile_smem_r<8>(sizeof(typename V2<R>::T));
        CK(cudaFuncSetAttribute(k_column_fd_tile_r<R, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        CK(cudaFuncSetAttribute(k_column_fd_tile_r<R, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        CK(cudaFuncSetAttribute(k_column_fd_tile_r<R, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        CK(cudaFuncSetAttribute(k_column_fd_tile_r<R, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        CK(cudaFuncSetAttribute(k_column_fd_tile_r<R, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        CK(cudaFuncSetAttribute(k_column_fd_tile_r<R, 6>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        CK(cudaFuncSetAttribute(k_column_fd_tile_r<R, 7>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        CK(cudaFuncSetAttribute(k_column_fd_tile_r<R, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        const int sp = (int)column_sp_tile_smem<4>(sizeof(typename V2<R>::T));
        CK(cudaFuncSetAttribute(k_column_sp_tile<R, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sp));
        CK(cudaFuncSetAttribute(k_column_sp_tile<R, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sp));
        CK(cudaFuncSetAttribute(k_column_sp_tile<R, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, sp));
        CK(cudaFuncSetAttribute(k_column_sp_tile<R, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, sp));
    }
    CK(cudaFuncSetAttribute(k_rhs_t_strip<R, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rhs_t_strip_smem<R>()));
    CK(cudaFuncSetAttribute(k_rhs_t_strip<R, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rhs_t_strip_smem<R>()));
    CK(cudaFuncSetAttribute(k_rhs_momentum_strip<R, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rhs_strip_smem<R>()));
    CK(cudaFuncSetAttribute(k_rhs_momentum_strip<R, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rhs_strip_smem<R>()));
    CK(cudaFuncSetAttribute(k_rhs_momentum_tiled<R, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rhs_tiled_smem<R>(1)));
    CK(cudaFuncSetAttribute(k_rhs_momentum_tiled<R, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rhs_tiled_smem<R>(1)));
    if (sizeof(R) == sizeof(float)) {
        CK(cudaFuncSetAttribute(k_rhs_momentum_tiled2<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rhs_tiled2_smem(1)));
        CK(cudaFuncSetAttribute(k_rhs_momentum_tiled2<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rhs_tiled2_smem(1)));

    }
    return HC_OK;
}

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------
static dim3 pt_block() { return dim3(32, 8, 1); }
static dim3 pt_grid(const Geo& g) { return dim3((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz); }

// The bottom ghost of T as T(-1) = tbs T(0) + tba: a fixed wall temperature (the
// reference, src/module_boundary.f90:176-183) gives tbs = -1, tba = 2 tbot; the
// fixed wall gradient dT/dz = tbot (tbc_bot = 1) gives tbs = 1, tba = -tbot dz_b(0).
static void t_ghost_bottom(const hc_handle* h, double& tbs, double& tba)
{
    if (h->p.tbc_bot) { tbs = 1.0; tba = -h->p.tbot * h->zhost[2][2]; }
    else { tbs = -1.0; tba = 2.0 * h->p.tbot; }
}
// The constants the wall ghosts of T add to the (0,0) mode of the T solve's
// source (src/module_poisson_solver.f90:575-582): the ghost's constant part times
// the coupling aa of the first level (cc of the last).
static void t_bc_src(const hc_handle* h, double rk_c, double& b0, double& b1)
{
    const hc_params& p = h->p;
    const double* DZ = h->zhost[0].data(); const double* DZT = h->zhost[1].data(); const double* DZB = h->zhost[2].data();
    const int ks = 2, ke = p.nz + 1;
    const double aa_t_zstr = -0.5 * rk_c * p.dt * p.alpha / DZ[ks] / DZB[ks];
    const double cc_t_zend = -0.5 * rk_c * p.dt * p.alpha / DZ[ke] / DZT[ke];
    b0 = p.tbc_bot ? aa_t_zstr * p.tbot * DZB[ks] : -2.0 * aa_t_zstr * p.tbot;
    b1 = -2.0 * cc_t_zend * p.ttop;
}

template <typename R> static Acc<R> make_acc(hc_handle* h)
{
    Acc<R> a;
    a.f.u = (const R*)h->fld[F_U]; a.f.v = (const R*)h->fld[F_V]; a.f.w = (const R*)h->fld[F_W];
    a.f.p = (const R*)h->fld[F_P]; a.f.t = (const R*)h->fld[F_T];
    a.g = h->g;
    double tbs, tba;
    t_ghost_bottom(h, tbs, tba);
    a.um = (R)h->p.u_mrf; a.tbs = (R)tbs; a.tba = (R)tba; a.ttop = (R)h->p.ttop;
    a.closed = h->p.ochannel == 0;
    a.su = a.sv = a.sw = a.sp = a.st = nullptr;
    a.kd = h->p.nz;
    return a;
}

template <typename R> static const typename V2<R>::T* fft_tw(hc_handle* h, int which)
{
    const typename V2<R>::T* t = (const typename V2<R>::T*)h->twt;
    return which == 0 ? t : (which == 1 ? t + h->g.nxh : t + h->g.nxh + h->g.ny);
}

// x then y forward transform of nf physical fields into half spectra
template <typename R> static int fft_forward(hc_handle* h, const R* const* in, typename V2<R>::T* const* out, int nf)
{
    typedef typename V2<R>::T T2;
    const int* halt = &h->sc->nan_flag;
    if (nf < 1 || nf > HC_FFT_MAXF) return HC_ERR_ARG;
    if (h->fft2d && !h->rec && nf <= HC_FFT_TMAXF) {
        F2Args<R> a;
        memset(&a, 0, sizeof(a));
        for (int f = 0; f < nf; ++f) { a.in[f] = in[f]; a.out[f] = out[f]; }
        a.nz = h->g.nz;
        a.twx = fft_tw<R>(h, 0); a.wp = fft_tw<R>(h, 2); a.twy = fft_tw<R>(h, 1);
        a.scale_x = (R)(1.0 / h->p.nx); a.scale_y = (R)(1.0 / h->p.ny); a.halt = halt;
        prof_begin(h, K_FFT2D_FWD);
        int rc = fft2d_dispatch<R>(h, 1, &a, nf);
        if (rc) return rc;
        CKL();
        return HC_OK;
    }
    if (h->fft_tx) {
        FxArgs<R> a;
        memset(&a, 0, sizeof(a));
        for (int f = 0; f < nf; ++f) { a.in[f] = in[f]; a.out[f] = out[f]; }
        a.nrows = (long long)h->g.ny * h->g.nz;
        a.tw = fft_tw<R>(h, 0); a.wp = fft_tw<R>(h, 2); a.scale = (R)(1.0 / h->p.nx); a.halt = halt;
        prof_begin(h, K_FFT_X_FWD);
        int rc = fft_t_dispatch<R>(h, h->g.nxh, 1, &a, dim3((unsigned)fft_t_xblocks<R>(h->g.nxh, a.nrows), nf, 1));
        if (rc) return rc;
        CKL();
    } else {
    FftXArgs<R> ax;
    memset(&ax, 0, sizeof(ax));
    for (int f = 0; f < nf; ++f) { ax.in[f] = in[f]; ax.out[f] = out[f]; }
    ax.nrows = (long long)h->g.ny * h->g.nz;
    ax.rows = h->rows_x; ax.pl = h->px; ax.wpack = h->wpack; ax.scale = 1.0 / h->p.nx; ax.halt = halt;
    dim3 gx((unsigned)((ax.nrows + ax.rows - 1) / ax.rows), nf, 1);
    prof_begin(h, K_FFT_X_FWD);
    { int lrc = hc_launch<FftXArgs<R>, k_fft_x_r2c<R>, k_fft_x_r2c_body<R>, 256, 1>(h, gx, dim3(256), h->smem_x, ax); if (lrc) return lrc; }
    CKL();
    }
    if (h->fft_ty) {
        FyArgs<R> a;
        memset(&a, 0, sizeof(a));
        for (int f = 0; f < nf; ++f) a.dst[f] = out[f];
        a.nxh = h->g.nxh; a.tw = fft_tw<R>(h, 1); a.scale = (R)(1.0 / h->p.ny); a.halt = halt;
        prof_begin(h, K_FFT_Y_FWD);
        int rc = fft_t_dispatch<R>(h, h->g.ny, 3, &a, dim3((h->g.nxh + fft_t_ytl<R>(h->g.ny) - 1) / fft_t_ytl<R>(h->g.ny), h->g.nz, nf));
        if (rc) return rc;
        CKL();
        return HC_OK;
    }
    FftYArgs<R> ay;
    memset(&ay, 0, sizeof(ay));
    for (int f = 0; f < nf; ++f) ay.data[f] = out[f];
    ay.nxh = h->g.nxh; ay.ny = h->g.ny; ay.tl = h->tl_y; ay.pl = h->py; ay.scale = 1.0 / h->p.ny; ay.halt = halt;
    dim3 gy((h->g.nxh + ay.tl - 1) / ay.tl, h->g.nz, nf);
    prof_begin(h, K_FFT_Y_FWD);
    { int lrc = hc_launch<FftYArgs<R>, k_fft_y<R, -1>, k_fft_y_body<R, -1>, 256, 1>(h, gy, dim3(256), h->smem_y, ay); if (lrc) return lrc; }
    CKL();
    (void)sizeof(T2);
    return HC_OK;
}

// y then x inverse transform of nf half spectra into physical fields, stored or
// (add[f] = 1) added. The y pass runs in place on in[f], or reads ysrc[f] and
// writes in[f] (which then serves as scratch) when ysrc is given.
template <typename R> static int fft_inverse(hc_handle* h, typename V2<R>::T* const* in, R* const* out, const int* add, int nf,
                                             const typename V2<R>::T* const* ysrc = nullptr)
{
    const int* halt = &h->sc->nan_flag;
    if (nf < 1 || nf > HC_FFT_MAXF) return HC_ERR_ARG;
    if (h->fft2d && !h->rec && nf <= HC_FFT_TMAXF) {
        // reads the spectra (ysrc, else in) and leaves them as they are
        F2Args<R> a;
        memset(&a, 0, sizeof(a));
        for (int f = 0; f < nf; ++f) { a.in[f] = ysrc ? ysrc[f] : in[f]; a.out[f] = out[f]; a.add[f] = add[f]; }
        a.nz = h->g.nz;
        a.twx = fft_tw<R>(h, 0); a.wp = fft_tw<R>(h, 2); a.twy = fft_tw<R>(h, 1);
        a.scale_x = (R)1; a.scale_y = (R)1; a.halt = halt;
        prof_begin(h, K_FFT2D_INV);
        int rc = fft2d_dispatch<R>(h, 2, &a, nf);
        if (rc) return rc;
        CKL();
        return HC_OK;
    }
    if (h->fft_ty) {
        FyArgs<R> a;
        memset(&a, 0, sizeof(a));
        for (int f = 0; f < nf; ++f) { a.dst[f] = in[f]; a.src[f] = ysrc ? ysrc[f] : nullptr; }
        a.nxh = h->g.nxh; a.tw = fft_tw<R>(h, 1); a.scale = (R)1; a.halt = halt;
        prof_begin(h, K_FFT_Y_INV);
        int rc = fft_t_dispatch<R>(h, h->g.ny, 4, &a, dim3((h->g.nxh + fft_t_ytl<R>(h->g.ny) - 1) / fft_t_ytl<R>(h->g.ny), h->g.nz, nf));
        if (rc) return rc;
        CKL();
    } else {
    FftYArgs<R> ay;
    memset(&ay, 0, sizeof(ay));
    for (int f = 0; f < nf; ++f) { ay.data[f] = in[f]; ay.src[f] = ysrc ? ysrc[f] : nullptr; }
    ay.nxh = h->g.nxh; ay.ny = h->g.ny; ay.tl = h->tl_y; ay.pl = h->py; ay.scale = 1.0; ay.halt = halt;
    dim3 gy((h->g.nxh + ay.tl - 1) / ay.tl, h->g.nz, nf);
    prof_begin(h, K_FFT_Y_INV);
    { int lrc = hc_launch<FftYArgs<R>, k_fft_y<R, 1>, k_fft_y_body<R, 1>, 256, 1>(h, gy, dim3(256), h->smem_y, ay); if (lrc) return lrc; }
    CKL();
    }
    if (h->fft_tx) {
        FxArgs<R> a;
        memset(&a, 0, sizeof(a));
        for (int f = 0; f < nf; ++f) { a.in[f] = in[f]; a.out[f] = out[f]; a.add[f] = add[f]; }
        a.nrows = (long long)h->g.ny * h->g.nz;
        a.tw = fft_tw<R>(h, 0); a.wp = fft_tw<R>(h, 2); a.scale = (R)1; a.halt = halt;
        prof_begin(h, K_FFT_X_INV);
        int rc = fft_t_dispatch<R>(h, h->g.nxh, 2, &a, dim3((unsigned)fft_t_xblocks<R>(h->g.nxh, a.nrows), nf, 1));
        if (rc) return rc;
        CKL();
        return HC_OK;
    }
    FftXInvArgs<R> ax;
    memset(&ax, 0, sizeof(ax));
    for (int f = 0; f < nf; ++f) { ax.in[f] = in[f]; ax.out[f] = out[f]; ax.add[f] = add[f]; }
    ax.nrows = (long long)h->g.ny * h->g.nz;
    ax.rows = h->rows_x; ax.pl = h->px; ax.wpack = h->wpack; ax.halt = halt;
    dim3 gx((unsigned)((ax.nrows + ax.rows - 1) / ax.rows), nf, 1);
    prof_begin(h, K_FFT_X_INV);
    { int lrc = hc_launch<FftXInvArgs<R>, k_fft_x_c2r<R>, k_fft_x_c2r_body<R>, 256, 1>(h, gx, dim3(256), h->smem_x, ax); if (lrc) return lrc; }
    CKL();
    return HC_OK;
}

static const double RKC1[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
static const double RKC2[3] = {0.0, -17.0 / 60.0, -5.0 / 12.0};
static const double RKC3[3] = {8.0 / 15.0, 2.0 / 15.0, 1.0 / 3.0};

template <typename R> static int launch_stats(hc_handle* h, int accumulate)
{
    StatsArgs<R> s;
    memset(&s, 0, sizeof(s));
    s.f.u = (const R*)h->fld[F_U]; s.f.v = (const R*)h->fld[F_V]; s.f.w = (const R*)h->fld[F_W];
    s.f.p = (const R*)h->fld[F_P]; s.f.t = (const R*)h->fld[F_T];
    s.g = h->g;
    if (h->p.cds != 3) { s.uhx_s = (const R*)h->fld[F_UHX]; s.vhy_s = (const R*)h->fld[F_VHY]; }
    for (int q = 0; q < 11; ++q) { s.mean[q] = h->mean[q]; s.win[q] = h->win[q]; }
    s.step = &h->sc->step;
    s.window = STATS_WINDOW;
    s.accumulate = accumulate;
    s.tdefer = h->tdefer ? &h->sc->tstat_n : nullptr;
    s.um = h->p.u_mrf; s.dt = h->p.dt;
    s.part = h->part_st;
    prof_begin(h, K_STATS);
    { int lrc = hc_launch<StatsArgs<R>, k_stats<R>, k_stats_body<R>, 256, StatsMinBlocks<R>::v>(
          h, dim3((unsigned)h->stx, (unsigned)h->sty), dim3(256), 0, s); if (lrc) return lrc; }
    CKL();
    return HC_OK;
}

static int launch_finalize(hc_handle* h, int nsub, int write_diag, int set_ubar = 1)
{
    FinalArgs f;
    memset(&f, 0, sizeof(f));
    f.sc = h->sc; f.part_div = h->part_div; f.stride = h->pd_stride; f.nsub = nsub;
    // FD RK3: the checks of sub-steps 1 and 2 run inside the next sub-step's RHS
    const long long nrhs = (long long)h->rhs_grid.x * h->rhs_grid.y * h->rhs_grid.z;
    // FD: sub-steps before the last are checked inside the next sub-step's RHS
    for (int q = 0; q < 3; ++q)
        f.nbq[q] = (h->div_in_rhs && q < nsub - 1) ? nrhs : h->nbd;
    f.part_st = h->part_st; f.nbs = h->nbs;
    f.nx = h->p.nx; f.ny = h->p.ny; f.nz = h->p.nz; f.lz = h->p.lz;
    f.dp_opt = h->p.dp_opt; f.diag = h->diag_dev; f.diag_cap = h->diag_cap; f.write_diag = write_diag;
    f.cds = h->p.cds;
    f.set_ubar = set_ubar;
    prof_begin(h, K_FINAL);
    { int lrc = hc_launch<FinalArgs, k_finalize, k_finalize_body, 256, 1>(h, dim3(1), dim3(256), 0, f); if (lrc) return lrc; }
    CKL();
    return HC_OK;
}

// Column solves: one warp per wavenumber pair while nz <= 256 (rows per lane
// K = ceil(nz/32)), else (or when tile[3] asks for it) one thread per pair.
template <typename R, int K> static int col_fd_k(hc_handle* h, const ColArgs<R>& ca)
{
    if (h->p.tile[3] == 2) {      // per-warp variant without the coalescing tiles
        const unsigned nb = (unsigned)((h->g.ncol + CW_WARPS - 1) / CW_WARPS);
        { int lrc = hc_launch<ColArgs<R>, k_column_fd_warp<R, K>, k_column_fd_warp_body<R, K>, CW_WARPS * 32, 4>(
              h, dim3(nb), dim3(CW_WARPS * 32), column_warp_smem<K>(), ca); if (lrc) return lrc; }
        CKL();
        return HC_OK;
    }
    const unsigned nb = (unsigned)((h->g.ncol + CT_COLS - 1) / CT_COLS);
    { int lrc = hc_launch<ColArgs<R>, k_column_fd_tile_r<R, K>, k_column_fd_tile_r_body<R, K>, CT_COLS * 32, 2>(
          h, dim3(nb), dim3(CT_COLS * 32), column_tile_smem_r<K>(sizeof(typename V2<R>::T)), ca); if (lrc) return lrc; }
    CKL();
    return HC_OK;
}
template <typename R> static int launch_column_fd(hc_handle* h, const ColArgs<R>& ca)
{
    const int K = (h->p.nz + 31) / 32;
    if (h->col_warp) {
        switch (K) {
        case 1: return col_fd_k<R, 1>(h, ca);
        case 2: return col_fd_k<R, 2>(h, ca);
        case 3: return col_fd_k<R, 3>(h, ca);
        case 4: return col_fd_k<R, 4>(h, ca);
        case 5: return col_fd_k<R, 5>(h, ca);
        case 6: return col_fd_k<R, 6>(h, ca);
        case 7: return col_fd_k<R, 7>(h, ca);
        case 8: return col_fd_k<R, 8>(h, ca);
        default: break;
        }
    }
    { int lrc = hc_launch<ColArgs<R>, k_column_fd<R>, k_column_fd_body<R>, 256, 1>(
          h, dim3((unsigned)((h->g.ncol + h->col_threads - 1) / h->col_threads)), dim3(h->col_threads), 0, ca); if (lrc) return lrc; }
    CKL();
    return HC_OK;
}
template <typename R, int K> static int col_t_k(hc_handle* h, const ColTArgs<R>& ct)
{
    const unsigned nb = (unsigned)((h->g.ncol + CT_COLS - 1) / CT_COLS);
    { int lrc = hc_launch<ColTArgs<R>, k_column_t_tile<R, K>, k_column_t_tile_body<R, K>, CT_COLS * 32, 2>(
          h, dim3(nb), dim3(CT_COLS * 32), column_t_tile_smem<K>(sizeof(typename V2<R>::T)), ct); if (lrc) return lrc; }
    CKL();
    return HC_OK;
}
template <typename R> static int launch_column_t(hc_handle* h, const ColTArgs<R>& ct)
{
    const int K = (h->p.nz + 31) / 32;
    if (h->col_warp) {
        switch (K) {
        case 1: return col_t_k<R, 1>(h, ct);
        case 2: return col_t_k<R, 2>(h, ct);
        case 3: return col_t_k<R, 3>(h, ct);
        case 4: return col_t_k<R, 4>(h, ct);
        case 5: return col_t_k<R, 5>(h, ct);
        case 6: return col_t_k<R, 6>(h, ct);
        case 7: return col_t_k<R, 7>(h, ct);
        case 8: return col_t_k<R, 8>(h, ct);
        default: break;
        }
    }
    { int lrc = hc_launch<ColTArgs<R>, k_column_t<R>, k_column_t_body<R>, 256, 1>(
          h, dim3((unsigned)((h->g.ncol + h->col_threads - 1) / h->col_threads)), dim3(h->col_threads), 0, ct); if (lrc) return lrc; }
    CKL();
    return HC_OK;
}

// recompute = 1: a sub-step re-run for the adjoint's tape -- no divergence
// check, no statistics snapshot, and the scalar update only when first = 1
template <typename R, int CDS> static int substep_fd(hc_handle* h, int sub, int recompute = 0, int first = 1)
{
    typedef typename V2<R>::T T2;
    const hc_params& p = h->p;
    const int* halt = &h->sc->nan_flag;
    double rk_a, rk_b, rk_c;
    if (p.dts == 2) { rk_a = RKC1[sub]; rk_b = RKC2[sub]; rk_c = RKC3[sub]; }
    else { rk_a = 1.5; rk_b = -0.5; rk_c = 1.0; }
    const int last = ((p.dts == 2) ? (sub == 2) : 1) && !recompute;

    ScalarArgs sa;
    sa.sc = h->sc; sa.sub = sub; sa.dt = p.dt; sa.dp_opt = p.dp_opt; sa.dpx_coef = h->dpx_coef; sa.um = p.u_mrf;
    sa.is_ri_var = p.is_ri_var; sa.ri_str = p.ri_str; sa.ri_end = p.ri_end; sa.imax = p.imax;
    if (!recompute || first) {
        prof_begin(h, K_BEGIN);
        { int lrc = hc_launch<ScalarArgs, k_substep_begin, k_substep_begin_body, 32, 1>(h, dim3(1), dim3(1), 0, sa); if (lrc) return lrc; }
        CKL();
    }

    // Rayleigh damping of the top layer (isdamp = 1), undamped copies kept for
    // the ghost reads of this sub-step's right-hand sides
    Acc<R> acc = make_acc<R>(h);
    if (p.isdamp == 1) {
        const int kd = p.nz - 1 - p.nzdamp;
        const long long lv = (long long)(p.nzdamp + 1) * h->g.nxy;
        FdDampArgs<R> da;
        const int fids[5] = {F_U, F_V, F_W, F_P, F_T};
        for (int f = 0; f < 5; ++f) { da.f[f] = (R*)h->fld[fids[f]]; da.stale[f] = (R*)h->dstale + f * lv; }
        da.mean = h->dmean; da.sig = h->dsig; da.g = h->g; da.kd = kd;
        prof_begin(h, K_SPEC_AUX);
        k_fd_damp_mean<R><<<dim3(p.nzdamp + 1, 5), 256, 0, h->st>>>(da);
        CKL();
        prof_begin(h, K_SPEC_AUX);
        k_fd_damp_apply<R><<<RED_BLOCKS, 256, 0, h->st>>>(da);
        CKL();
        acc.su = da.stale[0]; acc.sv = da.stale[1]; acc.sw = da.stale[2]; acc.sp = da.stale[3]; acc.st = da.stale[4];
        acc.kd = kd;
        // per-point RHS with the reference's ghost semantics of the damped layer
        MomArgs<R> mm;
        mm.a = acc;
        mm.ff = (R*)h->fld[F_FF]; mm.gg = (R*)h->fld[F_GG]; mm.hh = (R*)h->fld[F_HH];
        mm.qu = (R*)h->fld[F_QU]; mm.qv = (R*)h->fld[F_QV]; mm.qw = (R*)h->fld[F_QW];
        mm.uhx_s = last ? (R*)h->fld[F_UHX] : nullptr; mm.vhy_s = last ? (R*)h->fld[F_VHY] : nullptr;
        mm.rk_a = rk_a; mm.rk_b = rk_b; mm.rk_c = rk_c; mm.ph = h->ph; mm.sc = h->sc;
        mm.bfx = h->has_bf ? (const R*)h->bf[0] : nullptr;
        mm.bfy = (const R*)h->bf[1]; mm.bfz = (const R*)h->bf[2];
        prof_begin(h, K_RHS_MOM);
        k_rhs_momentum<R, CDS><<<pt_grid(h->g), pt_block(), 0, h->st>>>(mm);
        CKL();
    } else {
    // momentum RHS (SMEM-tiled, marching in k)
    RhsTArgs<R> m;
    m.f.u = (const R*)h->fld[F_U]; m.f.v = (const R*)h->fld[F_V]; m.f.w = (const R*)h->fld[F_W];
    m.f.p = (const R*)h->fld[F_P]; m.f.t = (const R*)h->fld[F_T];
    m.g = h->g;
    m.ff = (R*)h->fld[F_FF]; m.gg = (R*)h->fld[F_GG]; m.hh = (R*)h->fld[F_HH];
    m.qu = (R*)h->fld[F_QU]; m.qv = (R*)h->fld[F_QV]; m.qw = (R*)h->fld[F_QW];
    m.uhx_s = last ? (R*)h->fld[F_UHX] : nullptr; m.vhy_s = last ? (R*)h->fld[F_VHY] : nullptr;
    m.rk_a = rk_a; m.rk_b = rk_b; m.rk_c = rk_c; m.ph = h->ph; m.sc = h->sc;
    m.with_t = p.isscalar == 1;
    // the divergence check of the previous sub-step rides along (slot sub-1)
    m.part_div = (sub > 0 && h->div_in_rhs && !recompute) ? h->part_div + (long long)(sub - 1) * h->pd_stride * 3 : nullptr;
    m.kchunk = h->rhs_kc;
    m.zm = sizeof(R) == sizeof(float) ? (const void*)h->zm5 : (const void*)h->zm5d;
    m.bfx = h->has_bf ? (const R*)h->bf[0] : nullptr;
    m.bfy = (const R*)h->bf[1]; m.bfz = (const R*)h->bf[2];
    prof_begin(h, K_RHS_MOM);
    {
        int lrc;
        if (h->rhs_strip)                // products on strips (64 x 16 tiles)
            lrc = hc_launch<RhsTArgs<R>, k_rhs_momentum_strip<R, CDS>, k_rhs_momentum_strip_body<R, CDS>, RsCfg<R>::NT,
                            RsCfg<R>::MINB>(h, h->rhs_grid, dim3(RsCfg<R>::NT), rhs_strip_smem<R>(), m);
        else if constexpr (sizeof(R) == sizeof(float))      // FP32: two x points a thread (64 x 8 tiles)
            lrc = hc_launch<RhsTArgs<float>, k_rhs_momentum_tiled2<CDS>, k_rhs_momentum_tiled2_body<CDS>, 256, 2>(
                h, h->rhs_grid, dim3(256), rhs_tiled2_smem(m.with_t), m);
        else
            lrc = hc_launch<RhsTArgs<R>, k_rhs_momentum_tiled<R, CDS>, k_rhs_momentum_tiled_body<R, CDS>, 256,
                            RhsMinBlocks<R>::v>(h, h->rhs_grid, dim3(RT_TX * RT_TY), rhs_tiled_smem<R>(m.with_t), m);
        if (lrc) return lrc;
    }
    CKL();
    }

    T2* S[4] = {(T2*)h->spec[0], (T2*)h->spec[1], (T2*)h->spec[2], (T2*)h->spec[3]};
    const R* qin[3] = {(const R*)h->fld[F_QU], (const R*)h->fld[F_QV], (const R*)h->fld[F_QW]};
    int rc = fft_forward<R>(h, qin, S, 3);
    if (rc) return rc;

    ColArgs<R> ca;
    ca.qu = S[0]; ca.qv = S[1]; ca.qw = S[2]; ca.psi = S[3];
    ca.c = h->cc; ca.s = h->cs; ca.g = h->g;
    ca.rk_c = rk_c; ca.dt = p.dt; ca.nu = p.nu;
    {
        const double* DZ = h->zhost[0].data(); const double* DZT = h->zhost[1].data(); const double* DZB = h->zhost[2].data();
        const int ks = 2, ke = p.nz + 1;   // Fortran kstr3, kend3 at array index k-1
        double aa_u_zstr = -0.5 * rk_c * p.dt * p.nu / DZ[ks] / DZB[ks];
        ca.bcu0 = 2.0 * aa_u_zstr * p.u_mrf;
        ca.bcu1 = 0.0;
        if (p.ochannel == 0) {
            double cc_u_zend = -0.5 * rk_c * p.dt * p.nu / DZ[ke] / DZT[ke];
            ca.bcu1 = 2.0 * cc_u_zend * p.u_mrf;
        }
    }
    ca.halt = halt;
    prof_begin(h, K_COLUMN);
    rc = launch_column_fd<R>(h, ca);
    if (rc) return rc;

    R* outs[4] = {(R*)h->fld[F_U], (R*)h->fld[F_V], (R*)h->fld[F_W], (R*)h->fld[F_P]};
    const int add[4] = {0, 0, 0, 1};
    rc = fft_inverse<R>(h, S, outs, add, 4);
    if (rc) return rc;

    if (p.isscalar == 1) {
        TempArgs<R> ta;
        ta.a = make_acc<R>(h);
        if (p.isdamp == 1) { ta.a.st = acc.st; ta.a.kd = acc.kd; }   // t keeps its undamped ghosts
        ta.ss = (R*)h->fld[F_SS]; ta.qt = (R*)h->fld[F_QU];
        ta.rk_a = rk_a; ta.rk_b = rk_b; ta.rk_c = rk_c; ta.ph = h->ph;
        prof_begin(h, K_RHS_T);
        ta.kchunk = h->rhs_kc;
        ta.zm = sizeof(R) == sizeof(float) ? (const void*)h->zm5 : (const void*)h->zm5d;
        int lrc;
        if (h->rhs_strip && h->rhs_kc > 0 && p.isdamp == 0)    // fluxes on strips (64 x 16 tiles)
            lrc = hc_launch<TempArgs<R>, k_rhs_t_strip<R, CDS>, k_rhs_t_strip_body<R, CDS>, RsCfg<R>::NT, RsCfg<R>::MINB>(
                h, h->rhs_grid, dim3(RsCfg<R>::NT), rhs_t_strip_smem<R>(), ta);
        else
            lrc = hc_launch<TempArgs<R>, k_rhs_temperature<R, CDS>, k_rhs_temperature_body<R, CDS>, 256, 1>(
                h, pt_grid(h->g), pt_block(), 0, ta);
        if (lrc) return lrc;
        CKL();
        const R* tin[1] = {(const R*)h->fld[F_QU]};
        rc = fft_forward<R>(h, tin, S, 1);
        if (rc) return rc;
        ColTArgs<R> ct;
        ct.qt = S[0]; ct.c = h->cc; ct.s = h->cs; ct.g = h->g; ct.rk_c = rk_c; ct.halt = halt;
        ct.out = S[0]; ct.ltr = 0; ct.mtr = 0;
        t_bc_src(h, rk_c, ct.bct0, ct.bct1);
        prof_begin(h, K_COLUMN_T);
        rc = launch_column_t<R>(h, ct);
        if (rc) return rc;
        R* tout[1] = {(R*)h->fld[F_T]};
        const int add0[1] = {0};
        rc = fft_inverse<R>(h, S, tout, add0, 1);
        if (rc) return rc;
    }

    FieldsIn<R> fi;
    fi.u = (const R*)h->fld[F_U]; fi.v = (const R*)h->fld[F_V]; fi.w = (const R*)h->fld[F_W];
    fi.p = (const R*)h->fld[F_P]; fi.t = (const R*)h->fld[F_T];
    // the divergence check of this sub-step runs inside the next sub-step's RHS
    // (without damping, which changes the fields first); the last one has its own pass
    if (recompute || (!last && h->div_in_rhs)) return HC_OK;
    prof_begin(h, K_DIV);
    {
        DivArgs<R> da;
        da.f = fi; da.g = h->g; da.part = h->part_div + (long long)sub * h->pd_stride * 3;
        int lrc = hc_launch<DivArgs<R>, k_div_check<R, CDS>, k_div_check_body<R, CDS>, 256, DivMinBlocks<R>::v>(
            h, dim3((unsigned)h->nbd), dim3(256), 0, da);
        if (lrc) return lrc;
    }
    CKL();
    return HC_OK;
}

template <typename R, int CDS> static int step_fd(hc_handle* h)
{
    const int nsub = h->p.dts == 2 ? 3 : 1;
    for (int sub = 0; sub < nsub; ++sub) {
        int rc = substep_fd<R, CDS>(h, sub);
        if (rc) return rc;
    }
    int rc = launch_stats<R>(h, 1);
    if (rc) return rc;
    return launch_finalize(h, nsub, 1);
}

// ---------------------------------------------------------------------------
// pseudo-spectral sub-step (cds = 3), time_advancement_sp
// (src/module_navier_stokes.f90:371-517)
// ---------------------------------------------------------------------------
static int spec_kchunk(const hc_handle* h, long long columns)
{
    // enough blocks for about 8 per SM, chunks of 4..32 levels
    const long long blocks = (columns + 255) / 256;
    long long kc = blocks * h->p.nz / (8LL * 148);
    if (kc < 4) kc = 4;
    if (kc > 32) kc = 32;
    if (kc > h->p.nz) kc = h->p.nz;
    return (int)kc;
}

template <typename R> static DampTab spec_damp_tab(hc_handle* h)
{
    DampTab d;
    d.sig = h->p.isdamp == 1 ? h->dsig : nullptr;
    d.mean = h->dmean;
    return d;
}

// up to 128 levels (K <= 4) the tiled kernel: its FP64 registers for u*, v*, w*
// grow with K, and beyond that the warp kernel keeps them in shared memory
template <typename R, int K> static int col_sp_k(hc_handle* h, const SpColArgs<R>& a)
{
    if constexpr (K <= 4) {
        const unsigned nb = (unsigned)((h->g.ncol + CT_COLS - 1) / CT_COLS);
        k_column_sp_tile<R, K><<<nb, CT_COLS * 32, column_sp_tile_smem<K>(sizeof(typename V2<R>::T)), h->st>>>(a);
    } else {
        const unsigned nb = (unsigned)((h->g.ncol + CW_WARPS - 1) / CW_WARPS);
        k_column_sp_warp<R, K><<<nb, CW_WARPS * 32, column_warp_smem<K>(), h->st>>>(a);
    }
    CKL();
    return HC_OK;
}
template <typename R> static int launch_column_sp(hc_handle* h, const SpColArgs<R>& a)
{
    switch ((h->p.nz + 31) / 32) {
    case 1: return col_sp_k<R, 1>(h, a);
    case 2: return col_sp_k<R, 2>(h, a);
    case 3: return col_sp_k<R, 3>(h, a);
    case 4: return col_sp_k<R, 4>(h, a);
    case 5: return col_sp_k<R, 5>(h, a);
    case 6: return col_sp_k<R, 6>(h, a);
    case 7: return col_sp_k<R, 7>(h, a);
    case 8: return col_sp_k<R, 8>(h, a);
    default: break;
    }
    return HC_ERR_UNSUPPORTED;
}

template <typename R> static int substep_sp(hc_handle* h, int sub)
{
    typedef typename V2<R>::T T2;
    const hc_params& p = h->p;
    const Geo& g = h->g;
    const int* halt = &h->sc->nan_flag;
    double rk_a, rk_b, rk_c;
    if (p.dts == 2) { rk_a = RKC1[sub]; rk_b = RKC2[sub]; rk_c = RKC3[sub]; }
    else { rk_a = 1.5; rk_b = -0.5; rk_c = 1.0; }
    T2* S[NSP];
    R* Q[NSP];
    for (int q = 0; q < NSP; ++q) { S[q] = (T2*)h->sp[q]; Q[q] = (R*)h->sp[q]; }
    const double tpx = 2.0 * HC_PI / p.lx, tpy = 2.0 * HC_PI / p.ly;
    const DampTab dtab = spec_damp_tab<R>(h);
    const int ltr = (int)(p.nx / 3.0), mtr = (int)(p.ny / 3.0);
    int rc;

    ScalarArgs sa;
    sa.sc = h->sc; sa.sub = sub; sa.dt = p.dt; sa.dp_opt = p.dp_opt; sa.dpx_coef = h->dpx_coef; sa.um = p.u_mrf;
    sa.is_ri_var = p.is_ri_var; sa.ri_str = p.ri_str; sa.ri_end = p.ri_end; sa.imax = p.imax;
    prof_begin(h, K_BEGIN);
    k_substep_begin<<<1, 1, 0, h->st>>>(sa);
    CKL();

    // rayleigh_damping_spec on u, v, w, p, t: plane means of the damped levels
    if (p.isdamp == 1) {
        DampArgs<R> da;
        const int fs[5] = {SP_U, SP_V, SP_W, SP_P, SP_T};
        for (int f = 0; f < 5; ++f) da.f[f] = S[fs[f]];
        da.mean = h->dmean; da.g = g; da.kd = p.nz - 1 - p.nzdamp; da.halt = halt;
        prof_begin(h, K_SPEC_AUX);
        k_spec_damp_mean<R><<<dim3(p.nzdamp + 1, 5), 256, 0, h->st>>>(da);
        CKL();
    }
    // skew-symmetric form: physical images of the horizontal derivatives
    if (p.issk == 1) {
        DerivArgs<R> dv;
        dv.s[0] = S[SP_U]; dv.s[1] = S[SP_V]; dv.s[2] = S[SP_W];
        for (int f = 0; f < 6; ++f) dv.out[f] = S[SP_W0 + 8 + f];
        dv.dt = dtab; dv.g = g; dv.tpx = tpx; dv.tpy = tpy; dv.halt = halt;
        prof_begin(h, K_SPEC_AUX);
        k_spec_deriv<R><<<RED_BLOCKS, 256, 0, h->st>>>(dv);
        CKL();
        T2* din[6];
        R* dout[6];
        const int add0[6] = {0, 0, 0, 0, 0, 0};
        for (int f = 0; f < 6; ++f) { din[f] = S[SP_W0 + 8 + f]; dout[f] = Q[SP_W0 + 8 + f]; }
        if ((rc = fft_inverse<R>(h, din, dout, add0, 6))) return rc;
    }
    // physical products, then one batched forward transform
    {
        ProdArgs<R> pa;
        pa.u = (const R*)h->fld[F_U]; pa.v = (const R*)h->fld[F_V]; pa.w = (const R*)h->fld[F_W]; pa.t = (const R*)h->fld[F_T];
        for (int f = 0; f < 6; ++f) pa.d[f] = p.issk == 1 ? Q[SP_W0 + 8 + f] : nullptr;
        for (int f = 0; f < 8; ++f) pa.out[f] = Q[SP_W0 + f];
        for (int f = 0; f < 3; ++f) pa.bf[f] = h->has_bf ? (const R*)h->bf[f] : nullptr;
        pa.g = g; pa.sc = h->sc; pa.rdz = h->cc.rdz; pa.rdzt = h->cc.rdzt;
        pa.um = p.u_mrf; pa.fc = p.fc; pa.ug = p.ug; pa.vg = p.vg; pa.t_ref = p.t_ref; pa.ttop = p.ttop;
        t_ghost_bottom(h, pa.tbs, pa.tba);
        pa.inv_coe = 1.0 / (p.issk == 1 ? 0.5 : 1.0);
        pa.closed = p.ochannel == 0; pa.dp3 = p.dp_opt == 3; pa.scalar = p.isscalar == 1; pa.skew = p.issk == 1;
        pa.kchunk = spec_kchunk(h, g.nxy); pa.halt = halt;
        prof_begin(h, K_SPEC_PROD);
        k_spec_products<R><<<dim3((unsigned)((g.nxy + 255) / 256), (p.nz + pa.kchunk - 1) / pa.kchunk), 256, 0, h->st>>>(pa);
        CKL();
        const R* fin[8];
        T2* fout[8];
        for (int f = 0; f < 8; ++f) { fin[f] = Q[SP_W0 + f]; fout[f] = S[SP_W0 + f]; }
        if ((rc = fft_forward<R>(h, fin, fout, 8))) return rc;
    }
    // right-hand sides and new histories, mode by mode
    {
        AsmArgs<R> aa;
        aa.su = S[SP_U]; aa.sv = S[SP_V]; aa.sw = S[SP_W]; aa.sp = S[SP_P];
        for (int f = 0; f < 8; ++f) aa.F[f] = S[SP_W0 + f];
        aa.ff = S[SP_FF]; aa.gg = S[SP_GG]; aa.hh = S[SP_HH];
        aa.qu = S[SP_QU]; aa.qv = S[SP_QV]; aa.qw = S[SP_QW];
        aa.dt = dtab; aa.g = g; aa.tpx = tpx; aa.tpy = tpy;
        aa.rdz = h->cc.rdz; aa.rdzt = h->cc.rdzt; aa.rdzb = h->cc.rdzb;
        aa.rk_a = rk_a; aa.rk_b = rk_b; aa.rk_c = rk_c; aa.dtime = p.dt; aa.nu = p.nu; aa.um = p.u_mrf;
        aa.coe = p.issk == 1 ? 0.5 : 1.0;
        aa.closed = p.ochannel == 0; aa.kchunk = spec_kchunk(h, g.ncol); aa.halt = halt;
        prof_begin(h, K_SPEC_ASM);
        k_spec_assemble<R><<<dim3((unsigned)((g.ncol + 255) / 256), (p.nz + aa.kchunk - 1) / aa.kchunk), 256, 0, h->st>>>(aa);
        CKL();
    }
    // solves, projection, pressure update, truncation, divergence spectrum
    {
        SpColArgs<R> ca;
        memset(&ca, 0, sizeof(ca));
        ca.b.qu = S[SP_QU]; ca.b.qv = S[SP_QV]; ca.b.qw = S[SP_QW]; ca.b.psi = nullptr;
        ca.b.c = h->cc; ca.b.s = h->cs; ca.b.g = g;
        ca.b.rk_c = rk_c; ca.b.dt = p.dt; ca.b.nu = p.nu;
        const double* DZ = h->zhost[0].data(); const double* DZT = h->zhost[1].data(); const double* DZB = h->zhost[2].data();
        const int ks = 2, ke = p.nz + 1;
        ca.b.bcu0 = 2.0 * (-0.5 * rk_c * p.dt * p.nu / DZ[ks] / DZB[ks]) * p.u_mrf;
        ca.b.bcu1 = p.ochannel == 0 ? 2.0 * (-0.5 * rk_c * p.dt * p.nu / DZ[ke] / DZT[ke]) * p.u_mrf : 0.0;
        ca.b.halt = halt;
        ca.su = S[SP_U]; ca.sv = S[SP_V]; ca.sw = S[SP_W]; ca.sp = S[SP_P]; ca.phi = S[SP_PHI]; ca.div = S[SP_DIV];
        ca.dt = dtab; ca.ltr = ltr; ca.mtr = mtr;
        prof_begin(h, K_COLUMN);
        if ((rc = launch_column_sp<R>(h, ca))) return rc;
    }
    // physical u, v, w and the divergence image (y out of place into work fields)
    {
        const T2* ys[4] = {S[SP_U], S[SP_V], S[SP_W], S[SP_DIV]};
        T2* scr[4] = {S[SP_W0], S[SP_W0 + 1], S[SP_W0 + 2], S[SP_W0 + 3]};
        R* outs[4] = {(R*)h->fld[F_U], (R*)h->fld[F_V], (R*)h->fld[F_W], Q[SP_W0 + 3]};
        const int add0[4] = {0, 0, 0, 0};
        if ((rc = fft_inverse<R>(h, scr, outs, add0, 4, ys))) return rc;
    }
    if (p.isscalar == 1) {
        ProdTArgs<R> pt;
        pt.u = (const R*)h->fld[F_U]; pt.v = (const R*)h->fld[F_V]; pt.w = (const R*)h->fld[F_W]; pt.t = (const R*)h->fld[F_T];
        for (int f = 0; f < 3; ++f) pt.out[f] = Q[SP_W0 + 4 + f];
        t_ghost_bottom(h, pt.tbs, pt.tba);
        pt.g = g; pt.ttop = p.ttop; pt.kchunk = spec_kchunk(h, g.nxy); pt.halt = halt;
        prof_begin(h, K_SPEC_PROD);
        k_spec_products_t<R><<<dim3((unsigned)((g.nxy + 255) / 256), (p.nz + pt.kchunk - 1) / pt.kchunk), 256, 0, h->st>>>(pt);
        CKL();
        const R* fin[3] = {Q[SP_W0 + 4], Q[SP_W0 + 5], Q[SP_W0 + 6]};
        T2* fout[3] = {S[SP_W0 + 4], S[SP_W0 + 5], S[SP_W0 + 6]};
        if ((rc = fft_forward<R>(h, fin, fout, 3))) return rc;
        AsmTArgs<R> at;
        at.st = S[SP_T];
        for (int f = 0; f < 3; ++f) at.F[f] = S[SP_W0 + 4 + f];
        at.ss = S[SP_SS]; at.qt = S[SP_QU];
        at.dt = dtab; at.g = g; at.tpx = tpx; at.tpy = tpy;
        at.rdz = h->cc.rdz; at.rdzt = h->cc.rdzt; at.rdzb = h->cc.rdzb;
        at.rk_a = rk_a; at.rk_b = rk_b; at.rk_c = rk_c; at.dtime = p.dt; at.alpha = p.alpha; at.um = p.u_mrf;
        t_ghost_bottom(h, at.tbs, at.tba);
        at.ttop = p.ttop; at.kchunk = spec_kchunk(h, g.ncol); at.halt = halt;
        prof_begin(h, K_SPEC_ASM);
        k_spec_assemble_t<R><<<dim3((unsigned)((g.ncol + 255) / 256), (p.nz + at.kchunk - 1) / at.kchunk), 256, 0, h->st>>>(at);
        CKL();
        ColTArgs<R> ct;
        ct.qt = S[SP_QU]; ct.out = S[SP_T]; ct.ltr = ltr; ct.mtr = mtr;
        ct.c = h->cc; ct.s = h->cs; ct.g = g; ct.rk_c = rk_c; ct.halt = halt;
        t_bc_src(h, rk_c, ct.bct0, ct.bct1);
        prof_begin(h, K_COLUMN_T);
        if ((rc = launch_column_t<R>(h, ct))) return rc;
        const T2* ys[1] = {S[SP_T]};
        T2* scr[1] = {S[SP_W0]};
        R* tout[1] = {(R*)h->fld[F_T]};
        const int add0[1] = {0};
        if ((rc = fft_inverse<R>(h, scr, tout, add0, 1, ys))) return rc;
    }
    FieldsIn<R> fi;
    fi.u = (const R*)h->fld[F_U]; fi.v = (const R*)h->fld[F_V]; fi.w = (const R*)h->fld[F_W];
    fi.p = nullptr; fi.t = nullptr;
    prof_begin(h, K_DIV);
    k_spec_div_reduce<R><<<(unsigned)h->nbd, 256, 0, h->st>>>(Q[SP_W0 + 3], fi, g.n, h->part_div + (long long)sub * h->pd_stride * 3);
    CKL();
    return HC_OK;
}

template <typename R> static int step_sp(hc_handle* h)
{
    const int nsub = h->p.dts == 2 ? 3 : 1;
    for (int sub = 0; sub < nsub; ++sub) {
        int rc = substep_sp<R>(h, sub);
        if (rc) return rc;
    }
    int rc = launch_stats<R>(h, 1);
    if (rc) return rc;
    return launch_finalize(h, nsub, 1);
}

// set-up of the spectral state (src/module_navier_stokes.f90:61-129 with
// real_2_cmplx, spectral_truncation and cmplx_2_real of src/module_spectral.f90):
// spectra of u, v, w, p, t and the histories, truncation of the state spectra,
// and the truncated physical images.
template <typename R> static int init_sp(hc_handle* h)
{
    typedef typename V2<R>::T T2;
    const int fin_ids[9] = {F_U, F_V, F_W, F_P, F_T, F_FF, F_GG, F_HH, F_SS};
    const R* in[9];
    T2* out[9];
    for (int f = 0; f < 9; ++f) { in[f] = (const R*)h->fld[fin_ids[f]]; out[f] = (T2*)h->sp[SP_U + f]; }
    int rc = fft_forward<R>(h, in, out, 9);
    if (rc) return rc;
    TruncArgs<R> ta;
    for (int f = 0; f < 5; ++f) ta.f[f] = (T2*)h->sp[SP_U + f];
    ta.nf = 5; ta.g = h->g; ta.ltr = (int)(h->p.nx / 3.0); ta.mtr = (int)(h->p.ny / 3.0);
    prof_begin(h, K_SPEC_AUX);
    k_spec_truncate<R><<<RED_BLOCKS, 256, 0, h->st>>>(ta);
    CKL();
    const T2* ys[5];
    T2* scr[5];
    R* phys[5];
    const int add0[5] = {0, 0, 0, 0, 0};
    for (int f = 0; f < 5; ++f) {
        ys[f] = (const T2*)h->sp[SP_U + f];
        scr[f] = (T2*)h->sp[SP_W0 + f];
        phys[f] = (R*)h->fld[fin_ids[f]];
    }
    return fft_inverse<R>(h, scr, phys, add0, 5, ys);
}

// Physical image of a spectral-only quantity (p, phi, ff..ss) in work field 0.
template <typename R> static int spec_image(hc_handle* h, int sp_id, void** out)
{
    typedef typename V2<R>::T T2;
    const T2* ys[1] = {(const T2*)h->sp[sp_id]};
    T2* scr[1] = {(T2*)h->sp[SP_W0]};
    R* phys[1] = {(R*)h->sp[SP_W0]};
    const int add0[1] = {0};
    int rc = fft_inverse<R>(h, scr, phys, add0, 1, ys);
    if (rc) return rc;
    *out = h->sp[SP_W0];
    return HC_OK;
}

template <typename R> static int step_dispatch(hc_handle* h)
{
    if (h->p.cds == 1) return step_fd<R, 1>(h);
    if (h->p.cds == 2) return step_fd<R, 2>(h);
    return step_sp<R>(h);
}


// ---------------------------------------------------------------------------
// discrete adjoint of the FD step (hc_adjoint)
// ---------------------------------------------------------------------------
extern "C" {
static int graph_build(hc_handle* h);    // defined with the C-ABI below
}
struct AdjBufs {
    double* lam[4];      // adjoint of u, v, w, p at the current point of the sweep
    double* lh[3];       // adjoint of the histories ff, gg, hh
    double* lh2[3];      // the other half of the ping-pong pair for lh
    double* ax[8];       // adjoints of the eight interpolants of the current sub-step
    double* lq[3];       // lambda_q of the current sub-step (physical)
    double* lbf[3];      // body-force gradient
    double* lt;          // adjoint of T (temperature runs)
    double* ls; double* ls2;   // adjoint of the history ss, ping-pong pair
    double* nxt;         // u, v, w at the end of the segment being reversed (temperature runs)
    int nst, ntp;        // fields a checkpoint / a taped sub-step holds
    double* ckpt;        // checkpoint c: nst fields (u, v, w, p, ff, gg, hh[, t, ss]) at ckpt + nst c n
    double* tape;        // sub-step t of a segment: its start state u, v, w, p[, t] at tape + ntp t n
    double* fin;         // the final state, nst fields
};

static const int ADJ_STATE[9] = {F_U, F_V, F_W, F_P, F_FF, F_GG, F_HH, F_T, F_SS};
static const int ADJ_TAPE[5] = {F_U, F_V, F_W, F_P, F_T};

template <int K> static int col_adj_k(hc_handle* h, const ColAdjArgs& a)
{
    const unsigned nb = (unsigned)((h->g.ncol + CW_WARPS - 1) / CW_WARPS);
    k_column_fd_adj<K><<<nb, CW_WARPS * 32, 0, h->st>>>(a);
    CKL();
    return HC_OK;
}
static int launch_column_adj(hc_handle* h, const ColAdjArgs& a)
{
    switch ((h->p.nz + 31) / 32) {
    case 1: return col_adj_k<1>(h, a);
    case 2: return col_adj_k<2>(h, a);
    case 3: return col_adj_k<3>(h, a);
    case 4: return col_adj_k<4>(h, a);
    case 5: return col_adj_k<5>(h, a);
    case 6: return col_adj_k<6>(h, a);
    case 7: return col_adj_k<7>(h, a);
    case 8: return col_adj_k<8>(h, a);
    default: return HC_ERR_UNSUPPORTED;
    }
}

template <int K> static int col_t_adj_k(hc_handle* h, const ColTAdjArgs& a)
{
    const unsigned nb = (unsigned)((h->g.ncol + CW_WARPS - 1) / CW_WARPS);
    k_column_t_adj<K><<<nb, CW_WARPS * 32, 0, h->st>>>(a);
    CKL();
    return HC_OK;
}
static int launch_column_t_adj(hc_handle* h, const ColTAdjArgs& a)
{
    switch ((h->p.nz + 31) / 32) {
    case 1: return col_t_adj_k<1>(h, a);
    case 2: return col_t_adj_k<2>(h, a);
    case 3: return col_t_adj_k<3>(h, a);
    case 4: return col_t_adj_k<4>(h, a);
    case 5: return col_t_adj_k<5>(h, a);
    case 6: return col_t_adj_k<6>(h, a);
    case 7: return col_t_adj_k<7>(h, a);
    case 8: return col_t_adj_k<8>(h, a);
    default: return HC_ERR_UNSUPPORTED;
    }
}

// Adjoint of the temperature part of one FD sub-step (it runs after the
// momentum part in the forward step, so first here): on entry b.lt / b.ls hold
// the adjoints of T' and of the new history; on return b.lt holds the adjoint of
// the T the sub-step started from (the buoyancy share still to come from the
// momentum part), b.ls that of the old history, and the adjoints of the
// sub-step's velocities u', v', w' (nx[]) in b.lam have gained the advection terms.
template <int CDS> static int adj_substep_t(hc_handle* h, int sub, const double* const* st, const double* const* nx,
                                            AdjBufs& b)
{
    const hc_params& p = h->p;
    double rk_a, rk_b, rk_c;
    if (p.dts == 2) { rk_a = RKC1[sub]; rk_b = RKC2[sub]; rk_c = RKC3[sub]; }
    else { rk_a = 1.5; rk_b = -0.5; rk_c = 1.0; }
    double2* S0 = (double2*)h->spec[0];
    const double* lin[1] = {b.lt};
    double2* sout[1] = {S0};
    int rc = fft_forward<double>(h, lin, sout, 1);
    if (rc) return rc;
    ColTAdjArgs ct;
    ct.at = S0; ct.c = h->cc; ct.g = h->g; ct.rk_c = rk_c;
    prof_begin(h, K_ADJ_COLUMN);
    rc = launch_column_t_adj(h, ct);
    if (rc) return rc;
    double* lqt[1] = {b.lq[0]};
    const int add0[1] = {0};
    rc = fft_inverse<double>(h, sout, lqt, add0, 1);
    if (rc) return rc;
    AdjTArgs m;
    m.a = make_acc<double>(h);
    m.a.f.t = st[4]; m.a.f.u = nx[0]; m.a.f.v = nx[1]; m.a.f.w = nx[2];
    m.lqt = b.lq[0]; m.lss_out = b.ls; m.lss_prev = b.ls2;
    for (int f = 0; f < 3; ++f) { m.ax[f] = b.ax[f]; m.lvel[f] = b.lam[f]; }
    m.out_t = b.lt;
    m.rk_a = rk_a; m.rk_b = rk_b; m.rk_c = rk_c; m.ph = h->ph;
    prof_begin(h, K_ADJ_RHS);
    k_t_adj_interp<CDS><<<pt_grid(h->g), pt_block(), 0, h->st>>>(m);
    CKL();
    prof_begin(h, K_ADJ_RHS);
    k_t_adj_gather<CDS><<<pt_grid(h->g), pt_block(), 0, h->st>>>(m);
    CKL();
    double* t = b.ls; b.ls = b.ls2; b.ls2 = t;
    return HC_OK;
}

// Adjoint of one FD sub-step: on entry b.lam / b.lh (and b.lt / b.ls) hold the
// adjoints of the sub-step's outputs, on return those of its inputs (the state
// st[] it started from; nx[] is the u, v, w it produced).
template <int CDS> static int adj_substep(hc_handle* h, int sub, const double* const* st, const double* const* nx,
                                          AdjBufs& b)
{
    const hc_params& p = h->p;
    double rk_a, rk_b, rk_c;
    if (p.dts == 2) { rk_a = RKC1[sub]; rk_b = RKC2[sub]; rk_c = RKC3[sub]; }
    else { rk_a = 1.5; rk_b = -0.5; rk_c = 1.0; }
    if (p.isscalar == 1) {
        int rc = adj_substep_t<CDS>(h, sub, st, nx, b);
        if (rc) return rc;
    }
    double2* S[4] = {(double2*)h->spec[0], (double2*)h->spec[1], (double2*)h->spec[2], (double2*)h->spec[3]};
    // M^T = iFFT . C^H . FFT applied to the adjoints of (u', v', w', psi = p' - p)
    const double* lin[4] = {b.lam[0], b.lam[1], b.lam[2], b.lam[3]};
    int rc = fft_forward<double>(h, lin, S, 4);
    if (rc) return rc;
    ColAdjArgs ca;
    ca.au = S[0]; ca.av = S[1]; ca.aw = S[2]; ca.apsi = S[3];
    ca.c = h->cc; ca.g = h->g; ca.rk_c = rk_c; ca.dt = p.dt; ca.nu = p.nu;
    prof_begin(h, K_ADJ_COLUMN);
    rc = launch_column_adj(h, ca);
    if (rc) return rc;
    double* lq[3] = {b.lq[0], b.lq[1], b.lq[2]};
    const int add0[3] = {0, 0, 0};
    rc = fft_inverse<double>(h, S, lq, add0, 3);
    if (rc) return rc;
    // adjoint of the right-hand side: lambda_u, v, w are rewritten, lambda_p
    // keeps lambda_p' (p' = p + psi) and gains the pressure-gradient terms; the
    // history adjoints move to the other buffer of their pair
    AdjRhsArgs m;
    m.a = make_acc<double>(h);
    m.a.f.u = st[0]; m.a.f.v = st[1]; m.a.f.w = st[2]; m.a.f.p = st[3];
    for (int f = 0; f < 3; ++f) { m.lq[f] = b.lq[f]; m.lf_out[f] = b.lh[f]; m.lf_prev[f] = b.lh2[f]; m.lbf[f] = b.lbf[f]; }
    for (int f = 0; f < 8; ++f) m.ax[f] = b.ax[f];
    for (int f = 0; f < 4; ++f) m.out[f] = b.lam[f];
    m.out_t = p.isscalar == 1 ? b.lt : nullptr;
    m.got = p.got;
    m.rk_a = rk_a; m.rk_b = rk_b; m.rk_c = rk_c; m.ph = h->ph;
    prof_begin(h, K_ADJ_RHS);
    k_rhs_adj_interp<CDS><<<pt_grid(h->g), pt_block(), 0, h->st>>>(m);
    CKL();
    prof_begin(h, K_ADJ_RHS);
    k_rhs_adj_gather<CDS><<<pt_grid(h->g), pt_block(), 0, h->st>>>(m);
    CKL();
    for (int f = 0; f < 3; ++f) { double* t = b.lh[f]; b.lh[f] = b.lh2[f]; b.lh2[f] = t; }
    return HC_OK;
}

static int adj_copy_state(hc_handle* h, double* dst, int nf, int to_fields, const int* list = ADJ_STATE)
{
    const size_t fb = (size_t)h->g.n * sizeof(double);
    for (int f = 0; f < nf; ++f) {
        double* a = dst + (size_t)f * h->g.n;
        void* fld = h->fld[list[f]];
        if (to_fields) CK(cudaMemcpyAsync(fld, a, fb, cudaMemcpyDeviceToDevice, h->st));
        else CK(cudaMemcpyAsync(a, fld, fb, cudaMemcpyDeviceToDevice, h->st));
    }
    return HC_OK;
}

// Buffers of the adjoint inside the handle's allocation (layout fixed by
// hc_adjoint_forward: nseg checkpoints, a tape of one segment's sub-steps).
static AdjBufs adj_bufs(hc_handle* h)
{
    const long long n = h->g.n;
    AdjBufs b;
    double* q = h->adj_buf;
    for (int f = 0; f < 4; ++f) { b.lam[f] = q; q += n; }
    for (int f = 0; f < 3; ++f) { b.lh[f] = q; q += n; }
    for (int f = 0; f < 3; ++f) { b.lh2[f] = q; q += n; }
    for (int f = 0; f < 8; ++f) { b.ax[f] = q; q += n; }
    for (int f = 0; f < 3; ++f) { b.lq[f] = q; q += n; }
    for (int f = 0; f < 3; ++f) { b.lbf[f] = q; q += n; }
    b.lt = q; q += n;
    b.ls = q; q += n;
    b.ls2 = q; q += n;
    b.nxt = q; q += 3 * n;
    b.nst = h->p.isscalar == 1 ? 9 : 7;
    b.ntp = h->p.isscalar == 1 ? 5 : 4;
    b.ckpt = q; q += (size_t)b.nst * h->adj_nseg * n;
    b.tape = q; q += (size_t)b.ntp * h->adj_seglen * (h->p.dts == 2 ? 3 : 1) * n;
    b.fin = q;
    return b;
}

// Forward pass with a checkpoint every ckpt steps: the state and scalars at
// steps 0, ckpt, 2 ckpt, ... and at the end; the last segment also fills the
// tape (the start state of each of its sub-steps), so the reverse sweep starts
// without recomputation. The steps are plain steps (statistics and diagnostics
// advance as in hc_step), replayed from the step graph outside the last segment.
template <int CDS> static int adjoint_forward(hc_handle* h, AdjBufs& b)
{
    const int nsteps = h->adj_nsteps, ckpt = h->adj_ckpt, nseg = h->adj_nseg;
    const int nsub = h->p.dts == 2 ? 3 : 1;
    const long long n = h->g.n;
    const bool graph = !h->prof;
    int rc;
    if (graph && (rc = graph_build(h))) return rc;
    h->launches = 0;
    CK(cudaEventRecord(h->e0, h->st));
    for (int s = 0; s < nsteps; ++s) {
        const int seg = s / ckpt;
        if (s % ckpt == 0) {
            rc = adj_copy_state(h, b.ckpt + (size_t)seg * b.nst * n, b.nst, 0);
            if (rc) return rc;
            CK(cudaMemcpyAsync(h->adj_sc + seg, h->sc, sizeof(DevScalars), cudaMemcpyDeviceToDevice, h->st));
        }
        if (seg == nseg - 1) {
            const int t0 = (s - seg * ckpt) * nsub;
            for (int sub = 0; sub < nsub; ++sub) {
                rc = adj_copy_state(h, b.tape + (size_t)(t0 + sub) * b.ntp * n, b.ntp, 0, ADJ_TAPE);
                if (rc) return rc;
                rc = substep_fd<double, CDS>(h, sub);
                if (rc) return rc;
            }
            rc = launch_stats<double>(h, 1);
            if (rc) return rc;
            rc = launch_finalize(h, nsub, 1);
            if (rc) return rc;
        } else if (graph) {
            CK(cudaGraphLaunch(h->gexec, h->st));
            h->launches += h->graph_launches;
        } else {
            rc = step_fd<double, CDS>(h);
            if (rc) return rc;
        }
    }
    h->adj_tape_seg = nseg - 1;
    rc = adj_copy_state(h, b.fin, b.nst, 0);
    if (rc) return rc;
    CK(cudaMemcpyAsync(h->adj_sc + nseg, h->sc, sizeof(DevScalars), cudaMemcpyDeviceToDevice, h->st));
    CK(cudaEventRecord(h->e1, h->st));
    CK(cudaEventSynchronize(h->e1));
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, h->e0, h->e1));
    h->adj_ms[0] = ms;
    h->adj_launches[0] = h->launches;
    return HC_OK;
}

// One reverse segment of T sub-steps: with recompute, re-run the sub-steps from
// the restored checkpoint (copying each start state into the tape; the last one
// needs no re-run), then the sub-step adjoints from the last to the first.
template <int CDS> static int adj_segment(hc_handle* h, AdjBufs& b, int T, int recompute)
{
    const int nsub = h->p.dts == 2 ? 3 : 1;
    const long long n = h->g.n;
    int rc;
    if (recompute) {
        for (int t = 0; t < T; ++t) {
            rc = adj_copy_state(h, b.tape + (size_t)t * b.ntp * n, b.ntp, 0, ADJ_TAPE);
            if (rc) return rc;
            if (t == T - 1) break;
            rc = substep_fd<double, CDS>(h, t % nsub, 1, t == 0);
            if (rc) return rc;
        }
    }
    for (int t = T - 1; t >= 0; --t) {
        const double* st[5];
        const double* nx[3];
        for (int f = 0; f < b.ntp; ++f) st[f] = b.tape + ((size_t)t * b.ntp + f) * n;
        // the velocities the sub-step produced: the next sub-step's start, or the
        // segment's end staged in b.nxt
        for (int f = 0; f < 3; ++f) nx[f] = t + 1 < T ? b.tape + ((size_t)(t + 1) * b.ntp + f) * n : b.nxt + (size_t)f * n;
        rc = adj_substep<CDS>(h, t % nsub, st, nx, b);
        if (rc) return rc;
    }
    return HC_OK;
}

static void adj_graph_drop(hc_handle* h)
{
    for (int q = 0; q < ADJ_GRAPHS; ++q) {
        if (h->adj_gexec[q]) cudaGraphExecDestroy(h->adj_gexec[q]);
        h->adj_gexec[q] = nullptr;
        h->adj_gkey[q] = -1;
    }
}

// adj_segment through a CUDA graph, captured once per (T, recompute, which
// buffer of the history-adjoint pair is current) and replayed after that; the
// host-side pointer swaps of the sub-steps are repeated on replay.
template <int CDS> static int adj_segment_run(hc_handle* h, AdjBufs& b, int T, int recompute)
{
    if (h->prof) return adj_segment<CDS>(h, b, T, recompute);
    const int parity = b.lh[0] == h->adj_buf + 4 * h->g.n ? 0 : 1;
    const int key = (T * 2 + parity) * 2 + recompute;
    int slot = -1;
    for (int q = 0; q < ADJ_GRAPHS; ++q)
        if (h->adj_gkey[q] == key) slot = q;
    if (slot < 0) {
        slot = h->adj_gnext;
        h->adj_gnext = (h->adj_gnext + 1) % ADJ_GRAPHS;
        if (h->adj_gexec[slot]) cudaGraphExecDestroy(h->adj_gexec[slot]);
        h->adj_gexec[slot] = nullptr;
        h->adj_gkey[slot] = -1;
        const long long l0 = h->launches;
        CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
        int rc = adj_segment<CDS>(h, b, T, recompute);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(h->st, &g);
        if (rc || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            h->launches = l0;
            return rc ? rc : HC_ERR_CUDA;
        }
        h->adj_glaunch[slot] = h->launches - l0;
        h->launches = l0;
        e = cudaGraphInstantiate(&h->adj_gexec[slot], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) { h->adj_gexec[slot] = nullptr; return HC_ERR_CUDA; }
        h->adj_gkey[slot] = key;
    } else if (T & 1) {
        for (int f = 0; f < 3; ++f) { double* t = b.lh[f]; b.lh[f] = b.lh2[f]; b.lh2[f] = t; }
        if (h->p.isscalar == 1) { double* t = b.ls; b.ls = b.ls2; b.ls2 = t; }
    }
    CK(cudaGraphLaunch(h->adj_gexec[slot], h->st));
    h->launches += h->adj_glaunch[slot];
    return HC_OK;
}

// Reverse sweep over the segments, last first: restore the checkpoint and
// recompute where the tape does not hold the segment, then its sub-step
// adjoints. Ends with the final state and scalars of the forward pass restored.
template <int CDS> static int adjoint_reverse(hc_handle* h, AdjBufs& b)
{
    const int nsteps = h->adj_nsteps, ckpt = h->adj_ckpt, nseg = h->adj_nseg;
    const int nsub = h->p.dts == 2 ? 3 : 1;
    const long long n = h->g.n;
    int rc;
    h->launches = 0;
    CK(cudaEventRecord(h->e0, h->st));
    for (int seg = nseg - 1; seg >= 0; --seg) {
        const int s0 = seg * ckpt, s1 = (s0 + ckpt < nsteps ? s0 + ckpt : nsteps);
        const int recompute = h->adj_tape_seg != seg;
        if (recompute) {
            rc = adj_copy_state(h, b.ckpt + (size_t)seg * b.nst * n, b.nst, 1);
            if (rc) return rc;
            CK(cudaMemcpyAsync(h->sc, h->adj_sc + seg, sizeof(DevScalars), cudaMemcpyDeviceToDevice, h->st));
        }
        if (h->p.isscalar == 1) {
            // u, v, w at the segment's end: the next checkpoint, or the final state
            const double* end = seg == nseg - 1 ? b.fin : b.ckpt + (size_t)(seg + 1) * b.nst * n;
            CK(cudaMemcpyAsync(b.nxt, end, 3 * (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
        }
        rc = adj_segment_run<CDS>(h, b, (s1 - s0) * nsub, recompute);
        if (rc) return rc;
        h->adj_tape_seg = seg;
    }
    rc = adj_copy_state(h, b.fin, b.nst, 1);
    if (rc) return rc;
    CK(cudaMemcpyAsync(h->sc, h->adj_sc + nseg, sizeof(DevScalars), cudaMemcpyDeviceToDevice, h->st));
    CK(cudaEventRecord(h->e1, h->st));
    CK(cudaEventSynchronize(h->e1));
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, h->e0, h->e1));
    h->adj_ms[1] = ms;
    h->adj_launches[1] = h->launches;
    return HC_OK;
}

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

// ---------------------------------------------------------------------------
// ensemble: independent channels advanced together. FD members (no damping)
// advance through grouped launches: each member records the launches of one step
// (its own kernels, grids and arguments), and the n-th launch of every member is
// issued as one launch per distinct kernel variant over all members that run it
// (k_group), so a step takes a few dozen launches whatever the member count.
// Otherwise one graph per step holds a branch per member (the members' own
// streams, forked from and joined into the ensemble stream). Either way the
// step is replayed from a CUDA graph.
// ---------------------------------------------------------------------------
struct hc_ensemble {
    std::vector<hc_handle*> m;
    cudaStream_t st;
    cudaEvent_t e0, e1, fork;
    std::vector<cudaEvent_t> join;
    cudaGraphExec_t gexec;
    long long launches_per_step;
    double last_ms;
    std::vector<GroupLaunch> plan;     // grouped launches of one step (empty: branch graph)
    std::vector<cudaStream_t> side;    // branches for the independent groups of one position
    std::vector<cudaEvent_t> sev;
};

static void ensemble_free(hc_ensemble* e)
{
    for (size_t q = 0; q < e->side.size(); ++q) cudaStreamDestroy(e->side[q]);
    for (size_t q = 0; q < e->sev.size(); ++q) cudaEventDestroy(e->sev[q]);
    if (e->gexec) cudaGraphExecDestroy(e->gexec);
    for (size_t q = 0; q < e->join.size(); ++q) if (e->join[q]) cudaEventDestroy(e->join[q]);
    if (e->fork) cudaEventDestroy(e->fork);
    if (e->e0) cudaEventDestroy(e->e0);
    if (e->e1) cudaEventDestroy(e->e1);
    if (e->st) cudaStreamDestroy(e->st);
    delete e;
}

// The grouped plan of one ensemble step; 1 if some member's step cannot be
// recorded (spectral or damped members), then nothing is kept.
static int ensemble_plan(hc_ensemble* e)
{
    const int n = (int)e->m.size();
    std::vector<std::vector<GroupRec>> recs(n);
    size_t len = 0;
    for (int q = 0; q < n; ++q) {
        hc_handle* h = e->m[q];
        if (h->p.cds == 3 || h->p.isdamp == 1) return 1;
        const int prof = h->prof;
        const long long l0 = h->launches;
        h->prof = 0;
        h->rec = &recs[q];
        const int rc = h->rsz == sizeof(float) ? step_dispatch<float>(h) : step_dispatch<double>(h);
        h->rec = nullptr;
        h->prof = prof;
        h->launches = l0;
        if (rc != HC_OK) return 1;
        if (recs[q].size() > len) len = recs[q].size();
    }
    // the i-th launch of every member, grouped by kernel variant in member order
    for (size_t i = 0; i < len; ++i) {
        std::vector<const void*> keys;
        std::vector<std::vector<const GroupRec*>> groups;
        for (int q = 0; q < n; ++q) {
            if (i >= recs[q].size()) continue;
            const GroupRec* r = &recs[q][i];
            size_t g = 0;
            while (g < keys.size() && keys[g] != r->key) ++g;
            if (g == keys.size()) { keys.push_back(r->key); groups.emplace_back(); }
            groups[g].push_back(r);
        }
        for (size_t g = 0; g < groups.size(); ++g) {
            // at most cap members a launch
            const int cap = groups[g][0]->cap;
            for (size_t c0 = 0; c0 < groups[g].size(); c0 += (size_t)cap) {
                const int cnt = (int)std::min(groups[g].size() - c0, (size_t)cap);
                GroupLaunch gl;
                gl.pos = (int)i;
                if (groups[g][0]->build(groups[g].data() + c0, cnt, &gl) != 0) {
                    e->plan.clear();
                    cudaGetLastError();
                    return 1;
                }
                e->plan.push_back(std::move(gl));
            }
        }
    }
    return 0;
}

int hc_ensemble_create(hc_handle* const* members, int n, hc_ensemble** out)
{
    if (!members || n < 1 || !out) return HC_ERR_ARG;
    *out = nullptr;
    for (int q = 0; q < n; ++q) {
        if (!members[q]) return HC_ERR_ARG;
        if (!members[q]->initialized) return HC_ERR_STATE;
        if (members[q]->dev != members[0]->dev) return HC_ERR_ARG;
        for (int r = 0; r < q; ++r) if (members[r] == members[q]) return HC_ERR_ARG;
    }
    hc_ensemble* e = new hc_ensemble();
    e->st = nullptr; e->e0 = e->e1 = e->fork = nullptr; e->gexec = nullptr; e->launches_per_step = 0; e->last_ms = 0.0;
    e->m.assign(members, members + n);
    e->join.assign(n, nullptr);
    int rc = HC_OK;
    cudaGraph_t g = nullptr;
    long long total = 0;
    if (cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreate(&e->e0) != cudaSuccess || cudaEventCreate(&e->e1) != cudaSuccess) { rc = HC_ERR_CUDA; goto fail; }
    for (int q = 0; q < n; ++q)
        if (cudaEventCreateWithFlags(&e->join[q], cudaEventDisableTiming) != cudaSuccess) { rc = HC_ERR_CUDA; goto fail; }
    if (ensemble_plan(e) == 0) {
        // the groups of one position are independent: all but the first run on
        // side branches forked from and joined back into the ensemble stream
        size_t width = 1;
        for (size_t q = 0, w = 0; q < e->plan.size(); ++q) {
            w = (q > 0 && e->plan[q].pos == e->plan[q - 1].pos) ? w + 1 : 1;
            if (w > width) width = w;
        }
        for (size_t q = 1; q < width; ++q) {
            cudaStream_t sq;
            if (cudaStreamCreateWithFlags(&sq, cudaStreamNonBlocking) != cudaSuccess) { rc = HC_ERR_CUDA; goto fail; }
            e->side.push_back(sq);
        }
        for (size_t q = 0; q < 2 * width; ++q) {
            cudaEvent_t ev;
            if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) { rc = HC_ERR_CUDA; goto fail; }
            e->sev.push_back(ev);
        }
        if (cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) { rc = HC_ERR_CUDA; goto fail; }
        for (size_t q = 0; q < e->plan.size();) {
            size_t r = q;
            while (r < e->plan.size() && e->plan[r].pos == e->plan[q].pos) ++r;
            if (r - q > 1) cudaEventRecord(e->sev[0], e->st);
            for (size_t g = q; g < r; ++g) {
                cudaStream_t sg = g == q ? e->st : e->side[g - q - 1];
                if (g > q) cudaStreamWaitEvent(sg, e->sev[0], 0);
                if (e->plan[g].nblk) e->plan[g].run(e->plan[g], sg);
                if (g > q) { cudaEventRecord(e->sev[1 + (g - q - 1)], sg); cudaStreamWaitEvent(e->st, e->sev[1 + (g - q - 1)], 0); }
            }
            if (cudaGetLastError() != cudaSuccess) rc = HC_ERR_CUDA;
            q = r;
        }
        total = (long long)e->plan.size();
    } else {
    if (cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) { rc = HC_ERR_CUDA; goto fail; }
    cudaEventRecord(e->fork, e->st);
    for (int q = 0; q < n && rc == HC_OK; ++q) {
        hc_handle* h = e->m[q];
        const int prof = h->prof;
        h->prof = 0;
        const long long l0 = h->launches;
        cudaStreamWaitEvent(h->st, e->fork, 0);
        rc = h->rsz == sizeof(float) ? step_dispatch<float>(h) : step_dispatch<double>(h);
        total += h->launches - l0;
        h->launches = l0;
        h->prof = prof;
        cudaEventRecord(e->join[q], h->st);
        cudaStreamWaitEvent(e->st, e->join[q], 0);
    }
    }
    {
        cudaError_t ce = cudaStreamEndCapture(e->st, &g);
        if (rc == HC_OK && ce != cudaSuccess) rc = HC_ERR_CUDA;
    }
    if (rc != HC_OK) { if (g) cudaGraphDestroy(g); cudaGetLastError(); goto fail; }
    if (cudaGraphInstantiate(&e->gexec, g, 0) != cudaSuccess) { cudaGraphDestroy(g); e->gexec = nullptr; rc = HC_ERR_CUDA; goto fail; }
    cudaGraphDestroy(g);
    e->launches_per_step = total;
    *out = e;
    return HC_OK;
fail:
    ensemble_free(e);
    return rc;
}

int hc_ensemble_step(hc_ensemble* e, int nsteps)
{
    if (!e || nsteps < 0) return HC_ERR_ARG;
    for (size_t q = 0; q < e->m.size(); ++q) {
        DevScalars s;
        CK(cudaMemcpy(&s, e->m[q]->sc, sizeof(s), cudaMemcpyDeviceToHost));
        if (s.nan_flag) return HC_ERR_NAN;
    }
    CK(cudaEventRecord(e->e0, e->st));
    for (int n = 0; n < nsteps; ++n) CK(cudaGraphLaunch(e->gexec, e->st));
    CK(cudaEventRecord(e->e1, e->st));
    CK(cudaEventSynchronize(e->e1));
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, e->e0, e->e1));
    e->last_ms = ms;
    for (size_t q = 0; q < e->m.size(); ++q) {
        DevScalars s;
        CK(cudaMemcpy(&s, e->m[q]->sc, sizeof(s), cudaMemcpyDeviceToHost));
        if (s.nan_flag) return HC_ERR_NAN;
    }
    return HC_OK;
}

int hc_ensemble_last_ms(hc_ensemble* e, double* ms, long long* launches_per_step)
{
    if (!e) return HC_ERR_ARG;
    if (ms) *ms = e->last_ms;
    if (launches_per_step) *launches_per_step = e->launches_per_step;
    return HC_OK;
}

int hc_ensemble_destroy(hc_ensemble* e)
{
    if (!e) return HC_ERR_ARG;
    cudaStreamSynchronize(e->st);
    ensemble_free(e);
    return HC_OK;
}

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
