/*
 * hercules_b200.h -- C-ABI of the B200 (sm_100a) time-step engine for the
 * HERCULES channel / Ekman-layer DNS code.
 *
 * The reference advances its state through argument-less Fortran subroutines
 * that read and write module globals:
 *   - setup        src/module_navier_stokes.f90:53-129 (drive: get_mesh_param,
 *                  initiate_fields, update_ri(0), calculate_ubar, get_*_eqn_coeff,
 *                  spectral truncation for cds=3, update_boundary_*)
 *   - one step     src/module_navier_stokes.f90:142-165 (screen_cpu_time,
 *                  update_ri, time_advancement_fd / time_advancement_sp,
 *                  calculate_ubar)
 *   - outputs      src/module_navier_stokes.f90:169-203 read u,v,w,p,t,ff..ss and
 *                  the eleven mean_* accumulators.
 * This header replaces that seam with a handle-based, re-entrant-per-handle API.
 * All entry points return 0 (HC_OK) or a negative HC_ERR_* code; nothing here
 * prints or exits (the reference's `print` + `stop` become error codes).
 *
 * Host arrays are Fortran-ordered real(8): element (i,j,k) of the interior
 * (0-based, i fastest) lives at host[(i+g) + ld1*((j+g) + ld2*(k+g))] where g is
 * the ghost width the caller passes (2 for the reference's ghosted module arrays
 * of shape (nx+4,ny+4,nz+4), 0 for interior-only arrays).
 */
#ifndef HERCULES_B200_H
#define HERCULES_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- error codes -------------------------------------------------------- */
#define HC_OK               0
#define HC_ERR_ARG         -1   /* bad argument / null pointer                */
#define HC_ERR_PARAM       -2   /* parameter check failed (reference :254-270) */
#define HC_ERR_CUDA        -3   /* CUDA runtime error                         */
#define HC_ERR_NOMEM       -4   /* device allocation failed                   */
#define HC_ERR_NAN         -5   /* NaN detected (reference src/module_io.f90:135-140) */
#define HC_ERR_STATE       -6   /* call out of order (e.g. step before init)  */
#define HC_ERR_UNSUPPORTED -7   /* option combination not built               */
#define HC_ERR_SIZE        -8   /* size beyond a documented maximum           */

/* ---- precision modes ---------------------------------------------------- */
#define HC_PREC_FP64   0   /* every field, FFT and solve in real(8)            */
#define HC_PREC_MIXED  1   /* fields/stencils/FFTs FP32; Thomas, mean mode,
                              divergence check and reductions FP64             */

/* ---- field ids (hc_upload / hc_download) -------------------------------- */
#define HC_FIELD_U        0
#define HC_FIELD_V        1
#define HC_FIELD_W        2
#define HC_FIELD_P        3
#define HC_FIELD_T        4
#define HC_FIELD_FF       5
#define HC_FIELD_GG       6
#define HC_FIELD_HH       7
#define HC_FIELD_SS       8
#define HC_FIELD_PHI      9
#define HC_FIELD_MEAN_U  10   /* running sums, NOT divided by the step count */
#define HC_FIELD_MEAN_V  11
#define HC_FIELD_MEAN_W  12
#define HC_FIELD_MEAN_T  13
#define HC_FIELD_MEAN_UU 14
#define HC_FIELD_MEAN_VV 15
#define HC_FIELD_MEAN_WW 16
#define HC_FIELD_MEAN_UW 17
#define HC_FIELD_MEAN_VW 18
#define HC_FIELD_MEAN_TT 19
#define HC_FIELD_MEAN_TW 20
#define HC_NUM_FIELDS    21

/*
 * hc_params: POD mirror of the reference namelists &domain &modeling
 * &constants (src/module_parameters.f90:40-157). p_row/p_col and the &io group
 * stay with the host. `precision` selects HC_PREC_*.
 */
typedef struct hc_params {
    int    nx, ny, nz;
    double lx, ly, lz, zstretch;
    int    ochannel;          /* 0 closed channel, 1 open channel              */
    int    dp_opt;            /* 1 const friction, 2 const flow rate, 3 Ekman   */
    int    cds;               /* 1 FD2, 2 FD4, 3 pseudo-spectral                */
    int    issk;              /* skew-symmetric convection (cds=3)              */
    int    dts;               /* 1 AB2, 2 RK3                                   */
    int    isdamp, nzdamp;
    double cdamp;
    double nu, alpha, got, fc, ug, vg, dt;
    int    imax;
    double u_mrf;
    int    isscalar;
    double t_ref, tbot, ttop;
    int    is_ri_var;
    double ri_str, ri_end;
    int    precision;
    /* tile shapes, 0 = automatic (the autotuner in hercules_b200/autotune.py
     * writes these): [0] x-FFT rows per block (-1: the fused 2-D transform
     * kernels where a shape exists), [1] y-FFT lines per
     * block (a positive value selects the runtime-plan transforms), [2] momentum-RHS
     * levels per block, [3] column solve: 1 one thread per column, 2 one warp
     * per column without the coalescing tiles, >= 32 one thread per column with
     * that many threads a block */
    int    tile[4];
    /* bottom temperature condition (not in the reference, which fixes T): 0 the
     * wall temperature tbot (src/module_boundary.f90:176-183); 1 a fixed
     * wall-normal gradient dT/dz = tbot at the bottom wall, i.e. the fixed heat
     * flux alpha*tbot (tbot > 0 cools the fluid from below) */
    int    tbc_bot;
    int    reserved[2];
} hc_params;

/*
 * hc_diag: per-step diagnostics (reference screen_cpu_time src/module_io.f90:32-80,
 * screen_div_error :85-206 / screen_div_error_spec src/module_spectral.f90:899-1007,
 * calculate_ubar src/module_parameters.f90:513-546).
 * div_max keeps the reference's SIGNED value for cds=1,2 (src/module_io.f90:131-133)
 * and |div| for cds=3; div_*_sub hold each RK sub-step (only [0] for AB2).
 */
typedef struct hc_diag {
    double time_sim;        /* after the += dt of this step                  */
    double cfl;             /* CFL of the fields at the start of the step    */
    double div_avg;         /* final sub-step                                */
    double div_max;
    double div_hist_max;
    double ubar;            /* bulk velocity after the step (dp_opt=2), else 0 */
    double dpx_drive;       /* after the last sub-step                       */
    double got;             /* g/T0 used in the step                         */
    double div_avg_sub[3];
    double div_max_sub[3];
    int    nan_flag;
    int    step;            /* 1-based absolute step index                   */
} hc_diag;

typedef struct hc_handle hc_handle;

/* Create a handle on the current CUDA device: checks parameters exactly as
 * initiate_parameters (src/module_parameters.f90:254-270), computes the tanh
 * grid (get_mesh_param :432-508) and allocates device state, zero-filled as
 * initiate_fields (src/module_tools.f90:136-227). */
int hc_create(const hc_params* p, hc_handle** out);

/* Override the vertical grid with the host's own get_mesh_param arrays
 * (each of length nz+4, Fortran index k=1..nz+4 at [k-1]). */
int hc_set_grid(hc_handle* h, const double* dz, const double* l_t,
                const double* l_b, const double* dz_t, const double* dz_b);

/* Read back the vertical grid (each of length nz+4). */
int hc_get_grid(hc_handle* h, double* dz, double* l_t, double* l_b,
                double* dz_t, double* dz_b);

/* Copy one host field into the handle (replaces the reference's module array
 * before `drive` starts, e.g. read_init_fields src/module_tools.f90:260-316).
 * U is the frame-relative velocity held in the module array (u_file - u_mrf). */
int hc_upload(hc_handle* h, int field_id, const double* host,
              int ld1, int ld2, int ghost);

/* Copy one field out. Ghost cells of the destination are not written. */
int hc_download(hc_handle* h, int field_id, double* host,
                int ld1, int ld2, int ghost);

/* Finish the set-up part of drive (src/module_navier_stokes.f90:61-129):
 * update_ri(0), calculate_ubar (dp_opt=2), the forward FFT + 2/3 truncation of
 * all fields for cds=3, boundary conditions, CFL of the initial fields. */
int hc_initialize(hc_handle* h);

/* Advance nsteps steps (the body of the drive loop :142-165). `out` may be
 * NULL or point at nsteps hc_diag records. Stops early with HC_ERR_NAN after
 * the step in which a NaN appeared. */
int hc_step(hc_handle* h, int nsteps, hc_diag* out);

/* Scalars the host prints / checkpoints: time_sim, dpx_drive, ubar, got,
 * div_hist_max, completed step count. */
int hc_get_scalars(hc_handle* h, double* time_sim, double* dpx_drive,
                   double* ubar, double* got, double* div_hist_max, int* step);

/* Device-pointer variants for the PyTorch binding: `dev` is a contiguous
 * interior-only (nx,ny,nz) Fortran-order array on the handle's device, of the
 * handle's storage type (double for HC_PREC_FP64, float for HC_PREC_MIXED;
 * mean accumulators are always double). */
int hc_upload_dev(hc_handle* h, int field_id, const void* dev);
int hc_download_dev(hc_handle* h, int field_id, void* dev);

/* Time the last hc_step call spent on the device (CUDA events), ms. */
int hc_last_step_ms(hc_handle* h, double* ms);

/* Number of kernel launches the last hc_step issued. */
int hc_last_launch_count(hc_handle* h, long long* n);

/* Optional per-launch timing: with profiling on, hc_step brackets every kernel
 * launch with a CUDA-event pair on the handle's stream and sums the elapsed
 * times per kernel. No counterpart in the reference (it prints cpu_time only,
 * src/module_io.f90:72-75). */
int hc_set_profiling(hc_handle* h, int enable);

/* Per-kernel totals since profiling was enabled: names in 32-byte slots. */
int hc_kernel_profile(hc_handle* h, int max, char* names, double* total_ms,
                      long long* launches, int* count);

/* Divergence check of caller-owned device fields that allocates nothing. No
 * counterpart in the reference. It is for hosts that own all device memory and
 * let no library call cudaMalloc (for instance a Fortran code whose device arrays
 * come from its own arena or OpenACC data regions): u, v, w are the caller's
 * interior-only (nx,ny,nz) arrays of the storage type of p->precision, dz is the
 * host copy of the nz+4 vertical spacings, out_dev is 3 doubles in device memory
 * receiving {mean |div|, signed div at the largest |div|, NaN flag} exactly as
 * hc_step's divergence diagnostic computes them. Scratch lives in one fixed
 * array per device (about 61 KB, held until exit): nz <= 4096 and
 * nx*ny*nz < 2^31, else HC_ERR_SIZE. nx and ny must be even (nx >= 8, ny >= 4,
 * nz >= 3), else HC_ERR_PARAM; u, v, w and out_dev must be 8-byte aligned, else
 * HC_ERR_ARG; cds must be 1 or 2. All of these are checked before any device
 * work. The first call on a device looks up that array's address and keeps it
 * for the life of the process (do not call again on a device after
 * cudaDeviceReset); make it before any stream capture. Calls share the array,
 * so calls that overlap on the GPU (several streams or host threads) race with
 * each other. `stream` is a cudaStream_t (NULL for the default stream); the
 * call does not synchronise: dz is copied asynchronously on that stream, so if
 * it is page-locked host memory it must stay valid and unchanged until the
 * stream has passed the call. */
int hc_divergence_noalloc(const hc_params* p, const double* dz, const void* u,
                          const void* v, const void* w, double* out_dev, void* stream);

/* Body force, no counterpart in the reference: fx, fy, fz are interior-only
 * (nx,ny,nz) Fortran-order host arrays added to the explicit momentum terms ff,
 * gg, hh every sub-step (the FD right-hand side; on the spectral path through
 * their spectra). A NULL component is zero; all three NULL remove the force. */
int hc_set_body_force(hc_handle* h, const double* fx, const double* fy, const double* fz);

/* Advance hc_step through a CUDA graph of one whole step, captured on the first
 * call after enabling and replayed once per step (no counterpart in the
 * reference). Saves the per-kernel launch cost, which dominates small grids.
 * Ignored while profiling is on; hc_set_grid and hc_set_body_force drop the graph
 * (it is captured again on the next step). */
int hc_set_graph(hc_handle* h, int enable);

/* Ensemble of independent channels (no counterpart in the reference): one CUDA
 * graph per step holds a branch per member, each member's kernels on its own
 * stream, so small members run side by side. Members stay owned by the caller,
 * must be initialized, on one device, distinct, and not stepped on their own
 * while the ensemble lives. hc_ensemble_step advances every member nsteps steps
 * (their diagnostics ring on the device as in hc_step; read scalars with
 * hc_get_scalars) and returns HC_ERR_NAN if any member has seen a NaN. */
typedef struct hc_ensemble hc_ensemble;
int hc_ensemble_create(hc_handle* const* members, int n, hc_ensemble** out);
int hc_ensemble_step(hc_ensemble* e, int nsteps);
int hc_ensemble_last_ms(hc_ensemble* e, double* ms, long long* launches_per_step);
int hc_ensemble_destroy(hc_ensemble* e);

/* Discrete adjoint of FD steps (no counterpart in the reference), in two calls.
 * hc_adjoint_forward advances the handle by nsteps like hc_step (same final
 * fields, scalars and statistics), keeping a checkpoint of the state every ckpt
 * steps. hc_adjoint_reverse then returns the gradient of
 * J = <lu,u_N> + <lv,v_N> + <lw,w_N> + <lp,p_N> (the seeds, (nx,ny,nz) host
 * arrays, NULL = 0) with respect to the state the forward pass started from
 * (gu, gv, gw, gp) and to the body force (gbf: 3*nx*ny*nz, fx then fy then fz);
 * any output may be NULL. It recomputes one segment of ckpt steps at a time
 * from its checkpoint, leaves the handle in the forward pass's final state and
 * may be called again with other seeds. Any call that changes the state
 * (hc_step, hc_upload*, hc_initialize, hc_set_grid, hc_set_body_force)
 * invalidates the checkpoints (HC_ERR_STATE). Built for FP64 storage, cds = 1
 * or 2, dp_opt = 1 or 3, isdamp = 0, nz <= 256, and with temperature
 * (isscalar = 1) for a constant Richardson number (is_ri_var = 0); else
 * HC_ERR_UNSUPPORTED. With AB2 (dts = 1) the gradient with respect to the
 * starting histories is not returned. hc_adjoint is the two calls in one.
 * hc_adjoint_reverse_t adds the temperature: lt seeds <lt, t_N> in J and gt
 * receives the gradient with respect to the starting temperature (NULL = none;
 * either non-NULL without temperature is HC_ERR_ARG). */
int hc_adjoint_forward(hc_handle* h, int nsteps, int ckpt);
int hc_adjoint_reverse(hc_handle* h, const double* lu, const double* lv, const double* lw, const double* lp,
                       double* gu, double* gv, double* gw, double* gp, double* gbf);
int hc_adjoint_reverse_t(hc_handle* h, const double* lu, const double* lv, const double* lw, const double* lp,
                         const double* lt, double* gu, double* gv, double* gw, double* gp, double* gt, double* gbf);
int hc_adjoint(hc_handle* h, int nsteps, int ckpt, const double* lu, const double* lv, const double* lw,
               const double* lp, double* gu, double* gv, double* gw, double* gp, double* gbf);
/* Device time and kernel launches of the last adjoint forward pass and reverse
 * sweep (recomputation of the segments included). */
int hc_adjoint_last_ms(hc_handle* h, double* forward_ms, double* reverse_ms, long long* forward_launches,
                       long long* reverse_launches);

int hc_destroy(hc_handle* h);

const char* hc_error_string(int code);

#ifdef __cplusplus
}
#endif
#endif
