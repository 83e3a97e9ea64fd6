// hc_host_step.cuh -- host code of libhercules_b200 included by hc_api.cu (one translation
// unit: every kernel template is instantiated once): the launch helpers (transforms, statistics, finaliser, column solves) and the FD
// sub-step and step (time_advancement_fd).
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

// x then y forward transform of nf physical fields into half spectra (x_done:
// out already holds the x half spectra, only the y transform runs)
template <typename R> static int fft_forward(hc_handle* h, const R* const* in, typename V2<R>::T* const* out, int nf,
                                             bool x_done = false)
{
    typedef typename V2<R>::T T2;
    const int* halt = &h->sc->nan_flag;
    if (nf < 1 || nf > HC_FFT_MAXF) return HC_ERR_ARG;
    if (x_done && h->fft2d) return HC_ERR_ARG;
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
    if (x_done) {
    } else if (h->fft_tx) {
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
