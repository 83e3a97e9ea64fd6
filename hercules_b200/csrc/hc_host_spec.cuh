// hc_host_spec.cuh -- host code of libhercules_b200 included by hc_api.cu (one translation
// unit: every kernel template is instantiated once): the pseudo-spectral sub-step and step (time_advancement_sp) and the set-up of
// the spectral state.
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
    if (kc > SPEC_KCHUNK_MAX) kc = SPEC_KCHUNK_MAX;
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
        const unsigned nb = (unsigned)((h->g.ncol + SP_COLS - 1) / SP_COLS);
        k_column_sp_tile<R, K><<<nb, SP_COLS * 32, column_sp_tile_smem<K>(sizeof(typename V2<R>::T)), h->st>>>(a);
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
        pa.halt = halt;
        const R* fin[8];
        T2* fout[8];
        for (int f = 0; f < 8; ++f) { fin[f] = Q[SP_W0 + f]; fout[f] = S[SP_W0 + f]; }
        // pairs of points: the fields must be aligned to two values
        bool fx = h->spx && !h->rec;
        auto al = [&](const void* q) { return ((uintptr_t)q & (2 * sizeof(R) - 1)) == 0; };
        fx = fx && al(pa.u) && al(pa.v) && al(pa.w) && al(pa.t);
        for (int f = 0; f < 6; ++f) fx = fx && (!pa.d[f] || al(pa.d[f]));
        if (fx) {
            ProdFxArgs<R> fa;
            fa.p = pa;
            for (int f = 0; f < 8; ++f) fa.p.out[f] = (R*)S[SP_W0 + f];
            fa.p.kchunk = spx_kchunk(h);
            fa.tw = fft_tw<R>(h, 0); fa.wp = fft_tw<R>(h, 2); fa.scale = (R)(1.0 / p.nx);
            prof_begin(h, K_SPEC_PRODFX);
            if ((rc = spx_dispatch<R>(h, 1, &fa, dim3((unsigned)g.ny, (p.nz + fa.p.kchunk - 1) / fa.p.kchunk)))) return rc;
            CKL();
            if ((rc = fft_forward<R>(h, fin, fout, 8, true))) return rc;
        } else {
            pa.kchunk = spec_kchunk(h, g.nxy);
            prof_begin(h, K_SPEC_PROD);
            k_spec_products<R><<<dim3((unsigned)((g.nxy + 255) / 256), (p.nz + pa.kchunk - 1) / pa.kchunk), 256, 0, h->st>>>(pa);
            CKL();
            if ((rc = fft_forward<R>(h, fin, fout, 8))) return rc;
        }
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
        pt.g = g; pt.ttop = p.ttop; pt.halt = halt;
        const R* fin[3] = {Q[SP_W0 + 4], Q[SP_W0 + 5], Q[SP_W0 + 6]};
        T2* fout[3] = {S[SP_W0 + 4], S[SP_W0 + 5], S[SP_W0 + 6]};
        auto al = [&](const void* q) { return ((uintptr_t)q & (2 * sizeof(R) - 1)) == 0; };
        if (h->spx_t && !h->rec && al(pt.u) && al(pt.v) && al(pt.w) && al(pt.t)) {
            ProdTFxArgs<R> ta;
            ta.p = pt;
            for (int f = 0; f < 3; ++f) ta.p.out[f] = (R*)S[SP_W0 + 4 + f];
            ta.p.kchunk = spx_kchunk(h);
            ta.tw = fft_tw<R>(h, 0); ta.wp = fft_tw<R>(h, 2); ta.scale = (R)(1.0 / p.nx);
            prof_begin(h, K_SPEC_PRODFX);
            if ((rc = spx_t_dispatch<R>(h, 1, &ta, dim3((unsigned)g.ny, (p.nz + ta.p.kchunk - 1) / ta.p.kchunk)))) return rc;
            CKL();
            if ((rc = fft_forward<R>(h, fin, fout, 3, true))) return rc;
        } else {
            pt.kchunk = spec_kchunk(h, g.nxy);
            prof_begin(h, K_SPEC_PROD);
            k_spec_products_t<R><<<dim3((unsigned)((g.nxy + 255) / 256), (p.nz + pt.kchunk - 1) / pt.kchunk), 256, 0, h->st>>>(pt);
            CKL();
            if ((rc = fft_forward<R>(h, fin, fout, 3))) return rc;
        }
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
    const R* dv = Q[SP_W0 + 3];
    double* dp = h->part_div + (long long)sub * h->pd_stride * 3;
    auto a16 = [](const void* q) { return ((uintptr_t)q & 15) == 0; };
    if (a16(dv) && a16(fi.u) && a16(fi.v) && a16(fi.w))
        k_spec_div_reduce<R, 16 / sizeof(R)><<<(unsigned)h->nbd, 256, 0, h->st>>>(dv, fi, g.n, dp);
    else
        k_spec_div_reduce<R, 1><<<(unsigned)h->nbd, 256, 0, h->st>>>(dv, fi, g.n, dp);
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
