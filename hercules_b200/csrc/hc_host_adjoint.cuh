// hc_host_adjoint.cuh -- host code of libhercules_b200 included by hc_api.cu (one translation
// unit: every kernel template is instantiated once): the discrete adjoint of the FD step: buffers, the sub-step adjoints, the
// checkpointed forward pass and the reverse sweep (hc_adjoint_* below the C-ABI).
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
