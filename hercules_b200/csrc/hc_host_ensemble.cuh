// hc_host_ensemble.cuh -- host code of libhercules_b200 included by hc_api.cu (one translation
// unit: every kernel template is instantiated once): the ensemble C-ABI (hc_ensemble_*): grouped launches over the members and the
// per-step CUDA graph.
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
