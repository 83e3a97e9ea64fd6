// hc_host_fft.cuh -- host code of libhercules_b200 included by hc_api.cu (one translation
// unit: every kernel template is instantiated once): the transform dispatch: the compile-time-length x and y kernels, the fused 2-D
// transforms on thread-block clusters, the runtime-plan fallback, and the
// shared-memory limits the kernels need.
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
// fused 2-D transforms (hc_fft2d.cuh): persistent clusters of C CTAs over the (field, plane) pairs.
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
            if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::smem) != cudaSuccess) {
                cudaGetLastError();
                return HC_ERR_UNSUPPORTED;
            }
            if (C > 8 && cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
                cudaGetLastError();
                return HC_ERR_UNSUPPORTED;
            }
            int ncl = 0;
            cfg.gridDim = dim3(C);
            if (cudaOccupancyMaxActiveClusters(&ncl, k, &cfg) != cudaSuccess || ncl < 1) {
                cudaGetLastError();
                return HC_ERR_UNSUPPORTED;
            }
            h->f2_ncl[q] = ncl;
        }
        return HC_OK;
    }
    // persistent clusters: as many as are resident at once, at most one a plane
    const long long np = (long long)nf * h->g.nz;
    const long long ncl = std::min<long long>(np, h->f2_ncl[op == 1 ? 0 : 1]);
    F2Args<R> b = *a;
    b.nplanes = (int)np;
    cfg.gridDim = dim3((unsigned)(ncl * C));
    CK(cudaLaunchKernelEx(&cfg, op == 1 ? fwd : inv, b));
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

// ---------------------------------------------------------------------------
// the spectral products fused with their forward x transform (hc_spec.cuh):
// x half lengths with an instantiation
// ---------------------------------------------------------------------------
#define HC_SPX_LENGTHS(X) X(16) X(32) X(64) X(128) X(256)

// op 0: raise the shared-memory limit, note the resident blocks; 1: launch
template <typename R, int N> static int spx_op(hc_handle* h, int op, const ProdFxArgs<R>* a, dim3 grid)
{
    constexpr size_t sm = SpxCfg<R, N, HC_FFT_T_RMAX>::smem;
    // above 100 KB of shared memory (FP64 at nx/2 = 256) fewer than two blocks
    // fit an SM: the separate kernels run
    if constexpr (sm > 100 * 1024) {
        return HC_ERR_UNSUPPORTED;
    } else {
        void (*k)(ProdFxArgs<R>) = k_spec_products_fx<R, N, HC_FFT_T_RMAX>;
        if (op == 0) {
            if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess ||
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&h->spx_minb, k, SpxCfg<R, N, HC_FFT_T_RMAX>::NT, sm) != cudaSuccess ||
                h->spx_minb < 1) {
                cudaGetLastError();
                return HC_ERR_UNSUPPORTED;
            }
            return HC_OK;
        }
        k<<<grid, SpxCfg<R, N, HC_FFT_T_RMAX>::NT, sm, h->st>>>(*a);
        return HC_OK;
    }
}

template <typename R> static int spx_dispatch(hc_handle* h, int op, const ProdFxArgs<R>* a, dim3 grid)
{
    switch (h->g.nxh) {
#define HC_SPX_CASE(N) case N: return spx_op<R, N>(h, op, a, grid);
    HC_SPX_LENGTHS(HC_SPX_CASE)
#undef HC_SPX_CASE
    }
    return HC_ERR_UNSUPPORTED;
}

// the temperature products fused with their x transform: op 0 set up, 1 launch
template <typename R, int N> static int spx_t_op(hc_handle* h, int op, const ProdTFxArgs<R>* a, dim3 grid)
{
    constexpr size_t sm = SpxTCfg<R, N, HC_FFT_T_RMAX>::smem;
    if constexpr (sm > 100 * 1024) {
        return HC_ERR_UNSUPPORTED;
    } else {
        void (*k)(ProdTFxArgs<R>) = k_spec_products_t_fx<R, N, HC_FFT_T_RMAX>;
        if (op == 0) {
            if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess) {
                cudaGetLastError();
                return HC_ERR_UNSUPPORTED;
            }
            return HC_OK;
        }
        k<<<grid, SpxTCfg<R, N, HC_FFT_T_RMAX>::NT, sm, h->st>>>(*a);
        return HC_OK;
    }
}

template <typename R> static int spx_t_dispatch(hc_handle* h, int op, const ProdTFxArgs<R>* a, dim3 grid)
{
    switch (h->g.nxh) {
#define HC_SPX_CASE(N) case N: return spx_t_op<R, N>(h, op, a, grid);
    HC_SPX_LENGTHS(HC_SPX_CASE)
#undef HC_SPX_CASE
    }
    return HC_ERR_UNSUPPORTED;
}

// Levels a block of k_spec_products_fx: the chunk (4..SPEC_KCHUNK_MAX) whose
// grid of ny x chunks blocks fills its last wave best, each chunk's two extra
// start-up levels counted as extra reads
static int spx_kchunk(const hc_handle* h)
{
    const int nz = h->p.nz, ny = h->g.ny;
    const double slots = 148.0 * h->spx_minb;
    int best = nz < SPEC_KCHUNK_MAX ? nz : SPEC_KCHUNK_MAX;
    double bcost = 1e300;
    for (int kc = 4; kc <= SPEC_KCHUNK_MAX && kc <= nz; ++kc) {
        const double nb = (double)ny * ((nz + kc - 1) / kc);
        const double waves = nb / slots;
        const double cost = ceil(waves) / waves * (1.0 + 2.0 / kc);
        if (cost < bcost - 1e-12) { bcost = cost; best = kc; }
    }
    return best;
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
    // explicit tile sizes (tile[0], tile[1] > 0) select the runtime-length kernels;
    // tile[0] = -1 the fused 2-D transforms where a shape exists (measured slower
    // than the separate kernels at 512 x 384 x 256, so not the default)
    if (h->p.tile[0] < -1) return HC_ERR_PARAM;
    h->fft_tx = h->p.tile[0] <= 0 && fft_t_length_ok(nxh);
    h->fft_ty = h->p.tile[1] == 0 && fft_t_length_ok(ny);
    if (h->fft_tx || h->fft_ty) {
        int rc = h->rsz == sizeof(double) ? fft_t_setup<double>(h) : fft_t_setup<float>(h);
        if (rc != HC_OK) return rc;
    }
    // the fused transforms where a shape exists, when tile[0] = -1 asks for them
    h->fft2d = 0;
    if (h->fft_tx && h->fft_ty && h->p.tile[0] == -1) {
        const int rc = h->rsz == sizeof(double) ? fft2d_dispatch<double>(h, 0, nullptr, 0) : fft2d_dispatch<float>(h, 0, nullptr, 0);
        h->fft2d = rc == HC_OK;
    }
    // the spectral products with their x transform in one kernel: templated x
    // transforms of an instantiated length, the separate y transform after them
    h->spx = 0;
    if (h->p.cds == 3 && h->fft_tx && !h->fft2d) {
        const int rc = h->rsz == sizeof(double) ? spx_dispatch<double>(h, 0, nullptr, dim3())
                                                : spx_dispatch<float>(h, 0, nullptr, dim3());
        h->spx = rc == HC_OK;
    }
    h->spx_t = 0;
    if (h->spx && h->p.isscalar == 1) {
        const int rc = h->rsz == sizeof(double) ? spx_t_dispatch<double>(h, 0, nullptr, dim3())
                                                : spx_t_dispatch<float>(h, 0, nullptr, dim3());
        h->spx_t = rc == HC_OK;
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
