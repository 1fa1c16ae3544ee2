// Host side of the multilevel preconditioner (tb_multilevel.cuh): building
// the hierarchy on the device and launching one preconditioned iteration.
// Included by tb_system.cu inside its anonymous namespace.

void free_coarse(tb_system* s);
int keep_coarse_in_l2(tb_system* s);

inline int ml_cdiv(int a, int b) { return (a + b - 1) / b; }

MLGrid ml_grid(int L, int ny, int nx) {
    MLGrid g{};
    g.L = L;
    g.ny = ny;
    g.nx = nx;
    g.plane = (long long)ny * nx;
    g.n = (long long)L * g.plane;
    return g;
}

// Coarse grids, level 1 first: b x b aggregates of node columns per level
// (b = ml_aggregate_width of the level above) until at most 2048 unknowns
// remain (the last grid is inverted densely).  Each grid records the width
// that forms the next one (0 on the last).
std::vector<MLGrid> ml_grids(const Layout& L) {
    std::vector<MLGrid> out;
    int ny = ml_cdiv(L.R + 1, kMlAgg), nx = ml_cdiv(L.C + 1, kMlAgg);
    out.push_back(ml_grid(L.S + 1, ny, nx));
    while (out.back().n > 2048 && (ny > 1 || nx > 1)) {
        const int b = ml_aggregate_width((int)out.size(), out.front().ny, out.front().nx);
        out.back().b = b;
        ny = ml_cdiv(ny, b);
        nx = ml_cdiv(nx, b);
        out.push_back(ml_grid(L.S + 1, ny, nx));
    }
    return out;
}

// Fine pass: 32 x 8 node columns per block.  Coarse levels: one column per
// thread (z-line kernels), one node per thread (residual kernels).
dim3 ml_fine_grid(const Layout& L) { return dim3(ml_cdiv(L.Xp, kMlTile), ml_cdiv(L.R + 1, 8)); }
dim3 ml_column_grid(const MLGrid& g) { return dim3((unsigned)((g.plane + kMlThreads - 1) / kMlThreads)); }
dim3 ml_node_grid(const MLGrid& g) { return dim3(ml_cdiv(g.nx, kMlTile), ml_cdiv(g.ny, 8), g.L); }

void free_multilevel(tb_system* s) {
    dev_free(s, s->ml_zl);
    dev_free(s, s->ml_zi);
    dev_free(s, s->ml_w);
    const size_t c = s->ml.size();
    for (size_t l = 0; l < c; ++l) {
        tb_system::MLLevel& lv = s->ml[l];
        dev_free(s, lv.st);
        dev_free(s, lv.lf);
        dev_free(s, lv.ipd);
        dev_free(s, lv.x);
        if (l + 1 < c) {  // the coarsest level's R and y are coarse_rc and coarse_c
            dev_free(s, lv.R);
            dev_free(s, lv.y);
        }
    }
    s->ml.clear();
    s->ml_stages = 0;
    s->ml_staged = false;
}

int ensure_partials(tb_system* s, int blocks) {
    if (blocks <= s->partial_blocks) return TB_OK;
    dev_free(s, s->partials);
    TB_CHECK(alloc_n(s, &s->partials, (long long)blocks * 4));
    s->partial_blocks = blocks;
    return TB_OK;
}

// Dense coarse product c = Minv rc on `cl` (as the two-level step, without
// its restriction).
template <int MODE>
cudaError_t launch_coarse_apply(tb_system* s, bool pdl) {
    const CoarseLayout& cl = s->cl;
    static int per_sm[3] = {0, 0, 0};
    const size_t smem = sizeof(float) * (size_t)cl.ld;
    cudaError_t e = cudaSuccess;
    if (per_sm[MODE] == 0) {
        int n = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, coarse_apply<MODE>, kCoarseThreads, sizeof(float) * 8192);
        if (e != cudaSuccess) return e;
        per_sm[MODE] = std::max(n, 1);
    }
    constexpr int rows = kCoarseThreads / 32 / kCoarseSplit;
    const int grid = std::max(1, std::min({(cl.nc + rows - 1) / rows, s->partial_blocks, s->sms * per_sm[MODE]}));
    if (pdl)
        return launch_pdl(coarse_apply<MODE>, dim3(grid), dim3(kCoarseThreads), smem, s->stream,
                          (const float*)s->coarse_inv32, (const float*)s->coarse_rc, s->coarse_c, cl.nc, cl.ld, s->ctl,
                          s->partials, s->counter);
    coarse_apply<MODE><<<grid, kCoarseThreads, smem, s->stream>>>(s->coarse_inv32, s->coarse_rc, s->coarse_c, cl.nc,
                                                                  cl.ld, s->ctl, s->partials, s->counter);
    return cudaGetLastError();
}

template <typename... KArgs, typename... Args>
cudaError_t ml_launch(bool pdl, void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t stream, Args... args) {
    if (pdl) return launch_pdl(kernel, grid, block, 0, stream, args...);
    kernel<<<grid, block, 0, stream>>>(static_cast<KArgs>(args)...);
    return cudaGetLastError();
}

int ml_vcycle_kernels(const tb_system* s) {
    const int c = (int)s->ml.size();
    return c <= 1 ? 1 : 5 * (c - 1) + 1;
}

// One preconditioner action after the fine pass: the V-cycle over the coarse
// levels (MODE: ML_ITER / ML_START finish r.z at the top, ML_ONLY does not).
template <int NP, int MODE>
cudaError_t ml_vcycle(tb_system* s, bool pdl) {
    const int c = (int)s->ml.size();
    if (c == 1) {
        constexpr int CM = (MODE == ML_ITER) ? COARSE_ITERATE : (MODE == ML_START ? COARSE_START : COARSE_ONLY);
        return launch_coarse_apply<CM>(s, pdl);
    }
    SolveCtl* ctl = (MODE == ML_ONLY) ? nullptr : s->ctl;
    cudaError_t e = cudaSuccess;
    for (int l = 0; l + 1 < c && e == cudaSuccess; ++l) {
        const tb_system::MLLevel& lv = s->ml[l];
        const tb_system::MLLevel& dn = s->ml[l + 1];
        e = ml_launch(pdl, ml_presmooth<NP>, ml_column_grid(lv.g), dim3(kMlThreads), s->stream, (const float*)lv.R,
                      lv.x, (const float*)lv.lf, (const float*)lv.ipd, lv.g, (const SolveCtl*)ctl);
        if (e == cudaSuccess)
            e = ml_launch(pdl, lv.g.b == 4 ? ml_restrict<4> : ml_restrict<2>, ml_node_grid(lv.g), dim3(kMlThreads),
                          s->stream, (const float*)lv.st, (const float*)lv.R, (const float*)lv.x,
                          (const float*)lv.ipd, dn.R, lv.g, dn.g, (const SolveCtl*)ctl);
    }
    if (e == cudaSuccess) e = launch_coarse_apply<COARSE_ONLY>(s, pdl);
    for (int l = c - 2; l >= 0 && e == cudaSuccess; --l) {
        const tb_system::MLLevel& lv = s->ml[l];
        const tb_system::MLLevel& dn = s->ml[l + 1];
        e = ml_launch(pdl, ml_prolong,
                      dim3(ml_cdiv(lv.g.nx, kMlTile), ml_cdiv(lv.g.ny, 8), ml_cdiv(lv.g.L, kMlProlongPlanes)),
                      dim3(kMlThreads), s->stream, lv.x, (const float*)dn.y,
                      (const float*)lv.ipd, lv.g, dn.g, (const SolveCtl*)ctl);
        if (e == cudaSuccess)
            e = ml_launch(pdl, ml_residual, ml_node_grid(lv.g), dim3(kMlThreads), s->stream, (const float*)lv.st,
                          (const float*)lv.R, (const float*)lv.x, lv.y, lv.g, (const SolveCtl*)ctl);
        if (e != cudaSuccess) break;
        if (l == 0)
            e = ml_launch(pdl, ml_zsmooth<NP, MODE, true>, ml_column_grid(lv.g), dim3(kMlThreads), s->stream,
                          (const float*)lv.R, (const float*)lv.x, (const float*)lv.lf, (const float*)lv.ipd, lv.y,
                          lv.g, ctl, s->partials, s->counter);
        else
            e = ml_launch(pdl, ml_zsmooth<NP, MODE, false>, ml_column_grid(lv.g), dim3(kMlThreads), s->stream,
                          (const float*)lv.R, (const float*)lv.x, (const float*)lv.lf, (const float*)lv.ipd, lv.y,
                          lv.g, ctl, s->partials, s->counter);
    }
    return e;
}

// Dynamic shared memory of the staged fine pass: `stages` stages of four
// (S+1) x 8 x 32 boxes, and 128 bytes to align their base.
size_t ml_stage_smem(const Layout& L, int stages) {
    return (size_t)stages * 4 * (L.S + 1) * 8 * kMlTile * sizeof(float) + 128;
}
dim3 ml_stage_tiles(const Layout& L) { return dim3(ml_cdiv(L.Xp, kMlTile), ml_cdiv(L.R + 1, 8)); }

// Tensor maps and stage count of the staged fine pass: as many stages (at
// most kMlMaxStages) as fit beside the kernel's static shared memory, at
// least two; otherwise the form is not available on the board.  The solve
// keeps ml_update unless tb_set_ml_staging selects the staged form: on c3
// (71 M nodes) the staged kernel takes 0.328 ms per launch against 0.347-0.380
// ms (0.80 of the measured copy peak against 0.69-0.76), but the iteration as
// a whole is slower (652.7 against 621.7 ms per solve on one box; 698.5
// against 640.7 on another).  Its 214 KB of shared memory per SM changes the
// L1 / shared-memory split for the kernels that follow it; hinting those
// kernels back to a large L1 recovered part of it (698.5 -> 652.9 ms), and the
// same hints slowed the unstaged iteration (621.7 -> 664.4 ms).
template <int NP>
int ml_stage_setup_np(tb_system* s) {
    const Layout& L = s->lay;
    s->ml_stages = 0;
    s->ml_staged = false;
    const PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
    if (encode == nullptr || L.S + 1 > 256) return TB_OK;
    cudaFuncAttributes fa{};
    TB_CUDA(cudaFuncGetAttributes(&fa, ml_update_staged<NP>));
    int optin = 0;
    TB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, s->device));
    int stages = 0;
    for (int k = kMlMaxStages; k >= 2 && stages == 0; --k)
        if (fa.sharedSizeBytes + ml_stage_smem(L, k) <= (size_t)optin) stages = k;
    if (stages == 0) return TB_OK;
    auto map3 = [&](CUtensorMap* m, const float* base) {
        const cuuint64_t dims[3] = {(cuuint64_t)L.Xp, (cuuint64_t)(L.R + 1), (cuuint64_t)(L.S + 1)};
        const cuuint64_t strides[2] = {(cuuint64_t)L.Xp * sizeof(float), (cuuint64_t)L.Xp * (L.R + 1) * sizeof(float)};
        const cuuint32_t box[3] = {(cuuint32_t)kMlTile, 8u, (cuuint32_t)(L.S + 1)};
        const cuuint32_t estr[3] = {1, 1, 1};
        return encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, estr,
                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    };
    MLStageMaps m{};
    if (!(map3(&m.q, s->q32) && map3(&m.r, s->r32) && map3(&m.zl, s->ml_zl) && map3(&m.zi, s->ml_zi))) return TB_OK;
    m.err = s->stage_err;
    m.test_polls = 0;
    TB_CUDA(cudaFuncSetAttribute(ml_update_staged<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)ml_stage_smem(L, stages)));
    s->ml_maps = m;
    s->ml_stages = stages;
    s->ml_staged = false;
    return TB_OK;
}

int ml_stage_setup(tb_system* s) {
    if (s->ml_np <= 9) return ml_stage_setup_np<9>(s);
    if (s->ml_np <= 17) return ml_stage_setup_np<17>(s);
    return ml_stage_setup_np<33>(s);
}

template <int NP, int MODE>
cudaError_t ml_fine_pass(tb_system* s, bool pdl) {
    if (MODE == ML_ITER && s->ml_staged) {
        const dim3 tg = ml_stage_tiles(s->lay);
        const int tiles = (int)(tg.x * tg.y);
        const int grid = std::max(1, std::min(tiles, std::min(s->sms, s->partial_blocks)));
        const size_t smem = ml_stage_smem(s->lay, s->ml_stages);
        if (pdl)
            return launch_pdl(ml_update_staged<NP>, dim3(grid), dim3(kMlThreads), smem, s->stream, s->r32, s->ml_w,
                              s->ml[0].R, s->lay, s->pstride, s->ml[0].g, s->ctl, s->partials, s->counter,
                              s->clocks + 2, (int)tg.x, tiles, s->ml_stages, s->ml_maps);
        ml_update_staged<NP><<<grid, kMlThreads, smem, s->stream>>>(s->r32, s->ml_w, s->ml[0].R, s->lay, s->pstride,
                                                                     s->ml[0].g, s->ctl, s->partials, s->counter,
                                                                     s->clocks + 2, (int)tg.x, tiles, s->ml_stages,
                                                                     s->ml_maps);
        return cudaGetLastError();
    }
    return ml_launch(pdl, ml_update<NP, MODE>, ml_fine_grid(s->lay), dim3(kMlThreads), s->stream, s->r32,
                     (const float*)s->q32, (const double*)s->r64, s->x32, s->ml_w, s->ml[0].R, (const float*)s->ml_zl,
                     (const float*)s->ml_zi, s->lay, s->pstride, s->ml[0].g, s->ctl, s->partials, s->counter,
                     s->clocks + 2);
}

template <bool START>
cudaError_t ml_launch_direction(tb_system* s, bool pdl, const SolveCtl* ctl) {
    return ml_launch(pdl, ml_direction<START>, dim3(s->vec_blocks), dim3(kVecThreads), s->stream, s->p32, s->x32,
                     (const float*)s->ml_w, (const float*)s->ml[0].y, (const float*)s->ml_zi, s->nq, s->lay,
                     s->ml[0].g, s->special_mask, ctl);
}

// The multilevel part of one PCG iteration (after the operator), of the inner
// start (from r64) or of a bare preconditioner action (r32 -> p32).
template <int NP>
cudaError_t ml_step_np(tb_system* s, int mode, bool pdl) {
    cudaError_t e;
    if (mode == ML_ITER) {
        e = ml_fine_pass<NP, ML_ITER>(s, pdl);
        if (e == cudaSuccess) e = ml_vcycle<NP, ML_ITER>(s, pdl);
        if (e == cudaSuccess) e = ml_launch_direction<false>(s, pdl, s->ctl);
    } else if (mode == ML_START) {
        e = ml_fine_pass<NP, ML_START>(s, pdl);
        if (e == cudaSuccess) e = ml_vcycle<NP, ML_START>(s, pdl);
        if (e == cudaSuccess) e = ml_launch_direction<true>(s, pdl, s->ctl);
    } else {
        e = ml_fine_pass<NP, ML_ONLY>(s, pdl);
        if (e == cudaSuccess) e = ml_vcycle<NP, ML_ONLY>(s, pdl);
        if (e == cudaSuccess) e = ml_launch_direction<true>(s, pdl, nullptr);
    }
    return e;
}

// The multilevel part of an FP64 PCG iteration (after the FP64 operator and
// the norm-only update), or of its start (r64 = b - A x given).
template <int NP>
cudaError_t ml_step64_np(tb_system* s, bool start, bool pdl) {
    const dim3 vg(s->vec_blocks), vb(kVecThreads);
    cudaError_t e;
    if (start) {
        e = ml_fine_pass<NP, ML_START>(s, pdl);
        if (e == cudaSuccess) e = ml_vcycle<NP, ML_START>(s, pdl);
        if (e == cudaSuccess)
            e = ml_launch(pdl, ml_direction_f64<true>, vg, vb, s->stream, s->p64, (const float*)s->ml_w,
                          (const float*)s->ml[0].y, (const float*)s->ml_zi, s->nq, s->lay, s->ml[0].g, s->special_mask,
                          (const SolveCtl*)s->ctl);
        return e;
    }
    e = ml_fine_pass<NP, ML_PRE64>(s, pdl);
    if (e == cudaSuccess) e = ml_vcycle<NP, ML_ITER>(s, pdl);
    if (e == cudaSuccess)
        e = ml_launch(pdl, ml_direction_f64<false>, vg, vb, s->stream, s->p64, (const float*)s->ml_w,
                      (const float*)s->ml[0].y, (const float*)s->ml_zi, s->nq, s->lay, s->ml[0].g, s->special_mask,
                      (const SolveCtl*)s->ctl);
    return e;
}

cudaError_t ml_step64(tb_system* s, bool start, bool pdl) {
    if (s->ml_np <= 9) return ml_step64_np<9>(s, start, pdl);
    if (s->ml_np <= 17) return ml_step64_np<17>(s, start, pdl);
    return ml_step64_np<33>(s, start, pdl);
}

cudaError_t ml_step(tb_system* s, int mode, bool pdl) {
    if (s->ml_np <= 9) return ml_step_np<9>(s, mode, pdl);
    if (s->ml_np <= 17) return ml_step_np<17>(s, mode, pdl);
    return ml_step_np<33>(s, mode, pdl);
}

int ml_kernels_per_step(const tb_system* s) { return 2 + ml_vcycle_kernels(s); }

// Build the hierarchy: fine z-line factors; level 1 by 27 coloured FP64
// operator actions (same-coloured aggregates share no element), each summed
// over the free nodes of every aggregate; deeper levels from the stencil
// above; z-line factors and FP32 stencils per level; the dense inverse of the
// coarsest grid (blocked Gauss-Jordan, pivots checked).
int build_multilevel(tb_system* s) {
    const Layout& L = s->lay;
    if (L.S + 1 > kMlMaxPlanes)
        return fail(TB_EINVAL, "the multilevel preconditioner takes at most %d slabs", kMlMaxPlanes - 1);
    free_coarse(s);
    free_multilevel(s);
    const std::vector<MLGrid> grids = ml_grids(L);
    const int c = (int)grids.size();
    const MLGrid& gc = grids.back();
    if (gc.n > 8192) return fail(TB_EINVAL, "the coarsest multilevel grid has %lld unknowns", gc.n);
    // the fine pass indexes the node vectors, the coarse stencil kernels a
    // level's kMlStencil arrays, with 32-bit integers
    if ((long long)kMlStencil * grids[0].n >= (1LL << 31) || L.L >= (1LL << 31))
        return fail(TB_EINVAL, "the board is too large for the multilevel preconditioner (%lld first-level nodes)",
                    grids[0].n);
    s->ml.resize(c);
    TB_CHECK(alloc_n(s, &s->ml_zl, L.L));
    TB_CHECK(alloc_n(s, &s->ml_zi, L.L));
    TB_CHECK(alloc_n(s, &s->ml_w, L.L));
    TB_CUDA(cudaMemsetAsync(s->ml_w, 0, sizeof(float) * L.L, s->stream));
    CoarseLayout cl{};
    cl.b = kMlAgg;
    cl.layers = gc.L;
    cl.nby = gc.ny;
    cl.nbx = gc.nx;
    cl.nc = (int)gc.n;
    cl.ld = (cl.nc + 3) / 4 * 4;
    const long long nc = cl.nc, nn = nc * nc;
    TB_CHECK(alloc_n(s, &s->coarse_matrix, nn));
    TB_CHECK(alloc_n(s, &s->coarse_inv64, nn));
    TB_CHECK(alloc_n(s, &s->coarse_inv32, nc * cl.ld));
    TB_CHECK(alloc_n(s, &s->coarse_rc, cl.ld));
    TB_CHECK(alloc_n(s, &s->coarse_c, nc));
    TB_CUDA(cudaMemsetAsync(s->coarse_rc, 0, sizeof(float) * cl.ld, s->stream));  // pads stay zero
    std::vector<double*> st64(c, nullptr);
    for (int l = 0; l < c; ++l) {
        tb_system::MLLevel& lv = s->ml[l];
        lv.g = grids[l];
        const long long n = lv.g.n;
        TB_CHECK(alloc_n(s, &st64[l], kMlStencil * n));
        TB_CUDA(cudaMemsetAsync(st64[l], 0, sizeof(double) * kMlStencil * n, s->stream));
        TB_CHECK(alloc_n(s, &lv.x, n));
        if (l + 1 < c) {
            TB_CHECK(alloc_n(s, &lv.st, kMlStencil * n));
            TB_CHECK(alloc_n(s, &lv.lf, n));
            TB_CHECK(alloc_n(s, &lv.ipd, n));
            TB_CHECK(alloc_n(s, &lv.R, n));
            TB_CHECK(alloc_n(s, &lv.y, n));
        } else {
            lv.R = s->coarse_rc;
            lv.y = s->coarse_c;
        }
    }
    double* work = nullptr;
    TB_CHECK(alloc_n(s, &work, nn));
    cudaStream_t st = s->stream;
    int rc = TB_OK;
    auto check_launch = [&]() {
        if (rc == TB_OK && cudaGetLastError() != cudaSuccess) rc = fail(TB_ECUDA, "multilevel set-up launch failed");
    };
    const int sb = s->sms * 16;
    {
        const long long ncol = (long long)(L.R + 1) * L.Xp;
        ml_fine_factors<<<grid_for(ncol, 128, sb), 128, 0, st>>>(s->ml_zl, s->ml_zi, s->diag64, s->rf64, s->kin64,
                                                                s->kz64, s->dims64, s->dims64 + L.S,
                                                                s->dims64 + L.S + L.C, L, s->pstride);
        s->kernel_launches += 1;
        check_launch();
    }
    CoarseLayout c1{};
    c1.b = kMlAgg;
    c1.layers = grids[0].L;
    c1.nby = grids[0].ny;
    c1.nbx = grids[0].nx;
    const int nb = grid_for(L.L, kVecThreads, sb);
    for (int colour = 0; colour < 27 && rc == TB_OK; ++colour) {
        coarse_indicator<<<nb, kVecThreads, 0, st>>>(s->b64, s->rf64, L, c1, colour);
        check_launch();
        if (rc != TB_OK) break;
        const ApplyParams<double> P = apply_params<double>(s, s->b64, s->r64, nullptr);
        rc = launch_apply<double, MODE_OPERATOR, EPI_STORE>(s, P);
        if (rc != TB_OK) break;
        ml_galerkin_gather<<<grid_for(grids[0].n, kVecThreads, sb), kVecThreads, 0, st>>>(st64[0], s->r64, s->rf64, L,
                                                                                         s->pstride, grids[0], colour);
        s->kernel_launches += 3;
        check_launch();
    }
    if (rc == TB_OK) {
        ml_mark_empty<<<grid_for(grids[0].n, kVecThreads, sb), kVecThreads, 0, st>>>(st64[0], grids[0].n);
        for (int l = 0; l + 1 < c; ++l)
            ml_coarsen<<<grid_for(grids[l + 1].n, 128, sb), 128, 0, st>>>(st64[l + 1], st64[l], grids[l],
                                                                          grids[l + 1]);
        for (int l = 0; l + 1 < c; ++l) {
            tb_system::MLLevel& lv = s->ml[l];
            ml_level_factors<<<grid_for(lv.g.plane, 128, sb), 128, 0, st>>>(lv.st, lv.lf, lv.ipd, st64[l], lv.g);
        }
        cudaMemsetAsync(s->coarse_matrix, 0, sizeof(double) * nn, st);
        ml_dense<<<grid_for(nc, 128, sb), 128, 0, st>>>(s->coarse_matrix, st64[c - 1], gc);
        cudaMemcpyAsync(work, s->coarse_matrix, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st);
        cudaMemsetAsync(s->d_err, 0, sizeof(int), st);
        s->kernel_launches += 2 + 2 * (c - 1);
        check_launch();
    }
    if (rc == TB_OK && gauss_jordan_invert(work, cl.nc, s->d_err, st) != cudaSuccess)
        rc = fail(TB_ECUDA, "coarse inversion launch failed");
    if (rc == TB_OK) {
        const int mb = grid_for(nn, kVecThreads, sb);
        coarse_symmetrize<<<mb, kVecThreads, 0, st>>>(work, s->coarse_inv64, s->coarse_inv32, cl.nc, cl.ld);
        s->kernel_launches += 1 + 4LL * ml_cdiv(cl.nc, kGjB);
        check_launch();
    }
    int err = 0;
    if (rc == TB_OK) {
        if (cudaMemcpyAsync(&err, s->d_err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            rc = fail(TB_ECUDA, "multilevel set-up failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    cudaStreamSynchronize(st);
    dev_free(s, work);
    for (double*& p : st64) dev_free(s, p);
    if (rc != TB_OK) return rc;
    if (err)
        return fail(TB_EINVAL,
                    "the coarsest operator is not positive definite; the fine operator must be SPD for the multilevel "
                    "preconditioner");
    s->cl = cl;
    const int planes = L.S + 1;
    s->ml_np = planes <= 9 ? 9 : (planes <= 17 ? 17 : 33);
    {
        const dim3 fg = ml_fine_grid(L), tg = ml_column_grid(grids[0]);
        TB_CHECK(ensure_partials(s, std::max((int)(fg.x * fg.y), (int)tg.x)));
    }
    TB_CHECK(ml_stage_setup(s));
    return keep_coarse_in_l2(s);
}
