// Batch / serving engine: many boards resident in HBM, solved together by the
// batched kernels of tb_batch.cuh, admitted and collected while others run.
//
// Included at the end of tb_system.cu (it shares its helpers).  One engine owns
//   - a compute stream that runs the graph chunks and every write to the
//     device table and schedule, so those writes are ordered with the chunks;
//   - an I/O stream for uploads, board preparation and downloads, which
//     overlap the chunks;
//   - a CUDA memory pool that keeps freed board memory for the next board, so
//     serving does no device allocation once warm;
//   - the admission budget: a board is admitted when its bytes fit.
// A graph chunk is the three outer-step kernels followed by kChunk PCG
// iterations (apply, update, direction) over the whole schedule; it is
// captured once and replayed, the schedule lives in device memory.

namespace {

constexpr int kEngineDepth = 2;  // graph chunks in flight

struct EngineBoard {
    long long ticket = 0;
    int slot = -1;
    Layout lay{};
    long long pstride = 0, sstride = 0, nq = 0;
    size_t bytes = 0;  // resident bytes (one pool allocation)
    void* block = nullptr;
    BatchInstance inst{};
    int tiles32[3] = {0, 0, 0};  // per FP32 tile height 8, 16, 32
    int gx32 = 0;
    int max_outer = 0;
    CoarseLayout cl{};  // nc = 0 without the two-level preconditioner
    bool reported = false;  // the host has seen it leave the loop
    ApplyMaps maps[3]{};    // host copy of its tensor maps (tile heights 8, 16, 32)
};

}  // namespace

struct tb_engine {
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;  // compute
    cudaStream_t io = nullptr;
    cudaMemPool_t pool = nullptr;
    cudaEvent_t io_done = nullptr;
    int capacity = 0, max_slabs = 0, rows32 = 0;
    int tma32 = 0;          // batched FP32 operator stages filled by tensor copies
    int staging = 0;        // requested staging: 0 timed (with the tile height), 1 cp.async, 2 tensor copies
    bool tma_ok = false;    // the tensor-map encoder is available
    ApplyMaps* d_maps = nullptr;  // 3 per slot
    int* d_stage_err = nullptr;   // set by an operator block that gave up waiting for its tiles
    int precond = 0;   // 0 Jacobi, 1 two-level for every board
    int max_nc = 0;    // largest coarse grid admitted (shared memory of batch_coarse)
    static constexpr int rows64 = 8;
    int grid32 = 0, grid64 = 0, gridv = 0, gridr = 0, gridc = 0;
    size_t smem32 = 0, smem64 = 0;
    long long budget = 0, in_use = 0;
    BatchInstance* d_table = nullptr;
    SolveCtl* d_ctl = nullptr;
    BatchOuter* d_outer = nullptr;
    BatchStatus* d_status = nullptr;
    BatchSchedule* d_sched = nullptr;
    unsigned int* d_counters = nullptr;  // 4 per slot
    BatchStatus* h_status = nullptr;     // pinned, kEngineDepth snapshots
    cudaEvent_t ev[kEngineDepth] = {nullptr, nullptr};
    int inflight = 0, head = 0;
    cudaGraphExec_t chunk = nullptr;
    std::vector<EngineBoard*> slots;
    std::map<long long, EngineBoard*> boards;
    std::vector<long long> finished;
    long long next_ticket = 1;
    int active = 0;  // boards in the schedule (resident and not yet seen finished)
    bool dirty = true;
    long long chunks = 0, kernel_launches = 0;
};

namespace {

int row_index(int rows) { return rows == 8 ? 0 : (rows == 16 ? 1 : 2); }

template <int ROWS, bool TMA>
int engine_grid_rows(tb_engine* e, size_t smem, int* per_sm) {
    TB_CUDA(cudaFuncSetAttribute(batch_apply32<ROWS, TMA>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    TB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, batch_apply32<ROWS, TMA>, 16 * ROWS, smem));
    return TB_OK;
}

size_t engine_smem32(int rows, int S) {
    if (rows == 8) return apply_smem_bytes<float, 8>(S);
    if (rows == 16) return apply_smem_bytes<float, 16>(S);
    return apply_smem_bytes<float, 32>(S);
}

int engine_grid32(tb_engine* e) {
    int per_sm = 0;
    const int rows = e->rows32;
    const size_t smem = engine_smem32(rows, e->max_slabs);
    const bool tma = e->tma32 != 0;
    int rc;
    if (rows == 8) rc = tma ? engine_grid_rows<8, true>(e, smem, &per_sm) : engine_grid_rows<8, false>(e, smem, &per_sm);
    else if (rows == 16)
        rc = tma ? engine_grid_rows<16, true>(e, smem, &per_sm) : engine_grid_rows<16, false>(e, smem, &per_sm);
    else rc = tma ? engine_grid_rows<32, true>(e, smem, &per_sm) : engine_grid_rows<32, false>(e, smem, &per_sm);
    TB_CHECK(rc);
    if (per_sm < 1) return fail(TB_EINVAL, "the %d-row batched operator does not fit an SM for %d slabs", rows, e->max_slabs);
    e->smem32 = smem;
    e->grid32 = per_sm * e->sms;
    return TB_OK;
}

int engine_launch_apply32(tb_engine* e) {
    const dim3 grid(e->grid32), block(16 * e->rows32);
    const size_t sm = e->smem32;
    if (e->tma32) {
        if (e->rows32 == 8) batch_apply32<8, true><<<grid, block, sm, e->stream>>>(e->d_table, e->d_sched);
        else if (e->rows32 == 16) batch_apply32<16, true><<<grid, block, sm, e->stream>>>(e->d_table, e->d_sched);
        else batch_apply32<32, true><<<grid, block, sm, e->stream>>>(e->d_table, e->d_sched);
    } else {
        if (e->rows32 == 8) batch_apply32<8><<<grid, block, sm, e->stream>>>(e->d_table, e->d_sched);
        else if (e->rows32 == 16) batch_apply32<16><<<grid, block, sm, e->stream>>>(e->d_table, e->d_sched);
        else batch_apply32<32><<<grid, block, sm, e->stream>>>(e->d_table, e->d_sched);
    }
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ECUDA;
}

int engine_capture(tb_engine* e) {
    if (e->chunk) cudaGraphExecDestroy(e->chunk);
    e->chunk = nullptr;
    cudaGraph_t graph = nullptr;
    TB_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    int rc = TB_OK;
    batch_outer_finish<<<e->gridv, kVecThreads, 0, e->stream>>>(e->d_table, e->d_sched);
    batch_residual64<tb_engine::rows64><<<e->grid64, 16 * tb_engine::rows64, e->smem64, e->stream>>>(e->d_table,
                                                                                                   e->d_sched);
    batch_inner_start<<<e->gridv, kVecThreads, 0, e->stream>>>(e->d_table, e->d_sched);
    if (cudaGetLastError() != cudaSuccess) rc = TB_ECUDA;
    for (int i = 0; i < kChunk && rc == TB_OK; ++i) {
        rc = engine_launch_apply32(e);
        if (rc != TB_OK) break;
        batch_update32<<<e->gridv, kVecThreads, 0, e->stream>>>(e->d_table, e->d_sched);
        if (e->precond) {
            batch_restrict<<<e->gridr, 256, 0, e->stream>>>(e->d_table, e->d_sched);
            batch_coarse<<<e->gridc, 256, sizeof(float) * 2048, e->stream>>>(e->d_table, e->d_sched);
        }
        batch_direction32<<<e->gridv, kVecThreads, 0, e->stream>>>(e->d_table, e->d_sched);
        if (cudaGetLastError() != cudaSuccess) rc = TB_ECUDA;
    }
    const cudaError_t end = cudaStreamEndCapture(e->stream, &graph);
    if (rc != TB_OK || end != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return fail(TB_ECUDA, "capturing the batch chunk failed");
    }
    const cudaError_t inst = cudaGraphInstantiate(&e->chunk, graph, 0);
    cudaGraphDestroy(graph);
    if (inst != cudaSuccess) return fail(TB_ECUDA, "batch graph instantiation failed: %s", cudaGetErrorString(inst));
    return TB_OK;
}

int engine_kernels_per_chunk(const tb_engine* e) { return 3 + (e->precond ? 5 : 3) * kChunk; }

void engine_free(tb_engine* e) {
    if (!e) return;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    if (e->io) cudaStreamSynchronize(e->io);
    for (auto& kv : e->boards) {
        if (kv.second->block) cudaFreeAsync(kv.second->block, e->stream);
        delete kv.second;
    }
    e->boards.clear();
    if (e->stream) cudaStreamSynchronize(e->stream);
    if (e->chunk) cudaGraphExecDestroy(e->chunk);
    for (void* p : {(void*)e->d_table, (void*)e->d_ctl, (void*)e->d_outer, (void*)e->d_status, (void*)e->d_sched,
                    (void*)e->d_counters, (void*)e->d_maps, (void*)e->d_stage_err})
        if (p) cudaFree(p);
    if (e->h_status) cudaFreeHost(e->h_status);
    for (cudaEvent_t ev : e->ev)
        if (ev) cudaEventDestroy(ev);
    if (e->io_done) cudaEventDestroy(e->io_done);
    if (e->pool) cudaMemPoolDestroy(e->pool);
    if (e->io) cudaStreamDestroy(e->io);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

int engine_create(int device, const tb_engine_config* c, tb_engine** out) {
    if (!c) return fail(TB_EINVAL, "engine config is NULL");
    if (c->capacity < 1 || c->capacity > kBatchMax) return fail(TB_EINVAL, "capacity must be in [1, %d]", kBatchMax);
    if (c->max_slabs < 1 || c->max_slabs > 256) return fail(TB_EINVAL, "max_slabs must be in [1, 256]");
    if (c->tile_rows != 0 && c->tile_rows != 8 && c->tile_rows != 16 && c->tile_rows != 32)
        return fail(TB_EINVAL, "tile_rows must be 0 (autotune), 8, 16 or 32");
    if (c->budget_bytes <= 0) return fail(TB_EINVAL, "budget_bytes must be positive");
    if (c->preconditioner != 0 && c->preconditioner != 1)
        return fail(TB_EINVAL, "preconditioner must be 0 (Jacobi) or 1 (two-level)");
    if (c->staging < 0 || c->staging > 2) return fail(TB_EINVAL, "staging must be 0 (timed), 1 (cp.async) or 2 (TMA)");
    int count = 0;
    TB_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) return fail(TB_EINVAL, "CUDA device %d is outside [0, %d)", device, count);
    TB_CUDA(cudaSetDevice(device));
    tb_engine* e = new tb_engine();
    *out = e;
    e->device = device;
    e->capacity = c->capacity;
    e->max_slabs = c->max_slabs;
    e->rows32 = c->tile_rows;
    e->budget = c->budget_bytes;
    e->precond = c->preconditioner;
    e->slots.assign(e->capacity, nullptr);
    cudaDeviceGetAttribute(&e->sms, cudaDevAttrMultiProcessorCount, device);
    TB_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    TB_CUDA(cudaStreamCreateWithFlags(&e->io, cudaStreamNonBlocking));
    TB_CUDA(cudaEventCreateWithFlags(&e->io_done, cudaEventDisableTiming));
    for (cudaEvent_t& ev : e->ev) TB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        TB_CUDA(cudaMemPoolCreate(&e->pool, &props));
        unsigned long long keep = ~0ULL;  // freed board memory stays in the pool
        TB_CUDA(cudaMemPoolSetAttribute(e->pool, cudaMemPoolAttrReleaseThreshold, &keep));
    }
    const int cap = e->capacity;
    TB_CUDA(cudaMalloc(&e->d_table, sizeof(BatchInstance) * cap));
    TB_CUDA(cudaMalloc(&e->d_ctl, sizeof(SolveCtl) * cap));
    TB_CUDA(cudaMalloc(&e->d_outer, sizeof(BatchOuter) * cap));
    TB_CUDA(cudaMalloc(&e->d_status, sizeof(BatchStatus) * cap));
    TB_CUDA(cudaMalloc(&e->d_sched, sizeof(BatchSchedule)));
    TB_CUDA(cudaMalloc(&e->d_counters, sizeof(unsigned int) * 4 * cap));
    TB_CUDA(cudaMemsetAsync(e->d_table, 0, sizeof(BatchInstance) * cap, e->stream));
    TB_CUDA(cudaMemsetAsync(e->d_ctl, 0, sizeof(SolveCtl) * cap, e->stream));
    TB_CUDA(cudaMemsetAsync(e->d_outer, 0, sizeof(BatchOuter) * cap, e->stream));
    TB_CUDA(cudaMemsetAsync(e->d_status, 0, sizeof(BatchStatus) * cap, e->stream));
    TB_CUDA(cudaMemsetAsync(e->d_sched, 0, sizeof(BatchSchedule), e->stream));
    TB_CUDA(cudaMemsetAsync(e->d_counters, 0, sizeof(unsigned int) * 4 * cap, e->stream));
    TB_CUDA(cudaMalloc(&e->d_maps, sizeof(ApplyMaps) * 3 * cap));
    TB_CUDA(cudaMalloc(&e->d_stage_err, sizeof(int)));
    TB_CUDA(cudaMemsetAsync(e->d_stage_err, 0, sizeof(int), e->stream));
    e->tma_ok = tensor_map_encoder() != nullptr;
    e->staging = c->staging;
    if (e->staging == 2 && !e->tma_ok) return fail(TB_ENOTSUP, "tensor-copy staging is not available");
    e->tma32 = e->staging == 2 ? 1 : 0;
    {
        void* h = nullptr;
        TB_CUDA(cudaMallocHost(&h, sizeof(BatchStatus) * cap * kEngineDepth));
        e->h_status = static_cast<BatchStatus*>(h);
        std::memset(h, 0, sizeof(BatchStatus) * cap * kEngineDepth);
    }
    // FP64 residual and vector kernels: fixed shapes.
    e->smem64 = apply_smem_bytes<double, tb_engine::rows64>(e->max_slabs);
    TB_CUDA(cudaFuncSetAttribute(batch_residual64<tb_engine::rows64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)e->smem64));
    int per_sm = 0;
    TB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_residual64<tb_engine::rows64>,
                                                          16 * tb_engine::rows64, e->smem64));
    if (per_sm < 1) return fail(TB_EINVAL, "the batched FP64 residual does not fit an SM for %d slabs", e->max_slabs);
    e->grid64 = per_sm * e->sms;
    e->gridv = 8 * e->sms;
    e->gridr = 8 * e->sms;  // 8 warps per block, one patch per warp
    e->gridc = 8 * e->sms;
    TB_CHECK(set_smem_attributes(device, e->max_slabs));  // the FP64 actions of the coarse set-up
    if (e->rows32 != 0) {
        TB_CHECK(engine_grid32(e));
        TB_CHECK(engine_capture(e));
    }
    TB_CUDA(cudaStreamSynchronize(e->stream));
    return TB_OK;
}

// Bytes one board holds while resident, and the transient bytes of its
// preparation (input staging, FP64 diagonal, the coarse matrix and its
// Gauss-Jordan workspace); nc = 0 without the two-level preconditioner.
void board_bytes(const Layout& L, int max_items, int nc, size_t* resident, size_t* transient) {
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t nn = (size_t)nc * nc;
    const size_t ld = (size_t)(nc + 3) / 4 * 4;
    const size_t geo = (size_t)(2 * L.S + 2 * L.C + 2 * L.R);
    size_t r = 0;
    r += 2 * al(4 * (size_t)L.LE) + 2 * al(8 * (size_t)L.LE);  // kin, kz in FP32 and FP64
    r += 6 * al(4 * (size_t)L.L);                               // rf32 dinv32 x32 r32 p32 q32
    r += 4 * al(8 * (size_t)L.L);                               // rf64 b64 x64 r64
    r += al(4 * geo) + al(8 * geo) + al(4 * (size_t)(L.S + 1));
    r += al(32 * (size_t)max_items);                            // partials
    if (nc > 0) r += al(4 * nc * ld) + 2 * al(4 * ld);        // Minv (FP32, padded rows), R, c
    *resident = r;
    *transient = al(8 * (size_t)L.E) * 2 + al(8 * (size_t)L.N) * 3 + al((size_t)L.N) + al(8 * geo) +
                 al(8 * (size_t)L.L) * 2 + 512;
    if (nc > 0) *transient += 2 * al(8 * nn) + al(32 * (size_t)nc);
}

Layout layout_of(const tb_system_desc* d) {
    Layout L{};
    L.S = d->slabs;
    L.R = d->rows;
    L.C = d->cols;
    L.Xp = (int)round_up(L.C + 1, 4);
    L.Xe = (int)round_up(L.C, 4);
    L.N = (long long)(L.S + 1) * (L.R + 1) * (L.C + 1);
    L.L = (long long)(L.S + 1) * (L.R + 1) * L.Xp;
    L.E = (long long)L.S * L.R * L.C;
    L.LE = (long long)L.S * L.R * L.Xe;
    return L;
}

int board_items(const Layout& L, int nc, int* tiles32, int* gx32, int* tiles64, int* gx64, int* chunks) {
    *gx32 = apply_grid_x(L.C);
    tiles32[0] = *gx32 * apply_grid_y(8, L.R);
    tiles32[1] = *gx32 * apply_grid_y(16, L.R);
    tiles32[2] = *gx32 * apply_grid_y(32, L.R);
    *gx64 = apply_grid_x(L.C);
    *tiles64 = *gx64 * apply_grid_y(tb_engine::rows64, L.R);
    *chunks = (int)((L.L / 4 + kBatchChunkQuads - 1) / kBatchChunkQuads);
    const int coarse_items = (nc + kCoarseRows - 1) / kCoarseRows;
    return std::max(std::max(std::max(tiles32[0], *tiles64), *chunks), coarse_items);
}

template <typename T>
T* carve(char*& cursor, size_t count) {
    T* p = reinterpret_cast<T*>(cursor);
    cursor += (sizeof(T) * count + 255) / 256 * 256;
    return p;
}

int engine_build_schedule(tb_engine* e) {
    BatchSchedule s{};
    const int ri = row_index(e->rows32 == 0 ? 16 : e->rows32);
    s.tile32[0] = s.tile64[0] = s.chunk[0] = s.patch[0] = s.crow[0] = 0;
    // Boards with the most slabs first: their operator tiles cost the most, and
    // the operator hands tiles out in schedule order.
    std::vector<int> order;
    for (int slot = 0; slot < e->capacity; ++slot)
        if (e->slots[slot] && !e->slots[slot]->reported) order.push_back(slot);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return e->slots[a]->lay.S > e->slots[b]->lay.S; });
    int n = 0;
    for (const int slot : order) {
        const EngineBoard* b = e->slots[slot];
        s.slot[n] = slot;
        s.tile32[n + 1] = s.tile32[n] + b->tiles32[ri];
        s.tile64[n + 1] = s.tile64[n] + b->inst.tiles64;
        s.chunk[n + 1] = s.chunk[n] + b->inst.chunks;
        s.patch[n + 1] = s.patch[n] + b->cl.nc;
        s.crow[n + 1] = s.crow[n] + b->inst.coarse_items;
        ++n;
    }
    s.n = n;
    e->active = n;
    batch_set_schedule<<<1, 256, 0, e->stream>>>(s, e->d_sched);
    TB_CUDA(cudaGetLastError());
    e->kernel_launches += 1;
    e->dirty = false;
    return TB_OK;
}

// Rewrite the FP32 tile counts of every resident board for the current tile height.
__global__ void batch_set_tiles(BatchInstance* table, int slot, int gx, int tiles) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        table[slot].gx32 = gx;
        table[slot].tiles32 = tiles;
    }
}

int engine_apply_rows(tb_engine* e) {
    const int ri = row_index(e->rows32);
    for (EngineBoard* b : e->slots) {
        if (!b) continue;
        b->inst.gx32 = b->gx32;
        b->inst.tiles32 = b->tiles32[ri];
        batch_set_tiles<<<1, 32, 0, e->stream>>>(e->d_table, b->slot, b->gx32, b->tiles32[ri]);
        TB_CUDA(cudaGetLastError());
        e->kernel_launches += 1;
    }
    e->dirty = true;
    return TB_OK;
}

// Batched FP32 operator with the store epilogue over every resident board, for timing.
template <int ROWS, bool TMA>
__global__ void __launch_bounds__(16 * ROWS, ApplyOccupancy<float, ROWS>::min_blocks)
    batch_apply32_store(const BatchInstance* __restrict__ table, const BatchSchedule* __restrict__ sched) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ ItemMap m;
    __shared__ __align__(16) unsigned char p_raw[sizeof(ApplyParams<float>)];
    ApplyParams<float>* const sP = reinterpret_cast<ApplyParams<float>*>(p_raw);
    load_items<ITEMS_TILE32>(sched, m);
    const int total = m.prefix[m.n];
    int seq = 0;
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int k = find_board(m, t);
        const BatchInstance* I = table + m.slot[k];
        copy_params(sP, &I->a32);
        __syncthreads();
        const int lt = t - m.prefix[k];
        float dot = 0.f;
        double rmax = 0.0;
        if (apply_tile<float, MODE_OPERATOR, EPI_STORE, ROWS, TMA>(*sP, lt % I->gx32, lt / I->gx32, smem_raw, dot, rmax,
                                                                  false, 0, 1 << 30,
                                                                  TMA ? I->maps + maps_index(ROWS) : nullptr,
                                                                  &seq, true) == TILE_ABORTED)
            break;
    }
}

template <int ROWS, bool TMA>
int engine_time_rows(tb_engine* e, float* ms, int reps = 5) {
    const size_t smem = engine_smem32(ROWS, e->max_slabs);
    TB_CUDA(cudaFuncSetAttribute(batch_apply32_store<ROWS, TMA>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    int per_sm = 0;
    TB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_apply32_store<ROWS, TMA>, 16 * ROWS, smem));
    if (per_sm < 1) {
        *ms = 1e30f;
        return TB_OK;
    }
    cudaEvent_t t0, t1;
    TB_CUDA(cudaEventCreate(&t0));
    TB_CUDA(cudaEventCreate(&t1));
    const dim3 grid(per_sm * e->sms), block(16 * ROWS);
    batch_apply32_store<ROWS, TMA><<<grid, block, smem, e->stream>>>(e->d_table, e->d_sched);  // warm-up
    TB_CUDA(cudaEventRecord(t0, e->stream));
    for (int i = 0; i < reps; ++i)
        batch_apply32_store<ROWS, TMA><<<grid, block, smem, e->stream>>>(e->d_table, e->d_sched);
    TB_CUDA(cudaEventRecord(t1, e->stream));
    TB_CUDA(cudaGetLastError());
    TB_CUDA(cudaEventSynchronize(t1));
    TB_CUDA(cudaEventElapsedTime(ms, t0, t1));
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    e->kernel_launches += 1 + reps;
    return TB_OK;
}

// A block of the tensor-copy staging gave up waiting for its tiles.
int engine_check_stage(tb_engine* e) {
    int err = 0;
    TB_CUDA(cudaMemcpyAsync(&err, e->d_stage_err, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
    TB_CUDA(cudaStreamSynchronize(e->stream));
    if (err != 0) return fail(TB_ETIMEOUT, "a batched operator block gave up waiting for its staged tiles");
    return TB_OK;
}

int engine_time_current(tb_engine* e, float* ms, int reps = 5) {
    if (e->tma32) {
        if (e->rows32 == 8) return engine_time_rows<8, true>(e, ms, reps);
        if (e->rows32 == 16) return engine_time_rows<16, true>(e, ms, reps);
        return engine_time_rows<32, true>(e, ms, reps);
    }
    if (e->rows32 == 8) return engine_time_rows<8, false>(e, ms, reps);
    if (e->rows32 == 16) return engine_time_rows<16, false>(e, ms, reps);
    return engine_time_rows<32, false>(e, ms, reps);
}

// Tile height and staging of the batched FP32 operator: time each height,
// with cp.async and (where the encoder is available) tensor-copy staging,
// over the resident boards (store epilogue, which only writes the dead q
// vector) and keep the fastest.  Runs once, before the first chunk.
int engine_autotune(tb_engine* e) {
    const int heights[3] = {8, 16, 32};
    float best_ms = 0.f;
    int best = 16, best_tma = 0;
    bool first = true;
    for (int i = 0; i < 3; ++i) {
        e->rows32 = heights[i];
        TB_CHECK(engine_apply_rows(e));
        TB_CHECK(engine_build_schedule(e));
        const int tma_lo = e->staging == 2 ? 1 : 0, tma_hi = (e->staging == 0 && e->tma_ok) || e->staging == 2 ? 1 : 0;
        for (int tma = tma_lo; tma <= tma_hi; ++tma) {
            e->tma32 = tma;
            float ms = 0.f;
            TB_CHECK(engine_time_current(e, &ms));
            if (first || ms < best_ms) {
                best_ms = ms;
                best = heights[i];
                best_tma = tma;
                first = false;
            }
        }
    }
    e->tma32 = best_tma;
    TB_CHECK(engine_check_stage(e));
    e->rows32 = best;
    TB_CHECK(engine_apply_rows(e));
    TB_CHECK(engine_grid32(e));
    TB_CHECK(engine_capture(e));
    return TB_OK;
}

int engine_submit(tb_engine* e, const tb_system_desc* d, const double* rhs, const double* x0,
                  const tb_mpir_config* cfg, long long* ticket) {
    TB_CHECK(check_desc(d));
    if (!rhs || !cfg || !ticket) return fail(TB_EINVAL, "NULL argument");
    if (!(cfg->relative_tolerance >= 0.0) || !(cfg->absolute_tolerance >= 0.0) ||
        !(cfg->inner_relative_tolerance > 0.0 && cfg->inner_relative_tolerance < 1.0) ||
        cfg->max_outer_iterations < 1 || cfg->max_inner_iterations < 1)
        return fail(TB_EINVAL, "invalid MPIR configuration");
    if (d->slabs > e->max_slabs) return fail(TB_EINVAL, "board has %d slabs; the engine admits at most %d", d->slabs, e->max_slabs);
    const Layout L = layout_of(d);
    if (L.L / 4 > (long long)INT32_MAX * kBatchChunkQuads / 2) return fail(TB_EINVAL, "board too large for the engine");
    int slot = -1;
    for (int i = 0; i < e->capacity; ++i)
        if (!e->slots[i]) {
            slot = i;
            break;
        }
    if (slot < 0) return fail(TB_ENOMEM, "every engine slot is taken");
    EngineBoard tmp;
    if (e->precond) tmp.cl = coarse_layout(L, 0);
    const int nc = tmp.cl.nc;
    int tiles64 = 0, gx64 = 0, chunks = 0, gx32 = 0;
    const int max_items = board_items(L, nc, tmp.tiles32, &gx32, &tiles64, &gx64, &chunks);
    size_t resident = 0, transient = 0;
    board_bytes(L, max_items, nc, &resident, &transient);
    if (e->in_use + (long long)(resident + transient) > e->budget)
        return fail(TB_ENOMEM, "board needs %zu bytes; %lld of %lld are in use", resident + transient, e->in_use, e->budget);
    double bn2 = 0.0;
    {
        double acc[4] = {0, 0, 0, 0};
        long long n = 0;
        for (; n + 4 <= L.N; n += 4)
            for (int k = 0; k < 4; ++k) acc[k] += rhs[n + k] * rhs[n + k];
        for (; n < L.N; ++n) acc[0] += rhs[n] * rhs[n];
        bn2 = (acc[0] + acc[1]) + (acc[2] + acc[3]);
    }
    const double bnorm = std::sqrt(bn2);
    if (!std::isfinite(bnorm)) return fail(TB_ENONFINITE, "rhs must contain only finite values");

    EngineBoard* b = new EngineBoard(tmp);
    b->lay = L;
    b->slot = slot;
    b->pstride = (long long)(L.R + 1) * L.Xp;
    b->sstride = (long long)L.R * L.Xe;
    b->nq = L.L / 4;
    b->bytes = resident;
    b->gx32 = gx32;
    b->max_outer = cfg->max_outer_iterations;
    void* stage = nullptr;
    void* coarse_work = nullptr;
    auto cleanup = [&](int code) {
        if (coarse_work) cudaFreeAsync(coarse_work, e->io);
        if (stage) cudaFreeAsync(stage, e->io);
        if (b->block) cudaFreeAsync(b->block, e->io);
        cudaStreamSynchronize(e->io);
        delete b;
        return code;
    };
#define TB_ENGINE_CUDA(call)                                                                              \
    do {                                                                                                  \
        const cudaError_t err_ = (call);                                                                  \
        if (err_ != cudaSuccess) {                                                                        \
            fail(err_ == cudaErrorMemoryAllocation ? TB_ENOMEM : TB_ECUDA, "%s failed: %s", #call,       \
                 cudaGetErrorString(err_));                                                               \
            return cleanup(err_ == cudaErrorMemoryAllocation ? TB_ENOMEM : TB_ECUDA);                     \
        }                                                                                                 \
    } while (0)
    TB_ENGINE_CUDA(cudaMallocFromPoolAsync(&b->block, resident, e->pool, e->io));
    const size_t coarse_bytes = nc > 0 ? sizeof(double) * (2 * (size_t)nc * nc + 4 * (size_t)nc) : 0;
    TB_ENGINE_CUDA(cudaMallocFromPoolAsync(&stage, transient - coarse_bytes, e->pool, e->io));
    TB_ENGINE_CUDA(cudaMemsetAsync(b->block, 0, resident, e->io));
    const long long geo = 2LL * L.S + 2LL * L.C + 2LL * L.R;
    char* cur = static_cast<char*>(b->block);
    float* kin32 = carve<float>(cur, L.LE);
    float* kz32 = carve<float>(cur, L.LE);
    double* kin64 = carve<double>(cur, L.LE);
    double* kz64 = carve<double>(cur, L.LE);
    float* rf32 = carve<float>(cur, L.L);
    float* dinv32 = carve<float>(cur, L.L);
    float* x32 = carve<float>(cur, L.L);
    float* r32 = carve<float>(cur, L.L);
    float* p32 = carve<float>(cur, L.L);
    float* q32 = carve<float>(cur, L.L);
    double* rf64 = carve<double>(cur, L.L);
    double* b64 = carve<double>(cur, L.L);
    double* x64 = carve<double>(cur, L.L);
    double* r64 = carve<double>(cur, L.L);
    float* geo32 = carve<float>(cur, geo);
    double* geo64 = carve<double>(cur, geo);
    int* flags = carve<int>(cur, L.S + 1);
    double* partials = carve<double>(cur, 4 * (size_t)max_items);
    float* minv32 = nc > 0 ? carve<float>(cur, (size_t)nc * tmp.cl.ld) : nullptr;
    float* rc = nc > 0 ? carve<float>(cur, tmp.cl.ld) : nullptr;  // pads stay zero (block cleared)
    float* cvec = nc > 0 ? carve<float>(cur, tmp.cl.ld) : nullptr;

    // Device table entry.
    BatchInstance& I = b->inst;
    auto fill = [&](auto& P, auto* x, auto* y, const auto* bb, const auto* kin, const auto* kz, const auto* rf,
                    const auto* g) {
        P.x = x;
        P.y = y;
        P.b = bb;
        P.kin = kin;
        P.kz = kz;
        P.rf = rf;
        P.plane_flags = flags;
        P.gzt = g;
        P.gzi = g + L.S;
        P.hx = g + 2 * L.S;
        P.ihx = g + 2 * L.S + L.C;
        P.hy = g + 2 * L.S + 2 * L.C;
        P.ihy = g + 2 * L.S + 2 * L.C + L.R;
        P.partials = nullptr;
        P.counter = nullptr;
        P.ctl = e->d_ctl + slot;
        P.clock = nullptr;
        P.S = L.S;
        P.R = L.R;
        P.C = L.C;
        P.Xp = L.Xp;
        P.Xe = L.Xe;
        P.pstride = b->pstride;
        P.sstride = b->sstride;
    };
    fill(I.a32, (const float*)p32, q32, (const float*)nullptr, (const float*)kin32, (const float*)kz32,
         (const float*)rf32, (const float*)geo32);
    fill(I.a64, (const double*)x64, r64, (const double*)b64, (const double*)kin64, (const double*)kz64,
         (const double*)rf64, (const double*)geo64);
    I.x32 = x32;
    I.r32 = r32;
    I.p32 = p32;
    I.q32 = q32;
    I.dinv32 = dinv32;
    I.x64 = x64;
    I.r64 = r64;
    I.partials = partials;
    I.counter = e->d_counters + 4 * slot;
    I.ctl = e->d_ctl + slot;
    I.outer = e->d_outer + slot;
    I.status = e->d_status + slot;
    I.nq = b->nq;
    I.gx32 = gx32;
    I.tiles32 = b->tiles32[row_index(e->rows32 == 0 ? 16 : e->rows32)];
    I.gx64 = gx64;
    I.tiles64 = tiles64;
    I.chunks = chunks;
    I.cl = b->cl;
    I.twolevel = nc > 0 ? 1 : 0;
    I.coarse_items = (nc + kCoarseRows - 1) / kCoarseRows;
    I.minv = minv32;
    I.rc = rc;
    I.cvec = cvec;
    I.lay = L;
    I.maps = nullptr;
    if (e->tma_ok) {
        if (!encode_operator_maps(b->maps, p32, rf32, kin32, kz32, L, e->d_stage_err))
            return cleanup(fail(TB_ECUDA, "tensor maps of the board's operator fields were refused"));
        TB_ENGINE_CUDA(cudaMemcpyAsync(e->d_maps + 3 * slot, b->maps, sizeof(b->maps), cudaMemcpyHostToDevice, e->io));
        I.maps = e->d_maps + 3 * slot;
    }

    char* sc = static_cast<char*>(stage);
    double* st_kin = carve<double>(sc, L.E);
    double* st_kz = carve<double>(sc, L.E);
    double* st_robin = carve<double>(sc, L.N);
    double* st_rhs = carve<double>(sc, L.N);
    double* st_x0 = carve<double>(sc, L.N);
    uint8_t* st_free = carve<uint8_t>(sc, L.N);
    double* st_geo = carve<double>(sc, geo);  // thickness, pitch_x, pitch_y
    double* st_diag = carve<double>(sc, L.L);
    double* st_dinv = carve<double>(sc, L.L);
    int* st_err = carve<int>(sc, 2);  // [0] diagonal, [1] coarse operator

    std::vector<double> g64(geo), dims(L.S + L.C + L.R);
    for (int i = 0; i < L.S; ++i) {
        g64[i] = d->slab_thickness_m[i] / 16.0;
        g64[L.S + i] = 1.0 / (16.0 * d->slab_thickness_m[i]);
        dims[i] = d->slab_thickness_m[i];
    }
    for (int i = 0; i < L.C; ++i) {
        g64[2 * L.S + i] = d->pitch_x_m[i];
        g64[2 * L.S + L.C + i] = 1.0 / d->pitch_x_m[i];
        dims[L.S + i] = d->pitch_x_m[i];
    }
    for (int i = 0; i < L.R; ++i) {
        g64[2 * L.S + 2 * L.C + i] = d->pitch_y_m[i];
        g64[2 * L.S + 2 * L.C + L.R + i] = 1.0 / d->pitch_y_m[i];
        dims[L.S + L.C + i] = d->pitch_y_m[i];
    }
    std::vector<float> g32(g64.begin(), g64.end());
    const cudaMemcpyKind h2d = cudaMemcpyHostToDevice;
    TB_ENGINE_CUDA(cudaMemcpyAsync(geo64, g64.data(), sizeof(double) * geo, h2d, e->io));
    TB_ENGINE_CUDA(cudaMemcpyAsync(geo32, g32.data(), sizeof(float) * geo, h2d, e->io));
    TB_ENGINE_CUDA(cudaMemcpyAsync(st_geo, dims.data(), sizeof(double) * dims.size(), h2d, e->io));
    TB_ENGINE_CUDA(cudaMemcpyAsync(st_kin, d->k_in, sizeof(double) * L.E, h2d, e->io));
    TB_ENGINE_CUDA(cudaMemcpyAsync(st_kz, d->k_z, sizeof(double) * L.E, h2d, e->io));
    TB_ENGINE_CUDA(cudaMemcpyAsync(st_robin, d->robin_total, sizeof(double) * L.N, h2d, e->io));
    TB_ENGINE_CUDA(cudaMemcpyAsync(st_free, d->free_nodes, (size_t)L.N, h2d, e->io));
    TB_ENGINE_CUDA(cudaMemcpyAsync(st_rhs, rhs, sizeof(double) * L.N, h2d, e->io));
    if (x0) TB_ENGINE_CUDA(cudaMemcpyAsync(st_x0, x0, sizeof(double) * L.N, h2d, e->io));
    TB_ENGINE_CUDA(cudaMemsetAsync(st_err, 0, 2 * sizeof(int), e->io));
    const int eb = grid_for(L.LE, kVecThreads, e->sms * 16);
    const int nb = grid_for(L.L, kVecThreads, e->sms * 16);
    pack_elements<<<eb, kVecThreads, 0, e->io>>>(kin64, kin32, st_kin, L);
    pack_elements<<<eb, kVecThreads, 0, e->io>>>(kz64, kz32, st_kz, L);
    build_rf<<<nb, kVecThreads, 0, e->io>>>(rf64, rf32, flags, st_robin, st_free, L);
    build_diagonal<<<nb, kVecThreads, 0, e->io>>>(st_diag, st_dinv, dinv32, st_err, kin64, kz64, rf64, st_geo,
                                                  st_geo + L.S, st_geo + L.S + L.C, L);
    pack_nodes<double, double><<<nb, kVecThreads, 0, e->io>>>(b64, st_rhs, L);
    TB_ENGINE_CUDA(cudaGetLastError());
    e->kernel_launches += 5;
    if (nc > 0) {
        // Two-level set-up (reference two_level.py:62-134): Z^T A Z from 27
        // coloured FP64 actions with x64 / r64 as scratch, Gauss-Jordan
        // inverse, FP32 copy; the same kernels as a single system's.
        const CoarseLayout& cl = b->cl;
        const long long nn = (long long)nc * nc;
        TB_ENGINE_CUDA(cudaMallocFromPoolAsync(&coarse_work, sizeof(double) * (2 * nn + 4 * (long long)nc), e->pool,
                                               e->io));
        double* M = static_cast<double*>(coarse_work);
        double* W = M + nn;
        double* R = W + nn;
        double* counts = R + nc;
        const int mb = grid_for(nn, kVecThreads, e->sms * 16);
        const dim3 agrid(apply_grid_x(L.C), apply_grid_y(8, L.R));
        const size_t asmem = apply_smem_bytes<double, 8>(L.S);
        TB_ENGINE_CUDA(cudaMemsetAsync(M, 0, sizeof(double) * nn, e->io));
        coarse_indicator<<<nb, kVecThreads, 0, e->io>>>(x64, rf64, L, cl, -1);
        coarse_restrict<double><<<nc, 128, 0, e->io>>>(x64, rf64, counts, L, cl, b->pstride, nullptr);
        for (int colour = 0; colour < 27; ++colour) {
            coarse_indicator<<<nb, kVecThreads, 0, e->io>>>(x64, rf64, L, cl, colour);
            apply_kernel<double, MODE_OPERATOR, EPI_STORE, 8><<<agrid, TileShape<8>::threads, asmem, e->io>>>(I.a64, ApplyMaps{});
            coarse_restrict<double><<<nc, 128, 0, e->io>>>(r64, rf64, R, L, cl, b->pstride, nullptr);
            coarse_scatter<<<(nc + 127) / 128, 128, 0, e->io>>>(M, R, cl, colour);
        }
        coarse_fix_empty<<<mb, kVecThreads, 0, e->io>>>(M, counts, nc);
        TB_ENGINE_CUDA(cudaMemcpyAsync(W, M, sizeof(double) * nn, cudaMemcpyDeviceToDevice, e->io));
        TB_ENGINE_CUDA(gauss_jordan_invert(W, nc, st_err + 1, e->io));
        coarse_symmetrize<<<mb, kVecThreads, 0, e->io>>>(W, M, minv32, nc, cl.ld);
        TB_ENGINE_CUDA(cudaGetLastError());
        TB_ENGINE_CUDA(cudaFreeAsync(coarse_work, e->io));
        coarse_work = nullptr;
        TB_ENGINE_CUDA(cudaMemsetAsync(x64, 0, sizeof(double) * L.L, e->io));
        TB_ENGINE_CUDA(cudaMemsetAsync(r64, 0, sizeof(double) * L.L, e->io));
        e->kernel_launches += 2 + 4 * 27 + 2 + 4LL * ((nc + kGjB - 1) / kGjB);
    }
    if (x0) {
        pack_nodes<double, double><<<nb, kVecThreads, 0, e->io>>>(x64, st_x0, L);
        TB_ENGINE_CUDA(cudaGetLastError());
        e->kernel_launches += 1;
    }
    int errs[2] = {0, 0};
    TB_ENGINE_CUDA(cudaMemcpyAsync(errs, st_err, sizeof(errs), cudaMemcpyDeviceToHost, e->io));
    TB_ENGINE_CUDA(cudaFreeAsync(stage, e->io));
    stage = nullptr;
    TB_ENGINE_CUDA(cudaStreamSynchronize(e->io));
    if (errs[0]) {
        fail(TB_EINVAL, "every free node must have positive conductance");
        return cleanup(TB_EINVAL);
    }
    if (errs[1]) {
        fail(TB_EINVAL, "the coarse operator is not positive definite; the fine operator must be SPD for the "
                        "two-level preconditioner");
        return cleanup(TB_EINVAL);
    }
#undef TB_ENGINE_CUDA

    BatchOuter o{};
    o.bscale = bnorm > 0.0 ? bnorm : 1.0;
    o.target = cfg->absolute_tolerance + cfg->relative_tolerance * o.bscale;
    o.inner_tol = cfg->inner_relative_tolerance;
    o.max_inner = cfg->max_inner_iterations;
    o.max_outer = cfg->max_outer_iterations;
    o.rel = 1.0;
    b->ticket = e->next_ticket++;
    batch_admit<<<1, 32, 0, e->stream>>>(I, o, b->ticket, e->d_table, slot);
    TB_CUDA(cudaGetLastError());
    e->kernel_launches += 1;
    e->slots[slot] = b;
    e->boards[b->ticket] = b;
    e->in_use += (long long)resident;
    e->dirty = true;
    *ticket = b->ticket;
    return TB_OK;
}

// Read the oldest snapshot in flight and note the boards that left the loop.
int engine_retire_oldest(tb_engine* e) {
    const int k = (e->head - e->inflight + kEngineDepth) % kEngineDepth;
    TB_CUDA(cudaEventSynchronize(e->ev[k]));
    e->inflight -= 1;
    const BatchStatus* snap = e->h_status + (size_t)k * e->capacity;
    for (int s = 0; s < e->capacity; ++s) {
        EngineBoard* b = e->slots[s];
        if (!b || b->reported || snap[s].ticket != b->ticket) continue;
        if (snap[s].phase == PH_DONE || snap[s].phase == PH_FAILED) {
            b->reported = true;
            e->finished.push_back(b->ticket);
            e->dirty = true;
        }
    }
    return TB_OK;
}

int engine_step(tb_engine* e, int* finished) {
    if (e->rows32 == 0) {
        bool any = false;
        for (EngineBoard* b : e->slots) any = any || (b && !b->reported);
        if (any) {
            while (e->inflight > 0) TB_CHECK(engine_retire_oldest(e));
            TB_CHECK(engine_autotune(e));
        }
    }
    if (e->dirty) TB_CHECK(engine_build_schedule(e));
    if (e->active > 0 && e->chunk) {
        TB_CUDA(cudaGraphLaunch(e->chunk, e->stream));
        e->kernel_launches += engine_kernels_per_chunk(e);
        e->chunks += 1;
        TB_CUDA(cudaMemcpyAsync(e->h_status + (size_t)e->head * e->capacity, e->d_status,
                                sizeof(BatchStatus) * e->capacity, cudaMemcpyDeviceToHost, e->stream));
        TB_CUDA(cudaEventRecord(e->ev[e->head], e->stream));
        e->head = (e->head + 1) % kEngineDepth;
        e->inflight += 1;
    }
    while (e->inflight >= kEngineDepth || (e->inflight > 0 && e->active == 0)) TB_CHECK(engine_retire_oldest(e));
    if (finished) *finished = (int)e->finished.size();
    return TB_OK;
}

// Device time of one batched FP32 operator launch over every board in the
// schedule (store epilogue), averaged over `reps` launches after a warm-up.
int engine_time_apply(tb_engine* e, int reps, double* ms) {
    while (e->inflight > 0) TB_CHECK(engine_retire_oldest(e));
    if (e->dirty) TB_CHECK(engine_build_schedule(e));
    if (e->rows32 == 0) {
        if (e->active == 0) return fail(TB_EINVAL, "no resident board to time");
        TB_CHECK(engine_autotune(e));
        TB_CHECK(engine_build_schedule(e));
    }
    float total = 0.f;
    TB_CHECK(engine_time_current(e, &total, reps));
    TB_CHECK(engine_check_stage(e));
    *ms = total / reps;
    return TB_OK;
}

int engine_collect(tb_engine* e, long long ticket, double* x, tb_mpir_result* res, tb_mpir_step* hist, int cap) {
    const auto it = e->boards.find(ticket);
    if (it == e->boards.end()) return fail(TB_EINVAL, "unknown ticket %lld", ticket);
    EngineBoard* b = it->second;
    if (!b->reported) return fail(TB_EINVAL, "board %lld has not finished", ticket);
    const Layout& L = b->lay;
    BatchOuter o;
    BatchStatus st;
    TB_CUDA(cudaMemcpyAsync(&o, e->d_outer + b->slot, sizeof(o), cudaMemcpyDeviceToHost, e->io));
    TB_CUDA(cudaMemcpyAsync(&st, e->d_status + b->slot, sizeof(st), cudaMemcpyDeviceToHost, e->io));
    if (x) {
        void* tmp = nullptr;
        TB_CUDA(cudaMallocFromPoolAsync(&tmp, sizeof(double) * (size_t)L.N, e->pool, e->io));
        const int nb = grid_for(L.N, kVecThreads, e->sms * 16);
        unpack_nodes<double, double><<<nb, kVecThreads, 0, e->io>>>(static_cast<double*>(tmp), b->inst.x64, L);
        TB_CUDA(cudaGetLastError());
        e->kernel_launches += 1;
        TB_CUDA(cudaMemcpyAsync(x, tmp, sizeof(double) * (size_t)L.N, cudaMemcpyDeviceToHost, e->io));
        TB_CUDA(cudaFreeAsync(tmp, e->io));
    }
    TB_CUDA(cudaEventRecord(e->io_done, e->io));
    TB_CUDA(cudaEventSynchronize(e->io_done));
    // Release in compute-stream order: the slot goes idle and its memory back to the pool.
    TB_CUDA(cudaStreamWaitEvent(e->stream, e->io_done, 0));
    batch_release<<<1, 32, 0, e->stream>>>(e->d_status + b->slot);
    TB_CUDA(cudaGetLastError());
    e->kernel_launches += 1;
    TB_CUDA(cudaFreeAsync(b->block, e->stream));
    e->slots[b->slot] = nullptr;
    e->in_use -= (long long)b->bytes;
    e->boards.erase(it);
    e->finished.erase(std::remove(e->finished.begin(), e->finished.end(), ticket), e->finished.end());
    const int max_outer = b->max_outer;
    delete b;
    if (res) {
        std::memset(res, 0, sizeof(*res));
        res->converged = o.converged;
        res->outer_iterations = o.converged ? o.outer : max_outer;
        res->inner_iterations = o.inner_total;
        res->high_operator_applications = o.high;
        res->low_operator_applications = o.low;
        res->relative_residual = o.rel;
        res->history_length = std::min(std::min(o.nhist, kBatchHist), std::max(cap, 0));
    }
    if (hist) {
        for (int i = 0; i < o.nhist && i < kBatchHist && i < cap; ++i) {
            hist[i].outer_iteration = i + 1;
            hist[i].high_relative_residual = o.hist[i][0];
            hist[i].inner_iterations = (int)o.hist[i][1];
            hist[i].inner_relative_residual = o.hist[i][2];
        }
    }
    if (st.phase == PH_FAILED) {
        TB_CHECK(engine_check_stage(e));
        return fail(TB_ENOTSPD, "inner PCG requires a finite symmetric positive-definite operator");
    }
    return TB_OK;
}

}  // namespace

extern "C" {

int tb_engine_create(int32_t device, const tb_engine_config* config, tb_engine** out) {
    if (!out) return fail(TB_EINVAL, "out is NULL");
    *out = nullptr;
    tb_engine* e = nullptr;
    const int rc = engine_create(device, config, &e);
    if (rc != TB_OK) {
        engine_free(e);
        return rc;
    }
    *out = e;
    return TB_OK;
}

int tb_engine_destroy(tb_engine* engine) {
    engine_free(engine);
    return TB_OK;
}

int tb_engine_footprint(const tb_system_desc* desc, int32_t preconditioner, int64_t* resident, int64_t* transient) {
    if (!desc || desc->slabs < 1 || desc->rows < 1 || desc->cols < 1) return fail(TB_EINVAL, "invalid board shape");
    const Layout L = layout_of(desc);
    const int nc = preconditioner == 1 ? coarse_layout(L, 0).nc : 0;
    int t32[3], gx32, t64, gx64, chunks;
    const int items = board_items(L, nc, t32, &gx32, &t64, &gx64, &chunks);
    size_t r = 0, t = 0;
    board_bytes(L, items, nc, &r, &t);
    if (resident) *resident = (int64_t)r;
    if (transient) *transient = (int64_t)t;
    return TB_OK;
}

int tb_engine_submit(tb_engine* e, const tb_system_desc* desc, const double* rhs, const double* x0,
                     const tb_mpir_config* config, int64_t* ticket) {
    if (!e || !ticket) return fail(TB_EINVAL, "NULL argument");
    TB_CUDA(cudaSetDevice(e->device));
    long long t = 0;
    TB_CHECK(engine_submit(e, desc, rhs, x0, config, &t));
    *ticket = t;
    return TB_OK;
}

int tb_engine_step(tb_engine* e, int32_t* finished) {
    if (!e) return fail(TB_EINVAL, "engine is NULL");
    TB_CUDA(cudaSetDevice(e->device));
    int n = 0;
    TB_CHECK(engine_step(e, &n));
    if (finished) *finished = n;
    return TB_OK;
}

int tb_engine_finished(tb_engine* e, int64_t* tickets, int32_t capacity, int32_t* count) {
    if (!e || !count) return fail(TB_EINVAL, "NULL argument");
    const int n = std::min((int)e->finished.size(), std::max(capacity, 0));
    for (int i = 0; i < n && tickets; ++i) tickets[i] = e->finished[i];
    *count = (int)e->finished.size();
    return TB_OK;
}

int tb_engine_collect(tb_engine* e, int64_t ticket, double* x, tb_mpir_result* result, tb_mpir_step* history,
                      int32_t history_capacity) {
    if (!e) return fail(TB_EINVAL, "engine is NULL");
    TB_CUDA(cudaSetDevice(e->device));
    return engine_collect(e, ticket, x, result, history, history_capacity);
}

int tb_engine_time_apply(tb_engine* e, int32_t launches, double* ms_per_launch) {
    if (!e || !ms_per_launch || launches < 1) return fail(TB_EINVAL, "invalid argument");
    TB_CUDA(cudaSetDevice(e->device));
    return engine_time_apply(e, launches, ms_per_launch);
}

int tb_engine_stream(const tb_engine* e, void** stream) {
    if (!e || !stream) return fail(TB_EINVAL, "NULL argument");
    *stream = static_cast<void*>(e->stream);
    return TB_OK;
}

int tb_engine_staging(const tb_engine* e, int32_t* staging) {
    if (!e || !staging) return fail(TB_EINVAL, "NULL argument");
    *staging = e->tma32 ? 2 : 1;
    return TB_OK;
}

int tb_engine_info(const tb_engine* e, int64_t* info8) {
    if (!e || !info8) return fail(TB_EINVAL, "NULL argument");
    info8[0] = (int64_t)e->boards.size();
    info8[1] = e->active;
    info8[2] = e->in_use;
    info8[3] = e->budget;
    info8[4] = e->chunks;
    info8[5] = e->kernel_launches;
    info8[6] = e->rows32;
    info8[7] = e->capacity;
    return TB_OK;
}

}  // extern "C"
