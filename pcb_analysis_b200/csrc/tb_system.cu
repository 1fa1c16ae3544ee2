// Host side of libthermal_b200.so: the device-resident system, the MPIR
// outer loop and the CUDA-graph chunks of the inner PCG, behind the C ABI of
// include/thermal_b200.h.
//
// Control flow of one MPIR solve (reference solver.py:580-698,
// hex_q1.cpp:837-925): the FP64 residual r = b - A x, its norm and its peak are
// one fused kernel (apply<double> with the residual epilogue); the host reads
// back three scalars per outer step and decides.  The inner FP32 PCG
// (solver.py:151-232) runs as CUDA-graph chunks of kChunk iterations, each
// iteration = apply<float> with the p.Ap epilogue, the fused update and the
// direction kernel; every kernel reads the solve's scalars from device memory
// and returns at once when the PCG has stopped, so chunks can be queued ahead
// and the host only polls the state between chunks.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <thread>
#include <vector>

#include "../../include/thermal_b200.h"
#include "tb_apply.cuh"
#include "tb_batch.cuh"
#include "tb_coarse.cuh"
#include "tb_dc.cuh"
#include "tb_multilevel.cuh"
#include "tb_prep.cuh"
#include "tb_reduce.cuh"
#include "tb_types.h"
#include "tb_vec.cuh"
#include "tb_warp_apply.cuh"

// Scratch of the allocation-free residual entry point (layout next to
// static_scratch_base): 8192 tiles x 4 doubles of partials, a 256-byte
// counter slot and a 256-byte scalar slot.
static __device__ __align__(256) unsigned char g_static_scratch[8192 * 4 * 8 + 512];

using namespace tb;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

#define TB_CUDA(call)                                                                                     \
    do {                                                                                                  \
        const cudaError_t err_ = (call);                                                                  \
        if (err_ != cudaSuccess) {                                                                        \
            const int code_ = (err_ == cudaErrorMemoryAllocation) ? TB_ENOMEM : TB_ECUDA;                 \
            return fail(code_, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(err_), __FILE__, __LINE__); \
        }                                                                                                 \
    } while (0)

#define TB_CHECK(expr)            \
    do {                          \
        const int rc_ = (expr);   \
        if (rc_ != TB_OK) return rc_; \
    } while (0)

constexpr int kChunk = 16;  // PCG iterations per graph launch

// One instantiated chunk of kChunk PCG iterations.  In timing mode the chunk
// also records an event before every apply and after every iteration, so the
// device time of each kernel inside the solve can be read back.
struct ChunkSlot {
    cudaGraphExec_t exec = nullptr;
    bool timed = false;
    cudaEvent_t ev[2 * kChunk + 1] = {};
};

long long round_up(long long v, long long m) { return (v + m - 1) / m * m; }

}  // namespace

// How the FP32 operator is launched: the z-marching tile kernel with a tile
// height (one block per tile, or kind 2: one wave of blocks sharing the
// board's tile planes evenly), or the warp-marching kernel with ZW z groups of
// SL slabs per lane and bands of `band` node rows.  The FP64 kernels always
// use z-march tiles of the plan's height.
struct ApplyPlan {
    int kind = 0;  // 0 z-march tiles, 1 warp march, 2 balanced z-march
    int rows = 16;
    int zw = 0, sl = 0, band = 0;
    int tma = 0;  // z-march kinds: stages filled by tensor copies (1) or per-thread cp.async (0)
    int stages = kStages;  // kind 0 with tensor copies: kStages (two planes in flight) or kDeepStages (three)
};

struct tb_system {
    int device = 0;
    cudaStream_t stream = nullptr;
    Layout lay{};
    long long pstride = 0, sstride = 0, nq = 0;
    ApplyPlan plan;  // FP32 operator launch shape (chosen by the autotuner)
    ApplyMaps maps[3]{};   // tensor maps of p32, rf32, kin32, kz32 per tile height 8, 16, 32 (tensor-copy staging)
    bool maps_ok = false;  // the maps are encoded (thermal systems)
    int* stage_err = nullptr;  // device word a block sets when it gave up waiting for its tiles
    int vec_blocks = 0;
    int sms = 148;
    size_t bytes = 0;
    std::vector<void*> allocations;

    // coefficients and masks
    float *kin32 = nullptr, *kz32 = nullptr, *rf32 = nullptr, *dinv32 = nullptr;
    double *kin64 = nullptr, *kz64 = nullptr, *rf64 = nullptr, *diag64 = nullptr, *dinv64 = nullptr;
    float* geo32 = nullptr;   // gzt[S] gzi[S] hx[C] ihx[C] hy[R] ihy[R]
    std::vector<float> h_geo32;            // host copy (per-slab factors go into kernel parameters)
    unsigned long long special_mask = 0;   // bit z: plane z has Robin or fixed nodes (planes < 64)
    double* geo64 = nullptr;
    double* dims64 = nullptr;  // slab thickness (S), pitch_x (C), pitch_y (R): the diagonal's operands
    int* plane_flags = nullptr;
    int* d_err = nullptr;
    // iterates
    float *x32 = nullptr, *r32 = nullptr, *p32 = nullptr, *q32 = nullptr;
    double *b64 = nullptr, *x64 = nullptr, *r64 = nullptr, *p64 = nullptr, *q64 = nullptr;
    // flat staging for host I/O
    void* stage = nullptr;
    size_t stage_bytes = 0;
    // reductions and scalars
    double* partials = nullptr;  // partial_blocks x 4 doubles
    int partial_blocks = 0;
    unsigned int* counter = nullptr;
    SolveCtl* ctl = nullptr;
    SolveCtl* h_ctl = nullptr;  // pinned, 2 slots
    KernelClock* clocks = nullptr;  // [0] FP32 apply (p.Ap), [1] FP64 apply (residual / PCG), [2] multilevel fine pass
    // graphs: two chunk slots per precision, kept in flight alternately
    ChunkSlot slots32[2], slots64[2];
    cudaEvent_t ev[2] = {nullptr, nullptr};
    // timing (tb_set_timing): [0] FP32 apply, [1] FP64 apply, [2] PCG vector kernels, [3] whole solve calls
    bool timing = false;
    double ms[4] = {0, 0, 0, 0};
    long long launches[4] = {0, 0, 0, 0};
    cudaEvent_t tev[2] = {nullptr, nullptr};
    long long kernel_launches = 0;  // every kernel of this library launched for this system
    // two-level preconditioner (precond == 1): coarse grid, Galerkin matrix,
    // its inverse (FP64 and the FP32 copy the inner PCG uses), R = Z^T r, c
    int precond = 0;
    CoarseLayout cl{};
    double *coarse_matrix = nullptr, *coarse_inv64 = nullptr;
    float *coarse_inv32 = nullptr, *coarse_rc = nullptr, *coarse_c = nullptr;
    // multilevel preconditioner (precond == 2): the fine z-line factors (l, 1/p)
    // and T^-1 r, and the coarse levels 1..c; the coarsest is inverted densely
    // into coarse_inv32 (its R and y are coarse_rc and coarse_c)
    struct MLLevel {
        MLGrid g{};
        float *st = nullptr, *lf = nullptr, *ipd = nullptr, *R = nullptr, *x = nullptr, *y = nullptr;
    };
    float *ml_zl = nullptr, *ml_zi = nullptr, *ml_w = nullptr;
    std::vector<MLLevel> ml;
    int ml_np = 0;  // plane bucket of the column kernels (9, 17 or 33)
    // the staged fine pass of the inner PCG (ml_update_staged): tensor maps of
    // q32, r32, ml_zl and ml_zi (box 32 x 8 x (S+1)), its stage count (0: not
    // available on this board) and whether the iterations use it
    MLStageMaps ml_maps{};
    int ml_stages = 0;
    bool ml_staged = false;
    // the plain FP64 PCG preconditioned by the multilevel operator (set for
    // the call of tb_solve_pcg_f64_ml*), and the kind the FP64 graphs hold
    bool pcg64_ml = false, slots64_ml = false;
    // problem terms of a system made by tb_system_create_problem (flat node
    // order): node flags, loads, Robin terms, C / dt, fixed values, and each
    // convection boundary's lumped weights for its removed heat
    bool problem = false;
    // layered DC systems (tb_dc_system_create): physics 1, node bits, via tables
    int physics = 0;  // 0 thermal hexahedra, 1 layered DC sheets and vias
    uint8_t* dc_mask = nullptr;
    long long* via_other = nullptr;
    int *via_slot = nullptr, *via_start = nullptr;
    float* via_g32 = nullptr;
    double* via_g64 = nullptr;
    float *dc_colh32 = nullptr, *dc_colih32 = nullptr;  // h_x, 1/h_x per element column, padded to Xp
    double *dc_colh64 = nullptr, *dc_colih64 = nullptr;
    int via_nodes = 0;
    uint8_t* node_flags = nullptr;
    uint8_t* elem_active = nullptr;  // NULL when every element exists
    double *load = nullptr, *robin_only = nullptr, *robin_total = nullptr, *robin_rhs = nullptr;
    double *capacity = nullptr, *fixed_value = nullptr;
    bool capacity_positive = false;
    double total_load = 0.0;
    struct Boundary {
        int kind = 0;
        double* w = nullptr;
        double* rw = nullptr;
        long long offset = 0, count = 0;  // node range the weights cover
        double rw_sum = 0.0;
    };
    std::vector<Boundary> boundaries;
    double* sum_partials = nullptr;
    int sum_blocks = 0;
    double* extrema = nullptr;  // {min, max} of a post-processed temperature (made on first use)
    double* sums = nullptr;  // 2 doubles per reduction
};

namespace {

// Device memory of the systems comes from one stream-ordered memory pool per
// device, which keeps up to kPoolKeepBytes of freed memory for the next
// system.  A create / solve / destroy loop (one system per solve, as the
// reference's solve_thermal_conduction works) then makes no cudaMalloc /
// cudaFree driver calls in steady state; their latency varies from
// milliseconds to a second with the driver's page-table work.  A 71 M-node
// board with its multilevel hierarchy peaks near 17 GB during set-up, so the
// pool keeps 48 GB (a quarter of a B200's HBM) rather than trimming to a
// smaller figure at every synchronisation.
constexpr unsigned long long kPoolKeepBytes = 48ULL << 30;

int system_pool(int device, cudaMemPool_t* out) {
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lock(mu);
    const auto it = pools.find(device);
    if (it != pools.end()) {
        *out = it->second;
        return TB_OK;
    }
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    TB_CUDA(cudaMemPoolCreate(&pool, &props));
    unsigned long long keep = kPoolKeepBytes;
    TB_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    pools[device] = pool;
    *out = pool;
    return TB_OK;
}

// Stream-ordered allocation on the system's stream, complete on return (the
// memory may be touched from any stream or by synchronous copies).
int pool_alloc(tb_system* s, void** ptr, size_t bytes) {
    cudaMemPool_t pool = nullptr;
    TB_CHECK(system_pool(s->device, &pool));
    void* p = nullptr;
    const cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, pool, s->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? TB_ENOMEM : TB_ECUDA, "device allocation of %zu bytes failed: %s",
                    bytes, cudaGetErrorString(e));
    }
    TB_CUDA(cudaStreamSynchronize(s->stream));
    *ptr = p;
    return TB_OK;
}

int dev_alloc(tb_system* s, void** ptr, size_t bytes) {
    void* p = nullptr;
    TB_CHECK(pool_alloc(s, &p, bytes));
    s->allocations.push_back(p);
    s->bytes += bytes;
    *ptr = p;
    return TB_OK;
}

// Free one allocation made by dev_alloc.
template <typename T>
void dev_free(tb_system* s, T*& ptr) {
    if (ptr == nullptr) return;
    void* p = static_cast<void*>(ptr);
    for (size_t i = 0; i < s->allocations.size(); ++i) {
        if (s->allocations[i] == p) {
            s->allocations.erase(s->allocations.begin() + (long)i);
            break;
        }
    }
    cudaFreeAsync(p, s->stream);
    ptr = nullptr;
}

template <typename T>
int alloc_n(tb_system* s, T** ptr, long long n) {
    return dev_alloc(s, reinterpret_cast<void**>(ptr), (size_t)std::max<long long>(n, 1) * sizeof(T));
}

int ensure_stage(tb_system* s, size_t bytes) {
    if (s->stage_bytes >= bytes) return TB_OK;
    if (s->stage) {
        cudaFreeAsync(s->stage, s->stream);
        s->bytes -= s->stage_bytes;
        s->stage = nullptr;
        s->stage_bytes = 0;
    }
    TB_CHECK(pool_alloc(s, &s->stage, bytes));
    s->stage_bytes = bytes;
    s->bytes += bytes;
    return TB_OK;
}

int grid_for(long long work, int threads, int cap) {
    long long b = (work + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return (int)b;
}

#include "tb_hostio.inl"

template <typename T>
ApplyParams<T> apply_params(const tb_system* s, const T* x, T* y, const T* b);

template <>
ApplyParams<float> apply_params<float>(const tb_system* s, const float* x, float* y, const float* b) {
    ApplyParams<float> P{};
    const int S = s->lay.S, R = s->lay.R, C = s->lay.C;
    P.x = x;
    P.y = y;
    P.b = b;
    P.kin = s->kin32;
    P.kz = s->kz32;
    P.rf = s->rf32;
    P.plane_flags = s->plane_flags;
    P.gzt = s->geo32;
    P.gzi = s->geo32 + S;
    P.hx = s->geo32 + 2 * S;
    P.ihx = s->geo32 + 2 * S + C;
    P.hy = s->geo32 + 2 * S + 2 * C;
    P.ihy = s->geo32 + 2 * S + 2 * C + R;
    P.partials = s->partials;
    P.counter = s->counter;
    P.ctl = s->ctl;
    P.clock = s->clocks;
    P.S = S;
    P.R = R;
    P.C = C;
    P.Xp = s->lay.Xp;
    P.Xe = s->lay.Xe;
    P.pstride = s->pstride;
    P.sstride = s->sstride;
    return P;
}

template <>
ApplyParams<double> apply_params<double>(const tb_system* s, const double* x, double* y, const double* b) {
    ApplyParams<double> P{};
    const int S = s->lay.S, R = s->lay.R, C = s->lay.C;
    P.x = x;
    P.y = y;
    P.b = b;
    P.kin = s->kin64;
    P.kz = s->kz64;
    P.rf = s->rf64;
    P.plane_flags = s->plane_flags;
    P.gzt = s->geo64;
    P.gzi = s->geo64 + S;
    P.hx = s->geo64 + 2 * S;
    P.ihx = s->geo64 + 2 * S + C;
    P.hy = s->geo64 + 2 * S + 2 * C;
    P.ihy = s->geo64 + 2 * S + 2 * C + R;
    P.partials = s->partials;
    P.counter = s->counter;
    P.ctl = s->ctl;
    P.clock = s->clocks + 1;
    P.S = S;
    P.R = R;
    P.C = C;
    P.Xp = s->lay.Xp;
    P.Xe = s->lay.Xe;
    P.pstride = s->pstride;
    P.sstride = s->sstride;
    return P;
}

constexpr int kTileRows[3] = {8, 16, 32};
constexpr int rows_index(int rows) { return rows == 8 ? 0 : (rows == 16 ? 1 : 2); }

// Launch with programmatic stream serialization: the kernel may be scheduled
// while its predecessor on the stream is still finishing, and waits for it at
// its griddepcontrol.wait (in-graph this becomes a programmatic edge).
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                       Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

inline int apply_grid_y(int rows_variant, int R) { return (R + 1 + rows_variant - 2) / (rows_variant - 1); }
inline int apply_grid_x(int C) { return (C + 1 + kOutX - 1) / kOutX; }

template <typename T, int MODE, int EPI, int ROWS, bool TMA = false, int STAGES = kStages>
int launch_apply_rows(tb_system* s, const ApplyParams<T>& P, bool pdl) {
    const dim3 grid(apply_grid_x(s->lay.C), apply_grid_y(ROWS, s->lay.R));
    const size_t smem = apply_smem_bytes<T, ROWS, STAGES>(s->lay.S);
    if (pdl) {
        TB_CUDA(launch_pdl(apply_kernel<T, MODE, EPI, ROWS, TMA, STAGES>, grid, dim3(TileShape<ROWS>::threads), smem,
                           s->stream, P, s->maps[rows_index(ROWS)]));
    } else {
        apply_kernel<T, MODE, EPI, ROWS, TMA, STAGES>
            <<<grid, TileShape<ROWS>::threads, smem, s->stream>>>(P, s->maps[rows_index(ROWS)]);
        TB_CUDA(cudaGetLastError());
    }
    return TB_OK;
}

// The balanced one-wave launch (plan kind 2): as many blocks as fit on the
// device at once, each writing an equal share of the board's (tile, plane)
// pairs.
template <int MODE, int EPI, int ROWS, bool TMA = false>
int launch_split_rows(tb_system* s, const ApplyParams<float>& P, bool pdl) {
    const int gx = apply_grid_x(s->lay.C);
    const int tiles = gx * apply_grid_y(ROWS, s->lay.R);
    const size_t smem = apply_smem_bytes<float, ROWS>(s->lay.S);
    int per_sm = 0;
    TB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, apply_split_kernel<float, MODE, EPI, ROWS, TMA>,
                                                          TileShape<ROWS>::threads, smem));
    const long long work = (long long)tiles * (s->lay.S + 1);
    const int blocks = (int)std::max<long long>(
        1, std::min<long long>({work, (long long)s->sms * std::max(per_sm, 1), (long long)s->partial_blocks}));
    const dim3 grid(blocks);
    if (pdl) {
        TB_CUDA(launch_pdl(apply_split_kernel<float, MODE, EPI, ROWS, TMA>, grid, dim3(TileShape<ROWS>::threads), smem,
                           s->stream, P, gx, tiles, s->maps[rows_index(ROWS)]));
    } else {
        apply_split_kernel<float, MODE, EPI, ROWS, TMA>
            <<<grid, TileShape<ROWS>::threads, smem, s->stream>>>(P, gx, tiles, s->maps[rows_index(ROWS)]);
        TB_CUDA(cudaGetLastError());
    }
    return TB_OK;
}

// FP64 tiles of 32 rows would need more shared memory than a block may have
// (four pipeline stages of 69 KB); the FP64 kernels, which run once per outer
// step, use at most 16 rows.
// ------------------------------------------------------------- warp march
using WarpKernel = void (*)(const WarpApplyParams);

template <int EPI>
WarpKernel warp_kernel_for(int zw, int sl) {
#define TB_WARP_CASE(Z, L) \
    if (zw == Z && sl == L) return warp_apply_kernel<Z, L, EPI>;
    TB_WARP_CASE(1, 1) TB_WARP_CASE(1, 2) TB_WARP_CASE(1, 3) TB_WARP_CASE(1, 4)
    TB_WARP_CASE(2, 2) TB_WARP_CASE(2, 3) TB_WARP_CASE(2, 4) TB_WARP_CASE(2, 5) TB_WARP_CASE(2, 6)
    TB_WARP_CASE(2, 7) TB_WARP_CASE(2, 8)
    TB_WARP_CASE(4, 2) TB_WARP_CASE(4, 3) TB_WARP_CASE(4, 4) TB_WARP_CASE(4, 5) TB_WARP_CASE(4, 6)
    TB_WARP_CASE(4, 7) TB_WARP_CASE(4, 8)
#undef TB_WARP_CASE
    return nullptr;
}

// Warp-march shapes that cover S slabs: for each z-group count, the smallest
// instantiated slab count per lane.
std::vector<std::pair<int, int>> warp_shapes(int S, unsigned long long special_mask, long long field_elements) {
    std::vector<std::pair<int, int>> out;
    if (S > kWarpMaxSlabs || S + 1 > 64) return out;
    // the warp kernel holds Robin / fixed marks of the bottom and top planes only
    const unsigned long long faces = 1ULL | (1ULL << S);
    if (special_mask & ~faces) return out;
    if (field_elements >= (1LL << 31)) return out;  // its offsets are 32-bit
    for (const int zw : {1, 2, 4}) {
        const int sl = (S + zw - 1) / zw;
        for (int l = sl; l <= 8; ++l) {
            if (warp_kernel_for<EPI_STORE>(zw, l) != nullptr) {
                out.emplace_back(zw, l);
                break;
            }
        }
    }
    return out;
}

inline int warp_colw(int zw, int C) { return (C + 1 + (32 / zw - 1) - 1) / (32 / zw - 1); }
inline int warp_units(int zw, int band, int R, int C) { return warp_colw(zw, C) * ((R + 1 + band - 1) / band); }

int warp_params(const tb_system* s, const float* x, float* y, WarpApplyParams* W) {
    const Layout& L = s->lay;
    if (L.S > kWarpMaxSlabs) return fail(TB_EINVAL, "warp-march operator supports at most %d slabs", kWarpMaxSlabs);
    std::memset(W, 0, sizeof(*W));
    W->x = x;
    W->y = y;
    W->kin = s->kin32;
    W->kz = s->kz32;
    W->rf = s->rf32;
    W->hx = s->geo32 + 2 * L.S;
    W->ihx = s->geo32 + 2 * L.S + L.C;
    W->hy = s->geo32 + 2 * L.S + 2 * L.C;
    W->ihy = s->geo32 + 2 * L.S + 2 * L.C + L.R;
    W->partials = s->partials;
    W->counter = s->counter;
    W->ctl = s->ctl;
    W->clock = s->clocks;
    for (int i = 0; i < L.S; ++i) {
        W->tz[i] = s->h_geo32[i];
        W->iz[i] = s->h_geo32[L.S + i];
    }
    W->special_lo = (s->special_mask & 1ULL) ? 1 : 0;
    W->special_hi = ((s->special_mask >> L.S) & 1ULL) ? 1 : 0;
    W->pstride = s->pstride;
    W->sstride = s->sstride;
    W->S = L.S;
    W->R = L.R;
    W->C = L.C;
    W->Xp = L.Xp;
    W->Xe = L.Xe;
    W->ncolw = warp_colw(s->plan.zw, L.C);
    W->band = s->plan.band;
    W->nband = (L.R + 1 + s->plan.band - 1) / s->plan.band;
    return TB_OK;
}

template <int EPI>
int launch_warp(tb_system* s, const float* x, float* y, bool pdl) {
    WarpApplyParams W;
    TB_CHECK(warp_params(s, x, y, &W));
    const WarpKernel k = warp_kernel_for<EPI>(s->plan.zw, s->plan.sl);
    if (k == nullptr) return fail(TB_EINVAL, "no warp-march kernel for %d groups of %d slabs", s->plan.zw, s->plan.sl);
    const int units = W.ncolw * W.nband;
    const dim3 grid((units + kWarpBlockWarps - 1) / kWarpBlockWarps), block(32 * kWarpBlockWarps);
    if (pdl) {
        TB_CUDA(launch_pdl(k, grid, block, 0, s->stream, W));
    } else {
        k<<<grid, block, 0, s->stream>>>(W);
        TB_CUDA(cudaGetLastError());
    }
    return TB_OK;
}

// The layered DC operator, y-marching: warps of 31 node quads (plus a halo
// lane) march down bands of node rows; the band height is chosen so that the
// grid is about one wave of resident warps (a taller band loads fewer halo
// rows, a shorter one gives more warps).
template <typename T, int MODE, int EPI>
int launch_dc(tb_system* s, const ApplyParams<T>& P, bool pdl) {
    static int per_sm = 0;  // per instantiation
    if (per_sm == 0) {
        int n = 0;
        TB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dc_march_kernel<T, MODE, EPI>, kDcThreads, 0));
        per_sm = std::max(n, 1);
    }
    DcParams<T> D{};
    D.A = P;
    D.mask = s->dc_mask;
    if constexpr (sizeof(T) == 4) {
        D.colh = s->dc_colh32;
        D.colih = s->dc_colih32;
    } else {
        D.colh = s->dc_colh64;
        D.colih = s->dc_colih64;
    }
    D.vias.slot = s->via_slot;
    D.vias.start = s->via_start;
    D.vias.other = s->via_other;
    if constexpr (sizeof(T) == 4) D.vias.g = s->via_g32;
    else D.vias.g = s->via_g64;
    D.vias.count = s->via_nodes;
    const Layout& L = s->lay;
    const int layers = L.S + 1, rows = L.R + 1, qrow = L.Xp / 4;
    const int warps_per_block = kDcThreads / 32;
    const int nseg = (qrow + 30) / 31;
    const long long target = (long long)s->sms * per_sm * warps_per_block;
    long long nband = std::max<long long>(1, std::min<long long>(rows, (target + (long long)layers * nseg - 1) /
                                                                            ((long long)layers * nseg)));
    int band = (int)((rows + nband - 1) / nband);
    band = std::max(band, 4);
    nband = (rows + band - 1) / band;
    long long blocks = ((long long)layers * nband * nseg + warps_per_block - 1) / warps_per_block;
    while (blocks > s->partial_blocks) {  // one reduction partial per block
        band *= 2;
        nband = (rows + band - 1) / band;
        blocks = ((long long)layers * nband * nseg + warps_per_block - 1) / warps_per_block;
    }
    if (pdl) {
        TB_CUDA(launch_pdl(dc_march_kernel<T, MODE, EPI>, dim3((unsigned)blocks), dim3(kDcThreads), 0, s->stream, D,
                           nseg, (int)nband, band));
    } else {
        dc_march_kernel<T, MODE, EPI><<<(unsigned)blocks, kDcThreads, 0, s->stream>>>(D, nseg, (int)nband, band);
        TB_CUDA(cudaGetLastError());
    }
    return TB_OK;
}

template <typename T, int MODE, int EPI>
int launch_apply(tb_system* s, const ApplyParams<T>& P, bool pdl = false) {
    if (s->physics == 1) return launch_dc<T, MODE, EPI>(s, P, pdl);
    if constexpr (sizeof(T) == 4 && MODE == MODE_OPERATOR && (EPI == EPI_STORE || EPI == EPI_DOT)) {
        if (s->plan.kind == 1) return launch_warp<EPI>(s, P.x, P.y, pdl);
        const bool tma = s->plan.tma != 0;
        if (tma && !(s->maps_ok && P.x == s->p32)) return fail(TB_EINVAL, "tensor maps do not cover this operand");
        if (s->plan.kind == 2) {
            if (s->plan.rows == 8)
                return tma ? launch_split_rows<MODE, EPI, 8, true>(s, P, pdl) : launch_split_rows<MODE, EPI, 8>(s, P, pdl);
            if (s->plan.rows == 32)
                return tma ? launch_split_rows<MODE, EPI, 32, true>(s, P, pdl)
                           : launch_split_rows<MODE, EPI, 32>(s, P, pdl);
            return tma ? launch_split_rows<MODE, EPI, 16, true>(s, P, pdl) : launch_split_rows<MODE, EPI, 16>(s, P, pdl);
        }
        if (tma && s->plan.stages == kDeepStages) {
            if (s->plan.rows == 8) return launch_apply_rows<T, MODE, EPI, 8, true, kDeepStages>(s, P, pdl);
            return launch_apply_rows<T, MODE, EPI, 16, true, kDeepStages>(s, P, pdl);
        }
        if (tma) {
            if (s->plan.rows == 8) return launch_apply_rows<T, MODE, EPI, 8, true>(s, P, pdl);
            if (s->plan.rows == 32) return launch_apply_rows<T, MODE, EPI, 32, true>(s, P, pdl);
            return launch_apply_rows<T, MODE, EPI, 16, true>(s, P, pdl);
        }
    }
    const int rows = s->plan.rows;
    if (rows == 8) return launch_apply_rows<T, MODE, EPI, 8>(s, P, pdl);
    if constexpr (sizeof(T) == 4) {
        if (rows == 32) return launch_apply_rows<T, MODE, EPI, 32>(s, P, pdl);
    }
    return launch_apply_rows<T, MODE, EPI, 16>(s, P, pdl);
}

template <typename T, int MODE, int EPI, int ROWS, bool TMA = false, int STAGES = kStages>
int smem_attribute(int S) {
    TB_CUDA(cudaFuncSetAttribute(apply_kernel<T, MODE, EPI, ROWS, TMA, STAGES>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)apply_smem_bytes<T, ROWS, STAGES>(S)));
    return TB_OK;
}

template <int EPI, int ROWS, bool TMA = false>
int split_smem_attribute(int S) {
    TB_CUDA(cudaFuncSetAttribute(apply_split_kernel<float, MODE_OPERATOR, EPI, ROWS, TMA>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)apply_smem_bytes<float, ROWS>(S)));
    return TB_OK;
}

template <int ROWS>
int smem_attributes_rows(int S) {
    TB_CHECK((smem_attribute<float, MODE_OPERATOR, EPI_STORE, ROWS>(S)));
    TB_CHECK((smem_attribute<float, MODE_OPERATOR, EPI_DOT, ROWS>(S)));
    TB_CHECK((split_smem_attribute<EPI_STORE, ROWS>(S)));
    TB_CHECK((split_smem_attribute<EPI_DOT, ROWS>(S)));
    TB_CHECK((smem_attribute<float, MODE_OPERATOR, EPI_STORE, ROWS, true>(S)));
    TB_CHECK((smem_attribute<float, MODE_OPERATOR, EPI_DOT, ROWS, true>(S)));
    TB_CHECK((split_smem_attribute<EPI_STORE, ROWS, true>(S)));
    TB_CHECK((split_smem_attribute<EPI_DOT, ROWS, true>(S)));
    if constexpr (ROWS <= 16) {
        TB_CHECK((smem_attribute<float, MODE_OPERATOR, EPI_STORE, ROWS, true, kDeepStages>(S)));
        TB_CHECK((smem_attribute<float, MODE_OPERATOR, EPI_DOT, ROWS, true, kDeepStages>(S)));
    }
    if constexpr (ROWS <= 16) {
        TB_CHECK((smem_attribute<double, MODE_OPERATOR, EPI_STORE, ROWS>(S)));
        TB_CHECK((smem_attribute<double, MODE_OPERATOR, EPI_DOT, ROWS>(S)));
        TB_CHECK((smem_attribute<double, MODE_OPERATOR, EPI_RESIDUAL, ROWS>(S)));
        TB_CHECK((smem_attribute<double, MODE_STIFFNESS, EPI_STORE, ROWS>(S)));
    }
    return TB_OK;
}

// The dynamic shared memory of the apply kernels grows with the slab count;
// the attribute is per device and per kernel, so it is raised to the largest
// slab count seen on each device.
int set_smem_attributes(int device, int S) {
    static std::mutex mu;
    static int max_slabs[64] = {0};
    std::lock_guard<std::mutex> lock(mu);
    if (device < 0 || device >= 64) return fail(TB_EINVAL, "device index out of range");
    if (S <= max_slabs[device]) return TB_OK;
    TB_CHECK(smem_attributes_rows<8>(S));
    TB_CHECK(smem_attributes_rows<16>(S));
    TB_CHECK(smem_attributes_rows<32>(S));
    max_slabs[device] = S;
    return TB_OK;
}

int read_ctl(tb_system* s, SolveCtl* out) {
    TB_CUDA(cudaMemcpyAsync(s->h_ctl, s->ctl, sizeof(SolveCtl), cudaMemcpyDeviceToHost, s->stream));
    TB_CUDA(cudaStreamSynchronize(s->stream));
    *out = *s->h_ctl;
    return TB_OK;
}

void release_slot(ChunkSlot& slot) {
    if (slot.exec) cudaGraphExecDestroy(slot.exec);
    slot.exec = nullptr;
    for (cudaEvent_t& e : slot.ev) {
        if (e) cudaEventDestroy(e);
        e = nullptr;
    }
    slot.timed = false;
}

// During stream capture a plain cudaEventRecord only marks a dependency; the
// external flag makes it an event-record node whose time can be read back.
int record_node(cudaEvent_t ev, cudaStream_t stream) {
    return cudaEventRecordWithFlags(ev, stream, cudaEventRecordExternal) == cudaSuccess ? TB_OK : TB_ECUDA;
}

// Restriction R = Z^T r and coarse step c = Minv R of the two-level
// preconditioner, on the system's stream (PDL launches).
template <int MODE>
cudaError_t launch_coarse_step(tb_system* s, bool pdl) {
    const CoarseLayout& cl = s->cl;
    const SolveCtl* state = (MODE == COARSE_ONLY) ? nullptr : s->ctl;
    cudaError_t e;
    if (pdl) {
        e = launch_pdl(coarse_restrict<float>, dim3(cl.nc), dim3(128), 0, s->stream, (const float*)s->r32,
                       (const float*)s->dinv32, s->coarse_rc, s->lay, cl, s->pstride, state);
    } else {
        coarse_restrict<float><<<cl.nc, 128, 0, s->stream>>>(s->r32, s->dinv32, s->coarse_rc, s->lay, cl, s->pstride,
                                                              state);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return e;
    // One wave of resident blocks (8 rows each per pass), one partial per block.
    static int per_sm[3] = {0, 0, 0};  // per instantiation
    const size_t smem = sizeof(float) * (size_t)cl.ld;
    if (per_sm[MODE] == 0) {
        int n = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, coarse_apply<MODE>, kCoarseThreads, sizeof(float) * 8192);
        if (e != cudaSuccess) return e;
        per_sm[MODE] = std::max(n, 1);
    }
    constexpr int rows = kCoarseThreads / 32 / kCoarseSplit;
    const int grid = std::max(1, std::min({(cl.nc + rows - 1) / rows, s->partial_blocks, s->sms * per_sm[MODE]}));
    if (pdl) {
        e = launch_pdl(coarse_apply<MODE>, dim3(grid), dim3(kCoarseThreads), smem, s->stream,
                       (const float*)s->coarse_inv32, (const float*)s->coarse_rc, s->coarse_c, cl.nc, cl.ld, s->ctl,
                       s->partials, s->counter);
    } else {
        coarse_apply<MODE><<<grid, kCoarseThreads, smem, s->stream>>>(s->coarse_inv32, s->coarse_rc, s->coarse_c, cl.nc,
                                                                      cl.ld, s->ctl, s->partials, s->counter);
        e = cudaGetLastError();
    }
    return e;
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();

#include "tb_multilevel.inl"

int build_chunk(tb_system* s, bool f64, bool timed, ChunkSlot* slot) {
    release_slot(*slot);
    if (timed) {
        for (cudaEvent_t& e : slot->ev) TB_CUDA(cudaEventCreate(&e));
    }
    cudaGraph_t graph = nullptr;
    TB_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    int rc = TB_OK;
    if (timed) rc = record_node(slot->ev[0], s->stream);
    for (int i = 0; i < kChunk && rc == TB_OK; ++i) {
        if (f64) {
            const ApplyParams<double> P = apply_params<double>(s, s->p64, s->q64, nullptr);
            rc = launch_apply<double, MODE_OPERATOR, EPI_DOT>(s, P, !timed);
        } else {
            const ApplyParams<float> P = apply_params<float>(s, s->p32, s->q32, nullptr);
            rc = launch_apply<float, MODE_OPERATOR, EPI_DOT>(s, P, !timed);
        }
        if (rc == TB_OK && timed) rc = record_node(slot->ev[2 * i + 1], s->stream);
        if (rc != TB_OK) break;
        const dim3 vg(s->vec_blocks), vb(kVecThreads);
        cudaError_t e1, e2;
        if (f64 && s->pcg64_ml) {
            e1 = launch_pdl(pcg_update_f64_norm, vg, vb, 0, s->stream, s->x64, s->r64, (const double*)s->p64,
                            (const double*)s->q64, s->nq, s->ctl, s->partials, s->counter);
            e2 = (e1 == cudaSuccess) ? ml_step64(s, false, true) : e1;
        } else if (f64) {
            e1 = launch_pdl(pcg_update_f64, vg, vb, 0, s->stream, s->x64, s->r64, s->p64, s->q64, s->dinv64, s->nq,
                            s->ctl, s->partials, s->counter);
            e2 = launch_pdl(pcg_direction_f64, vg, vb, 0, s->stream, s->p64, s->r64, s->dinv64, s->nq, s->ctl);
        } else if (s->precond == 2) {
            e1 = ml_step(s, ML_ITER, true);
            e2 = cudaSuccess;
        } else if (s->precond == 1) {
            e1 = launch_pdl(pcg_update_f32<true>, vg, vb, 0, s->stream, s->r32, (const float*)s->q32,
                            (const float*)s->dinv32, s->nq, s->ctl, s->partials, s->counter);
            if (e1 == cudaSuccess) e1 = launch_coarse_step<COARSE_ITERATE>(s, true);
            e2 = launch_pdl(pcg_direction_2l<false>, vg, vb, 0, s->stream, s->p32, s->x32, (const float*)s->r32,
                            (const float*)s->dinv32, (const float*)s->coarse_c, s->nq, s->lay, s->cl,
                            (const SolveCtl*)s->ctl);
        } else {
            e1 = launch_pdl(pcg_update_f32<false>, vg, vb, 0, s->stream, s->r32, (const float*)s->q32,
                            (const float*)s->dinv32, s->nq, s->ctl, s->partials, s->counter);
            e2 = launch_pdl(pcg_direction_f32, vg, vb, 0, s->stream, s->p32, s->x32, (const float*)s->r32,
                            (const float*)s->dinv32, s->nq, (const SolveCtl*)s->ctl);
        }
        rc = (e1 == cudaSuccess && e2 == cudaSuccess) ? TB_OK : TB_ECUDA;
        if (rc == TB_OK && timed) rc = record_node(slot->ev[2 * i + 2], s->stream);
    }
    const cudaError_t e = cudaStreamEndCapture(s->stream, &graph);
    if (rc != TB_OK) {
        if (graph) cudaGraphDestroy(graph);
        return fail(rc, "capturing the PCG chunk failed");
    }
    if (e != cudaSuccess) return fail(TB_ECUDA, "graph capture failed: %s", cudaGetErrorString(e));
    const cudaError_t e2 = cudaGraphInstantiate(&slot->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e2 != cudaSuccess) return fail(TB_ECUDA, "graph instantiation failed: %s", cudaGetErrorString(e2));
    slot->timed = timed;
    return TB_OK;
}

int ensure_slots(tb_system* s, bool f64) {
    if (f64 && s->slots64_ml != s->pcg64_ml) {
        for (int k = 0; k < 2; ++k) release_slot(s->slots64[k]);
        s->slots64_ml = s->pcg64_ml;
    }
    ChunkSlot* slots = f64 ? s->slots64 : s->slots32;
    for (int k = 0; k < 2; ++k) {
        if (slots[k].exec == nullptr || slots[k].timed != s->timing) TB_CHECK(build_chunk(s, f64, s->timing, &slots[k]));
    }
    return TB_OK;
}

// Device time of the first `worked` iterations of a finished timed chunk.
int accumulate_chunk(tb_system* s, const ChunkSlot& slot, int worked, bool f64) {
    if (s->launches[f64 ? 1 : 0] < 0) return TB_OK;
    for (int i = 0; i < worked && i < kChunk; ++i) {
        float a = 0.f, v = 0.f;
        if (cudaEventElapsedTime(&a, slot.ev[2 * i], slot.ev[2 * i + 1]) != cudaSuccess ||
            cudaEventElapsedTime(&v, slot.ev[2 * i + 1], slot.ev[2 * i + 2]) != cudaSuccess) {
            cudaGetLastError();  // timing unavailable: report nothing rather than fail the solve
            s->launches[f64 ? 1 : 0] = -1;
            return TB_OK;
        }
        s->ms[f64 ? 1 : 0] += a;
        s->launches[f64 ? 1 : 0] += 1;
        s->ms[2] += v;
        s->launches[2] += 2;
    }
    return TB_OK;
}

int check_stage(tb_system* s);

int kernels_per_iteration(const tb_system* s, bool f64) {
    if (f64 && s->pcg64_ml) return 2 + ml_kernels_per_step(s);
    if (!f64 && s->precond == 2) return 1 + ml_kernels_per_step(s);
    return (!f64 && s->precond == 1) ? 5 : 3;
}

// Run PCG chunks until the device state leaves ST_RUNNING.  Two chunks are in
// flight: the next one is queued before the state after the previous one is
// read, and the kernels of a finished PCG return at once.  Those returns are
// not free (on c3 a finished iteration's 34 launches still take about 0.18
// ms), so when the residual's decay since the previous chunk says that the
// chunk in flight will reach the tolerance with a quarter of its iterations
// to spare, no further chunk is queued until its state has been read.  A
// wrong guess costs one host round trip; the iterations themselves, and so
// the results, do not depend on it.
int run_pcg(tb_system* s, bool f64, SolveCtl* out) {
    TB_CHECK(ensure_slots(s, f64));
    ChunkSlot* slots = f64 ? s->slots64 : s->slots32;
    SolveCtl start;
    TB_CHECK(read_ctl(s, &start));
    if (start.state != ST_RUNNING) {
        *out = start;
        return TB_OK;
    }
    auto launch = [&](const int k) -> int {
        TB_CUDA(cudaGraphLaunch(slots[k].exec, s->stream));
        s->kernel_launches += kernels_per_iteration(s, f64) * kChunk;
        TB_CUDA(cudaMemcpyAsync(&s->h_ctl[k], s->ctl, sizeof(SolveCtl), cudaMemcpyDeviceToHost, s->stream));
        TB_CUDA(cudaEventRecord(s->ev[k], s->stream));
        return TB_OK;
    };
    TB_CHECK(launch(0));
    TB_CHECK(launch(1));
    int oldest = 0, in_flight = 2;
    int prev_apps = start.applications;
    double prev_rel = -1.0;
    int prev_it = 0;
    for (long long chunks = 2;; ++chunks) {
        TB_CUDA(cudaEventSynchronize(s->ev[oldest]));
        const SolveCtl seen = s->h_ctl[oldest];
        --in_flight;
        if (s->timing) TB_CHECK(accumulate_chunk(s, slots[oldest], seen.applications - prev_apps, f64));
        prev_apps = seen.applications;
        if (seen.state != ST_RUNNING) break;
        bool hold = false;
        if (in_flight == 1 && prev_rel > 0.0 && seen.rel > 0.0 && seen.rel < prev_rel && seen.iterations > prev_it &&
            seen.tol > 0.0) {
            const double slope = std::log(seen.rel / prev_rel) / (double)(seen.iterations - prev_it);
            const double need = std::log(seen.tol / seen.rel) / slope;  // iterations still to go, by the decay seen
            hold = need < 0.75 * kChunk;
        }
        prev_rel = seen.rel;
        prev_it = seen.iterations;
        if (in_flight == 0) {  // the held chunk did not finish: refill both slots, oldest first
            TB_CHECK(launch(oldest));
            TB_CHECK(launch(oldest ^ 1));
            in_flight = 2;
        } else if (hold) {
            oldest ^= 1;  // wait for the chunk in flight
        } else {
            TB_CHECK(launch(oldest));
            ++in_flight;
            oldest ^= 1;
        }
        if (chunks > (1LL << 40)) return fail(TB_ETIMEOUT, "PCG did not stop");
    }
    TB_CUDA(cudaStreamSynchronize(s->stream));
    TB_CUDA(cudaMemcpy(out, s->ctl, sizeof(SolveCtl), cudaMemcpyDeviceToHost));
    if (out->state == ST_STAGE_TIMEOUT) return check_stage(s) == TB_OK ? fail(TB_ETIMEOUT, "operator staging timed out")
                                                                       : TB_ETIMEOUT;
    return TB_OK;
}

int check_desc(const tb_system_desc* d) {
    if (d == nullptr) return fail(TB_EINVAL, "system description is NULL");
    if (d->slabs < 1 || d->rows < 1 || d->cols < 1) return fail(TB_EINVAL, "element grid must be positive");
    if (!d->slab_thickness_m || !d->pitch_x_m || !d->pitch_y_m || !d->k_in || !d->k_z || !d->robin_total ||
        !d->free_nodes)
        return fail(TB_EINVAL, "system arrays are missing");
    const long long nodes = (long long)(d->slabs + 1) * (d->rows + 1) * (d->cols + 1);
    if (nodes > (1LL << 31) * 4) return fail(TB_EINVAL, "grid too large");
    auto positive = [](const double* v, int n) {
        for (int i = 0; i < n; ++i)
            if (!(std::isfinite(v[i]) && v[i] > 0.0)) return false;
        return true;
    };
    if (!positive(d->slab_thickness_m, d->slabs)) return fail(TB_EINVAL, "slab thicknesses must be finite and positive");
    if (!positive(d->pitch_x_m, d->cols)) return fail(TB_EINVAL, "pitch_x_m must be finite and positive");
    if (!positive(d->pitch_y_m, d->rows)) return fail(TB_EINVAL, "pitch_y_m must be finite and positive");
    const long long elements = (long long)d->slabs * d->rows * d->cols;
    for (long long e = 0; e < elements; ++e) {
        if (!(std::isfinite(d->k_in[e]) && d->k_in[e] >= 0.0 && std::isfinite(d->k_z[e]) && d->k_z[e] >= 0.0))
            return fail(TB_EINVAL, "conductivities must be finite and non-negative");
    }
    for (long long n = 0; n < nodes; ++n) {
        if (d->free_nodes[n] && !(std::isfinite(d->robin_total[n]) && d->robin_total[n] >= 0.0))
            return fail(TB_EINVAL, "robin_total must be finite and non-negative on free nodes");
    }
    return TB_OK;
}

// Launch-shape autotuner.  The FP32 operator comes as z-marching tiles of 8,
// 16 or 32 element rows, or as the warp-marching kernel with 1, 2 or 4 z
// groups per warp and bands of 4 to 64 node rows.  Which one is fastest
// depends on how the board's work fills the 148 SMs against the halo
// overheads of small tiles and short bands.  At system creation every
// candidate's FP32 apply is timed on the board itself (three interleaved
// rounds of 2 warm-up and 5 timed launches, the fastest round counting), and
// the winner is cached per (device, slabs, row bucket, column bucket), buckets
// being quarter-octaves of the node counts.
int size_bucket(int n) { return (int)std::lround(4.0 * std::log2((double)std::max(n, 1))); }

std::vector<ApplyPlan> plan_candidates(const Layout& L, unsigned long long special_mask, bool maps_ok) {
    std::vector<ApplyPlan> out;
    for (const int kind : {0, 2}) {
        for (const int rows : kTileRows) {
            for (int tma = 0; tma <= (maps_ok ? 1 : 0); ++tma) {
                ApplyPlan p;
                p.kind = kind;
                p.rows = rows;
                p.tma = tma;
                out.push_back(p);
                if (kind == 0 && tma == 1 && rows <= 16) {  // the deeper tensor-copy pipeline
                    p.stages = kDeepStages;
                    out.push_back(p);
                }
            }
        }
    }
    for (const auto& shape : warp_shapes(L.S, special_mask, L.L)) {
        for (const int band : {4, 8, 16, 32, 64}) {
            if (band > 4 && (L.R + 1) < band) break;
            ApplyPlan p;
            p.kind = 1;
            p.rows = 8;
            p.zw = shape.first;
            p.sl = shape.second;
            p.band = band;
            out.push_back(p);
        }
    }
    return out;
}

int autotune_tile(tb_system* s) {
    static std::mutex mu;
    static std::map<std::tuple<int, int, int, int, int, int>, ApplyPlan> cache;
    // The warp march only serves boards whose Robin / fixed nodes sit on the
    // bottom and top planes, so that is part of the key.
    const int faces_only = warp_shapes(s->lay.S, s->special_mask, s->lay.L).empty() ? 0 : 1;
    const auto key =
        std::make_tuple(s->device, s->lay.S, size_bucket(s->lay.R + 1), size_bucket(s->lay.C + 1), faces_only,
                        s->maps_ok ? 1 : 0);
    {
        std::lock_guard<std::mutex> lock(mu);
        const auto it = cache.find(key);
        if (it != cache.end()) {
            s->plan = it->second;
            return TB_OK;
        }
    }
    float best = 1e30f, best_rows_ms = 1e30f;
    int best_rows = 16;
    ApplyPlan best_plan;
    const ApplyParams<float> P = apply_params<float>(s, s->p32, s->q32, nullptr);
    // Each candidate is timed as the solve runs it: the p.Ap action launched
    // by programmatic dependent launch right after the direction update that
    // writes p, and measured by the action's own device clock (first block
    // past its dependency wait to the last block's end, the figure the solve
    // reports).  Three interleaved rounds of 2 warm-up and 5 timed actions,
    // each candidate's fastest round kept: the candidates are often within a
    // few percent of each other.  A small kernel re-arms the solve state
    // before each pair (a zero p makes p.Ap zero, which stops a solve).  The
    // clock's running totals are put back afterwards.
    KernelClock saved{};
    TB_CUDA(cudaMemcpyAsync(&saved, s->clocks, sizeof(saved), cudaMemcpyDeviceToHost, s->stream));
    TB_CUDA(cudaStreamSynchronize(s->stream));
    const dim3 vg(s->vec_blocks), vb(kVecThreads);
    auto pair = [&]() -> int {
        set_ctl<<<1, 32, 0, s->stream>>>(s->ctl, 0.0, 1 << 30, 1.0, 0.0);
        TB_CUDA(cudaGetLastError());
        TB_CUDA(launch_pdl(pcg_direction_f32, vg, vb, 0, s->stream, s->p32, s->x32, (const float*)s->r32,
                           (const float*)s->dinv32, s->nq, (const SolveCtl*)s->ctl));
        TB_CHECK((launch_apply<float, MODE_OPERATOR, EPI_DOT>(s, P, true)));
        s->kernel_launches += 3;
        return TB_OK;
    };
    const std::vector<ApplyPlan> cands = plan_candidates(s->lay, s->special_mask, s->maps_ok);
    std::vector<float> fastest(cands.size(), 1e30f);
    for (int round = 0; round < 3; ++round) {
        for (size_t c = 0; c < cands.size(); ++c) {
            s->plan = cands[c];
            for (int i = 0; i < 2; ++i) TB_CHECK(pair());
            KernelClock c0{}, c1{};
            TB_CUDA(cudaMemcpyAsync(&c0, s->clocks, sizeof(c0), cudaMemcpyDeviceToHost, s->stream));
            for (int i = 0; i < 5; ++i) TB_CHECK(pair());
            TB_CUDA(cudaMemcpyAsync(&c1, s->clocks, sizeof(c1), cudaMemcpyDeviceToHost, s->stream));
            TB_CUDA(cudaStreamSynchronize(s->stream));
            const unsigned long long n = c1.count - c0.count;
            const float ms = n > 0 ? (float)((double)(c1.total_ns - c0.total_ns) * 1e-6 / (double)n) : 1e30f;
            fastest[c] = std::min(fastest[c], ms);
        }
    }
    TB_CUDA(cudaMemcpyAsync(s->clocks, &saved, sizeof(saved), cudaMemcpyHostToDevice, s->stream));
    TB_CUDA(cudaMemsetAsync(s->ctl, 0, sizeof(SolveCtl), s->stream));
    TB_CUDA(cudaStreamSynchronize(s->stream));
    for (size_t c = 0; c < cands.size(); ++c) {
        const ApplyPlan& cand = cands[c];
        const float ms = fastest[c];
        if (ms < best) {
            best = ms;
            best_plan = cand;
        }
        if (cand.kind == 0 && cand.tma == 0 && ms < best_rows_ms) {
            best_rows_ms = ms;
            best_rows = cand.rows;
        }
    }
    if (best_plan.kind == 1) best_plan.rows = best_rows;  // the tile height also serves the FP64 kernels
    s->plan = best_plan;
    TB_CHECK(check_stage(s));
    std::lock_guard<std::mutex> lock(mu);
    cache[key] = best_plan;
    return TB_OK;
}

// Tensor maps of the FP32 fields the operator stages (ApplyMaps): 3D maps of
// the padded node fields (S+1, R+1, Xp) and element fields (S, R, Xe), boxes
// of one stage's tiles, zero fill outside the field.  The encoder is the
// driver's cuTensorMapEncodeTiled, reached through the runtime so that the
// library needs no link against the driver library.  Without it (or when a
// map is refused) the system keeps the cp.async staging only.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
        cudaGetLastError();
    });
    return encode;
}

// The three map sets (tile heights 8, 16, 32) of one board's FP32 operator
// fields: the operand x and the Robin/fixed field (S+1, R+1, Xp), the element
// fields (S, R, Xe).  False when the encoder or a map is refused.
bool encode_operator_maps(ApplyMaps (&maps)[3], const float* x, const float* rf, const float* kin, const float* kz,
                          const Layout& L, int* err) {
    const PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
    if (encode == nullptr) return false;
    auto map3 = [&](CUtensorMap* m, const float* base, int d0, int d1, int d2, int box0, int box1) {
        const cuuint64_t dims[3] = {(cuuint64_t)d0, (cuuint64_t)d1, (cuuint64_t)d2};
        const cuuint64_t strides[2] = {(cuuint64_t)d0 * sizeof(float), (cuuint64_t)d0 * d1 * sizeof(float)};
        const cuuint32_t box[3] = {(cuuint32_t)box0, (cuuint32_t)box1, 1};
        const cuuint32_t estr[3] = {1, 1, 1};
        return encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, estr,
                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    };
    bool ok = true;
    for (int i = 0; i < 3; ++i) {  // the box is one stage's tile, so its height is the tile height's
        const int rows = kTileRows[i];
        ApplyMaps& m = maps[i];
        ok = ok && map3(&m.x, x, L.Xp, L.R + 1, L.S + 1, kTileW, rows + 1);
        ok = ok && map3(&m.rf, rf, L.Xp, L.R + 1, L.S + 1, kTileW, rows + 1);
        ok = ok && map3(&m.kin, kin, L.Xe, L.R, L.S, 64, rows);
        ok = ok && map3(&m.kz, kz, L.Xe, L.R, L.S, 64, rows);
        m.err = err;
    }
    return ok;
}

int encode_apply_maps(tb_system* s) {
    s->maps_ok = encode_operator_maps(s->maps, s->p32, s->rf32, s->kin32, s->kz32, s->lay, s->stage_err);
    return TB_OK;
}

// A block of the tensor-copy staging that gave up waiting for its tiles set
// the error word: the action is incomplete.
int check_stage(tb_system* s) {
    int err = 0;
    TB_CUDA(cudaMemcpyAsync(&err, s->stage_err, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    TB_CUDA(cudaStreamSynchronize(s->stream));
    if (err != 0) {
        TB_CUDA(cudaMemsetAsync(s->stage_err, 0, sizeof(int), s->stream));
        return fail(TB_ETIMEOUT, "a block of the operator or of the staged fine pass gave up waiting for its staged tiles");
    }
    return TB_OK;
}

// First half of system creation: the device, stream, layout, every solver
// array and the geometry factors.  The board's coefficients follow in
// finish_system, from device arrays.
int begin_system(int slabs, int rows, int cols, const double* thick, const double* px, const double* py, int device,
                 tb_system** out, int element_layers = -1) {
    int count = 0;
    TB_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) return fail(TB_EINVAL, "CUDA device %d is outside [0, %d)", device, count);
    TB_CUDA(cudaSetDevice(device));

    tb_system* s = new tb_system();
    *out = s;
    s->device = device;
    TB_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    TB_CUDA(cudaEventCreateWithFlags(&s->ev[0], cudaEventDisableTiming));
    TB_CUDA(cudaEventCreateWithFlags(&s->ev[1], cudaEventDisableTiming));
    Layout& L = s->lay;
    L.S = slabs;
    L.R = rows;
    L.C = cols;
    L.Xp = (int)round_up(L.C + 1, 4);
    L.Xe = (int)round_up(L.C, 4);
    L.N = (long long)(L.S + 1) * (L.R + 1) * (L.C + 1);
    L.L = (long long)(L.S + 1) * (L.R + 1) * L.Xp;
    const int el = element_layers < 0 ? L.S : element_layers;  // the DC sheets: one element layer per node layer
    L.E = (long long)el * L.R * L.C;
    L.LE = (long long)el * L.R * L.Xe;
    s->pstride = (long long)(L.R + 1) * L.Xp;
    s->sstride = (long long)L.R * L.Xe;
    s->nq = L.L / 4;
    TB_CHECK(set_smem_attributes(device, L.S));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    s->sms = sms;
    s->vec_blocks = grid_for(s->nq, kVecThreads, sms * 8);
    int max_blocks = std::max(apply_grid_x(L.C) * apply_grid_y(8, L.R), s->vec_blocks);
    for (const auto& shape : warp_shapes(L.S, 0, L.L)) {
        const int units = warp_units(shape.first, 4, L.R, L.C);
        max_blocks = std::max(max_blocks, (units + kWarpBlockWarps - 1) / kWarpBlockWarps);
    }

    TB_CHECK(alloc_n(s, &s->kin32, L.LE));
    TB_CHECK(alloc_n(s, &s->kz32, L.LE));
    TB_CHECK(alloc_n(s, &s->kin64, L.LE));
    TB_CHECK(alloc_n(s, &s->kz64, L.LE));
    TB_CHECK(alloc_n(s, &s->rf32, L.L));
    TB_CHECK(alloc_n(s, &s->rf64, L.L));
    TB_CHECK(alloc_n(s, &s->dinv32, L.L));
    TB_CHECK(alloc_n(s, &s->diag64, L.L));
    TB_CHECK(alloc_n(s, &s->dinv64, L.L));
    TB_CHECK(alloc_n(s, &s->geo32, 2 * L.S + 2 * L.C + 2 * L.R));
    TB_CHECK(alloc_n(s, &s->geo64, 2 * L.S + 2 * L.C + 2 * L.R));
    TB_CHECK(alloc_n(s, &s->dims64, (long long)L.S + L.C + L.R));
    TB_CHECK(alloc_n(s, &s->plane_flags, L.S + 1));
    TB_CHECK(alloc_n(s, &s->d_err, 1));
    TB_CHECK(alloc_n(s, &s->stage_err, 1));
    TB_CHECK(alloc_n(s, &s->x32, L.L));
    TB_CHECK(alloc_n(s, &s->r32, L.L));
    TB_CHECK(alloc_n(s, &s->p32, L.L));
    TB_CHECK(alloc_n(s, &s->q32, L.L));
    TB_CHECK(alloc_n(s, &s->b64, L.L));
    TB_CHECK(alloc_n(s, &s->x64, L.L));
    TB_CHECK(alloc_n(s, &s->r64, L.L));
    TB_CHECK(alloc_n(s, &s->partials, (long long)max_blocks * 4));
    s->partial_blocks = max_blocks;
    TB_CHECK(alloc_n(s, &s->counter, 1));
    TB_CHECK(alloc_n(s, &s->ctl, 1));
    TB_CHECK(alloc_n(s, &s->clocks, 3));
    {
        void* h = nullptr;
        TB_CUDA(cudaMallocHost(&h, 2 * sizeof(SolveCtl)));
        s->h_ctl = static_cast<SolveCtl*>(h);
        std::memset(s->h_ctl, 0, 2 * sizeof(SolveCtl));
    }
    TB_CUDA(cudaMemsetAsync(s->counter, 0, sizeof(unsigned int), s->stream));
    TB_CUDA(cudaMemsetAsync(s->ctl, 0, sizeof(SolveCtl), s->stream));
    {
        const KernelClock init[3] = {{~0ULL, 0, 0, 0}, {~0ULL, 0, 0, 0}, {~0ULL, 0, 0, 0}};
        TB_CUDA(cudaMemcpyAsync(s->clocks, init, sizeof(init), cudaMemcpyHostToDevice, s->stream));
    }
    TB_CUDA(cudaMemsetAsync(s->plane_flags, 0, sizeof(int) * (L.S + 1), s->stream));
    TB_CUDA(cudaMemsetAsync(s->d_err, 0, sizeof(int), s->stream));
    TB_CUDA(cudaMemsetAsync(s->stage_err, 0, sizeof(int), s->stream));
    if (element_layers < 0) TB_CHECK(encode_apply_maps(s));  // the layered DC sheets use their own kernel
    for (float* v : {s->x32, s->r32, s->p32, s->q32}) TB_CUDA(cudaMemsetAsync(v, 0, sizeof(float) * L.L, s->stream));
    for (double* v : {s->b64, s->x64, s->r64}) TB_CUDA(cudaMemsetAsync(v, 0, sizeof(double) * L.L, s->stream));

    // Geometry: gzt = h_z/16, gzi = 1/(16 h_z), h_x, 1/h_x, h_y, 1/h_y; and the
    // raw thickness | pitch_x | pitch_y, the operands of the diagonal.
    std::vector<double> g64(2 * L.S + 2 * L.C + 2 * L.R);
    for (int i = 0; i < L.S; ++i) {
        g64[i] = thick[i] / 16.0;
        g64[L.S + i] = 1.0 / (16.0 * thick[i]);
    }
    for (int i = 0; i < L.C; ++i) {
        g64[2 * L.S + i] = px[i];
        g64[2 * L.S + L.C + i] = 1.0 / px[i];
    }
    for (int i = 0; i < L.R; ++i) {
        g64[2 * L.S + 2 * L.C + i] = py[i];
        g64[2 * L.S + 2 * L.C + L.R + i] = 1.0 / py[i];
    }
    std::vector<float> g32(g64.begin(), g64.end());
    s->h_geo32 = g32;
    std::vector<double> dims(thick, thick + L.S);
    dims.insert(dims.end(), px, px + L.C);
    dims.insert(dims.end(), py, py + L.R);
    TB_CUDA(cudaMemcpyAsync(s->geo64, g64.data(), sizeof(double) * g64.size(), cudaMemcpyHostToDevice, s->stream));
    TB_CUDA(cudaMemcpyAsync(s->geo32, g32.data(), sizeof(float) * g32.size(), cudaMemcpyHostToDevice, s->stream));
    TB_CUDA(cudaMemcpyAsync(s->dims64, dims.data(), sizeof(double) * dims.size(), cudaMemcpyHostToDevice, s->stream));
    // the host vectors above must outlive the copies
    TB_CUDA(cudaStreamSynchronize(s->stream));
    return TB_OK;
}

// Second half: FP32/FP64 conductivities, the Robin/fixed field, the diagonal
// and the launch shape, from flat device arrays (k_in, k_z per element,
// Robin totals and the free mask per node).
int finish_system(tb_system* s, const double* d_kin, const double* d_kz, const double* d_robin, const uint8_t* d_free) {
    const Layout& L = s->lay;
    const int eb = grid_for(L.LE, kVecThreads, s->sms * 16);
    const int nb = grid_for(L.L, kVecThreads, s->sms * 16);
    pack_elements<<<eb, kVecThreads, 0, s->stream>>>(s->kin64, s->kin32, d_kin, L);
    pack_elements<<<eb, kVecThreads, 0, s->stream>>>(s->kz64, s->kz32, d_kz, L);
    build_rf<<<nb, kVecThreads, 0, s->stream>>>(s->rf64, s->rf32, s->plane_flags, d_robin, d_free, L);
    build_diagonal<<<nb, kVecThreads, 0, s->stream>>>(s->diag64, s->dinv64, s->dinv32, s->d_err, s->kin64, s->kz64,
                                                      s->rf64, s->dims64, s->dims64 + L.S, s->dims64 + L.S + L.C, L);
    TB_CUDA(cudaGetLastError());
    s->kernel_launches += 4;
    int err = 0;
    TB_CUDA(cudaMemcpyAsync(&err, s->d_err, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    TB_CUDA(cudaStreamSynchronize(s->stream));
    if (err) return fail(TB_EINVAL, "every free node must have positive conductance");
    {
        std::vector<int> flags(L.S + 1);
        TB_CUDA(cudaMemcpy(flags.data(), s->plane_flags, sizeof(int) * (L.S + 1), cudaMemcpyDeviceToHost));
        s->special_mask = 0;
        for (int z = 0; z <= L.S && z < 64; ++z)
            if (flags[z]) s->special_mask |= (1ULL << z);
    }
    TB_CHECK(autotune_tile(s));
    return TB_OK;
}

int create_impl(const tb_system_desc* d, int device, tb_system** out) {
    TB_CHECK(check_desc(d));
    TB_CHECK(begin_system(d->slabs, d->rows, d->cols, d->slab_thickness_m, d->pitch_x_m, d->pitch_y_m, device, out));
    tb_system* s = *out;
    const Layout& L = s->lay;
    // Staging: k_in, k_z (E doubles each), robin (N doubles), free (N bytes).
    const size_t need = sizeof(double) * (2 * (size_t)L.E + (size_t)L.N) + (size_t)L.N + 64;
    TB_CHECK(ensure_stage(s, need));
    double* st_kin = static_cast<double*>(s->stage);
    double* st_kz = st_kin + L.E;
    double* st_robin = st_kz + L.E;
    uint8_t* st_free = reinterpret_cast<uint8_t*>(st_robin + L.N);
    TB_CHECK(host_to_device(s, st_kin, d->k_in, sizeof(double) * L.E));
    TB_CHECK(host_to_device(s, st_kz, d->k_z, sizeof(double) * L.E));
    TB_CHECK(host_to_device(s, st_robin, d->robin_total, sizeof(double) * L.N));
    TB_CHECK(host_to_device(s, st_free, d->free_nodes, (size_t)L.N));
    return finish_system(s, st_kin, st_kz, st_robin, st_free);
}

void destroy_impl(tb_system* s) {
    if (s == nullptr) return;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (int k = 0; k < 2; ++k) {
        release_slot(s->slots32[k]);
        release_slot(s->slots64[k]);
    }
    for (cudaEvent_t e : s->tev)
        if (e) cudaEventDestroy(e);
    if (s->stream) {  // back to the device's pool, in stream order
        for (void* p : s->allocations) cudaFreeAsync(p, s->stream);
        if (s->stage) cudaFreeAsync(s->stage, s->stream);
        cudaStreamSynchronize(s->stream);
    }
    if (s->h_ctl) cudaFreeHost(s->h_ctl);
    for (cudaEvent_t e : s->ev)
        if (e) cudaEventDestroy(e);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

// Copy a flat host or device node array into a padded device field.
template <typename T>
int load_nodes(tb_system* s, T* dst, const T* src, bool src_on_device) {
    const Layout& L = s->lay;
    const int nb = grid_for(L.L, kVecThreads, 148 * 16);
    const T* flat = src;
    if (!src_on_device) {
        TB_CHECK(ensure_stage(s, sizeof(T) * (size_t)L.N));
        TB_CHECK(host_to_device(s, s->stage, src, sizeof(T) * L.N));
        flat = static_cast<const T*>(s->stage);
    }
    pack_nodes<T, T><<<nb, kVecThreads, 0, s->stream>>>(dst, flat, L);
    TB_CUDA(cudaGetLastError());
    s->kernel_launches += 1;
    return TB_OK;
}

template <typename T>
int store_nodes(tb_system* s, T* dst, const T* src, bool dst_on_device) {
    const Layout& L = s->lay;
    const int nb = grid_for(L.N, kVecThreads, 148 * 16);
    if (dst_on_device) {
        unpack_nodes<T, T><<<nb, kVecThreads, 0, s->stream>>>(dst, src, L);
        TB_CUDA(cudaGetLastError());
        s->kernel_launches += 1;
        return TB_OK;
    }
    TB_CHECK(ensure_stage(s, sizeof(T) * (size_t)L.N));
    unpack_nodes<T, T><<<nb, kVecThreads, 0, s->stream>>>(static_cast<T*>(s->stage), src, L);
    TB_CUDA(cudaGetLastError());
    s->kernel_launches += 1;
    TB_CHECK(device_to_host(s, dst, s->stage, sizeof(T) * L.N));
    TB_CUDA(cudaStreamSynchronize(s->stream));
    return TB_OK;
}

int norm2(tb_system* s, const double* v, double* out) {
    norm2_f64<<<s->vec_blocks, kVecThreads, 0, s->stream>>>(v, s->nq, s->ctl, s->partials, s->counter);
    TB_CUDA(cudaGetLastError());
    s->kernel_launches += 1;
    SolveCtl c;
    TB_CHECK(read_ctl(s, &c));
    *out = c.norm2;
    return TB_OK;
}

// r64 = b64 - A x64, returns ||r||^2 and max |r|.
int residual64(tb_system* s, double* res2, double* peak) {
    const ApplyParams<double> P = apply_params<double>(s, s->x64, s->r64, s->b64);
    if (s->timing) TB_CUDA(cudaEventRecord(s->tev[0], s->stream));
    TB_CHECK((launch_apply<double, MODE_OPERATOR, EPI_RESIDUAL>(s, P)));
    if (s->timing) TB_CUDA(cudaEventRecord(s->tev[1], s->stream));
    s->kernel_launches += 1;
    SolveCtl c;
    TB_CHECK(read_ctl(s, &c));
    if (s->timing) {
        float ms = 0.f;
        TB_CUDA(cudaEventElapsedTime(&ms, s->tev[0], s->tev[1]));
        s->ms[1] += ms;
        s->launches[1] += 1;
    }
    *res2 = c.res2;
    *peak = c.peak;
    return TB_OK;
}

int mpir_impl(tb_system* s, const tb_mpir_config* cfg, tb_mpir_result* res, tb_mpir_step* hist, int cap) {
    if (cfg == nullptr || res == nullptr) return fail(TB_EINVAL, "config and result must not be NULL");
    if (!(cfg->relative_tolerance >= 0.0) || !(cfg->absolute_tolerance >= 0.0) ||
        !(cfg->inner_relative_tolerance > 0.0 && cfg->inner_relative_tolerance < 1.0) ||
        cfg->max_outer_iterations < 1 || cfg->max_inner_iterations < 1)
        return fail(TB_EINVAL, "invalid MPIR configuration");
    std::memset(res, 0, sizeof(*res));
    double bn2 = 0.0;
    TB_CHECK(norm2(s, s->b64, &bn2));
    const double rhs_norm = std::sqrt(bn2);
    if (!std::isfinite(rhs_norm)) return fail(TB_ENONFINITE, "rhs must contain only finite values");
    const double scale = rhs_norm > 0.0 ? rhs_norm : 1.0;
    const double target = cfg->absolute_tolerance + cfg->relative_tolerance * scale;
    int high = 0, low = 0, total_inner = 0, nhist = 0;
    double relative = 1.0;
    bool converged = false;
    int outer = 0;
    for (outer = 0; outer <= cfg->max_outer_iterations; ++outer) {
        double res2 = 0.0, peak = 0.0;
        TB_CHECK(residual64(s, &res2, &peak));
        ++high;
        const double rnorm = std::sqrt(res2);
        relative = rnorm / scale;
        if (rnorm <= target) {
            converged = true;
            break;
        }
        if (outer == cfg->max_outer_iterations) break;
        // power-of-two scale: max |r| * 2^-e in [0.5, 1)
        double pscale = 1.0;
        if (peak > 0.0 && std::isfinite(peak)) {
            int e = 0;
            std::frexp(peak, &e);
            pscale = std::ldexp(1.0, -e);
        }
        set_ctl<<<1, 32, 0, s->stream>>>(s->ctl, cfg->inner_relative_tolerance, cfg->max_inner_iterations, pscale, 0.0);
        if (s->precond == 2) {
            TB_CUDA(ml_step(s, ML_START, false));
            s->kernel_launches += ml_kernels_per_step(s);
        } else if (s->precond == 1) {
            inner_start_f32<true><<<s->vec_blocks, kVecThreads, 0, s->stream>>>(
                s->r64, s->x32, s->r32, s->p32, s->dinv32, s->nq, s->ctl, s->partials, s->counter);
            TB_CUDA(cudaGetLastError());
            TB_CUDA(launch_coarse_step<COARSE_START>(s, false));
            pcg_direction_2l<true><<<s->vec_blocks, kVecThreads, 0, s->stream>>>(
                s->p32, nullptr, s->r32, s->dinv32, s->coarse_c, s->nq, s->lay, s->cl, s->ctl);
            TB_CUDA(cudaGetLastError());
            s->kernel_launches += 5;
        } else {
            inner_start_f32<false><<<s->vec_blocks, kVecThreads, 0, s->stream>>>(
                s->r64, s->x32, s->r32, s->p32, s->dinv32, s->nq, s->ctl, s->partials, s->counter);
            TB_CUDA(cudaGetLastError());
            s->kernel_launches += 2;
        }
        SolveCtl c;
        TB_CHECK(run_pcg(s, false, &c));
        if (c.state == ST_NOT_SPD) return fail(TB_ENOTSPD, "inner PCG requires a finite symmetric positive-definite operator");
        mpir_finish<<<s->vec_blocks, kVecThreads, 0, s->stream>>>(s->x64, s->x32, s->p32, s->nq, s->ctl);
        TB_CUDA(cudaGetLastError());
        s->kernel_launches += 1;
        total_inner += c.iterations;
        low += c.applications;
        if (hist && nhist < cap) {
            hist[nhist].outer_iteration = outer + 1;
            hist[nhist].high_relative_residual = relative;
            hist[nhist].inner_iterations = c.iterations;
            hist[nhist].inner_relative_residual = (c.state == ST_ZERO_RHS) ? 0.0 : c.rel;
        }
        ++nhist;
    }
    res->converged = converged ? 1 : 0;
    res->outer_iterations = converged ? outer : cfg->max_outer_iterations;
    res->inner_iterations = total_inner;
    res->high_operator_applications = high;
    res->low_operator_applications = low;
    res->relative_residual = relative;
    res->history_length = std::min(nhist, cap);
    return TB_OK;
}

// ------------------------------------------------------------ two-level
int cdiv(int a, int b) { return (a + b - 1) / b; }

// Coarse grid of the two-level preconditioner: the smallest patch width >= 4
// whose grid has at most 2048 patches, as the reference chooses it
// (two_level.py:36-50), unless the caller fixes the width.
CoarseLayout coarse_layout(const Layout& L, int block) {
    const int layers = L.S + 1, rows = L.R + 1, cols = L.C + 1;
    int b = block;
    if (b <= 0) {
        b = 4;
        while ((long long)layers * cdiv(rows, b) * cdiv(cols, b) > 2048 && b < std::max(rows, cols)) ++b;
    }
    CoarseLayout cl{};
    cl.b = b;
    cl.layers = layers;
    cl.nby = cdiv(rows, b);
    cl.nbx = cdiv(cols, b);
    cl.nc = layers * cl.nby * cl.nbx;
    cl.ld = (cl.nc + 3) / 4 * 4;
    return cl;
}

// The FP32 coarse inverse is read whole once per inner iteration while the
// vector kernels stream some 200 MB past L2, so it is marked persisting in
// L2 through the system stream's access-policy window (captured into the
// chunk graphs).  The set-aside is a limit of this process's context: it is
// raised to fit the inverse (up to the device maximum) and ends with the
// process.  Without two-level the window is cleared.
int keep_coarse_in_l2(tb_system* s) {
    cudaStreamAttrValue attr{};
    size_t bytes = 0;
    if (s->coarse_inv32 != nullptr) bytes = sizeof(float) * (size_t)s->cl.nc * (size_t)s->cl.ld;
    int max_window = 0, max_persist = 0;
    cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, s->device);
    cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, s->device);
    if (bytes == 0 || max_window <= 0 || max_persist <= 0) {
        attr.accessPolicyWindow.num_bytes = 0;
        TB_CUDA(cudaStreamSetAttribute(s->stream, cudaStreamAttributeAccessPolicyWindow, &attr));
        return TB_OK;
    }
    const size_t window = std::min(bytes, (size_t)max_window);
    size_t limit = 0;
    TB_CUDA(cudaDeviceGetLimit(&limit, cudaLimitPersistingL2CacheSize));
    const size_t want = std::min(window, (size_t)max_persist);
    if (limit < want) TB_CUDA(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want));
    TB_CUDA(cudaDeviceGetLimit(&limit, cudaLimitPersistingL2CacheSize));
    attr.accessPolicyWindow.base_ptr = s->coarse_inv32;
    attr.accessPolicyWindow.num_bytes = window;
    attr.accessPolicyWindow.hitRatio = std::min(1.0f, (float)((double)limit / (double)window));
    attr.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    attr.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    TB_CUDA(cudaStreamSetAttribute(s->stream, cudaStreamAttributeAccessPolicyWindow, &attr));
    return TB_OK;
}

void free_coarse(tb_system* s) {
    dev_free(s, s->coarse_matrix);
    dev_free(s, s->coarse_inv64);
    dev_free(s, s->coarse_inv32);
    dev_free(s, s->coarse_rc);
    dev_free(s, s->coarse_c);
}

// Build Z^T A Z (27 coloured FP64 actions), its symmetrised inverse (Gauss-
// Jordan) and the FP32 copy (reference two_level.py:62-134, 152-199).
int build_coarse(tb_system* s, int block) {
    const Layout& L = s->lay;
    if (block < 0) return fail(TB_EINVAL, "coarse_block_nodes must be positive");
    const CoarseLayout cl = coarse_layout(L, block);
    if (cl.nc > 8192)
        return fail(TB_EINVAL, "a patch width of %d gives %d coarse unknowns; at most 8192 are supported", cl.b, cl.nc);
    free_coarse(s);
    const long long nc = cl.nc, nn = nc * nc;
    TB_CHECK(alloc_n(s, &s->coarse_matrix, nn));
    TB_CHECK(alloc_n(s, &s->coarse_inv64, nn));
    TB_CHECK(alloc_n(s, &s->coarse_inv32, nc * cl.ld));
    TB_CHECK(alloc_n(s, &s->coarse_rc, cl.ld));
    TB_CHECK(alloc_n(s, &s->coarse_c, nc));
    double* work = nullptr;  // Gauss-Jordan workspace, then scratch vectors
    double* vecs = nullptr;  // R, counts, row k, column k
    TB_CHECK(alloc_n(s, &work, nn));
    TB_CHECK(alloc_n(s, &vecs, 4 * nc));
    double* R = vecs;
    double* counts = vecs + nc;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
    const int nb = grid_for(L.L, kVecThreads, sms * 16);
    const int mb = grid_for(nn, kVecThreads, sms * 16);
    const int cb = cdiv((int)nc, 128);
    cudaStream_t st = s->stream;
    int rc = TB_OK;
    auto check_launch = [&]() {
        if (rc == TB_OK && cudaGetLastError() != cudaSuccess) rc = fail(TB_ECUDA, "coarse set-up launch failed");
    };
    cudaMemsetAsync(s->coarse_matrix, 0, sizeof(double) * nn, st);
    cudaMemsetAsync(s->coarse_rc, 0, sizeof(float) * cl.ld, st);  // the pads of R stay zero
    cudaMemsetAsync(s->d_err, 0, sizeof(int), st);
    coarse_indicator<<<nb, kVecThreads, 0, st>>>(s->b64, s->rf64, L, cl, -1);
    coarse_restrict<double><<<cl.nc, 128, 0, st>>>(s->b64, s->rf64, counts, L, cl, s->pstride, nullptr);
    s->kernel_launches += 2;
    check_launch();
    for (int colour = 0; colour < 27 && rc == TB_OK; ++colour) {
        coarse_indicator<<<nb, kVecThreads, 0, st>>>(s->b64, s->rf64, L, cl, colour);
        check_launch();
        if (rc != TB_OK) break;
        const ApplyParams<double> P = apply_params<double>(s, s->b64, s->r64, nullptr);
        rc = launch_apply<double, MODE_OPERATOR, EPI_STORE>(s, P);
        if (rc != TB_OK) break;
        coarse_restrict<double><<<cl.nc, 128, 0, st>>>(s->r64, s->rf64, R, L, cl, s->pstride, nullptr);
        coarse_scatter<<<cb, 128, 0, st>>>(s->coarse_matrix, R, cl, colour);
        s->kernel_launches += 4;
        check_launch();
    }
    if (rc == TB_OK) {
        coarse_fix_empty<<<mb, kVecThreads, 0, st>>>(s->coarse_matrix, counts, cl.nc);
        cudaMemcpyAsync(work, s->coarse_matrix, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st);
        if (rc == TB_OK && gauss_jordan_invert(work, cl.nc, s->d_err, st) != cudaSuccess)
            rc = fail(TB_ECUDA, "coarse inversion launch failed");
        coarse_symmetrize<<<mb, kVecThreads, 0, st>>>(work, s->coarse_inv64, s->coarse_inv32, cl.nc, cl.ld);
        s->kernel_launches += 2 + 4LL * cdiv(cl.nc, kGjB);
        check_launch();
    }
    int err = 0;
    if (rc == TB_OK) {
        if (cudaMemcpyAsync(&err, s->d_err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            rc = fail(TB_ECUDA, "coarse set-up failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    cudaStreamSynchronize(st);
    dev_free(s, work);
    dev_free(s, vecs);
    if (rc != TB_OK) return rc;
    if (err)
        return fail(TB_EINVAL,
                    "the coarse operator is not positive definite; the fine operator must be SPD for the two-level "
                    "preconditioner");
    s->cl = cl;
    return keep_coarse_in_l2(s);
}

int set_preconditioner(tb_system* s, int kind, int block) {
    if (kind < 0 || kind > 2)
        return fail(TB_EINVAL, "preconditioner kind must be 0 (Jacobi), 1 (two-level) or 2 (multilevel)");
    if (kind == 2 && s->physics != 0) return fail(TB_EINVAL, "the multilevel preconditioner is built for thermal systems");
    TB_CUDA(cudaStreamSynchronize(s->stream));
    for (int k = 0; k < 2; ++k) {  // the chunk graphs hold the old kernels and buffers
        release_slot(s->slots32[k]);
        release_slot(s->slots64[k]);
    }
    s->precond = 0;
    free_multilevel(s);
    if (kind == 0) {
        free_coarse(s);
        s->cl = CoarseLayout{};
        return keep_coarse_in_l2(s);
    }
    if (kind == 2) {
        TB_CHECK(build_multilevel(s));
        s->precond = 2;
        return TB_OK;
    }
    TB_CHECK(build_coarse(s, block));
    s->precond = 1;
    return TB_OK;
}

// New lumped Robin totals (Robin conductance + C / dt of a transient step,
// or the Newton linearisation of radiation) on the resident system, from a
// flat device array: rf, the plane flags, the Jacobi diagonal and, for the
// two-level preconditioner, the coarse operator are rebuilt on the device;
// the free mask is kept.
int refresh_robin(tb_system* s, const double* d_robin) {
    const Layout& L = s->lay;
    TB_CUDA(cudaMemsetAsync(s->plane_flags, 0, sizeof(int) * (L.S + 1), s->stream));
    TB_CUDA(cudaMemsetAsync(s->d_err, 0, sizeof(int), s->stream));
    const int nb = grid_for(L.L, kVecThreads, s->sms * 16);
    update_rf<<<nb, kVecThreads, 0, s->stream>>>(s->rf64, s->rf32, s->plane_flags, d_robin, L);
    build_diagonal<<<nb, kVecThreads, 0, s->stream>>>(s->diag64, s->dinv64, s->dinv32, s->d_err, s->kin64, s->kz64,
                                                      s->rf64, s->dims64, s->dims64 + L.S, s->dims64 + L.S + L.C, L);
    TB_CUDA(cudaGetLastError());
    s->kernel_launches += 2;
    int err = 0;
    TB_CUDA(cudaMemcpyAsync(&err, s->d_err, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    std::vector<int> flags(L.S + 1);
    TB_CUDA(cudaMemcpyAsync(flags.data(), s->plane_flags, sizeof(int) * (L.S + 1), cudaMemcpyDeviceToHost, s->stream));
    TB_CUDA(cudaStreamSynchronize(s->stream));
    if (err) return fail(TB_EINVAL, "every free node must have positive conductance");
    const unsigned long long old_mask = s->special_mask;
    s->special_mask = 0;
    for (int z = 0; z <= L.S && z < 64; ++z)
        if (flags[z]) s->special_mask |= (1ULL << z);
    for (int k = 0; k < 2; ++k) {  // the chunk graphs hold the old launch shape
        release_slot(s->slots32[k]);
        release_slot(s->slots64[k]);
    }
    if (s->special_mask != old_mask) TB_CHECK(autotune_tile(s));
    if (s->precond == 1) TB_CHECK(set_preconditioner(s, 1, s->cl.b));
    if (s->precond == 2) TB_CHECK(set_preconditioner(s, 2, 0));
    return TB_OK;
}

int set_robin_impl(tb_system* s, const double* robin) {
    const Layout& L = s->lay;
    if (s->physics != 0) return fail(TB_EINVAL, "a layered DC system has no Robin terms");
    if (s->problem)
        return fail(TB_EINVAL, "a system made from a problem takes new boundaries through tb_set_convection and "
                               "tb_set_capacity");
    for (long long n = 0; n < L.N; ++n)
        if (!(std::isfinite(robin[n]) && robin[n] >= 0.0))
            return fail(TB_EINVAL, "robin_total must be finite and non-negative");
    TB_CUDA(cudaStreamSynchronize(s->stream));
    TB_CHECK(ensure_stage(s, sizeof(double) * (size_t)L.N));
    TB_CHECK(host_to_device(s, s->stage, robin, sizeof(double) * L.N));
    return refresh_robin(s, static_cast<const double*>(s->stage));
}

int ensure_f64_pcg(tb_system* s) {
    if (s->p64) return TB_OK;
    TB_CHECK(alloc_n(s, &s->p64, s->lay.L));
    TB_CHECK(alloc_n(s, &s->q64, s->lay.L));
    TB_CUDA(cudaMemsetAsync(s->p64, 0, sizeof(double) * s->lay.L, s->stream));
    TB_CUDA(cudaMemsetAsync(s->q64, 0, sizeof(double) * s->lay.L, s->stream));
    return TB_OK;
}

int pcg64_impl(tb_system* s, double rtol, double atol, int max_it, tb_pcg_result* res) {
    if (res == nullptr) return fail(TB_EINVAL, "result must not be NULL");
    if (!(rtol >= 0.0) || !(atol >= 0.0) || max_it < 1) return fail(TB_EINVAL, "invalid PCG configuration");
    TB_CHECK(ensure_f64_pcg(s));
    std::memset(res, 0, sizeof(*res));
    double bn2 = 0.0;
    TB_CHECK(norm2(s, s->b64, &bn2));
    const double bnorm = std::sqrt(bn2);
    if (!std::isfinite(bnorm)) return fail(TB_ENONFINITE, "rhs must contain only finite values");
    const double scale = bnorm > 0.0 ? bnorm : 1.0;
    const double target = atol + rtol * scale;
    // PCG to the recursive target, then restarts from the iterate while the
    // true residual is above it (recursive and true residuals drift apart on
    // stiff stacks); at most 8 restarts.
    int total = 0;
    double true_norm = 0.0;
    for (int restart = 0;; ++restart) {
        double res2 = 0.0, peak = 0.0;
        TB_CHECK(residual64(s, &res2, &peak));
        true_norm = std::sqrt(res2);
        if (true_norm <= target || total >= max_it || restart > 8) break;
        set_ctl<<<1, 32, 0, s->stream>>>(s->ctl, target / scale, max_it - total, 1.0, scale);
        if (s->pcg64_ml) {
            TB_CUDA(ml_step64(s, true, false));
            s->kernel_launches += 1 + ml_kernels_per_step(s);
        } else {
            pcg_start_f64<<<s->vec_blocks, kVecThreads, 0, s->stream>>>(s->r64, s->p64, s->dinv64, s->nq, s->ctl,
                                                                         s->partials, s->counter);
            TB_CUDA(cudaGetLastError());
            s->kernel_launches += 2;
        }
        SolveCtl c;
        TB_CHECK(run_pcg(s, true, &c));
        if (c.state == ST_NOT_SPD) return fail(TB_ENOTSPD, "PCG requires a finite symmetric positive-definite operator");
        total += c.iterations;
        if (c.iterations == 0 && c.state != ST_RUNNING && c.state != ST_MAXIT) break;
    }
    res->iterations = total;
    res->relative_residual = true_norm / scale;
    res->converged = (true_norm <= target) ? 1 : 0;
    return TB_OK;
}

int finish_call_timing(tb_system* s, cudaEvent_t t0, cudaEvent_t t1) {
    TB_CUDA(cudaEventRecord(t1, s->stream));
    TB_CUDA(cudaEventSynchronize(t1));
    float ms = 0.f;
    TB_CUDA(cudaEventElapsedTime(&ms, t0, t1));
    s->ms[3] += ms;
    s->launches[3] += 1;
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    return TB_OK;
}

// ------------------------------------------------------ problem systems
// A board given as its problem (geometry, conductivities, masks, loads and
// convection boundaries) is prepared on the device: node masks, loads,
// lumped Robin terms, then the same solver arrays as tb_system_create.  The
// right-hand side and the post-processing of a solve run on the device too.

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

// Bytes of the element or plane fields of one convection boundary.
long long convection_field_count(const tb_convection_desc& c, const Layout& L) {
    return c.kind == TB_CONVECTION_FACE ? (long long)L.R * L.C : L.E;
}

int check_convection(const tb_convection_desc* c, int count) {
    if (count < 0 || count > TB_MAX_CONVECTION) return fail(TB_EINVAL, "at most %d convection boundaries", TB_MAX_CONVECTION);
    if (count > 0 && c == nullptr) return fail(TB_EINVAL, "convection boundaries are missing");
    for (int b = 0; b < count; ++b) {
        const tb_convection_desc& d = c[b];
        if (d.kind == TB_CONVECTION_FACE) {
            if (d.side != 0 && d.side != 1) return fail(TB_EINVAL, "side must be 0 (bottom) or 1 (top)");
        } else if (d.kind == TB_CONVECTION_EXPOSED) {
            if (d.direction_count < 1 || d.direction_count > 6)
                return fail(TB_EINVAL, "exposed-face convection needs 1 to 6 directions");
            int seen = 0;
            for (int k = 0; k < d.direction_count; ++k) {
                const int dir = d.directions[k];
                if (dir < 0 || dir > 5 || (seen >> dir) & 1) return fail(TB_EINVAL, "directions must be unique, 0..5");
                seen |= 1 << dir;
            }
        } else {
            return fail(TB_EINVAL, "convection kind must be TB_CONVECTION_FACE or TB_CONVECTION_EXPOSED");
        }
        if (!d.coefficient_field && !(std::isfinite(d.coefficient_w_per_m2_k) && d.coefficient_w_per_m2_k >= 0.0))
            return fail(TB_EINVAL, "film coefficient must be finite and non-negative");
        if (!d.ambient_field && !std::isfinite(d.ambient_temperature_k))
            return fail(TB_EINVAL, "ambient temperature must be finite");
    }
    return TB_OK;
}

int check_problem(const tb_problem_desc* d) {
    if (d == nullptr) return fail(TB_EINVAL, "problem description is NULL");
    if (d->slabs < 1 || d->rows < 1 || d->cols < 1) return fail(TB_EINVAL, "element grid must be positive");
    if (!d->slab_thickness_m || !d->pitch_x_m || !d->pitch_y_m || !d->k_in || !d->k_z)
        return fail(TB_EINVAL, "geometry or conductivity arrays are missing");
    const long long nodes = (long long)(d->slabs + 1) * (d->rows + 1) * (d->cols + 1);
    if (nodes > (1LL << 31) * 4) return fail(TB_EINVAL, "grid too large");
    auto positive = [](const double* v, int n) {
        for (int i = 0; i < n; ++i)
            if (!(std::isfinite(v[i]) && v[i] > 0.0)) return false;
        return true;
    };
    if (!positive(d->slab_thickness_m, d->slabs)) return fail(TB_EINVAL, "slab thicknesses must be finite and positive");
    if (!positive(d->pitch_x_m, d->cols)) return fail(TB_EINVAL, "pitch_x_m must be finite and positive");
    if (!positive(d->pitch_y_m, d->rows)) return fail(TB_EINVAL, "pitch_y_m must be finite and positive");
    if (d->fixed_mask && !d->fixed_temperature_k) return fail(TB_EINVAL, "fixed temperatures are missing");
    if (d->source_entries < 0 || (d->source_entries > 0 && (!d->source_nodes || !d->source_node_w)))
        return fail(TB_EINVAL, "heat source entries are missing");
    for (int i = 0; i < d->source_entries; ++i) {
        if (d->source_nodes[i] < 0 || d->source_nodes[i] >= nodes)
            return fail(TB_EINVAL, "heat source node %lld lies outside the grid", (long long)d->source_nodes[i]);
        if (!std::isfinite(d->source_node_w[i])) return fail(TB_EINVAL, "heat source power must be finite");
    }
    return check_convection(d->convection, d->convection_count);
}

// Read and clear the validation bits of the prep kernels.
int take_prep_errors(tb_system* s) {
    int err = 0;
    TB_CUDA(cudaMemcpyAsync(&err, s->d_err, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    TB_CUDA(cudaStreamSynchronize(s->stream));
    TB_CUDA(cudaMemsetAsync(s->d_err, 0, sizeof(int), s->stream));
    if (err & kErrConductivity) return fail(TB_EINVAL, "conductivities must be finite and non-negative");
    if (err & kErrCoefficient) return fail(TB_EINVAL, "film coefficient must be finite and non-negative");
    if (err & kErrAmbient) return fail(TB_EINVAL, "ambient temperature must be finite");
    if (err & kErrHeat) return fail(TB_EINVAL, "heat loads must be finite");
    if (err & kErrFixed) return fail(TB_EINVAL, "fixed temperatures must be finite");
    if (err & kErrCapacity) return fail(TB_EINVAL, "capacity_per_s must be finite and non-negative");
    return TB_OK;
}

// Sum over blocks of a two-quantity pass into s->sums[slot], slot .. slot+1.
int finish_pass(tb_system* s, int blocks, int slot) {
    finish_sums<<<1, 32, 0, s->stream>>>(s->sum_partials, blocks, 2, s->sums + slot);
    TB_CUDA(cudaGetLastError());
    s->kernel_launches += 1;
    return TB_OK;
}

// (Re)build the lumped Robin terms of `count` boundaries into robin_only /
// robin_rhs / robin_total and each boundary's own weights.  The coefficient
// and ambient fields are copied through `scratch` (device, scratch_bytes).
int lump_boundaries(tb_system* s, const tb_convection_desc* conv, int count, unsigned char* scratch,
                    size_t scratch_bytes) {
    const Layout& L = s->lay;
    for (auto& b : s->boundaries) {
        dev_free(s, b.w);
        dev_free(s, b.rw);
    }
    s->boundaries.assign((size_t)count, tb_system::Boundary{});
    if (s->sums) dev_free(s, s->sums);
    TB_CHECK(alloc_n(s, &s->sums, 2 * (long long)(count + 2)));
    TB_CUDA(cudaMemsetAsync(s->robin_only, 0, sizeof(double) * L.N, s->stream));
    TB_CUDA(cudaMemsetAsync(s->robin_rhs, 0, sizeof(double) * L.N, s->stream));
    const long long plane = (long long)(L.R + 1) * (L.C + 1);
    const int nb = grid_for(L.N, kVecThreads, s->sms * 16);
    size_t used = 0;
    for (int b = 0; b < count; ++b) {
        const tb_convection_desc& c = conv[b];
        ConvectionTerm t{};
        t.kind = c.kind == TB_CONVECTION_FACE ? 0 : 1;
        t.side = c.side;
        t.ndir = c.direction_count;
        for (int k = 0; k < 6; ++k) t.dirs[k] = k < c.direction_count ? c.directions[k] : 0;
        t.coef = c.coefficient_w_per_m2_k;
        t.amb = c.ambient_temperature_k;
        const long long fc = convection_field_count(c, L);
        const double* fields[2] = {c.coefficient_field, c.ambient_field};
        const double* dev_fields[2] = {nullptr, nullptr};
        for (int f = 0; f < 2; ++f) {
            if (!fields[f]) continue;
            const size_t bytes = sizeof(double) * (size_t)fc;
            if (used + bytes > scratch_bytes) return fail(TB_EINVAL, "internal: convection scratch too small");
            double* dst = reinterpret_cast<double*>(scratch + used);
            used = align256(used + bytes);
            TB_CHECK(host_to_device(s, dst, fields[f], bytes));
            check_field<<<grid_for(fc, kVecThreads, s->sms * 8), kVecThreads, 0, s->stream>>>(
                dst, fc, f == 0 ? 1 : 0, f == 0 ? kErrCoefficient : kErrAmbient, s->d_err);
            s->kernel_launches += 1;
            dev_fields[f] = dst;
        }
        t.coef_field = dev_fields[0];
        t.amb_field = dev_fields[1];
        tb_system::Boundary& bd = s->boundaries[(size_t)b];
        bd.kind = t.kind;
        if (t.kind == 0) {
            bd.offset = (long long)(t.side ? L.S : 0) * plane;
            bd.count = plane;
            TB_CHECK(alloc_n(s, &bd.w, plane));
            TB_CHECK(alloc_n(s, &bd.rw, plane));
            lump_outer_face<<<grid_for(plane, kVecThreads, s->sms * 16), kVecThreads, 0, s->stream>>>(
                bd.w, bd.rw, s->robin_only, s->robin_rhs, t, s->elem_active, s->dims64 + L.S, s->dims64 + L.S + L.C,
                L);
        } else {
            bd.offset = 0;
            bd.count = L.N;
            TB_CHECK(alloc_n(s, &bd.w, L.N));
            TB_CHECK(alloc_n(s, &bd.rw, L.N));
            lump_exposed_faces<<<nb, kVecThreads, 0, s->stream>>>(bd.w, bd.rw, s->robin_only, s->robin_rhs, t,
                                                                 s->elem_active, s->dims64, s->dims64 + L.S,
                                                                 s->dims64 + L.S + L.C, L);
        }
        TB_CUDA(cudaGetLastError());
        s->kernel_launches += 1;
        // sum of R T_amb of this boundary, the constant part of its removed heat
        const int blocks = std::min(s->sum_blocks, grid_for(bd.count, kSumThreads, s->sum_blocks));
        dot_sums<<<blocks, kSumThreads, 0, s->stream>>>(s->sum_partials, nullptr, bd.rw, bd.count);
        TB_CUDA(cudaGetLastError());
        s->kernel_launches += 1;
        TB_CHECK(finish_pass(s, blocks, 2 * (b + 2)));
    }
    prep_robin_total<<<nb, kVecThreads, 0, s->stream>>>(s->robin_total, s->robin_only, s->capacity, L.N);
    TB_CUDA(cudaGetLastError());
    s->kernel_launches += 1;
    std::vector<double> sums(2 * (size_t)(count + 2));
    TB_CUDA(cudaMemcpyAsync(sums.data(), s->sums, sizeof(double) * sums.size(), cudaMemcpyDeviceToHost, s->stream));
    TB_CUDA(cudaStreamSynchronize(s->stream));
    for (int b = 0; b < count; ++b) s->boundaries[(size_t)b].rw_sum = sums[2 * (size_t)(b + 2) + 1];
    return take_prep_errors(s);
}

size_t convection_scratch_bytes(const tb_convection_desc* conv, int count, const Layout& L) {
    size_t bytes = 0;
    for (int b = 0; b < count; ++b) {
        const size_t one = align256(sizeof(double) * (size_t)convection_field_count(conv[b], L));
        if (conv[b].coefficient_field) bytes += one;
        if (conv[b].ambient_field) bytes += one;
    }
    return bytes;
}

// C / dt per node (NULL: steady); validates, uploads and flags whether any is positive.
int upload_capacity(tb_system* s, const double* capacity) {
    const Layout& L = s->lay;
    if (capacity == nullptr) {
        if (s->capacity) dev_free(s, s->capacity);
        s->capacity_positive = false;
        return TB_OK;
    }
    bool positive = false;
    for (long long n = 0; n < L.N; ++n) {
        if (!(std::isfinite(capacity[n]) && capacity[n] >= 0.0))
            return fail(TB_EINVAL, "capacity_per_s must be finite and non-negative");
        positive = positive || capacity[n] > 0.0;
    }
    if (!s->capacity) TB_CHECK(alloc_n(s, &s->capacity, L.N));
    TB_CHECK(host_to_device(s, s->capacity, capacity, sizeof(double) * L.N));
    TB_CUDA(cudaStreamSynchronize(s->stream));  // the host array may go away after the call
    s->capacity_positive = positive;
    return TB_OK;
}

int create_problem_impl(const tb_problem_desc* d, int device, tb_system** out) {
    TB_CHECK(check_problem(d));
    TB_CHECK(begin_system(d->slabs, d->rows, d->cols, d->slab_thickness_m, d->pitch_x_m, d->pitch_y_m, device, out));
    tb_system* s = *out;
    s->problem = true;
    const Layout& L = s->lay;
    TB_CHECK(alloc_n(s, &s->node_flags, L.N));
    TB_CHECK(alloc_n(s, &s->load, L.N));
    TB_CHECK(alloc_n(s, &s->robin_only, L.N));
    TB_CHECK(alloc_n(s, &s->robin_total, L.N));
    TB_CHECK(alloc_n(s, &s->robin_rhs, L.N));
    TB_CHECK(alloc_n(s, &s->fixed_value, L.N));
    s->sum_blocks = s->sms * 4;
    TB_CHECK(alloc_n(s, &s->sum_partials, (long long)s->sum_blocks * 4));
    if (d->active) {
        TB_CHECK(alloc_n(s, &s->elem_active, L.E));
        TB_CHECK(host_to_device(s, s->elem_active, d->active, (size_t)L.E));
    }
    TB_CHECK(upload_capacity(s, d->capacity_per_s));

    // Staging: k_in, k_z, element heat (E doubles each), fixed values, nodal
    // heat (N doubles each), fixed mask and free mask (N bytes each), the
    // sorted heat-source entries and the convection fields.
    const int ns = d->source_entries;
    size_t off = 0;
    auto carve = [&](size_t bytes) {
        const size_t at = off;
        off = align256(off + bytes);
        return at;
    };
    const size_t o_kin = carve(sizeof(double) * (size_t)L.E);
    const size_t o_kz = carve(sizeof(double) * (size_t)L.E);
    const size_t o_eh = d->element_heat_w ? carve(sizeof(double) * (size_t)L.E) : 0;
    const size_t o_ft = d->fixed_mask ? carve(sizeof(double) * (size_t)L.N) : 0;
    const size_t o_nh = d->nodal_heat_w ? carve(sizeof(double) * (size_t)L.N) : 0;
    const size_t o_fm = d->fixed_mask ? carve((size_t)L.N) : 0;
    const size_t o_free = carve((size_t)L.N);
    const size_t o_src_n = carve(sizeof(long long) * (size_t)std::max(ns, 1));
    const size_t o_src_v = carve(sizeof(double) * (size_t)std::max(ns, 1));
    const size_t o_conv = off;
    const size_t conv_bytes = convection_scratch_bytes(d->convection, d->convection_count, L);
    TB_CHECK(ensure_stage(s, o_conv + conv_bytes + 256));
    unsigned char* st = static_cast<unsigned char*>(s->stage);
    double* st_kin = reinterpret_cast<double*>(st + o_kin);
    double* st_kz = reinterpret_cast<double*>(st + o_kz);
    double* st_eh = d->element_heat_w ? reinterpret_cast<double*>(st + o_eh) : nullptr;
    double* st_ft = d->fixed_mask ? reinterpret_cast<double*>(st + o_ft) : nullptr;
    double* st_nh = d->nodal_heat_w ? reinterpret_cast<double*>(st + o_nh) : nullptr;
    uint8_t* st_fm = d->fixed_mask ? st + o_fm : nullptr;
    uint8_t* st_free = st + o_free;
    long long* st_src_n = reinterpret_cast<long long*>(st + o_src_n);
    double* st_src_v = reinterpret_cast<double*>(st + o_src_v);
    TB_CHECK(host_to_device(s, st_kin, d->k_in, sizeof(double) * L.E));
    TB_CHECK(host_to_device(s, st_kz, d->k_z, sizeof(double) * L.E));
    if (st_eh) TB_CHECK(host_to_device(s, st_eh, d->element_heat_w, sizeof(double) * L.E));
    if (st_ft)
        TB_CHECK(host_to_device(s, st_ft, d->fixed_temperature_k, sizeof(double) * L.N));
    if (st_nh) TB_CHECK(host_to_device(s, st_nh, d->nodal_heat_w, sizeof(double) * L.N));
    if (st_fm) TB_CHECK(host_to_device(s, st_fm, d->fixed_mask, (size_t)L.N));
    // heat-source entries sorted by node, stable in source order
    std::vector<long long> src_n((size_t)ns);
    std::vector<double> src_v((size_t)ns);
    if (ns > 0) {
        std::vector<int> order((size_t)ns);
        for (int i = 0; i < ns; ++i) order[(size_t)i] = i;
        std::stable_sort(order.begin(), order.end(),
                         [&](int a, int b) { return d->source_nodes[a] < d->source_nodes[b]; });
        for (int i = 0; i < ns; ++i) {
            src_n[(size_t)i] = d->source_nodes[order[(size_t)i]];
            src_v[(size_t)i] = d->source_node_w[order[(size_t)i]];
        }
        TB_CUDA(cudaMemcpyAsync(st_src_n, src_n.data(), sizeof(long long) * ns, cudaMemcpyHostToDevice, s->stream));
        TB_CUDA(cudaMemcpyAsync(st_src_v, src_v.data(), sizeof(double) * ns, cudaMemcpyHostToDevice, s->stream));
    }

    const int eb = grid_for(L.E, kVecThreads, s->sms * 16);
    const int nb = grid_for(L.N, kVecThreads, s->sms * 16);
    check_elements<<<eb, kVecThreads, 0, s->stream>>>(st_kin, st_kz, st_eh, s->d_err, L.E);
    check_nodes<<<nb, kVecThreads, 0, s->stream>>>(st_nh, st_fm, st_ft, nullptr, s->d_err, L.N);
    prep_nodes<<<nb, kVecThreads, 0, s->stream>>>(s->node_flags, st_free, s->fixed_value, s->elem_active, st_fm, st_ft,
                                                  L);
    prep_load<<<nb, kVecThreads, 0, s->stream>>>(s->load, st_nh, st_eh, L);
    if (ns > 0) prep_sources<<<(ns + 255) / 256, 256, 0, s->stream>>>(s->load, st_src_n, st_src_v, ns);
    TB_CUDA(cudaGetLastError());
    s->kernel_launches += 4 + (ns > 0 ? 1 : 0);
    {
        const int blocks = std::min(s->sum_blocks, grid_for(L.N, kSumThreads, s->sum_blocks));
        TB_CHECK(alloc_n(s, &s->sums, 4));
        dot_sums<<<blocks, kSumThreads, 0, s->stream>>>(s->sum_partials, nullptr, s->load, L.N);
        TB_CUDA(cudaGetLastError());
        s->kernel_launches += 1;
        TB_CHECK(finish_pass(s, blocks, 0));
        double sums[2] = {0.0, 0.0};
        TB_CUDA(cudaMemcpyAsync(sums, s->sums, sizeof(sums), cudaMemcpyDeviceToHost, s->stream));
        TB_CUDA(cudaStreamSynchronize(s->stream));
        s->total_load = sums[1];
    }
    TB_CHECK(take_prep_errors(s));
    TB_CHECK(lump_boundaries(s, d->convection, d->convection_count, st + o_conv, conv_bytes + 256));
    // robin_total holds the Robin totals on every node; the solver arrays take them with the free mask
    return finish_system(s, st_kin, st_kz, s->robin_total, st_free);
}

int require_problem(tb_system* s) {
    if (!s) return fail(TB_EINVAL, "system is NULL");
    if (!s->problem) return fail(TB_EINVAL, "the system was not made from a problem (tb_system_create_problem)");
    return TB_OK;
}

// Upload an optional flat node array into the stage at byte offset `at`.
int stage_nodes(tb_system* s, const double* host, size_t at, const double** dev) {
    *dev = nullptr;
    if (!host) return TB_OK;
    double* dst = reinterpret_cast<double*>(static_cast<unsigned char*>(s->stage) + at);
    TB_CHECK(host_to_device(s, dst, host, sizeof(double) * (size_t)s->lay.N));
    *dev = dst;
    return TB_OK;
}

// The right-hand side for a reference temperature.  `on_device`: the
// previous temperature and the output are flat device arrays (the output is
// written in place, nothing crosses to the host); otherwise both are host
// arrays, staged through the system's buffer.
int build_rhs_impl(tb_system* s, double reference, const double* previous, double* rhs_out, bool on_device = false) {
    const Layout& L = s->lay;
    if (!std::isfinite(reference)) return fail(TB_EINVAL, "reference_temperature_k must be finite");
    if (s->capacity_positive && !previous) return fail(TB_EINVAL, "a transient operator needs previous_temperature_k");
    const size_t nbytes = align256(sizeof(double) * (size_t)L.N);
    TB_CUDA(cudaStreamSynchronize(s->stream));
    const double* prev = nullptr;
    double* rhs = nullptr;
    if (on_device) {
        prev = previous;
        rhs = rhs_out;
    } else {
        TB_CHECK(ensure_stage(s, 2 * nbytes));
        TB_CHECK(stage_nodes(s, previous, 0, &prev));
        rhs = reinterpret_cast<double*>(static_cast<unsigned char*>(s->stage) + nbytes);
    }
    const int pb = grid_for(L.L, kVecThreads, s->sms * 16);
    const int nb = grid_for(L.N, kVecThreads, s->sms * 16);
    prep_shifted<<<pb, kVecThreads, 0, s->stream>>>(s->b64, s->fixed_value, s->node_flags, reference, L);
    TB_CUDA(cudaGetLastError());
    const ApplyParams<double> P = apply_params<double>(s, s->b64, s->r64, nullptr);
    TB_CHECK((launch_apply<double, MODE_STIFFNESS, EPI_STORE>(s, P)));
    prep_rhs<<<nb, kVecThreads, 0, s->stream>>>(rhs, s->load, s->robin_rhs, s->robin_total, s->capacity, prev,
                                                s->fixed_value, s->node_flags, s->r64, reference, L);
    TB_CUDA(cudaGetLastError());
    s->kernel_launches += 3;
    if (rhs_out && !on_device) TB_CHECK(device_to_host(s, rhs_out, rhs, sizeof(double) * L.N));
    TB_CUDA(cudaStreamSynchronize(s->stream));
    return TB_OK;
}

// Post-processing of a temperature field.  The field is a host array, or,
// with `rise_on_device`, a flat device array of the rise over `reference`
// (the solve's own solution): T = rise + reference is formed on the device,
// as the host would form it, and never crosses to the host and back.
int postprocess_impl(tb_system* s, const double* temperature, const double* previous, double* flux_out,
                     double* convective_out, double* budget3, double* residual_out, bool rise_on_device = false,
                     double reference = 0.0, double* temperature_out = nullptr, double* extrema_out = nullptr) {
    const Layout& L = s->lay;
    if (!temperature) return fail(TB_EINVAL, "temperature is NULL");
    if (rise_on_device && !std::isfinite(reference)) return fail(TB_EINVAL, "reference_temperature_k must be finite");
    const size_t nbytes = align256(sizeof(double) * (size_t)L.N);
    const size_t fbytes = align256(sizeof(double) * 3 * (size_t)L.E);
    TB_CUDA(cudaStreamSynchronize(s->stream));
    TB_CHECK(ensure_stage(s, 3 * nbytes + (flux_out ? fbytes : 0)));
    unsigned char* st = static_cast<unsigned char*>(s->stage);
    const double* t = nullptr;
    const double* prev = nullptr;
    if (rise_on_device) {
        double* shifted = reinterpret_cast<double*>(st);
        shift_nodes<<<grid_for(L.N, kVecThreads, s->sms * 16), kVecThreads, 0, s->stream>>>(shifted, temperature,
                                                                                            reference, L.N);
        TB_CUDA(cudaGetLastError());
        s->kernel_launches += 1;
        t = shifted;
        if (extrema_out) {
            if (!s->extrema) TB_CHECK(alloc_n(s, &s->extrema, 2));
            const int blocks = std::min(s->partial_blocks, grid_for(L.N, 256, s->sms * 8));
            node_extrema<<<blocks, 256, 0, s->stream>>>(shifted, s->node_flags, L.N, s->partials, s->counter,
                                                        s->extrema);
            TB_CUDA(cudaGetLastError());
            s->kernel_launches += 1;
            TB_CUDA(cudaMemcpyAsync(extrema_out, s->extrema, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
        }
        if (temperature_out) TB_CHECK(device_to_host(s, temperature_out, shifted, sizeof(double) * (size_t)L.N));
    } else {
        TB_CHECK(stage_nodes(s, temperature, 0, &t));
    }
    TB_CHECK(stage_nodes(s, previous, nbytes, &prev));
    double* residual = residual_out ? reinterpret_cast<double*>(st + 2 * nbytes) : nullptr;
    double* flux = flux_out ? reinterpret_cast<double*>(st + 3 * nbytes) : nullptr;
    // conduction K T
    TB_CHECK(load_nodes<double>(s, s->b64, t, true));
    const ApplyParams<double> P = apply_params<double>(s, s->b64, s->r64, nullptr);
    TB_CHECK((launch_apply<double, MODE_STIFFNESS, EPI_STORE>(s, P)));
    const int count = (int)s->boundaries.size();
    {
        const int blocks = std::min(s->sum_blocks, grid_for(L.N, kSumThreads, s->sum_blocks));
        post_nodes<<<blocks, kSumThreads, 0, s->stream>>>(residual, s->sum_partials, t, s->r64, s->robin_only,
                                                          s->robin_rhs, s->load, s->capacity, prev, s->node_flags, L);
        TB_CUDA(cudaGetLastError());
        s->kernel_launches += 2;
        TB_CHECK(finish_pass(s, blocks, 0));
    }
    for (int b = 0; b < count; ++b) {
        const tb_system::Boundary& bd = s->boundaries[(size_t)b];
        const int blocks = std::min(s->sum_blocks, grid_for(bd.count, kSumThreads, s->sum_blocks));
        dot_sums<<<blocks, kSumThreads, 0, s->stream>>>(s->sum_partials, bd.w, t + bd.offset, bd.count);
        TB_CUDA(cudaGetLastError());
        s->kernel_launches += 1;
        TB_CHECK(finish_pass(s, blocks, 2 * (b + 2)));
    }
    if (flux) {
        element_flux<<<grid_for(L.E, kVecThreads, s->sms * 16), kVecThreads, 0, s->stream>>>(
            flux, t, s->kin64, s->kz64, s->dims64, s->dims64 + L.S, s->dims64 + L.S + L.C, s->elem_active, L);
        TB_CUDA(cudaGetLastError());
        s->kernel_launches += 1;
        TB_CHECK(device_to_host(s, flux_out, flux, sizeof(double) * 3 * L.E));
    }
    if (residual) TB_CHECK(device_to_host(s, residual_out, residual, sizeof(double) * L.N));
    std::vector<double> sums(2 * (size_t)(count + 2));
    TB_CUDA(cudaMemcpyAsync(sums.data(), s->sums, sizeof(double) * sums.size(), cudaMemcpyDeviceToHost, s->stream));
    TB_CUDA(cudaStreamSynchronize(s->stream));
    if (convective_out)
        for (int b = 0; b < count; ++b) convective_out[b] = sums[2 * (size_t)(b + 2)] - s->boundaries[(size_t)b].rw_sum;
    if (budget3) {
        budget3[0] = s->total_load;
        budget3[1] = sums[0];
        budget3[2] = sums[1];
    }
    return TB_OK;
}

// ------------------------------------------------------- layered DC systems
// The reference's LayeredDCSystem / MatrixFreePCBOperator preparation
// (pcb.py:275-400, layered_dc_system.cpp): active nodes (the corners of
// active elements and the via ends), fixed nodes (not active, the reference
// node, the Dirichlet nodes), sheet conductance sigma t per element, the via
// lists per node, then the free mask, rf and the diagonal on the device.
int check_dc(const tb_dc_desc* d) {
    if (d == nullptr) return fail(TB_EINVAL, "DC description is NULL");
    if (d->layers < 1 || d->rows < 1 || d->cols < 1) return fail(TB_EINVAL, "element grid must be positive");
    if (!d->layer_thickness_m || !d->pitch_x_m || !d->pitch_y_m || !d->conductivity_s_per_m || !d->element_active)
        return fail(TB_EINVAL, "mesh arrays are missing");
    const long long nodes = (long long)d->layers * (d->rows + 1) * (d->cols + 1);
    if (nodes > (1LL << 31) * 4) return fail(TB_EINVAL, "grid too large");
    auto positive = [](const double* v, long long n) {
        for (long long i = 0; i < n; ++i)
            if (!(std::isfinite(v[i]) && v[i] > 0.0)) return false;
        return true;
    };
    if (!positive(d->layer_thickness_m, d->layers)) return fail(TB_EINVAL, "layer thicknesses must be finite and positive");
    if (!positive(d->pitch_x_m, d->cols)) return fail(TB_EINVAL, "pitch_x_m must be finite and positive");
    if (!positive(d->pitch_y_m, d->rows)) return fail(TB_EINVAL, "pitch_y_m must be finite and positive");
    if (!positive(d->conductivity_s_per_m, (long long)d->layers * d->rows * d->cols))
        return fail(TB_EINVAL, "conductivity must be finite and positive");
    if (d->via_count < 0 || (d->via_count > 0 && (!d->via_lower || !d->via_upper || !d->via_conductance_s)))
        return fail(TB_EINVAL, "via arrays are missing");
    const long long plane = (long long)(d->rows + 1) * (d->cols + 1);
    for (int v = 0; v < d->via_count; ++v) {
        const long long a = d->via_lower[v], b = d->via_upper[v];
        if (a < 0 || a >= nodes || b < 0 || b >= nodes) return fail(TB_EINVAL, "via %d has an end outside the grid", v);
        if (a / plane == b / plane) return fail(TB_EINVAL, "a via must connect different layers");
        if (!(std::isfinite(d->via_conductance_s[v]) && d->via_conductance_s[v] > 0.0))
            return fail(TB_EINVAL, "via conductance must be finite and positive");
    }
    if (d->reference_node < -1 || d->reference_node >= nodes) return fail(TB_EINVAL, "reference_node lies outside the grid");
    if (d->dirichlet_count < 0 || (d->dirichlet_count > 0 && !d->dirichlet_nodes))
        return fail(TB_EINVAL, "Dirichlet nodes are missing");
    for (int i = 0; i < d->dirichlet_count; ++i)
        if (d->dirichlet_nodes[i] < 0 || d->dirichlet_nodes[i] >= nodes)
            return fail(TB_EINVAL, "a Dirichlet node lies outside the grid");
    if (d->reference_node < 0 && d->dirichlet_count == 0)
        return fail(TB_EINVAL, "pass a reference_node or dirichlet_nodes to fix the potential");
    return TB_OK;
}

int create_dc_impl(const tb_dc_desc* d, int device, tb_system** out) {
    TB_CHECK(check_dc(d));
    const int Ly = d->layers, R = d->rows, C = d->cols;
    const long long plane = (long long)(R + 1) * (C + 1), nodes = (long long)Ly * plane;
    // masks on the host, in the reference's node order
    std::vector<uint8_t> active((size_t)nodes, 0), fixed((size_t)nodes, 0);
    for (int l = 0; l < Ly; ++l)
        for (int y = 0; y < R; ++y)
            for (int x = 0; x < C; ++x) {
                if (!d->element_active[((long long)l * R + y) * C + x]) continue;
                const long long n = (long long)l * plane + (long long)y * (C + 1) + x;
                active[(size_t)n] = active[(size_t)(n + 1)] = 1;
                active[(size_t)(n + C + 1)] = active[(size_t)(n + C + 2)] = 1;
            }
    for (int v = 0; v < d->via_count; ++v) active[(size_t)d->via_lower[v]] = active[(size_t)d->via_upper[v]] = 1;
    for (long long n = 0; n < nodes; ++n) fixed[(size_t)n] = active[(size_t)n] ? 0 : 1;
    if (d->reference_node >= 0) {
        if (!active[(size_t)d->reference_node])
            return fail(TB_EINVAL, "reference_node must lie on active copper or a via endpoint");
        fixed[(size_t)d->reference_node] = 1;
    }
    for (int i = 0; i < d->dirichlet_count; ++i) {
        if (!active[(size_t)d->dirichlet_nodes[i]])
            return fail(TB_EINVAL, "dirichlet_nodes must lie on active copper or via endpoints");
        fixed[(size_t)d->dirichlet_nodes[i]] = 1;
    }
    // the solver layout takes the layers as node planes (S = layers - 1 slabs)
    TB_CHECK(begin_system(Ly - 1, R, C, d->layer_thickness_m, d->pitch_x_m, d->pitch_y_m, device, out, Ly));
    tb_system* s = *out;
    s->physics = 1;
    const Layout& L = s->lay;
    auto padded = [&](long long n) {
        const long long line = n / (C + 1);
        return line * L.Xp + (n - line * (C + 1));
    };
    // node bits: free, via end, active
    std::vector<uint8_t> mask((size_t)L.L, 0);
    for (long long n = 0; n < nodes; ++n)
        mask[(size_t)padded(n)] = (uint8_t)((fixed[(size_t)n] ? 0 : kDcFree) | (active[(size_t)n] ? 4 : 0));
    // via lists: per node, its vias as the lower end (via order), then as the upper end
    std::map<long long, std::vector<std::pair<long long, double>>> lists;
    for (int v = 0; v < d->via_count; ++v)
        lists[padded(d->via_lower[v])].emplace_back(padded(d->via_upper[v]), d->via_conductance_s[v]);
    for (int v = 0; v < d->via_count; ++v)
        lists[padded(d->via_upper[v])].emplace_back(padded(d->via_lower[v]), d->via_conductance_s[v]);
    std::vector<long long> vnode, vother;
    std::vector<int> vstart(1, 0);
    std::vector<double> vg64;
    std::vector<float> vg32;
    for (const auto& kv : lists) {
        vnode.push_back(kv.first);
        mask[(size_t)kv.first] |= kDcVia;
        for (const auto& e : kv.second) {
            vother.push_back(e.first);
            vg64.push_back(e.second);
            vg32.push_back((float)e.second);
        }
        vstart.push_back((int)vother.size());
    }
    s->via_nodes = (int)vnode.size();
    TB_CHECK(alloc_n(s, &s->dc_mask, L.L));
    TB_CHECK(alloc_n(s, &s->via_slot, L.L));
    TB_CHECK(alloc_n(s, &s->via_start, (long long)vstart.size()));
    TB_CHECK(alloc_n(s, &s->via_other, std::max<long long>(1, (long long)vother.size())));
    TB_CHECK(alloc_n(s, &s->via_g64, std::max<long long>(1, (long long)vg64.size())));
    TB_CHECK(alloc_n(s, &s->via_g32, std::max<long long>(1, (long long)vg32.size())));
    {
        std::vector<double> h64((size_t)L.Xp, 0.0), ih64((size_t)L.Xp, 0.0);
        std::vector<float> h32((size_t)L.Xp, 0.f), ih32((size_t)L.Xp, 0.f);
        for (int x = 0; x < C; ++x) {
            h64[(size_t)x] = d->pitch_x_m[x];
            ih64[(size_t)x] = 1.0 / d->pitch_x_m[x];
            h32[(size_t)x] = (float)h64[(size_t)x];
            ih32[(size_t)x] = (float)ih64[(size_t)x];
        }
        TB_CHECK(alloc_n(s, &s->dc_colh64, L.Xp));
        TB_CHECK(alloc_n(s, &s->dc_colih64, L.Xp));
        TB_CHECK(alloc_n(s, &s->dc_colh32, L.Xp));
        TB_CHECK(alloc_n(s, &s->dc_colih32, L.Xp));
        TB_CUDA(cudaMemcpy(s->dc_colh64, h64.data(), sizeof(double) * L.Xp, cudaMemcpyHostToDevice));
        TB_CUDA(cudaMemcpy(s->dc_colih64, ih64.data(), sizeof(double) * L.Xp, cudaMemcpyHostToDevice));
        TB_CUDA(cudaMemcpy(s->dc_colh32, h32.data(), sizeof(float) * L.Xp, cudaMemcpyHostToDevice));
        TB_CUDA(cudaMemcpy(s->dc_colih32, ih32.data(), sizeof(float) * L.Xp, cudaMemcpyHostToDevice));
    }
    // sheet conductance (sigma t) active, in the reference's rounding order
    std::vector<double> sheet((size_t)L.E);
    for (int l = 0; l < Ly; ++l)
        for (long long e = 0; e < (long long)R * C; ++e) {
            const long long i = (long long)l * R * C + e;
            sheet[(size_t)i] = (d->conductivity_s_per_m[i] * d->layer_thickness_m[l]) * (d->element_active[i] ? 1.0 : 0.0);
        }
    TB_CHECK(ensure_stage(s, sizeof(double) * (size_t)L.E + 64));
    TB_CHECK(host_to_device(s, s->stage, sheet.data(), sizeof(double) * L.E));
    TB_CUDA(cudaMemcpyAsync(s->dc_mask, mask.data(), (size_t)L.L, cudaMemcpyHostToDevice, s->stream));
    std::vector<int> slots((size_t)L.L, -1);
    for (size_t i = 0; i < vnode.size(); ++i) slots[(size_t)vnode[i]] = (int)i;
    TB_CUDA(cudaMemcpyAsync(s->via_slot, slots.data(), sizeof(int) * (size_t)L.L, cudaMemcpyHostToDevice, s->stream));
    if (!vnode.empty()) {
        TB_CUDA(cudaMemcpyAsync(s->via_other, vother.data(), sizeof(long long) * vother.size(),
                                cudaMemcpyHostToDevice, s->stream));
        TB_CUDA(cudaMemcpyAsync(s->via_g64, vg64.data(), sizeof(double) * vg64.size(), cudaMemcpyHostToDevice,
                                s->stream));
        TB_CUDA(cudaMemcpyAsync(s->via_g32, vg32.data(), sizeof(float) * vg32.size(), cudaMemcpyHostToDevice,
                                s->stream));
    }
    TB_CUDA(cudaMemcpyAsync(s->via_start, vstart.data(), sizeof(int) * vstart.size(), cudaMemcpyHostToDevice,
                            s->stream));
    const int eb = grid_for(L.LE, kVecThreads, s->sms * 16);
    const int nb = grid_for(L.L, kVecThreads, s->sms * 16);
    pack_elements<<<eb, kVecThreads, 0, s->stream>>>(s->kin64, s->kin32, static_cast<const double*>(s->stage), L);
    dc_build_rf<<<nb, kVecThreads, 0, s->stream>>>(s->rf64, s->rf32, s->dc_mask, L.L);
    DcVias<double> vias{s->via_slot, s->via_start, s->via_other, s->via_g64, s->via_nodes};
    dc_build_diagonal<<<nb, kVecThreads, 0, s->stream>>>(s->diag64, s->dinv64, s->dinv32, s->d_err, s->kin64,
                                                         s->dc_mask, s->dims64 + L.S, s->dims64 + L.S + L.C, vias,
                                                         Ly, R, C, L.Xp, L.Xe);
    TB_CUDA(cudaGetLastError());
    s->kernel_launches += 3;
    int err = 0;
    TB_CUDA(cudaMemcpyAsync(&err, s->d_err, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    TB_CUDA(cudaStreamSynchronize(s->stream));
    if (err) return fail(TB_EINVAL, "every free node must have positive conductivity coupling");
    s->special_mask = 0;
    return TB_OK;
}

// ------------------------------------------------- allocation-free scratch
// Scratch of tb_residual_f64_device_static, the entry point for callers that
// may not allocate device memory (their memory belongs to another allocator,
// or cudaMalloc's implicit synchronisation is not acceptable where they run):
// the block partials of the residual epilogue (4 doubles per tile), its ticket
// counter and the scalars the last block finishes, in one statically
// allocated device array that every GPU loading this library holds until the
// process exits.  Every system on a device shares it.
constexpr int kStaticMaxTiles = 8192;
constexpr size_t kStaticCounterOffset = (size_t)kStaticMaxTiles * 4 * sizeof(double);  // 256 KiB of partials
constexpr size_t kStaticCtlOffset = kStaticCounterOffset + 256;
constexpr size_t kStaticScratchBytes = kStaticCtlOffset + 256;
static_assert(sizeof(g_static_scratch) == kStaticScratchBytes, "layout matches the array");
static_assert(sizeof(SolveCtl) <= 256, "the scalars fit their 256-byte slot");
static_assert(offsetof(SolveCtl, peak) == offsetof(SolveCtl, res2) + sizeof(double), "res2 and peak are adjacent");

// Device address of g_static_scratch on `device` (the current device),
// looked up once per device.  The lookup may load the module on first use,
// so the first call on a device must not fall inside a stream capture.
int static_scratch_base(int device, unsigned char** out) {
    static std::mutex mu;
    static std::map<int, unsigned char*> bases;
    std::lock_guard<std::mutex> lock(mu);
    const auto it = bases.find(device);
    if (it != bases.end()) {
        *out = it->second;
        return TB_OK;
    }
    void* p = nullptr;
    TB_CUDA(cudaGetSymbolAddress(&p, g_static_scratch));
    if (p == nullptr || (reinterpret_cast<uintptr_t>(p) & 255u) != 0)
        return fail(TB_ECUDA, "static scratch is not 256-byte aligned");
    bases[device] = static_cast<unsigned char*>(p);
    *out = static_cast<unsigned char*>(p);
    return TB_OK;
}

}  // namespace

// ===================================================================== C ABI
extern "C" {

const char* tb_version(void) { return "thermal_b200 0.1 (sm_100a)"; }

const char* tb_last_error(void) { return g_last_error.c_str(); }

int tb_device_count(int32_t* count) {
    if (!count) return fail(TB_EINVAL, "count is NULL");
    int n = 0;
    const cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        cudaGetLastError();
        n = 0;
    }
    *count = n;
    return TB_OK;
}

int tb_system_create(const tb_system_desc* desc, int32_t device, tb_system** out) {
    if (!out) return fail(TB_EINVAL, "out is NULL");
    *out = nullptr;
    tb_system* s = nullptr;
    const int rc = create_impl(desc, device, &s);
    if (rc != TB_OK) {
        destroy_impl(s);
        return rc;
    }
    *out = s;
    return TB_OK;
}

int tb_system_destroy(tb_system* system) {
    destroy_impl(system);
    return TB_OK;
}

int tb_system_info(const tb_system* s, int64_t* nodes, int64_t* device_bytes) {
    if (!s) return fail(TB_EINVAL, "system is NULL");
    if (nodes) *nodes = s->lay.N;
    if (device_bytes) *device_bytes = (int64_t)s->bytes;
    return TB_OK;
}

static int apply_any(tb_system* s, const void* x, void* y, bool f64, bool dev, bool stiffness) {
    if (!s || !x || !y) return fail(TB_EINVAL, "NULL argument");
    TB_CUDA(cudaSetDevice(s->device));
    if (f64) {
        TB_CHECK(load_nodes<double>(s, s->b64, static_cast<const double*>(x), dev));
        const ApplyParams<double> P = apply_params<double>(s, s->b64, s->r64, nullptr);
        if (stiffness)
            TB_CHECK((launch_apply<double, MODE_STIFFNESS, EPI_STORE>(s, P)));
        else
            TB_CHECK((launch_apply<double, MODE_OPERATOR, EPI_STORE>(s, P)));
        TB_CHECK(store_nodes<double>(s, static_cast<double*>(y), s->r64, dev));
    } else {
        TB_CHECK(load_nodes<float>(s, s->p32, static_cast<const float*>(x), dev));
        const ApplyParams<float> P = apply_params<float>(s, s->p32, s->q32, nullptr);
        TB_CHECK((launch_apply<float, MODE_OPERATOR, EPI_STORE>(s, P)));
        TB_CHECK(check_stage(s));
        TB_CHECK(store_nodes<float>(s, static_cast<float*>(y), s->q32, dev));
    }
    s->kernel_launches += 1;
    if (dev) TB_CUDA(cudaStreamSynchronize(s->stream));
    return TB_OK;
}

int tb_apply_f32(tb_system* s, const float* x, float* y) { return apply_any(s, x, y, false, false, false); }
int tb_apply_f64(tb_system* s, const double* x, double* y) { return apply_any(s, x, y, true, false, false); }
int tb_apply_f32_device(tb_system* s, const float* x, float* y) { return apply_any(s, x, y, false, true, false); }
int tb_apply_f64_device(tb_system* s, const double* x, double* y) { return apply_any(s, x, y, true, true, false); }
int tb_stiffness_f64(tb_system* s, const double* x, double* y) { return apply_any(s, x, y, true, false, true); }

int tb_diagonal(tb_system* s, double* diagonal) {
    if (!s || !diagonal) return fail(TB_EINVAL, "NULL argument");
    TB_CUDA(cudaSetDevice(s->device));
    return store_nodes<double>(s, diagonal, s->diag64, false);
}

static int solve_mpir_any(tb_system* s, const double* rhs, double* x, const tb_mpir_config* cfg, tb_mpir_result* res,
                          tb_mpir_step* hist, int32_t cap, bool dev) {
    if (!s || !rhs || !x) return fail(TB_EINVAL, "NULL argument");
    TB_CUDA(cudaSetDevice(s->device));
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    if (s->timing) {
        TB_CUDA(cudaEventCreate(&t0));
        TB_CUDA(cudaEventCreate(&t1));
        TB_CUDA(cudaEventRecord(t0, s->stream));
    }
    TB_CHECK(load_nodes<double>(s, s->b64, rhs, dev));
    TB_CHECK(load_nodes<double>(s, s->x64, x, dev));
    TB_CHECK(mpir_impl(s, cfg, res, hist, hist ? cap : 0));
    TB_CHECK(store_nodes<double>(s, x, s->x64, dev));
    if (dev) TB_CUDA(cudaStreamSynchronize(s->stream));
    if (s->timing) TB_CHECK(finish_call_timing(s, t0, t1));
    return TB_OK;
}

int tb_solve_mpir(tb_system* s, const double* rhs, double* x, const tb_mpir_config* cfg, tb_mpir_result* res,
                  tb_mpir_step* hist, int32_t cap) {
    return solve_mpir_any(s, rhs, x, cfg, res, hist, cap, false);
}

int tb_solve_mpir_device(tb_system* s, const double* rhs, double* x, const tb_mpir_config* cfg, tb_mpir_result* res,
                         tb_mpir_step* hist, int32_t cap) {
    return solve_mpir_any(s, rhs, x, cfg, res, hist, cap, true);
}

static int pcg64_any(tb_system* s, const double* rhs, double* x, double rtol, double atol, int32_t max_it,
                     tb_pcg_result* res, bool dev) {
    if (!s || !rhs || !x) return fail(TB_EINVAL, "NULL argument");
    TB_CUDA(cudaSetDevice(s->device));
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    if (s->timing) {
        TB_CUDA(cudaEventCreate(&t0));
        TB_CUDA(cudaEventCreate(&t1));
        TB_CUDA(cudaEventRecord(t0, s->stream));
    }
    TB_CHECK(load_nodes<double>(s, s->b64, rhs, dev));
    TB_CHECK(load_nodes<double>(s, s->x64, x, dev));
    TB_CHECK(pcg64_impl(s, rtol, atol, max_it, res));
    TB_CHECK(store_nodes<double>(s, x, s->x64, dev));
    if (dev) TB_CUDA(cudaStreamSynchronize(s->stream));
    if (s->timing) TB_CHECK(finish_call_timing(s, t0, t1));
    return TB_OK;
}

static int pcg64_ml_any(tb_system* s, const double* rhs, double* x, double rtol, double atol, int32_t max_it,
                        tb_pcg_result* res, bool dev) {
    if (!s) return fail(TB_EINVAL, "system is NULL");
    if (s->precond != 2) return fail(TB_EINVAL, "the multilevel preconditioner is not set");
    s->pcg64_ml = true;
    const int rc = pcg64_any(s, rhs, x, rtol, atol, max_it, res, dev);
    s->pcg64_ml = false;
    return rc;
}

int tb_solve_pcg_f64_ml(tb_system* s, const double* rhs, double* x, double rtol, double atol, int32_t max_it,
                        tb_pcg_result* res) {
    return pcg64_ml_any(s, rhs, x, rtol, atol, max_it, res, false);
}

int tb_solve_pcg_f64_ml_device(tb_system* s, const double* rhs, double* x, double rtol, double atol, int32_t max_it,
                               tb_pcg_result* res) {
    return pcg64_ml_any(s, rhs, x, rtol, atol, max_it, res, true);
}

int tb_solve_pcg_f64(tb_system* s, const double* rhs, double* x, double rtol, double atol, int32_t max_it,
                     tb_pcg_result* res) {
    return pcg64_any(s, rhs, x, rtol, atol, max_it, res, false);
}

int tb_solve_pcg_f64_device(tb_system* s, const double* rhs, double* x, double rtol, double atol, int32_t max_it,
                            tb_pcg_result* res) {
    return pcg64_any(s, rhs, x, rtol, atol, max_it, res, true);
}

int tb_set_timing(tb_system* s, int32_t enabled) {
    if (!s) return fail(TB_EINVAL, "system is NULL");
    TB_CUDA(cudaSetDevice(s->device));
    s->timing = enabled != 0;
    for (int i = 0; i < 4; ++i) {
        s->ms[i] = 0.0;
        s->launches[i] = 0;
    }
    if (s->timing && s->tev[0] == nullptr) {
        TB_CUDA(cudaEventCreate(&s->tev[0]));
        TB_CUDA(cudaEventCreate(&s->tev[1]));
    }
    return TB_OK;
}

int tb_set_apply_plan(tb_system* s, const int32_t* plan5) {
    if (!s || !plan5) return fail(TB_EINVAL, "NULL argument");
    ApplyPlan p;
    p.kind = plan5[0];
    p.rows = plan5[1];
    p.zw = plan5[2];
    p.sl = plan5[3];
    p.band = plan5[4];
    if (p.rows != 8 && p.rows != 16 && p.rows != 32) return fail(TB_EINVAL, "tile rows must be 8, 16 or 32");
    if (p.kind != 1) {  // z-march kinds: plan5[2] selects the staging, plan5[3] the stage count (0: default)
        p.tma = p.zw;
        p.stages = p.sl == 0 ? kStages : p.sl;
        p.zw = p.sl = p.band = 0;
        if (p.tma != 0 && p.tma != 1) return fail(TB_EINVAL, "z-march staging must be 0 (cp.async) or 1 (tensor copies)");
        if (p.tma == 1 && !s->maps_ok) return fail(TB_ENOTSUP, "tensor-copy staging is not available for this system");
        if (p.stages != kStages && !(p.stages == kDeepStages && p.kind == 0 && p.tma == 1 && p.rows <= 16))
            return fail(TB_EINVAL, "%d stages are built for tensor-copy z-march tiles of 8 or 16 rows only",
                        kDeepStages);
    }
    if (p.kind == 1) {
        if (warp_kernel_for<EPI_STORE>(p.zw, p.sl) == nullptr || p.band < 1 || s->lay.S > p.zw * p.sl)
            return fail(TB_EINVAL, "no warp-march kernel for %d groups of %d slabs covering %d slabs", p.zw, p.sl, s->lay.S);
        const int units = warp_units(p.zw, p.band, s->lay.R, s->lay.C);
        int max_blocks = std::max(apply_grid_x(s->lay.C) * apply_grid_y(8, s->lay.R), s->vec_blocks);
        for (const auto& shape : warp_shapes(s->lay.S, 0, s->lay.L))
            max_blocks = std::max(max_blocks, (warp_units(shape.first, 4, s->lay.R, s->lay.C) + 3) / 4);
        if (warp_shapes(s->lay.S, s->special_mask, s->lay.L).empty())
            return fail(TB_EINVAL, "the warp-march kernel needs Robin / fixed nodes on the bottom and top planes only");
        if ((units + kWarpBlockWarps - 1) / kWarpBlockWarps > max_blocks) return fail(TB_EINVAL, "band too small");
    } else if (p.kind != 0 && p.kind != 2) {
        return fail(TB_EINVAL, "plan kind must be 0 (z-march), 1 (warp march) or 2 (balanced z-march)");
    }
    TB_CUDA(cudaSetDevice(s->device));
    TB_CUDA(cudaStreamSynchronize(s->stream));
    s->plan = p;
    for (int k = 0; k < 2; ++k) {  // captured chunks hold the old launch shape
        release_slot(s->slots32[k]);
        release_slot(s->slots64[k]);
    }
    return TB_OK;
}

int tb_get_apply_plan(const tb_system* s, int32_t* plan5) {
    if (!s || !plan5) return fail(TB_EINVAL, "NULL argument");
    plan5[0] = s->plan.kind;
    plan5[1] = s->plan.rows;
    plan5[2] = s->plan.kind == 1 ? s->plan.zw : s->plan.tma;
    plan5[3] = s->plan.kind == 1 ? s->plan.sl : (s->plan.stages == kStages ? 0 : s->plan.stages);
    plan5[4] = s->plan.band;
    return TB_OK;
}

int tb_set_tile_rows(tb_system* s, int32_t rows) {
    if (!s) return fail(TB_EINVAL, "system is NULL");
    const int32_t plan5[5] = {0, rows, 0, 0, 0};
    return tb_set_apply_plan(s, plan5);
}

int tb_get_kernel_clocks(tb_system* s, int32_t n, double* ns, int64_t* counts) {
    if (!s) return fail(TB_EINVAL, "system is NULL");
    if (n < 0 || n > 3) return fail(TB_EINVAL, "there are 3 kernel clocks");
    TB_CUDA(cudaSetDevice(s->device));
    KernelClock c[3];
    TB_CUDA(cudaMemcpyAsync(c, s->clocks, sizeof(c), cudaMemcpyDeviceToHost, s->stream));
    TB_CUDA(cudaStreamSynchronize(s->stream));
    for (int i = 0; i < n; ++i) {
        if (ns) ns[i] = (double)c[i].total_ns;
        if (counts) counts[i] = (int64_t)c[i].count;
    }
    return TB_OK;
}

int tb_get_kernel_clock(tb_system* s, double* ns2, int64_t* count2) {
    if (!s) return fail(TB_EINVAL, "system is NULL");
    TB_CUDA(cudaSetDevice(s->device));
    KernelClock c[2];
    TB_CUDA(cudaMemcpyAsync(c, s->clocks, sizeof(c), cudaMemcpyDeviceToHost, s->stream));
    TB_CUDA(cudaStreamSynchronize(s->stream));
    for (int i = 0; i < 2; ++i) {
        if (ns2) ns2[i] = (double)c[i].total_ns;
        if (count2) count2[i] = (int64_t)c[i].count;
    }
    return TB_OK;
}

int tb_set_stage_test(tb_system* s, int32_t polls) {
    if (!s) return fail(TB_EINVAL, "system is NULL");
    if (polls < 0) return fail(TB_EINVAL, "polls must be non-negative");
    if (!s->maps_ok) return fail(TB_EINVAL, "this system has no tensor-copy staging");
    TB_CUDA(cudaSetDevice(s->device));
    TB_CUDA(cudaStreamSynchronize(s->stream));
    for (ApplyMaps& m : s->maps) m.test_polls = polls;
    s->ml_maps.test_polls = polls;
    for (int k = 0; k < 2; ++k) {  // the graphs hold the maps by value
        release_slot(s->slots32[k]);
        release_slot(s->slots64[k]);
    }
    return TB_OK;
}

int tb_set_ml_staging(tb_system* s, int32_t staged) {
    if (!s) return fail(TB_EINVAL, "system is NULL");
    if (staged != 0 && staged != 1) return fail(TB_EINVAL, "staged must be 0 or 1");
    if (staged == 1 && (s->precond != 2 || s->ml_stages < 2))
        return fail(TB_ENOTSUP, "the staged fine pass is not available for this system");
    if (s->precond == 2 && s->ml_staged != (staged == 1)) {
        TB_CUDA(cudaSetDevice(s->device));
        TB_CUDA(cudaStreamSynchronize(s->stream));
        s->ml_staged = staged == 1;
        for (int k = 0; k < 2; ++k) {  // the graphs hold the launch form
            release_slot(s->slots32[k]);
            release_slot(s->slots64[k]);
        }
    }
    return TB_OK;
}

int tb_get_ml_staging(const tb_system* s, int32_t* staged) {
    if (!s || !staged) return fail(TB_EINVAL, "NULL argument");
    *staged = (s->precond == 2 && s->ml_staged) ? 1 : 0;
    return TB_OK;
}

int tb_get_tile_rows(const tb_system* s, int32_t* rows) {
    if (!s || !rows) return fail(TB_EINVAL, "NULL argument");
    *rows = s->plan.rows;
    return TB_OK;
}

int tb_system_stream(const tb_system* s, void** stream) {
    if (!s || !stream) return fail(TB_EINVAL, "NULL argument");
    *stream = static_cast<void*>(s->stream);
    return TB_OK;
}

int tb_get_launch_count(const tb_system* s, int64_t* count) {
    if (!s || !count) return fail(TB_EINVAL, "NULL argument");
    *count = s->kernel_launches;
    return TB_OK;
}

int tb_get_timing(const tb_system* s, double* ms4, int64_t* launches4) {
    if (!s) return fail(TB_EINVAL, "system is NULL");
    for (int i = 0; i < 4; ++i) {
        if (ms4) ms4[i] = s->ms[i];
        if (launches4) launches4[i] = s->launches[i];
    }
    return TB_OK;
}

int tb_set_robin(tb_system* s, const double* robin_total) {
    if (!s || !robin_total) return fail(TB_EINVAL, "NULL argument");
    TB_CUDA(cudaSetDevice(s->device));
    return set_robin_impl(s, robin_total);
}

int tb_system_create_problem(const tb_problem_desc* desc, int32_t device, tb_system** out) {
    if (!out) return fail(TB_EINVAL, "out is NULL");
    *out = nullptr;
    tb_system* s = nullptr;
    const int rc = create_problem_impl(desc, device, &s);
    if (rc != TB_OK) {
        destroy_impl(s);
        return rc;
    }
    *out = s;
    return TB_OK;
}

int tb_set_convection(tb_system* s, const tb_convection_desc* convection, int32_t count) {
    TB_CHECK(require_problem(s));
    TB_CUDA(cudaSetDevice(s->device));
    TB_CHECK(check_convection(convection, count));
    TB_CUDA(cudaStreamSynchronize(s->stream));
    const size_t bytes = convection_scratch_bytes(convection, count, s->lay) + 256;
    TB_CHECK(ensure_stage(s, bytes));
    TB_CHECK(lump_boundaries(s, convection, count, static_cast<unsigned char*>(s->stage), bytes));
    return refresh_robin(s, s->robin_total);
}

int tb_set_capacity(tb_system* s, const double* capacity_per_s) {
    TB_CHECK(require_problem(s));
    TB_CUDA(cudaSetDevice(s->device));
    TB_CUDA(cudaStreamSynchronize(s->stream));
    TB_CHECK(upload_capacity(s, capacity_per_s));
    const Layout& L = s->lay;
    prep_robin_total<<<grid_for(L.N, kVecThreads, s->sms * 16), kVecThreads, 0, s->stream>>>(
        s->robin_total, s->robin_only, s->capacity, L.N);
    TB_CUDA(cudaGetLastError());
    s->kernel_launches += 1;
    return refresh_robin(s, s->robin_total);
}

int tb_get_prepared(tb_system* s, double* robin_only, double* robin_total, double* robin_rhs, double* load,
                    uint8_t* free_nodes, uint8_t* active_nodes) {
    TB_CHECK(require_problem(s));
    TB_CUDA(cudaSetDevice(s->device));
    const Layout& L = s->lay;
    const size_t bytes = sizeof(double) * (size_t)L.N;
    const double* src[4] = {s->robin_only, s->robin_total, s->robin_rhs, s->load};
    double* dst[4] = {robin_only, robin_total, robin_rhs, load};
    for (int k = 0; k < 4; ++k)
        if (dst[k]) TB_CUDA(cudaMemcpyAsync(dst[k], src[k], bytes, cudaMemcpyDeviceToHost, s->stream));
    std::vector<uint8_t> flags;
    if (free_nodes || active_nodes) {
        flags.resize((size_t)L.N);
        TB_CUDA(cudaMemcpyAsync(flags.data(), s->node_flags, (size_t)L.N, cudaMemcpyDeviceToHost, s->stream));
    }
    TB_CUDA(cudaStreamSynchronize(s->stream));
    for (long long n = 0; n < (long long)flags.size(); ++n) {
        if (free_nodes) free_nodes[n] = (flags[(size_t)n] & kNodeFixed) ? 0 : 1;
        if (active_nodes) active_nodes[n] = (flags[(size_t)n] & kNodeActive) ? 1 : 0;
    }
    return TB_OK;
}

int tb_get_boundary_weights(tb_system* s, int32_t index, double* weights, double* rhs_weights) {
    TB_CHECK(require_problem(s));
    if (index < 0 || index >= (int)s->boundaries.size()) return fail(TB_EINVAL, "boundary index out of range");
    TB_CUDA(cudaSetDevice(s->device));
    const Layout& L = s->lay;
    const tb_system::Boundary& bd = s->boundaries[(size_t)index];
    double* dst[2] = {weights, rhs_weights};
    const double* src[2] = {bd.w, bd.rw};
    for (int k = 0; k < 2; ++k) {
        if (!dst[k]) continue;
        std::fill(dst[k], dst[k] + L.N, 0.0);
        TB_CUDA(cudaMemcpyAsync(dst[k] + bd.offset, src[k], sizeof(double) * (size_t)bd.count, cudaMemcpyDeviceToHost,
                                s->stream));
    }
    TB_CUDA(cudaStreamSynchronize(s->stream));
    return TB_OK;
}

int tb_build_rhs(tb_system* s, double reference_temperature_k, const double* previous_temperature_k, double* rhs) {
    TB_CHECK(require_problem(s));
    TB_CUDA(cudaSetDevice(s->device));
    return build_rhs_impl(s, reference_temperature_k, previous_temperature_k, rhs);
}

int tb_postprocess(tb_system* s, const double* temperature_k, const double* previous_temperature_k,
                   double* heat_flux, double* convective_heat, double* budget3, double* residual) {
    TB_CHECK(require_problem(s));
    TB_CUDA(cudaSetDevice(s->device));
    return postprocess_impl(s, temperature_k, previous_temperature_k, heat_flux, convective_heat, budget3, residual);
}

int tb_build_rhs_device(tb_system* s, double reference_temperature_k, const double* previous_temperature_k,
                        double* rhs) {
    TB_CHECK(require_problem(s));
    if (!rhs) return fail(TB_EINVAL, "rhs is NULL");
    TB_CUDA(cudaSetDevice(s->device));
    return build_rhs_impl(s, reference_temperature_k, previous_temperature_k, rhs, true);
}

int tb_postprocess_rise_device(tb_system* s, const double* rise, double reference_temperature_k,
                               const double* previous_temperature_k, double* heat_flux, double* convective_heat,
                               double* budget3, double* residual, double* temperature_k, double* extrema2) {
    TB_CHECK(require_problem(s));
    TB_CUDA(cudaSetDevice(s->device));
    return postprocess_impl(s, rise, previous_temperature_k, heat_flux, convective_heat, budget3, residual, true,
                            reference_temperature_k, temperature_k, extrema2);
}

int tb_download(tb_system* s, void* host, const void* device_array, size_t bytes) {
    if (!s || (bytes > 0 && (!host || !device_array))) return fail(TB_EINVAL, "NULL argument");
    TB_CUDA(cudaSetDevice(s->device));
    TB_CUDA(cudaStreamSynchronize(s->stream));
    return device_to_host(s, host, device_array, bytes);
}

int tb_dc_system_create(const tb_dc_desc* desc, int32_t device, tb_system** out) {
    if (!out) return fail(TB_EINVAL, "out is NULL");
    *out = nullptr;
    tb_system* s = nullptr;
    const int rc = create_dc_impl(desc, device, &s);
    if (rc != TB_OK) {
        destroy_impl(s);
        return rc;
    }
    *out = s;
    return TB_OK;
}

int tb_dc_post(tb_system* s, const double* potential, double* field, double* element_loss) {
    if (!s || !potential || !field || !element_loss) return fail(TB_EINVAL, "NULL argument");
    if (s->physics != 1) return fail(TB_EINVAL, "not a layered DC system (tb_dc_system_create)");
    TB_CUDA(cudaSetDevice(s->device));
    const Layout& L = s->lay;
    const int layers = L.S + 1;
    const long long E = (long long)layers * L.R * L.C;
    // staging: the potential (N), then field (2E) and loss (E), read back in one copy
    TB_CHECK(ensure_stage(s, sizeof(double) * (size_t)(L.N + 3 * E)));
    double* d_pot = static_cast<double*>(s->stage);
    double* d_out = d_pot + L.N;
    TB_CHECK(host_to_device(s, d_pot, potential, sizeof(double) * L.N));
    const int nb = grid_for(E, kDcThreads, 148 * 8);
    dc_post_kernel<<<nb, kDcThreads, 0, s->stream>>>(d_pot, s->kin64, s->dims64 + L.S, s->dims64 + L.S + L.C, layers,
                                                     L.R, L.C, L.Xe, d_out, d_out + 2 * E);
    TB_CUDA(cudaGetLastError());
    s->kernel_launches += 1;
    TB_CHECK(device_to_host(s, field, d_out, sizeof(double) * 2 * E));
    TB_CHECK(device_to_host(s, element_loss, d_out + 2 * E, sizeof(double) * E));
    TB_CUDA(cudaStreamSynchronize(s->stream));
    return TB_OK;
}

int tb_dc_get_masks(tb_system* s, uint8_t* active_nodes, uint8_t* free_nodes) {
    if (!s) return fail(TB_EINVAL, "system is NULL");
    if (s->physics != 1) return fail(TB_EINVAL, "not a layered DC system (tb_dc_system_create)");
    TB_CUDA(cudaSetDevice(s->device));
    const Layout& L = s->lay;
    std::vector<uint8_t> mask((size_t)L.L);
    TB_CUDA(cudaMemcpyAsync(mask.data(), s->dc_mask, (size_t)L.L, cudaMemcpyDeviceToHost, s->stream));
    TB_CUDA(cudaStreamSynchronize(s->stream));
    const int cols = L.C + 1;
    for (long long n = 0; n < L.N; ++n) {
        const long long line = n / cols;
        const uint8_t m = mask[(size_t)(line * L.Xp + (n - line * cols))];
        if (active_nodes) active_nodes[n] = (m & 4) ? 1 : 0;
        if (free_nodes) free_nodes[n] = (m & kDcFree) ? 1 : 0;
    }
    return TB_OK;
}

int tb_set_preconditioner(tb_system* s, int32_t kind, int32_t coarse_block_nodes) {
    if (!s) return fail(TB_EINVAL, "system is NULL");
    TB_CUDA(cudaSetDevice(s->device));
    return set_preconditioner(s, kind, coarse_block_nodes);
}

int tb_get_preconditioner(const tb_system* s, int32_t* info5) {
    if (!s || !info5) return fail(TB_EINVAL, "NULL argument");
    info5[0] = s->precond;
    info5[1] = s->cl.b;
    info5[2] = s->cl.layers;
    info5[3] = s->cl.nby;
    info5[4] = s->cl.nbx;
    return TB_OK;
}

int tb_get_multilevel(const tb_system* s, int32_t* dims, int32_t cap, int32_t* count) {
    if (!s || !count) return fail(TB_EINVAL, "NULL argument");
    if (s->precond != 2) return fail(TB_EINVAL, "the multilevel preconditioner is not set");
    *count = (int32_t)s->ml.size();
    for (int l = 0; l < (int)s->ml.size() && l < cap && dims; ++l) {
        dims[3 * l] = s->ml[l].g.L;
        dims[3 * l + 1] = s->ml[l].g.ny;
        dims[3 * l + 2] = s->ml[l].g.nx;
    }
    return TB_OK;
}

int tb_get_multilevel_stencil(tb_system* s, int32_t level, float* stencil) {
    if (!s || !stencil) return fail(TB_EINVAL, "NULL argument");
    if (s->precond != 2) return fail(TB_EINVAL, "the multilevel preconditioner is not set");
    if (level < 1 || level >= (int)s->ml.size())
        return fail(TB_EINVAL, "level %d has no stored stencil (levels 1..%d do)", level, (int)s->ml.size() - 1);
    TB_CUDA(cudaSetDevice(s->device));
    const tb_system::MLLevel& lv = s->ml[level - 1];
    TB_CUDA(cudaMemcpyAsync(stencil, lv.st, sizeof(float) * kMlStencil * lv.g.n, cudaMemcpyDeviceToHost, s->stream));
    TB_CUDA(cudaStreamSynchronize(s->stream));
    return TB_OK;
}

int tb_get_coarse(tb_system* s, double* matrix, double* inverse) {
    if (!s) return fail(TB_EINVAL, "system is NULL");
    if (s->precond != 1 && s->precond != 2) return fail(TB_EINVAL, "no coarse operator is set");
    TB_CUDA(cudaSetDevice(s->device));
    const size_t bytes = sizeof(double) * (size_t)s->cl.nc * s->cl.nc;
    if (matrix) TB_CUDA(cudaMemcpyAsync(matrix, s->coarse_matrix, bytes, cudaMemcpyDeviceToHost, s->stream));
    if (inverse) TB_CUDA(cudaMemcpyAsync(inverse, s->coarse_inv64, bytes, cudaMemcpyDeviceToHost, s->stream));
    TB_CUDA(cudaStreamSynchronize(s->stream));
    return TB_OK;
}

int tb_precondition_f32(tb_system* s, const float* x, float* y) {
    if (!s || !x || !y) return fail(TB_EINVAL, "NULL argument");
    if (s->precond != 1 && s->precond != 2) return fail(TB_EINVAL, "no two-level or multilevel preconditioner is set");
    TB_CUDA(cudaSetDevice(s->device));
    TB_CHECK(load_nodes<float>(s, s->r32, x, false));
    if (s->precond == 2) {
        TB_CUDA(ml_step(s, ML_ONLY, false));
        s->kernel_launches += ml_kernels_per_step(s);
        return store_nodes<float>(s, y, s->p32, false);
    }
    TB_CUDA(launch_coarse_step<COARSE_ONLY>(s, false));
    pcg_direction_2l<true><<<s->vec_blocks, kVecThreads, 0, s->stream>>>(s->p32, nullptr, s->r32, s->dinv32,
                                                                         s->coarse_c, s->nq, s->lay, s->cl, nullptr);
    TB_CUDA(cudaGetLastError());
    s->kernel_launches += 3;
    return store_nodes<float>(s, y, s->p32, false);
}

int tb_residual_f64_device_static(tb_system* s, const double* d_x, const double* d_b, double* d_r, double* norms2) {
    if (!s || !d_x || !d_b || !d_r || !norms2) return fail(TB_EINVAL, "NULL argument");
    if (s->physics != 0) return fail(TB_ENOTSUP, "the static-scratch residual serves the thermal operator only");
    TB_CUDA(cudaSetDevice(s->device));
    // FP64 tiles are 8 or 16 rows high (launch_apply caps 32 at 16).
    const int rows = (s->plan.rows == 8) ? 8 : 16;
    const long long tiles = (long long)apply_grid_x(s->lay.C) * apply_grid_y(rows, s->lay.R);
    if (tiles > kStaticMaxTiles)
        return fail(TB_EINVAL, "board needs %lld operator tiles; the static scratch holds %d", tiles, kStaticMaxTiles);
    unsigned char* base = nullptr;
    TB_CHECK(static_scratch_base(s->device, &base));
    TB_CHECK(load_nodes<double>(s, s->x64, d_x, true));
    TB_CHECK(load_nodes<double>(s, s->b64, d_b, true));
    ApplyParams<double> P = apply_params<double>(s, s->x64, s->r64, s->b64);
    P.partials = reinterpret_cast<double*>(base);
    P.counter = reinterpret_cast<unsigned int*>(base + kStaticCounterOffset);
    P.ctl = reinterpret_cast<SolveCtl*>(base + kStaticCtlOffset);
    P.clock = nullptr;
    TB_CUDA(cudaMemsetAsync(P.counter, 0, sizeof(unsigned int), s->stream));
    TB_CHECK((launch_apply<double, MODE_OPERATOR, EPI_RESIDUAL>(s, P)));
    s->kernel_launches += 1;
    TB_CHECK(store_nodes<double>(s, d_r, s->r64, true));
    double out[2] = {0.0, 0.0};  // res2, peak: adjacent in SolveCtl
    TB_CUDA(cudaMemcpyAsync(out, &P.ctl->res2, sizeof(out), cudaMemcpyDeviceToHost, s->stream));
    TB_CUDA(cudaStreamSynchronize(s->stream));
    norms2[0] = out[0];
    norms2[1] = out[1];
    return TB_OK;
}

}  // extern "C"

#include "tb_engine.inl"
