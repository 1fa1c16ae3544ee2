// Matrix-free trilinear (Q1) hexahedral conduction action on the layered grid.
//
// Operator (reference src/thermal/matrix_free_mpir_fem/operator.py:243-288,
// hex_q1.cpp:90-193):
//     y = where(free, K (x * free) + R x, x),   K = sum_e a_x U_x + a_y U_y + a_z U_z
// with U_x = M (x) M (x) S, U_y = M (x) S (x) M, U_z = S (x) M (x) M in the local
// corner order 4 dz + 2 dy + dx, S = [[1,-1],[-1,1]], M = [[2,1],[1,2]]/6.
//
// Element action in the Haar basis.  The 1D vectors [1,1] and [1,-1] are
// eigenvectors of both M (eigenvalues 1/2, 1/6) and S (0, 2), so the eight
// 3D sum/difference patterns v_m diagonalise U_x, U_y and U_z at once.  With
// u~_m = v_m . u (butterflies, no multiplies) the element action is
//     K_e u = sum_m (lambda_m / 8) u~_m v_m,
//     lambda/8:  SSD a_x/16   SDS a_y/16   DSS a_z/16      (pattern z,y,x)
//                SDD (a_x+a_y)/48  DSD (a_x+a_z)/48  DDS (a_y+a_z)/48
//                DDD (a_x+a_y+a_z)/144,  SSS 0.
// The forward transform works on differences, so a constant field maps to
// exactly zero and smooth fields keep their accuracy in FP32.
//
// Data movement.  A block owns a tile of element columns (64 x 16: x from
// X0-4, y from Y0-1) and marches along z through the S slabs.  Per node plane
// it stages the node tile, the Robin/fixed tile (on planes that have one) and
// the conductivity tiles of the slab below in shared memory -- by tensor
// copies (cp.async.bulk.tensor) that one thread issues onto a stage mbarrier,
// or by per-thread cp.async copies; four stages, two planes in flight ahead of
// the one in use -- takes the 2D (y,x) Haar transform of each
// element's face on that plane (shared by the slab below and the slab above),
// finishes the slab between the previous plane and this one with the z
// butterfly and the eigenvalue scaling, and keeps the upper-face result in
// registers until the next slab adds its lower-face part.  The corner
// contributions of one plane are summed per node in a fixed order (warp
// shuffle in x, shared memory in y), so the result is deterministic.  The
// block writes 60 x 15 output nodes; the one-element halo on the low x and y
// sides is recomputed by the neighbouring block.
//
// Conductivities are stored per element (k_in, k_z); the element factors
// a_x = k_in h_y h_z / h_x, a_y = k_in h_x h_z / h_y, a_z = k_z h_x h_y / h_z
// (mesh.py:276-293) are rebuilt from per-slab, per-row and per-column pitches.
#pragma once

#include <cuda.h>  // CUtensorMap (the type only; maps are encoded by the host)
#include <cuda_runtime.h>
#include <stdint.h>

#include "tb_reduce.cuh"
#include "tb_types.h"

namespace tb {

// Programmatic dependent launch: a kernel lets its successor start launching
// at once (launch_dependents) and waits for its predecessor's completion and
// memory (wait) only where it first reads what the predecessor wrote.  Both
// are no-ops for kernels launched without the programmatic attribute.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

constexpr int kTileW = 68;  // node tile width: node columns X0-4 .. X0+63
constexpr int kTileQ = 17;  // quads (4 nodes) per tile row
constexpr int kOutX = 60;   // output node columns per block
constexpr int kXchW = 64;

// Tile of ROWS element rows x 64 element columns, 16 * ROWS threads (4
// element columns each); it writes 60 x (ROWS - 1) nodes.
template <int ROWS>
struct TileShape {
    static constexpr int threads = 16 * ROWS;
    static constexpr int out_y = ROWS - 1;
    static constexpr int tile_h = ROWS + 1;  // node rows Y0-1 .. Y0+ROWS-1
    static constexpr int tile_size = tile_h * kTileW;
    static constexpr int quads = tile_h * kTileQ;
};

// Epilogues: store y; store y and reduce p.Ap (PCG); store b - y and reduce
// its norm and peak (FP64 residual).
enum { EPI_STORE = 0, EPI_DOT = 1, EPI_RESIDUAL = 2 };
enum { MODE_OPERATOR = 0, MODE_STIFFNESS = 1 };

template <typename T>
struct ApplyParams {
    const T* x;                // node field, padded (S+1, R+1, Xp)
    T* y;                      // output node field (the residual in EPI_RESIDUAL)
    const T* b;                // EPI_RESIDUAL: right-hand side
    const T* kin;              // element field, padded (S, R, Xe)
    const T* kz;
    const T* rf;               // node field: Robin total (>= 0) on free nodes, -1 on fixed ones
    const int* plane_flags;      // (S+1): nonzero when the plane holds a Robin term or a fixed node
    const T* gzt;              // (S) h_z / 16
    const T* gzi;              // (S) 1 / (16 h_z)
    const T* hx;               // (C)
    const T* ihx;              // (C)
    const T* hy;               // (R)
    const T* ihy;              // (R)
    double* partials;          // per-block accumulators (4 doubles per block)
    unsigned int* counter;     // last-block ticket
    SolveCtl* ctl;             // scalars of the running solve
    KernelClock* clock;        // device-time accounting of this kernel kind (may be null)
    int S, R, C, Xp, Xe;
    long long pstride;         // (R+1) * Xp
    long long sstride;         // R * Xe
};

template <typename T>
struct Quad {
    T v[4];
};

__device__ __forceinline__ Quad<float> ldg_quad(const float* p) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(p));
    return {{a.x, a.y, a.z, a.w}};
}
__device__ __forceinline__ Quad<double> ldg_quad(const double* p) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    return {{a.x, a.y, b.x, b.y}};
}
__device__ __forceinline__ void st_quad(float* p, const Quad<float>& q) {
    *reinterpret_cast<float4*>(p) = make_float4(q.v[0], q.v[1], q.v[2], q.v[3]);
}
__device__ __forceinline__ void st_quad(double* p, const Quad<double>& q) {
    reinterpret_cast<double2*>(p)[0] = make_double2(q.v[0], q.v[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(q.v[2], q.v[3]);
}
__device__ __forceinline__ Quad<float> lds_quad(const float* p) {
    const float4 a = *reinterpret_cast<const float4*>(p);
    return {{a.x, a.y, a.z, a.w}};
}
__device__ __forceinline__ Quad<double> lds_quad(const double* p) {
    const double2 a = reinterpret_cast<const double2*>(p)[0];
    const double2 b = reinterpret_cast<const double2*>(p)[1];
    return {{a.x, a.y, b.x, b.y}};
}
template <typename T>
__device__ __forceinline__ Quad<T> zero_quad() {
    return {{T(0), T(0), T(0), T(0)}};
}

// ------------------------------------------------------------ cp.async
// Asynchronous 16-byte global->shared copies (LDGSTS).  A copy whose source
// lies outside the field is issued with source size 0, which writes zeros.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    const int bytes = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// A quad of T (4 nodes or 4 elements) is 16 bytes in FP32, 32 bytes in FP64.
template <typename T>
__device__ __forceinline__ void cp_async_quad(T* smem, const T* gmem, bool valid) {
    cp_async16(smem, gmem, valid);
    if (sizeof(T) == 8) cp_async16(smem + 2, gmem + 2, valid);
}

constexpr int kStages = 4;  // default: plane p computes, p-1 is emitted, p+1 and p+2 are in flight
constexpr int kDeepStages = 5;  // the deeper tensor-copy shapes: three planes in flight

// Shared memory of one pipeline stage: node tile, Robin/fixed tile, and the
// k_in / k_z tiles of the slab below the plane.  Each part starts on a
// 128-byte boundary, where a tensor copy may write it.
template <typename T, int ROWS>
struct StageLayout {
    static constexpr int align = 128 / (int)sizeof(T);
    static constexpr int tile_pad = (TileShape<ROWS>::tile_size + align - 1) / align * align;
    static constexpr int x_off = 0;
    static constexpr int rf_off = tile_pad;
    static constexpr int kin_off = 2 * tile_pad;
    static constexpr int kz_off = kin_off + ROWS * 64;
    static constexpr int size = kz_off + ROWS * 64;  // in T, a multiple of 128 bytes
};

// ------------------------------------------------------------ tensor copies
// Tensor maps of the FP32 fields the operator stages, for the staging by the
// tensor memory accelerator (TMA): one thread per block copies a plane's
// tiles with cp.async.bulk.tensor and every thread waits on the stage's
// mbarrier.  Boxes: the node tile (68 x (ROWS+1) nodes from column X0-4, row
// Y0-1) of x and of the Robin/fixed field; the 64 x ROWS element tiles of k_in
// and k_z.  Parts of a box outside the field are filled with zeros, as the
// zero-size cp.async copies of the other staging do.  The box origin in x is
// X0-4 = 60 bx - 4 nodes, a multiple of 4 FP32 values (16 bytes), as a tensor
// copy requires.
struct ApplyMaps {
    CUtensorMap x;    // (S+1, R+1, Xp) node field staged as the operand
    CUtensorMap rf;   // (S+1, R+1, Xp) Robin total / fixed mark
    CUtensorMap kin;  // (S, R, Xe) element fields
    CUtensorMap kz;
    int* err;         // set to 1 when a block gave up waiting for its tiles
    // Test only (tb_set_stage_test): when > 0, the issuing thread arms each
    // stage barrier without issuing its copies and every wait gives up after
    // this many polls, so the give-up path runs with no copy in flight.
    int test_polls;
};

// Polls of a stage's mbarrier before a block gives up (each poll blocks for a
// hardware-defined slice): about a second in all, far beyond a copy's latency.
constexpr int kStageSpinLimit = 1 << 20;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred P1;\n mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n selp.b32 %0, 1, 0, P1;\n}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}
// Bounded wait for the phase `parity` of a stage's mbarrier to complete.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int polls = kStageSpinLimit) {
    for (int i = 0; i < polls; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// A tensor map written in global memory by an earlier copy (a slot's maps
// are rewritten when a new board takes the slot) is read by the tensor-copy
// unit through its own proxy: acquire it before the first copy that uses it.
__device__ __forceinline__ void tensormap_acquire(const CUtensorMap* map) {
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(reinterpret_cast<uint64_t>(map))
                 : "memory");
}

// 3D tile copy global -> shared, completing `bar`'s transaction count.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
        : "memory");
}

// Blocks per SM the FP32 kernels are compiled for (registers capped to fit):
// 4 x 128, 2 x 256 or 1 x 512 threads, so that the packed element math of a
// thread (about 120 registers) runs without spills.  The FP64 kernels run once per outer step and are not capped.
template <typename T, int ROWS>
struct ApplyOccupancy {
    static constexpr int min_blocks = sizeof(T) == 4 ? (ROWS == 8 ? 4 : (ROWS == 16 ? 2 : 1)) : 1;
};

// Dynamic shared memory of apply_kernel<T, ..., ROWS> for S slabs: the
// stages, the y exchange, one mbarrier per stage (used by the tensor-copy
// staging) and the per-slab tables.  The barriers sit at an offset that does
// not depend on S, because a block of the batched kernels walks boards of
// different slab counts with the same barriers.
template <typename T, int ROWS, int STAGES = kStages>
__host__ __device__ constexpr size_t apply_bar_offset() {
    return (size_t)STAGES * StageLayout<T, ROWS>::size * sizeof(T) + (size_t)ROWS * kXchW * sizeof(T);
}
template <typename T, int ROWS, int STAGES = kStages>
__host__ __device__ constexpr size_t apply_tables_offset() {
    return apply_bar_offset<T, ROWS, STAGES>() + STAGES * sizeof(unsigned long long);
}
template <typename T, int ROWS, int STAGES = kStages>
inline size_t apply_smem_bytes(int S) {
    const size_t tables = 2 * (size_t)S * sizeof(T) + (size_t)(S + 1) * sizeof(int);
    return (apply_tables_offset<T, ROWS, STAGES>() + tables + 15) / 16 * 16;
}
static_assert(apply_bar_offset<float, 8>() % 16 == 0 && apply_bar_offset<double, 16>() % 16 == 0,
              "barriers and tables stay 16-byte aligned");

// ---------------------------------------------------------- pair arithmetic
// Element columns 2q and 2q+1 of a thread travel as one pair.  FP32 pairs use
// the packed f32x2 datapath of sm_100 (one instruction per pair, each half
// rounded exactly as the scalar operation); FP64 pairs are two scalar
// operations.  a - b is fma(b, -1, a): exact before its single rounding.
template <typename T> struct PairOf;
template <> struct PairOf<float> { using type = float2; };
template <> struct PairOf<double> { using type = double2; };

__device__ __forceinline__ float2 pr_make(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ double2 pr_make(double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ float2 pr_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 pr_sub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 pr_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 pr_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ double2 pr_add(double2 a, double2 b) {
    return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
}
__device__ __forceinline__ double2 pr_sub(double2 a, double2 b) {
    return make_double2(__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y));
}
__device__ __forceinline__ double2 pr_mul(double2 a, double2 b) {
    return make_double2(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y));
}
__device__ __forceinline__ double2 pr_fma(double2 a, double2 b, double2 c) {
    return make_double2(__fma_rn(a.x, b.x, c.x), __fma_rn(a.y, b.y, c.y));
}

// The work of one tile (bx, by): stage its planes, run the element actions,
// write its output nodes.  Adds this thread's share of the tile's reduction
// (p.Ap, or ||b - Ax||^2 and max |b - Ax|) to `dot` and `rmax`.  Ends with a
// barrier, so a block may call it for several tiles in a row.
//
// Only node planes q0 .. q1-1 of the tile are written (0 <= q0 < q1 <= S+1).
// A plane's nodes need the slabs below and above it, so a range that starts
// at q0 > 0 also stages plane q0-1 and runs slab q0-1 for its upper-face
// part; every written value is the one the whole march writes, bit for bit.
//
// With `gate`, the tile first waits for the preceding launch (programmatic
// dependent launch) after loading the static tables and per-thread offsets,
// then returns TILE_SKIP without touching anything when an inner-product
// launch finds its solve no longer running (a value uniform across the grid).
//
// TMA selects the staging: per-thread cp.async copies (false), or tensor
// copies issued by thread 0 onto one mbarrier per stage (true; `maps` holds
// the tensor maps and `seq` counts the planes this block has staged so far,
// which fixes each stage's slot and mbarrier phase across the tiles of a
// block).  A block whose wait for a stage runs out sets the error word and
// the solve state, stops the tile after its copies in flight have landed (or
// a bounded wait for them has run out) and returns TILE_ABORTED.
enum { TILE_SKIP = 0, TILE_DONE = 1, TILE_ABORTED = 2 };

template <typename T, int MODE, int EPI, int ROWS, bool TMA = false, int STAGES = kStages>
__device__ __forceinline__ int apply_tile(const ApplyParams<T>& P, const int bx, const int by,
                                          unsigned char* smem_raw, T& dot, double& rmax, const bool gate,
                                          const int q0 = 0, const int q1 = 1 << 30,
                                          const ApplyMaps* maps = nullptr, int* seq = nullptr,
                                          const bool maps_in_global = false) {
    static_assert(!TMA || sizeof(T) == 4, "tensor-copy staging is built for the FP32 fields");
    static_assert(STAGES >= 4, "plane p is computed, p-1 emitted, and STAGES-2 planes are in flight");
    constexpr int AHEAD = STAGES - 2;  // planes staged ahead of the one computed
    using T2 = typename PairOf<T>::type;
    using Sh = TileShape<ROWS>;
    using St = StageLayout<T, ROWS>;
    T* const stage = reinterpret_cast<T*>(smem_raw);        // [STAGES][St::size]
    T* const xch = stage + STAGES * St::size;                // [ROWS][64] y-exchange
    const uint32_t bar0 = smem_u32(smem_raw + apply_bar_offset<T, ROWS, STAGES>());  // [STAGES] mbarriers
    T* const s_tz = reinterpret_cast<T*>(smem_raw + apply_tables_offset<T, ROWS, STAGES>());  // [S] h_z / 16
    T* const s_iz = s_tz + P.S;                              // [S] 1 / (16 h_z)
    int* const s_flag = reinterpret_cast<int*>(s_iz + P.S);  // [S+1] plane holds Robin / fixed nodes
    const int seq0 = TMA ? *seq : 0;
    const int tid = threadIdx.x;
    const int g = tid & 15;   // column group: element columns exb .. exb+3
    const int j = tid >> 4;   // element row of this thread in the tile
    const int X0 = bx * kOutX;
    const int Y0 = by * Sh::out_y;
    const int S = P.S, R = P.R, C = P.C, Xp = P.Xp;
    const int ey = Y0 - 1 + j;
    const int exb = X0 - 4 + 4 * g;
    const bool erow_ok = (ey >= 0) && (ey < R);
    const bool equad_ok = erow_ok && (exb >= 0) && (exb < P.Xe);

    for (int i = tid; i < S; i += Sh::threads) {
        s_tz[i] = P.gzt[i];
        s_iz[i] = P.gzi[i];
    }
    for (int i = tid; i <= S; i += Sh::threads) s_flag[i] = (MODE == MODE_OPERATOR) ? P.plane_flags[i] : 0;
    if constexpr (TMA) {
        if (seq0 == 0 && tid == 0) {  // first tile of this block: the barriers expect one arrival per phase
            for (int i = 0; i < STAGES; ++i) mbar_init(bar0 + 8 * i, 1);
            mbar_init_fence();
        }
        if (maps_in_global && tid == 0) {
            tensormap_acquire(&maps->x);
            tensormap_acquire(&maps->rf);
            tensormap_acquire(&maps->kin);
            tensormap_acquire(&maps->kz);
        }
    }

    // Per element column geometry: a_x/16 = k_in (h_z/16) (h_y/h_x),
    // a_y/16 = k_in (h_z/16) (h_x/h_y), a_z/16 = k_z (1/(16 h_z)) h_x h_y, and
    // (a_x + a_y)/48 = k_in (h_z/16) (h_y/h_x + h_x/h_y)/3.
    const T third = T(1) / T(3);
    T qx[4], qy[4], qxy[4], qz[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int ex = exb + k;
        if (erow_ok && ex >= 0 && ex < C) {
            const T hx = P.hx[ex], ihx = P.ihx[ex], hy = P.hy[ey], ihy = P.ihy[ey];
            qx[k] = hy * ihx;
            qy[k] = hx * ihy;
            qxy[k] = (qx[k] + qy[k]) * third;
            qz[k] = hx * hy;
        } else {
            qx[k] = T(0);
            qy[k] = T(0);
            qxy[k] = T(0);
            qz[k] = T(0);
        }
    }
    const T2 qx2[2] = {pr_make(qx[0], qx[1]), pr_make(qx[2], qx[3])};
    const T2 qy2[2] = {pr_make(qy[0], qy[1]), pr_make(qy[2], qy[3])};
    const T2 qxy2[2] = {pr_make(qxy[0], qxy[1]), pr_make(qxy[2], qxy[3])};
    const T2 qz2[2] = {pr_make(qz[0], qz[1]), pr_make(qz[2], qz[3])};
    const T2 third2 = pr_make(third, third);
    // Loop-invariant offsets of this thread: the (at most two) node-tile
    // quads it stages, its conductivity quad, its face-read and output slots.
    // (tid < threads <= quads, so the first quad always exists.)
    int so[2], go[2];
    bool qok[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const int q = tid + i * Sh::threads;
        const int tr = q / kTileQ, tc = (q % kTileQ) * 4;
        const int nr = Y0 - 1 + tr, nc = X0 - 4 + tc;
        qok[i] = (q < Sh::quads) && (nr >= 0) && (nr <= R) && (nc >= 0) && (nc < Xp);
        so[i] = (q < Sh::quads) ? tr * kTileW + tc : -1;
        go[i] = qok[i] ? nr * Xp + nc : 0;
    }
    const int gk = equad_ok ? ey * P.Xe + exb : 0;
    const int sface = j * kTileW + 4 * g;  // face rows j, j+1; the output row is j+1
    const bool out_ok = (j < Sh::out_y) && (g >= 1) && (Y0 + j <= R) && (exb < Xp);
    const int gout = out_ok ? (Y0 + j) * Xp + exb : 0;
    const int xrow = (j + 1 < ROWS ? j + 1 : ROWS - 1) * kXchW + 4 * g;  // exchange slot read (in range for all)

    if (gate) {
        pdl_wait();  // the predecessor's writes (the direction, the scalars) are visible from here on
        if (EPI == EPI_DOT && P.ctl->state != ST_RUNNING) return TILE_SKIP;  // whole grid skips
        if (EPI != EPI_STORE && P.clock != nullptr && threadIdx.x == 0) atomicMin(&P.clock->first, global_ns());
    }
    __syncthreads();  // tables ready

    const int p_first = q0 > 0 ? q0 - 1 : 0;  // first node plane staged
    const int p_last = q1 <= S ? q1 : S;       // last node plane staged

    // Stage of plane p, and (tensor copies) the phase of its mbarrier.  The
    // march keeps both as counters that advance by one plane (no division by
    // the stage count per plane); these give their starting values.
    auto slot = [&](const int p) { return TMA ? ((seq0 + p - p_first) % STAGES) : (p % STAGES); };
    auto phase = [&](const int p) { return (uint32_t)(((seq0 + p - p_first) / STAGES) & 1); };
    auto next_slot = [](const int sl) { return sl + 1 == STAGES ? 0 : sl + 1; };

    // Asynchronous staging of plane p (and of slab p-1 below it, when that
    // slab is computed) into stage `sl`, the plane's slot.
    auto issue = [&](const int p, const int sl) {
        T* const st = stage + sl * St::size;
        if constexpr (TMA) {
            if (tid == 0) {
                const uint32_t bar = bar0 + 8 * sl;
                constexpr uint32_t node_bytes = Sh::tile_size * sizeof(T);
                constexpr uint32_t elem_bytes = ROWS * 64 * sizeof(T);
                const bool special = s_flag[p] != 0;
                const bool slab = p > p_first;
                mbar_expect_tx(bar, node_bytes * (special ? 2u : 1u) + (slab ? 2u * elem_bytes : 0u));
                if (maps->test_polls > 0) return;  // test: the stage stays armed, nothing is copied
                tma_load_3d(st + St::x_off, &maps->x, X0 - 4, Y0 - 1, p, bar);
                if (special) tma_load_3d(st + St::rf_off, &maps->rf, X0 - 4, Y0 - 1, p, bar);
                if (slab) {
                    tma_load_3d(st + St::kin_off, &maps->kin, X0 - 4, Y0 - 1, p - 1, bar);
                    tma_load_3d(st + St::kz_off, &maps->kz, X0 - 4, Y0 - 1, p - 1, bar);
                }
            }
            return;
        }
        const T* const xb = P.x + (long long)p * P.pstride;
        const T* const rb = P.rf + (long long)p * P.pstride;
        const bool special = s_flag[p] != 0;
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            if (so[i] >= 0) {
                cp_async_quad(st + St::x_off + so[i], xb + go[i], qok[i]);
                if (special) cp_async_quad(st + St::rf_off + so[i], rb + go[i], qok[i]);
            }
        }
        if (p > p_first) {
            const long long kb = (long long)(p - 1) * P.sstride;
            const int sk = sface - 4 * j;  // = j * 64 + 4 g
            cp_async_quad(st + St::kin_off + sk, P.kin + kb + gk, equad_ok);
            cp_async_quad(st + St::kz_off + sk, P.kz + kb + gk, equad_ok);
        }
    };

    // Face transforms (SS, DS, SD, DD) of the plane below and the upper-face
    // contributions waiting for the next plane, as pairs of element columns.
    // Up[.][0] holds the DSS weight itself (its contribution to the plane
    // above enters with the opposite sign).
    T2 Fl[2][4], Up[2][4];
#pragma unroll
    for (int q = 0; q < 2; ++q)
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            Fl[q][m] = pr_make(T(0), T(0));
            Up[q][m] = pr_make(T(0), T(0));
        }

    // Sum one plane's Haar-domain contributions into nodes and write them
    // (`sl`: the plane's stage).
    auto emit_plane = [&](const int pl, const int sl, const T2 (&tot)[2][4]) {
        const T* const st = stage + sl * St::size;
        T2 c00[2], c01[2], c10[2], c11[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const T2 A = pr_add(tot[q][0], tot[q][1]);
            const T2 B = pr_sub(tot[q][0], tot[q][1]);
            const T2 Cc = pr_add(tot[q][2], tot[q][3]);
            const T2 D = pr_sub(tot[q][2], tot[q][3]);
            c00[q] = pr_add(A, Cc);
            c01[q] = pr_sub(A, Cc);
            c10[q] = pr_add(B, D);
            c11[q] = pr_sub(B, D);
        }
        T R0[5], R1[5];
        R0[0] = c00[0].x;
        R0[1] = c01[0].x + c00[0].y;
        R0[2] = c01[0].y + c00[1].x;
        R0[3] = c01[1].x + c00[1].y;
        R0[4] = c01[1].y;
        R1[0] = c10[0].x;
        R1[1] = c11[0].x + c10[0].y;
        R1[2] = c11[0].y + c10[1].x;
        R1[3] = c11[1].x + c10[1].y;
        R1[4] = c11[1].y;
        const T left0 = __shfl_up_sync(0xffffffffu, R0[4], 1);
        const T left1 = __shfl_up_sync(0xffffffffu, R1[4], 1);
        R0[0] += left0;
        R1[0] += left1;
        {
            Quad<T> w = {{R0[0], R0[1], R0[2], R0[3]}};
            st_quad(xch + j * kXchW + 4 * g, w);
        }
        __syncthreads();
        const Quad<T> other = lds_quad(xch + xrow);
        const Quad<T> xo = lds_quad(st + St::x_off + sface + kTileW);
        Quad<T> out;
        if (s_flag[pl] != 0) {
            const Quad<T> rr = lds_quad(st + St::rf_off + sface + kTileW);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const T acc = R1[k] + other.v[k];
                out.v[k] = (rr.v[k] < T(0)) ? xo.v[k] : acc + rr.v[k] * xo.v[k];
            }
        } else {
#pragma unroll
            for (int k = 0; k < 4; ++k) out.v[k] = R1[k] + other.v[k];
        }
        if (out_ok) {
            const long long node = (long long)pl * P.pstride + gout;
            if (EPI == EPI_RESIDUAL) {
                const Quad<T> bq = ldg_quad(P.b + node);
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    out.v[k] = bq.v[k] - out.v[k];
                    dot = fma(out.v[k], out.v[k], dot);
                    rmax = fmax(rmax, fabs((double)out.v[k]));
                }
            } else if (EPI == EPI_DOT) {
#pragma unroll
                for (int k = 0; k < 4; ++k) dot = fma(xo.v[k], out.v[k], dot);
            }
            st_quad(P.y + node, out);
        }
    };

    if constexpr (TMA) {
        // tensor copies write 128-byte aligned stage parts; a misplaced
        // dynamic shared memory window (uniform across the block) is reported
        // instead of being written
        if (smem_u32(smem_raw) & 127u) {
            if (tid == 0) {
                atomicExch(maps->err, 1);
                if (P.ctl != nullptr) P.ctl->state = ST_STAGE_TIMEOUT;
            }
            __syncthreads();
            return TILE_ABORTED;
        }
    }
#pragma unroll
    for (int k = 0; k < AHEAD; ++k) {  // one commit group per plane, issued or not
        if (p_first + k <= p_last) issue(p_first + k, slot(p_first + k));
        if constexpr (!TMA) cp_async_commit();
    }

    bool aborted = false;
    int sl_cur = slot(p_first);                // stage of plane p
    uint32_t ph_cur = phase(p_first);          // phase of its mbarrier
    int sl_ahead = slot(p_first + AHEAD);      // stage of plane p + AHEAD
    int sl_prev = sl_cur;                      // stage of plane p - 1 (once p > p_first)
    for (int p = p_first; p <= p_last; ++p) {
        if constexpr (TMA) {
            // every thread sees plane p's tiles land; the vote is also the
            // barrier after which every thread is done with plane p-2
            const int polls = maps->test_polls > 0 ? maps->test_polls : kStageSpinLimit;
            const bool ok = mbar_wait(bar0 + 8 * sl_cur, ph_cur, polls);
            if (!__syncthreads_and(ok)) {
                if (tid == 0) {  // let the copies in flight (planes p .. p+AHEAD-1) land before the block leaves
                    for (int k = AHEAD - 1; k >= 1; --k)
                        if (p + k <= p_last) mbar_wait(bar0 + 8 * slot(p + k), phase(p + k), polls);
                    mbar_wait(bar0 + 8 * sl_cur, ph_cur, polls);
                    atomicExch(maps->err, 1);
                    if (P.ctl != nullptr) P.ctl->state = ST_STAGE_TIMEOUT;
                }
                aborted = true;
                break;
            }
        } else {
            cp_async_wait<AHEAD - 1>();  // this thread's copies of plane p have landed
            __syncthreads();             // everybody's have, and every thread is done with plane p-2
        }
        if (p + AHEAD <= p_last) issue(p + AHEAD, sl_ahead);
        if constexpr (!TMA) cp_async_commit();

        const T* const st = stage + sl_cur * St::size;
        const bool special = s_flag[p] != 0;
        // Face transform of plane p for the four elements.  The fifth column
        // comes from the next lane's first one by a shuffle; the last group of
        // a row takes it from shared memory (read by every lane, selected).
        T2 F[2][4];
        {
            const T* r0 = st + St::x_off + sface;
            const T* r1 = r0 + kTileW;
            Quad<T> a4 = lds_quad(r0), c4 = lds_quad(r1);
            T a5s = r0[4], c5s = r1[4];
            if (special) {  // x * free: fixed nodes do not enter free rows
                const T* f0 = st + St::rf_off + sface;
                const Quad<T> fa = lds_quad(f0);
                const Quad<T> fc = lds_quad(f0 + kTileW);
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    a4.v[k] = (fa.v[k] < T(0)) ? T(0) : a4.v[k];
                    c4.v[k] = (fc.v[k] < T(0)) ? T(0) : c4.v[k];
                }
                a5s = (f0[4] < T(0)) ? T(0) : a5s;
                c5s = (f0[kTileW + 4] < T(0)) ? T(0) : c5s;
            }
            const T a5n = __shfl_down_sync(0xffffffffu, a4.v[0], 1);
            const T c5n = __shfl_down_sync(0xffffffffu, c4.v[0], 1);
            const T a[5] = {a4.v[0], a4.v[1], a4.v[2], a4.v[3], g == 15 ? a5s : a5n};
            const T c[5] = {c4.v[0], c4.v[1], c4.v[2], c4.v[3], g == 15 ? c5s : c5n};
            T A0[4], D0[4], A1[4], D1[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                A0[k] = a[k] + a[k + 1];
                D0[k] = a[k] - a[k + 1];
                A1[k] = c[k] + c[k + 1];
                D1[k] = c[k] - c[k + 1];
            }
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const T2 a0 = pr_make(A0[2 * q], A0[2 * q + 1]), d0 = pr_make(D0[2 * q], D0[2 * q + 1]);
                const T2 a1 = pr_make(A1[2 * q], A1[2 * q + 1]), d1 = pr_make(D1[2 * q], D1[2 * q + 1]);
                F[q][0] = pr_add(a0, a1);  // SS
                F[q][1] = pr_sub(a0, a1);  // DS (y difference)
                F[q][2] = pr_add(d0, d1);  // SD (x difference)
                F[q][3] = pr_sub(d0, d1);  // DD
            }
        }

        if (p > p_first) {
            const int s = p - 1;
            const T2 tz2 = pr_make(s_tz[s], s_tz[s]), iz2 = pr_make(s_iz[s], s_iz[s]);
            const Quad<T> kin_c = lds_quad(st + St::kin_off + sface - 4 * j);
            const Quad<T> kz_c = lds_quad(st + St::kz_off + sface - 4 * j);
            T2 tot[2][4];
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const T2 kin2 = pr_make(kin_c.v[2 * q], kin_c.v[2 * q + 1]);
                const T2 kz2 = pr_make(kz_c.v[2 * q], kz_c.v[2 * q + 1]);
                const T2 tk = pr_mul(kin2, tz2);
                const T2 ax = pr_mul(tk, qx2[q]);
                const T2 ay = pr_mul(tk, qy2[q]);
                const T2 cxy = pr_mul(tk, qxy2[q]);
                const T2 az = pr_mul(pr_mul(kz2, iz2), qz2[q]);
                const T2 az3 = pr_mul(az, third2);
                const T2 cxz = pr_fma(ax, third2, az3);
                const T2 cyz = pr_fma(ay, third2, az3);
                const T2 cxyz = pr_mul(pr_add(cxy, az3), third2);
                // z butterfly: pattern (z, face) with faces SS, DS, SD, DD
                const T2 sDS = pr_add(Fl[q][1], F[q][1]), sSD = pr_add(Fl[q][2], F[q][2]);
                const T2 sDD = pr_add(Fl[q][3], F[q][3]);
                const T2 dSS = pr_sub(Fl[q][0], F[q][0]), dDS = pr_sub(Fl[q][1], F[q][1]);
                const T2 dSD = pr_sub(Fl[q][2], F[q][2]), dDD = pr_sub(Fl[q][3], F[q][3]);
                const T2 wDSS = pr_mul(az, dSS);
                const T2 wSDS = pr_mul(ay, sDS), wDDS = pr_mul(cyz, dDS);
                const T2 wSSD = pr_mul(ax, sSD), wDSD = pr_mul(cxz, dSD);
                const T2 wSDD = pr_mul(cxy, sDD), wDDD = pr_mul(cxyz, dDD);
                // lower face (plane p-1) and upper face (plane p) contributions
                tot[q][0] = pr_sub(wDSS, Up[q][0]);
                tot[q][1] = pr_add(Up[q][1], pr_add(wSDS, wDDS));
                tot[q][2] = pr_add(Up[q][2], pr_add(wSSD, wDSD));
                tot[q][3] = pr_add(Up[q][3], pr_add(wSDD, wDDD));
                Up[q][0] = wDSS;
                Up[q][1] = pr_sub(wSDS, wDDS);
                Up[q][2] = pr_sub(wSSD, wDSD);
                Up[q][3] = pr_sub(wSDD, wDDD);
            }
            if (p - 1 >= q0) emit_plane(p - 1, sl_prev, tot);
        }
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
            for (int m = 0; m < 4; ++m) Fl[q][m] = F[q][m];
        sl_prev = sl_cur;
        sl_cur = next_slot(sl_cur);
        if (sl_cur == 0) ph_cur ^= 1u;
        sl_ahead = next_slot(sl_ahead);
    }
    if constexpr (!TMA) cp_async_wait<0>();
    __syncthreads();  // the exchange buffer of plane S-1 is still being read
    if constexpr (TMA) *seq = seq0 + (p_last - p_first + 1);
    if (aborted) return TILE_ABORTED;
    if (q1 > S) {
        T2 top[2][4];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            top[q][0] = pr_sub(pr_make(T(0), T(0)), Up[q][0]);
            top[q][1] = Up[q][1];
            top[q][2] = Up[q][2];
            top[q][3] = Up[q][3];
        }
        emit_plane(S, sl_prev, top);
    }
    __syncthreads();  // shared memory is free for the next tile
    return TILE_DONE;
}

// Grid epilogue of the p.Ap and residual launches: block partials, then the
// last block to finish merges them in block order and sets the scalars.
template <typename T, int EPI>
__device__ __forceinline__ void apply_reduce(const ApplyParams<T>& P, const T dot, const double rmax, const int nblocks,
                                             const int bid) {
    constexpr bool DOT = EPI == EPI_DOT;
    using Acc = typename AccOf<T>::type;
    __shared__ __align__(16) unsigned char red_scratch_raw[sizeof(Acc) * 32];
    Acc* const red_scratch = reinterpret_cast<Acc*>(red_scratch_raw);
    __shared__ double max_scratch[32];

    Acc accs[1];
    accs[0].s = dot;
    block_merge<1>(accs, red_scratch);
    double bmax = 0.0;
    if (EPI == EPI_RESIDUAL) bmax = block_max(rmax, max_scratch);
    if (threadIdx.x == 0) {
        acc_store(P.partials + (size_t)bid * 4, accs[0]);
        if (EPI == EPI_RESIDUAL) P.partials[(size_t)bid * 4 + 2] = bmax;
    }
    if (!last_block(P.counter)) return;
    Acc tot[1];
    grid_merge<1>(P.partials, nblocks, 4, tot, red_scratch, P.counter);
    double gmax = 0.0;
    if (EPI == EPI_RESIDUAL) {
        double m = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x) m = fmax(m, __ldcg(P.partials + (size_t)b * 4 + 2));
        gmax = block_max(m, max_scratch);
    }
    if (threadIdx.x == 0) {
        SolveCtl* ctl = P.ctl;
        if (DOT) {
            const double pq = tot[0].value();
            ctl->pq = pq;
            ctl->applications += 1;
            if (ctl->state == ST_STAGE_TIMEOUT) {
                // a block gave up on its tiles: p.Ap is incomplete, and the
                // state must keep saying why the PCG stopped
            } else if (!(isfinite(pq) && pq > 0.0)) {
                ctl->state = ST_NOT_SPD;
            } else {
                ctl->alpha = ctl->rz / pq;
            }
        } else {
            ctl->res2 = tot[0].value();
            ctl->peak = gmax;
        }
        if (P.clock != nullptr) {
            KernelClock* clk = P.clock;
            const unsigned long long first = atomicExch(&clk->first, ~0ULL);
            clk->total_ns += global_ns() - first;
            clk->count += 1;
        }
    }
}

// One block per tile.  With TMA the stages are filled by tensor copies (the
// maps are a __grid_constant__ parameter, whose address the copies take).
template <typename T, int MODE, int EPI, int ROWS, bool TMA = false, int STAGES = kStages>
__global__ void __launch_bounds__(16 * ROWS, ApplyOccupancy<T, ROWS>::min_blocks)
    apply_kernel(const ApplyParams<T> P, const __grid_constant__ ApplyMaps M) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    pdl_trigger();
    T dot = T(0);  // per-thread sum, merged with compensation across the grid
    double rmax = 0.0;
    int seq = 0;
    if (apply_tile<T, MODE, EPI, ROWS, TMA, STAGES>(P, blockIdx.x, blockIdx.y, smem_raw, dot, rmax, true, 0, 1 << 30,
                                                    &M, &seq) == TILE_SKIP)
        return;
    if (EPI == EPI_STORE) return;
    apply_reduce<T, EPI>(P, dot, rmax, gridDim.x * gridDim.y, blockIdx.y * gridDim.x + blockIdx.x);
}

// The same action with the work balanced over a grid of one wave.  The
// (tile, node plane) pairs of the board, tile-major, are split into gridDim.x
// contiguous ranges of (almost) equal length; a block writes its range, which
// may end inside one tile and continue in the next.  A board whose tile count
// is just above a multiple of the resident blocks (c2 at 8-row tiles: 666
// tiles on 592 slots) would otherwise run a second, nearly empty wave of
// whole tiles.
template <typename T, int MODE, int EPI, int ROWS, bool TMA = false>
__global__ void __launch_bounds__(16 * ROWS, ApplyOccupancy<T, ROWS>::min_blocks)
    apply_split_kernel(const ApplyParams<T> P, const int gx, const int tiles, const __grid_constant__ ApplyMaps M) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    pdl_trigger();
    T dot = T(0);
    double rmax = 0.0;
    const int planes = P.S + 1;
    const long long work = (long long)tiles * planes;
    const long long lo = (long long)blockIdx.x * work / gridDim.x;
    const long long hi = (long long)(blockIdx.x + 1) * work / gridDim.x;
    bool gate = true;
    int seq = 0;
    for (long long u = lo; u < hi;) {
        const int t = (int)(u / planes);
        const int q0 = (int)(u - (long long)t * planes);
        const int q1 = (int)((hi - u < (long long)(planes - q0)) ? q0 + (hi - u) : planes);
        const int st = apply_tile<T, MODE, EPI, ROWS, TMA>(P, t % gx, t / gx, smem_raw, dot, rmax, gate, q0, q1, &M,
                                                           &seq);
        if (st == TILE_SKIP) return;
        gate = false;
        if (st == TILE_ABORTED) break;  // the block's mbarrier phases are no longer in step with its tiles
        u += q1 - q0;
    }
    if (gate) {  // an empty range (more blocks than pairs) still orders itself after the predecessor
        pdl_wait();
        if (EPI == EPI_DOT && P.ctl->state != ST_RUNNING) return;
    }
    if (EPI == EPI_STORE) return;
    apply_reduce<T, EPI>(P, dot, rmax, gridDim.x, blockIdx.x);
}

}  // namespace tb
