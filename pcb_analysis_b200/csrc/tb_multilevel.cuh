// Multilevel preconditioner of the inner FP32 PCG:
//
//     M^-1 r = T^-1 r + Z_1 V_1(Z_1^T r)
//
// T is the z-line block of the operator: for every node column (y, x) the
// tridiagonal coupling of its nodes along z.  On copper stacks the two node
// planes of a thin copper slab are coupled some fifty times more strongly
// through the slab than along it, so point Jacobi leaves the in-plane error of
// such a plane pair almost unscaled; solving the column exactly (LDL^T, one
// forward and one backward sweep) removes that stiffness from the PCG.
//
// Z_1 aggregates 4 x 4 free nodes of one node layer (the reference's patch
// space of two_level.py with a patch width of 4), and the coarse operators
// are Galerkin products A_{l+1} = Z_l^T A_l Z_l down to a grid of at most 2048
// unknowns, whose dense inverse ends the hierarchy.  V_1 is one symmetric
// V-cycle over the coarse levels: damped z-line smoothing (omega = 2/3) before
// and after each coarse correction.  Every piece is a fixed linear map and
// the V-cycle is symmetric, so M is SPD and the PCG stays a plain PCG.  The
// two-level preconditioner's patch width grows with the board (a 2048 x 2048
// board needs patches 205 nodes wide to stay under 2048 unknowns), and its
// iteration count with it; this hierarchy keeps the patch width at 4 on every
// level, so the count stays nearly flat in the board size.
//
// Storage of a coarse level: node grid (L, ny, nx) without row padding; the
// symmetric 27-point stencil as the 14 upper coefficients A(i, i + d(o)),
// o = 9 (dz + 1) + 3 (dy + 1) + (dx + 1) in 13..26, one array per o; the lower
// ones are read from the neighbour, A(i, i + d(o)) = A(i + d(o), i) =
// st[26 - o](i + d(o)).  A coarse node whose aggregate holds no free node is
// empty: a unit row and column, marked by a negative z-line reciprocal and
// left out of every restriction and prolongation.
//
// Per inner iteration: ml_update (r -= alpha q, T^-1 r, Z_1^T r, r.r and
// r.T^-1 r in one pass over the node columns), then per coarse level a
// pre-smoothing (one thread per column) and a residual-with-restriction
// kernel (one thread per node), the dense coarse product, per level the
// prolongation and the residual (per node) and a post-smoothing kernel (per
// column; the top one finishes r.z and beta), and ml_direction (p = T^-1 r + Z_1 c + beta p,
// x += alpha p).
#pragma once

#include <cuda.h>  // CUtensorMap (the type only; maps are encoded by the host)
#include <cuda_runtime.h>
#include <stdint.h>

#include "tb_apply.cuh"
#include "tb_coarse.cuh"
#include "tb_reduce.cuh"
#include "tb_types.h"
#include "tb_vec.cuh"

namespace tb {

constexpr int kMlAgg = 4;        // aggregate width (nodes) along x and y from the fine grid to level 1
constexpr int kMlThreads = 256;  // 32 lanes along x, 8 warps along y
constexpr int kMlTile = 32;      // block tile: 32 node columns along x
constexpr int kMlMaxPlanes = 33;
constexpr float kMlOmega = 2.0f / 3.0f;
constexpr int kMlStencil = 14;   // stored coefficients per coarse node

// ML_ITER: an inner FP32 PCG iteration; ML_START: the inner start from the
// FP64 outer residual; ML_ONLY: a bare preconditioner action; ML_PRE64: the
// preconditioner of an FP64 PCG iteration (its residual read from r64).
enum { ML_ITER = 0, ML_START = 1, ML_ONLY = 2, ML_PRE64 = 3 };

struct MLGrid {
    int L, ny, nx;
    long long plane;  // ny * nx
    long long n;      // L * plane
    int b;            // width of the aggregates (b x b node columns) that form the next level; 0 on the coarsest
};

// Aggregate width from a level to the next: 4 x 4 from the fine grid to
// level 1 (the fine pass and the direction update are built for it); below,
// one width for every coarse level of the board: 2 x 2 when the first coarse
// grid is more than kMlWideSide node columns across, 4 x 4 otherwise.  On a
// large board the narrower aggregates keep every coarse operator close to the
// one above it, which cuts the iteration count (c3, 71 M nodes: 598 -> 468
// inner iterations, 0.74 -> 0.64 s); mixing the widths on one board measured
// worse (c3: 559 iterations with 2 x 2 only on grids wider than 200 columns).
// On a small board the extra levels cost more in launch latency than they
// save (c2, 3.4 M nodes: 464 -> 452 iterations but 0.056 -> 0.073 s).
constexpr int kMlWideSide = 200;
__host__ __device__ constexpr int ml_aggregate_width(int level, int ny1, int nx1) {  // ny1, nx1: level 1's grid
    return level == 0 ? kMlAgg : ((ny1 > kMlWideSide || nx1 > kMlWideSide) ? 2 : 4);
}

__device__ __forceinline__ long long ml_index(const MLGrid& g, int z, int y, int x) {
    return (long long)z * g.plane + (long long)y * g.nx + x;
}

// A(i, i + d(o)) of a coarse level from the symmetric half storage.
template <typename T>
__device__ __forceinline__ T ml_coef(const T* __restrict__ st, long long n, long long i, long long j, int o) {
    return (o >= 13) ? st[(long long)(o - 13) * n + i] : st[(long long)(13 - o) * n + j];
}

// sum_o A(i, j_o) v_j at node (z, y, x) of level g, in a fixed order (dz,
// dy, dx ascending).  INTERIOR: every neighbour exists (1 <= x <= nx-2 and
// the same for y and z), so no term is tested; otherwise the terms outside
// the grid are left out.  Both give the same sum for an interior node.
// Indices are 32-bit: a level's 14 stencil arrays hold fewer than 2^31
// values (checked at set-up).
template <bool INTERIOR>
__device__ __forceinline__ float ml_stencil_dot(const float* __restrict__ st, const float* __restrict__ v,
                                                const MLGrid& g, int z, int y, int x) {
    const int n = (int)g.n, plane = (int)g.plane, nx = g.nx;
    const int i = z * plane + y * nx + x;
    float acc = 0.f;
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz) {
        if (!INTERIOR && (z + dz < 0 || z + dz >= g.L)) continue;
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy) {
            if (!INTERIOR && (y + dy < 0 || y + dy >= g.ny)) continue;
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx) {
                if (!INTERIOR && (x + dx < 0 || x + dx >= nx)) continue;
                const int o = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
                const int j = i + dz * plane + dy * nx + dx;
                const float a = (o >= 13) ? __ldg(st + (o - 13) * n + i) : __ldg(st + (13 - o) * n + j);
                acc = fmaf(a, __ldg(v + j), acc);
            }
        }
    }
    return acc;
}

__device__ __forceinline__ bool ml_interior(const MLGrid& g, int z, int y, int x) {
    return x >= 1 && x + 1 < g.nx && y >= 1 && y + 1 < g.ny && z >= 1 && z + 1 < g.L;
}

// Last-block finish of a 2D grid's per-block accumulators.
template <int NA>
__device__ __forceinline__ bool ml_finish(Acc32 (&acc)[NA], Acc32* scratch, double* partials, unsigned int* counter,
                                          Acc32 (&tot)[NA]) {
    block_merge<NA>(acc, scratch);
    const int b = blockIdx.y * gridDim.x + blockIdx.x;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NA; ++k) acc_store(partials + (size_t)b * 4 + 2 * k, acc[k]);
    }
    if (!last_block(counter)) return false;
    grid_merge<NA>(partials, gridDim.x * gridDim.y, 4, tot, scratch, counter);
    return threadIdx.x == 0;
}

// ------------------------------------------------------------ fine level
// One pass over the fine node columns.  Thread (lane, warp) of block (bx, by)
// owns node column x = 32 bx + lane of node row y = 8 by + warp and walks the
// planes bottom to top:
//   ML_ITER:  r -= alpha q (the PCG update);  ML_START: r = f32(r64 * scale),
//   x = 0 (the inner start);  ML_ONLY: r as given (a preconditioner action);
//   ML_PRE64: r = f32(r64 * scale) of an FP64 PCG, left unwritten;
// the LDL^T forward sweep of the column block (g = r - l g_below, h = g / p,
// kept in registers), r.r and r.T^-1 r = sum g h (FMA chains per thread, compensated merges), and the
// partial aggregate sums of R_1 = Z_1^T r over the free nodes (lanes x ^ 1,
// x ^ 2); then the backward sweep w = h - l_above w_above, w = T^-1 r, from
// registers, and after one barrier the sums over the four rows of each
// aggregate, in that order.  Fixed rows carry a -1
// reciprocal (their block row is the identity, so w = r there); pads carry 0.
template <int NP, int MODE>
__global__ void __launch_bounds__(kMlThreads)
    ml_update(float* __restrict__ r, const float* __restrict__ q, const double* __restrict__ r64,
              float* __restrict__ x32, float* __restrict__ w, float* __restrict__ R1, const float* __restrict__ zl,
              const float* __restrict__ zi, Layout lay, long long pstride, MLGrid g1, SolveCtl* ctl,
              double* partials, unsigned int* counter, KernelClock* clock) {
    __shared__ __align__(16) unsigned char scratch_raw[sizeof(Acc32) * 2 * 32];
    __shared__ float s_part[NP][8][8];  // [plane][row of the block][aggregate column of the block]
    Acc32* const scratch = reinterpret_cast<Acc32*>(scratch_raw);
    pdl_enter();
    if ((MODE == ML_ITER || MODE == ML_PRE64) && ctl->state != ST_RUNNING) return;
    if (MODE == ML_ITER && clock != nullptr && threadIdx.x == 0) atomicMin(&clock->first, global_ns());
    const float alpha = (MODE == ML_ITER) ? (float)ctl->alpha : 0.f;
    const double scale = (MODE == ML_START || MODE == ML_PRE64) ? ctl->scale : 1.0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int x = blockIdx.x * kMlTile + lane;
    const int y = blockIdx.y * 8 + warp;
    const int np = lay.S + 1;
    const bool mine = (x < lay.Xp) && (y <= lay.R);
    // 32-bit node offsets: a fine vector holds fewer than 2^31 values (checked at set-up)
    const int col = y * lay.Xp + x, pst = (int)pstride;
    // All planes' loads first, at clamped (always valid) addresses and with no
    // branch between them, so that they are in flight together; then the
    // sweeps.  No barrier inside the plane loops: the per-plane partial sums
    // of the restriction wait in shared memory.
    const int colc = mine ? col : 0;
    float H[NP], Lz[NP], Ip[NP];  // r (then h of the forward sweep), the multipliers l, the reciprocals 1/p
#pragma unroll
    for (int z = 0; z < NP; ++z) {
        const int idx = (z < np ? z : np - 1) * pst + colc;
        if (MODE == ML_ITER) H[z] = fmaf(-alpha, q[idx], r[idx]);
        else if (MODE == ML_START || MODE == ML_PRE64) H[z] = (float)(r64[idx] * scale);
        else H[z] = r[idx];
        Lz[z] = zl[idx];
        Ip[z] = zi[idx];
    }
    float gp = 0.f;
    // r.r and r.T^-1 r = sum g h: both sums have non-negative terms (h = g |1/p|),
    // so a thread's plain FMA chain over its column loses no digits to
    // cancellation; the merges across threads and blocks are compensated.
    float rr = 0.f, gh = 0.f;
#pragma unroll
    for (int z = 0; z < NP; ++z) {
        if (z < np) {
            float s = 0.f;
            if (mine) {
                const int idx = z * pst + col;
                const float rv = H[z];
                if (MODE == ML_ITER || MODE == ML_START) r[idx] = rv;
                if (MODE == ML_START) x32[idx] = 0.f;
                const float l = Lz[z], ip = Ip[z];
                const float gg = fmaf(-l, gp, rv);
                const float h = gg * fabsf(ip);
                H[z] = h;
                gp = gg;
                if (ip >= 0.f) s = rv;
                if (MODE != ML_ONLY) {
                    rr = fmaf(rv, rv, rr);
                    gh = fmaf(gg, h, gh);
                }
            }
            s += __shfl_xor_sync(0xffffffffu, s, 1);
            s += __shfl_xor_sync(0xffffffffu, s, 2);
            if ((lane & 3) == 0) s_part[z][warp][lane >> 2] = s;
        }
    }
    if (mine) {
        float wn = 0.f;
#pragma unroll
        for (int z = NP - 1; z >= 0; --z) {
            if (z < np) {
                const float lup = (z + 1 < np) ? Lz[z + 1 < NP ? z + 1 : z] : 0.f;
                wn = fmaf(-lup, wn, H[z]);
                w[z * pst + col] = wn;
            }
        }
    }
    __syncthreads();
    // the block's aggregates: rows 2 by, 2 by + 1 of level 1, columns 8 bx .. 8 bx + 7, every plane
    for (int k = threadIdx.x; k < 16 * np; k += blockDim.x) {
        const int z = k >> 4, a_row = (k >> 3) & 1, a_col = k & 7;
        const int AY = blockIdx.y * 2 + a_row, AX = blockIdx.x * 8 + a_col;
        if (AY < g1.ny && AX < g1.nx) {
            const float(&b)[8][8] = s_part[z];
            const int w0 = 4 * a_row;
            R1[ml_index(g1, z, AY, AX)] = (b[w0][a_col] + b[w0 + 1][a_col]) + (b[w0 + 2][a_col] + b[w0 + 3][a_col]);
        }
    }
    if (MODE == ML_ONLY) return;
    Acc32 acc[2], tot[2];
    acc[0].s = rr;
    acc[1].s = gh;
    if (ml_finish<2>(acc, scratch, partials, counter, tot)) {
        if (MODE == ML_ITER) finalize_update_2l(ctl, tot[0].value(), tot[1].value());
        else if (MODE == ML_PRE64) ctl->rdr = tot[1].value();
        else finalize_start_2l(ctl, tot[0].value(), tot[1].value());
        if (MODE == ML_ITER && clock != nullptr) {  // device time: first block's start to the last block's end
            const unsigned long long first = atomicExch(&clock->first, ~0ULL);
            clock->total_ns += global_ns() - first;
            clock->count += 1;
        }
    }
}

// ------------------------------------------------- fine level, staged
// The fine pass of an inner PCG iteration (ML_ITER) as a persistent kernel
// fed by tensor copies.  ml_update's blocks load every plane of their
// columns and then compute, so an SM's loads come in bursts and HBM idles
// while its blocks compute.  Here one block per SM walks the 32 x 8 column
// tiles t = blockIdx.x + k gridDim.x; thread 0 copies a tile's q, r, l and
// 1/p boxes (32 x 8 columns x np planes each, zero outside the field) into
// one of `stages` shared-memory stages with cp.async.bulk.tensor onto the
// stage's mbarrier, stages - 1 tiles ahead of the tile computed, so that the
// copies stream without a pause.  Per column the arithmetic is ml_update's:
// r -= alpha q, the z-line sweeps, the partial aggregate sums of R_1 and the
// column's r.r and r.T^-1 r as plain FMA chains; the column sums then enter
// the thread's compensated accumulators, which merge across the block and
// the grid in a fixed order.  Every wait on a stage is bounded: a block that
// gives up lets its copies in flight land (bounded), sets the error word and
// the solve state, and still takes its part in the grid reduction.
constexpr int kMlMaxStages = 4;
struct MLStageMaps {
    CUtensorMap q, r, zl, zi;  // (S+1, R+1, Xp) node fields, box 32 x 8 x np
    int* err;                  // set to 1 when a block gave up waiting for its tiles
    int test_polls;            // test only: > 0 arms the stages without copies, waits give up after this many polls
};

template <int NP>
__global__ void __launch_bounds__(kMlThreads, 1)
    ml_update_staged(float* __restrict__ r, float* __restrict__ w, float* __restrict__ R1, Layout lay,
                     long long pstride, MLGrid g1, SolveCtl* ctl, double* partials, unsigned int* counter,
                     KernelClock* clock, int tiles_x, int tiles, int stages, const __grid_constant__ MLStageMaps M) {
    extern __shared__ __align__(128) unsigned char ml_stage_raw[];
    __shared__ __align__(16) unsigned char scratch_raw[sizeof(Acc32) * 2 * 32];
    __shared__ float s_part[NP][8][8];  // [plane][row of the tile][aggregate column of the tile]
    __shared__ __align__(8) unsigned long long s_bar[kMlMaxStages];
    Acc32* const scratch = reinterpret_cast<Acc32*>(scratch_raw);
    // tensor copies write 128-byte aligned boxes: the launch adds 128 bytes
    // to the stages so that their base can be rounded up
    float* const stage = reinterpret_cast<float*>(ml_stage_raw + ((128u - (smem_u32(ml_stage_raw) & 127u)) & 127u));
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int np = lay.S + 1, pst = (int)pstride;
    const int plane_box = kMlTile * 8;  // floats of one plane of a box
    const int stage_floats = 4 * np * plane_box;
    const uint32_t stage_bytes = (uint32_t)stage_floats * sizeof(float);
    const uint32_t bar0 = smem_u32(s_bar);
    const int ntiles = (int)blockIdx.x < tiles ? (tiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    const int polls = M.test_polls > 0 ? M.test_polls : kStageSpinLimit;
    if (tid == 0) {
        for (int i = 0; i < stages; ++i) mbar_init(bar0 + 8 * i, 1);
        mbar_init_fence();
    }
    pdl_enter();  // q and alpha come from the operator
    if (ctl->state != ST_RUNNING) return;  // uniform across the grid
    if (clock != nullptr && tid == 0) atomicMin(&clock->first, global_ns());
    __syncthreads();  // the barriers are initialised
    const float alpha = (float)ctl->alpha;

    // tile k of this block into stage k % stages
    auto issue = [&](const int k) {
        const int t = (int)blockIdx.x + k * (int)gridDim.x;
        const uint32_t bar = bar0 + 8 * (k % stages);
        mbar_expect_tx(bar, stage_bytes);
        if (M.test_polls > 0) return;  // test: the stage stays armed, nothing is copied
        const int tx = t % tiles_x, ty = t / tiles_x;
        float* const dst = stage + (k % stages) * stage_floats;
        tma_load_3d(dst, &M.q, tx * kMlTile, ty * 8, 0, bar);
        tma_load_3d(dst + np * plane_box, &M.r, tx * kMlTile, ty * 8, 0, bar);
        tma_load_3d(dst + 2 * np * plane_box, &M.zl, tx * kMlTile, ty * 8, 0, bar);
        tma_load_3d(dst + 3 * np * plane_box, &M.zi, tx * kMlTile, ty * 8, 0, bar);
    };
    if (tid == 0)
        for (int k = 0; k < stages - 1 && k < ntiles; ++k) issue(k);

    Acc32 acc[2];
    for (int k = 0; k < ntiles; ++k) {
        // the stage of tile k - 1 was released by the barrier that ended it
        if (tid == 0 && k + stages - 1 < ntiles) issue(k + stages - 1);
        const bool ok = mbar_wait(bar0 + 8 * (k % stages), (uint32_t)((k / stages) & 1), polls);
        if (!__syncthreads_and(ok)) {
            if (tid == 0) {  // let the copies in flight (tiles k .. k + stages - 2) land before the block goes on
                for (int j = k; j < k + stages - 1 && j < ntiles; ++j)
                    mbar_wait(bar0 + 8 * (j % stages), (uint32_t)((j / stages) & 1), polls);
                atomicExch(M.err, 1);
                ctl->state = ST_STAGE_TIMEOUT;
            }
            break;
        }
        const int t = (int)blockIdx.x + k * (int)gridDim.x;
        const int tx = t % tiles_x, ty = t / tiles_x;
        const int x = tx * kMlTile + lane, y = ty * 8 + warp;
        const bool mine = (x < lay.Xp) && (y <= lay.R);
        const int col = mine ? y * lay.Xp + x : 0;
        const float* const sq = stage + (k % stages) * stage_floats + warp * kMlTile + lane;
        const float* const sr = sq + np * plane_box;
        const float* const sl = sq + 2 * np * plane_box;
        const float* const si = sq + 3 * np * plane_box;
        float H[NP], Lz[NP];
        float gp = 0.f, rr = 0.f, gh = 0.f;
#pragma unroll
        for (int z = 0; z < NP; ++z) {
            if (z < np) {
                const float rv = fmaf(-alpha, sq[z * plane_box], sr[z * plane_box]);
                const float l = sl[z * plane_box], ip = si[z * plane_box];
                if (mine) r[z * pst + col] = rv;
                const float gg = fmaf(-l, gp, rv);
                const float h = gg * fabsf(ip);
                H[z] = h;
                Lz[z] = l;
                gp = gg;
                rr = fmaf(rv, rv, rr);
                gh = fmaf(gg, h, gh);
                // outside the field every staged value is zero, so s is too
                float s = (ip >= 0.f) ? rv : 0.f;
                s += __shfl_xor_sync(0xffffffffu, s, 1);
                s += __shfl_xor_sync(0xffffffffu, s, 2);
                if ((lane & 3) == 0) s_part[z][warp][lane >> 2] = s;
            }
        }
        if (mine) {
            float wn = 0.f;
#pragma unroll
            for (int z = NP - 1; z >= 0; --z) {
                if (z < np) {
                    const float lup = (z + 1 < np) ? Lz[z + 1 < NP ? z + 1 : z] : 0.f;
                    wn = fmaf(-lup, wn, H[z]);
                    w[z * pst + col] = wn;
                }
            }
        }
        Acc32 cr, cg;
        cr.s = rr;
        cg.s = gh;
        acc[0].merge(cr);
        acc[1].merge(cg);
        __syncthreads();  // the tile's partial sums are complete and its stage is free
        for (int i = tid; i < 16 * np; i += blockDim.x) {
            const int z = i >> 4, a_row = (i >> 3) & 1, a_col = i & 7;
            const int AY = ty * 2 + a_row, AX = tx * 8 + a_col;
            if (AY < g1.ny && AX < g1.nx) {
                const float(&b)[8][8] = s_part[z];
                const int w0 = 4 * a_row;
                R1[ml_index(g1, z, AY, AX)] = (b[w0][a_col] + b[w0 + 1][a_col]) + (b[w0 + 2][a_col] + b[w0 + 3][a_col]);
            }
        }
        // the next tile's s_part writes follow its stage vote, a barrier
    }
    Acc32 tot[2];
    if (ml_finish<2>(acc, scratch, partials, counter, tot)) {
        if (ctl->state != ST_STAGE_TIMEOUT) finalize_update_2l(ctl, tot[0].value(), tot[1].value());
        if (clock != nullptr) {  // device time: first block's start to the last block's end
            const unsigned long long first = atomicExch(&clock->first, ~0ULL);
            clock->total_ns += global_ns() - first;
            clock->count += 1;
        }
    }
}

// ------------------------------------------------- FP64 PCG, multilevel
// The plain FP64 PCG with the multilevel preconditioner: FP64 vectors, dots
// and updates; the preconditioner applied in FP32 to f32(r) (ML_PRE64 fine
// pass, V-cycle), its result widened to FP64.
//
// x += alpha p, r -= alpha q, r.r (FP64); the stopping test; r.z and beta
// follow from the preconditioner's kernels.
__global__ void __launch_bounds__(kVecThreads)
    pcg_update_f64_norm(double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
                        const double* __restrict__ q, long long nq, SolveCtl* ctl, double* partials,
                        unsigned int* counter) {
    __shared__ __align__(16) unsigned char scratch_raw[sizeof(Acc64) * 32];
    Acc64* const scratch = reinterpret_cast<Acc64*>(scratch_raw);
    pdl_enter();
    if (ctl->state != ST_RUNNING) return;
    const double alpha = ctl->alpha;
    Acc64 acc[1];
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < 2 * nq; i += stride) {
        double2 xv = reinterpret_cast<double2*>(x)[i];
        double2 rv = reinterpret_cast<double2*>(r)[i];
        const double2 pv = reinterpret_cast<const double2*>(p)[i];
        const double2 qv = reinterpret_cast<const double2*>(q)[i];
        xv.x = fma(alpha, pv.x, xv.x);
        xv.y = fma(alpha, pv.y, xv.y);
        rv.x = fma(-alpha, qv.x, rv.x);
        rv.y = fma(-alpha, qv.y, rv.y);
        reinterpret_cast<double2*>(x)[i] = xv;
        reinterpret_cast<double2*>(r)[i] = rv;
        acc[0].add_product(rv.x, rv.x);
        acc[0].add_product(rv.y, rv.y);
    }
    Acc64 tot[1];
    if (finish_partials<1>(acc, scratch, partials, counter, tot)) finalize_update_2l(ctl, tot[0].value(), ctl->rdr);
}

// p = f64(T^-1 r + Z_1 c) + beta p (START: without beta p).
template <bool START>
__global__ void __launch_bounds__(kVecThreads)
    ml_direction_f64(double* __restrict__ p, const float* __restrict__ w, const float* __restrict__ c1,
                     const float* __restrict__ zi, long long nq, Layout lay, MLGrid g1,
                     unsigned long long fixed_planes, const SolveCtl* ctl) {
    pdl_enter();
    if (ctl->state != ST_RUNNING) return;
    const double beta = START ? 0.0 : ctl->beta;
    const int qpl = lay.Xp / 4, rows = lay.R + 1;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += stride) {
        const long long line = i / qpl;
        const int q = (int)(i - line * qpl);
        const int z = (int)(line / rows);
        const int y = (int)(line - (long long)z * rows);
        const float4 wv = reinterpret_cast<const float4*>(w)[i];
        const float cv = c1[ml_index(g1, z, y / kMlAgg, q)];
        const int x0 = 4 * q;
        bool fr[4] = {x0 <= lay.C, x0 + 1 <= lay.C, x0 + 2 <= lay.C, x0 + 3 <= lay.C};
        if (z >= 64 || ((fixed_planes >> z) & 1ULL)) {
            const float4 m = reinterpret_cast<const float4*>(zi)[i];
            fr[0] = fr[0] && m.x >= 0.f;
            fr[1] = fr[1] && m.y >= 0.f;
            fr[2] = fr[2] && m.z >= 0.f;
            fr[3] = fr[3] && m.w >= 0.f;
        }
        const double z0 = (double)(wv.x + (fr[0] ? cv : 0.f)), z1 = (double)(wv.y + (fr[1] ? cv : 0.f));
        const double z2 = (double)(wv.z + (fr[2] ? cv : 0.f)), z3 = (double)(wv.w + (fr[3] ? cv : 0.f));
        double2* pp = reinterpret_cast<double2*>(p) + 2 * i;
        if (START) {
            pp[0] = make_double2(z0, z1);
            pp[1] = make_double2(z2, z3);
        } else {
            const double2 a = pp[0], b = pp[1];
            pp[0] = make_double2(fma(beta, a.x, z0), fma(beta, a.y, z1));
            pp[1] = make_double2(fma(beta, b.x, z2), fma(beta, b.y, z3));
        }
    }
}

// p = T^-1 r + Z_1 c + beta p on the fine level (START: without beta p);
// not START: x += alpha p first (the update's step, on the old p).  A quad
// of four nodes lies in one aggregate.  The free mask (sign of the z-line
// reciprocal) is read only on planes that hold a fixed node.
template <bool START>
__global__ void __launch_bounds__(kVecThreads)
    ml_direction(float* __restrict__ p, float* __restrict__ x, const float* __restrict__ w,
                 const float* __restrict__ c1, const float* __restrict__ zi, long long nq, Layout lay, MLGrid g1,
                 unsigned long long fixed_planes, const SolveCtl* ctl) {
    pdl_enter();
    if (ctl != nullptr && ctl->state != ST_RUNNING) return;
    const float beta = (START || ctl == nullptr) ? 0.f : (float)ctl->beta;
    const float alpha = (START || ctl == nullptr) ? 0.f : (float)ctl->alpha;
    const int qpl = lay.Xp / 4, rows = lay.R + 1;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long i0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long line0 = i0 / qpl;
    int q = (int)(i0 - line0 * qpl);
    int z = (int)(line0 / rows);
    int y = (int)(line0 - (long long)z * rows);
    const long long sline = stride / qpl;
    const int sq = (int)(stride - sline * qpl);
    const int sz = (int)(sline / rows);
    const int sy = (int)(sline - (long long)sz * rows);
    for (long long i = i0; i < nq; i += stride) {
        const float4 wv = reinterpret_cast<const float4*>(w)[i];
        const float cv = c1[ml_index(g1, z, y / kMlAgg, q)];
        const int x0 = 4 * q;
        bool fr[4] = {x0 <= lay.C, x0 + 1 <= lay.C, x0 + 2 <= lay.C, x0 + 3 <= lay.C};
        if (z >= 64 || ((fixed_planes >> z) & 1ULL)) {
            const float4 m = reinterpret_cast<const float4*>(zi)[i];
            fr[0] = fr[0] && m.x >= 0.f;
            fr[1] = fr[1] && m.y >= 0.f;
            fr[2] = fr[2] && m.z >= 0.f;
            fr[3] = fr[3] && m.w >= 0.f;
        }
        float4 zv = make_float4(wv.x + (fr[0] ? cv : 0.f), wv.y + (fr[1] ? cv : 0.f), wv.z + (fr[2] ? cv : 0.f),
                                wv.w + (fr[3] ? cv : 0.f));
        if (!START && ctl != nullptr) {
            const float4 pv = reinterpret_cast<const float4*>(p)[i];
            float4 xv = reinterpret_cast<const float4*>(x)[i];
            xv.x = fmaf(alpha, pv.x, xv.x);
            xv.y = fmaf(alpha, pv.y, xv.y);
            xv.z = fmaf(alpha, pv.z, xv.z);
            xv.w = fmaf(alpha, pv.w, xv.w);
            reinterpret_cast<float4*>(x)[i] = xv;
            zv.x = fmaf(beta, pv.x, zv.x);
            zv.y = fmaf(beta, pv.y, zv.y);
            zv.z = fmaf(beta, pv.z, zv.z);
            zv.w = fmaf(beta, pv.w, zv.w);
        }
        reinterpret_cast<float4*>(p)[i] = zv;
        q += sq;
        y += sy;
        z += sz;
        if (q >= qpl) {
            q -= qpl;
            ++y;
        }
        if (y >= rows) {
            y -= rows;
            ++z;
        }
    }
}

// ------------------------------------------------------------ coarse levels
// Two thread layouts: the z-line kernels give each thread one node column
// (all planes, a 1D grid over the columns); the residual kernels give each
// thread one node (block = 32 columns x 8 rows of one plane, grid.z = plane),
// so the 27-point stencils of a level run fully in parallel.

// x = omega T^-1 R on column c of level g (pre-smoothing from zero): every
// plane's loads first, at clamped addresses, then the sweeps.
template <int NP>
__device__ __forceinline__ void ml_presmooth_column(const float* __restrict__ R, float* __restrict__ xo,
                                                    const float* __restrict__ lf, const float* __restrict__ ipd,
                                                    const MLGrid& g, long long c) {
    float H[NP], Lz[NP], Ip[NP];
#pragma unroll
    for (int z = 0; z < NP; ++z) {
        const long long idx = (long long)(z < g.L ? z : g.L - 1) * g.plane + c;
        H[z] = R[idx];
        Lz[z] = lf[idx];
        Ip[z] = ipd[idx];
    }
    float gp = 0.f;
#pragma unroll
    for (int z = 0; z < NP; ++z) {
        if (z < g.L) {
            const float gg = fmaf(-Lz[z], gp, H[z]);
            H[z] = gg * fabsf(Ip[z]);
            gp = gg;
        }
    }
    float wn = 0.f;
#pragma unroll
    for (int z = NP - 1; z >= 0; --z) {
        if (z < g.L) {
            const float lup = (z + 1 < g.L) ? Lz[z + 1 < NP ? z + 1 : z] : 0.f;
            wn = fmaf(-lup, wn, H[z]);
            xo[(long long)z * g.plane + c] = kMlOmega * wn;
        }
    }
}

template <int NP>
__global__ void __launch_bounds__(kMlThreads)
    ml_presmooth(const float* __restrict__ R, float* __restrict__ xo, const float* __restrict__ lf,
                 const float* __restrict__ ipd, MLGrid g, const SolveCtl* ctl) {
    pdl_enter();
    if (ctl != nullptr && ctl->state != ST_RUNNING) return;
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.plane) return;
    ml_presmooth_column<NP>(R, xo, lf, ipd, g, c);
}

// Rc = Z^T (R - A x): the residual after pre-smoothing at every node, summed
// over the non-empty nodes of each B x B aggregate (lanes x ^ 1 (, x ^ 2),
// then the aggregate's B rows through shared memory).
// The restriction of one 32 x 8 node tile (bx, by) of plane z: its partial
// aggregate sums go through `s_part` (block shared memory, [8][kMlTile / B]);
// the block's threads all take part.  A caller that runs several tiles in a
// row must place a barrier between them.
template <int B>
__device__ __forceinline__ void ml_restrict_tile(const float* __restrict__ st, const float* __restrict__ R,
                                                 const float* __restrict__ xv, const float* __restrict__ ipd,
                                                 float* __restrict__ Rc, const MLGrid& g, const MLGrid& gc, int bx,
                                                 int by, int z, float (*s_part)[kMlTile / B]) {
    static_assert(B == 2 || B == 4, "aggregates are 2 x 2 or 4 x 4 node columns");
    constexpr int AX_PER_BLOCK = kMlTile / B, AY_PER_BLOCK = 8 / B;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int x = bx * kMlTile + lane, y = by * 8 + warp;
    float s = 0.f;
    if (x < g.nx && y < g.ny) {
        const long long idx = ml_index(g, z, y, x);
        if (ipd[idx] >= 0.f)
            s = R[idx] - (ml_interior(g, z, y, x) ? ml_stencil_dot<true>(st, xv, g, z, y, x)
                                                  : ml_stencil_dot<false>(st, xv, g, z, y, x));
    }
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    if (B == 4) s += __shfl_xor_sync(0xffffffffu, s, 2);
    if ((lane & (B - 1)) == 0) s_part[warp][lane / B] = s;
    __syncthreads();
    if (threadIdx.x < AX_PER_BLOCK * AY_PER_BLOCK) {
        const int a_row = threadIdx.x / AX_PER_BLOCK, a_col = threadIdx.x % AX_PER_BLOCK;
        const int AY = by * AY_PER_BLOCK + a_row, AX = bx * AX_PER_BLOCK + a_col;
        if (AY < gc.ny && AX < gc.nx) {
            const int w0 = B * a_row;
            float v;
            if (B == 4)
                v = (s_part[w0][a_col] + s_part[w0 + 1][a_col]) + (s_part[w0 + 2][a_col] + s_part[w0 + 3][a_col]);
            else
                v = s_part[w0][a_col] + s_part[w0 + 1][a_col];
            Rc[ml_index(gc, z, AY, AX)] = v;
        }
    }
}

template <int B>  // aggregate width g.b: 4 or 2
__global__ void __launch_bounds__(kMlThreads)
    ml_restrict(const float* __restrict__ st, const float* __restrict__ R, const float* __restrict__ xv,
                const float* __restrict__ ipd, float* __restrict__ Rc, MLGrid g, MLGrid gc, const SolveCtl* ctl) {
    __shared__ float s_part[8][kMlTile / B];
    pdl_enter();
    if (ctl != nullptr && ctl->state != ST_RUNNING) return;
    ml_restrict_tile<B>(st, R, xv, ipd, Rc, g, gc, blockIdx.x, blockIdx.y, blockIdx.z, s_part);
}

// x += Z c on the non-empty nodes of a level (c: the correction of the level
// below), before the level's residual.  One node column of kMlProlongPlanes
// planes per thread (block z index = group of planes), every load issued
// before the first store, so that a thread has several nodes' bytes in flight.
constexpr int kMlProlongPlanes = 4;
__device__ __forceinline__ void ml_prolong_column(float* __restrict__ xv, const float* __restrict__ cn,
                                                  const float* __restrict__ ipd, const MLGrid& g, const MLGrid& gc,
                                                  int z0, int y, int x) {
    float xs[kMlProlongPlanes], cs[kMlProlongPlanes], ps[kMlProlongPlanes];
#pragma unroll
    for (int k = 0; k < kMlProlongPlanes; ++k) {
        const int z = min(z0 + k, g.L - 1);  // clamped: valid addresses, stores guarded below
        xs[k] = xv[ml_index(g, z, y, x)];
        ps[k] = ipd[ml_index(g, z, y, x)];
        cs[k] = cn[ml_index(gc, z, y / g.b, x / g.b)];
    }
#pragma unroll
    for (int k = 0; k < kMlProlongPlanes; ++k)
        if (z0 + k < g.L && ps[k] >= 0.f) xv[ml_index(g, z0 + k, y, x)] = xs[k] + cs[k];
}

__global__ void __launch_bounds__(kMlThreads)
    ml_prolong(float* __restrict__ xv, const float* __restrict__ cn, const float* __restrict__ ipd, MLGrid g,
               MLGrid gc, const SolveCtl* ctl) {
    pdl_enter();
    if (ctl != nullptr && ctl->state != ST_RUNNING) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int x = blockIdx.x * kMlTile + lane, y = blockIdx.y * 8 + warp;
    if (x >= g.nx || y >= g.ny) return;
    ml_prolong_column(xv, cn, ipd, g, gc, blockIdx.z * kMlProlongPlanes, y, x);
}

// t = R - A y' at every node (y' the prolonged x), written to `t` (the
// level's output array, which ml_zsmooth then overwrites column by column).
__device__ __forceinline__ void ml_residual_node(const float* __restrict__ st, const float* __restrict__ R,
                                                 const float* __restrict__ xv, float* __restrict__ t,
                                                 const MLGrid& g, int z, int y, int x) {
    const long long idx = ml_index(g, z, y, x);
    t[idx] = R[idx] - (ml_interior(g, z, y, x) ? ml_stencil_dot<true>(st, xv, g, z, y, x)
                                               : ml_stencil_dot<false>(st, xv, g, z, y, x));
}

__global__ void __launch_bounds__(kMlThreads)
    ml_residual(const float* __restrict__ st, const float* __restrict__ R, const float* __restrict__ xv,
                float* __restrict__ t, MLGrid g, const SolveCtl* ctl) {
    pdl_enter();
    if (ctl != nullptr && ctl->state != ST_RUNNING) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int x = blockIdx.x * kMlTile + lane, y = blockIdx.y * 8 + warp, z = blockIdx.z;
    if (x >= g.nx || y >= g.ny) return;
    ml_residual_node(st, R, xv, t, g, z, y, x);
}

// Post-smoothing of column c: y = y' + omega T^-1 t with y' the prolonged x
// and t from ml_residual (read from `yo` before it is overwritten there);
// DOT: also acc += R.y over the column.
template <int NP, bool DOT>
__device__ __forceinline__ void ml_zsmooth_column(const float* __restrict__ R, const float* __restrict__ xv,
                                                  const float* __restrict__ lf, const float* __restrict__ ipd,
                                                  float* __restrict__ yo, const MLGrid& g, long long c, Acc32& acc) {
    float H[NP], Lz[NP], Ip[NP];  // loads of every plane first (clamped addresses), then the sweeps
#pragma unroll
    for (int z = 0; z < NP; ++z) {
        const long long idx = (long long)(z < g.L ? z : g.L - 1) * g.plane + c;
        H[z] = yo[idx];
        Lz[z] = lf[idx];
        Ip[z] = ipd[idx];
    }
    float gp = 0.f;
#pragma unroll
    for (int z = 0; z < NP; ++z) {
        if (z < g.L) {
            const float gg = fmaf(-Lz[z], gp, H[z]);
            H[z] = gg * fabsf(Ip[z]);
            gp = gg;
        }
    }
    float wn = 0.f;
#pragma unroll
    for (int z = NP - 1; z >= 0; --z) {
        if (z < g.L) {
            const long long idx = (long long)z * g.plane + c;
            const float lup = (z + 1 < g.L) ? Lz[z + 1 < NP ? z + 1 : z] : 0.f;
            wn = fmaf(-lup, wn, H[z]);
            const float yv = fmaf(kMlOmega, wn, xv[idx]);
            yo[idx] = yv;
            if (DOT) acc.add_product(R[idx], yv);
        }
    }
}

// Post-smoothing, one column per thread (ml_zsmooth_column).  At the top level (MODE != ML_ONLY) the last block also
// finishes r.z = r.T^-1 r + R.y and, for ML_ITER, beta and the iteration
// limit; ML_START sets r.z.
template <int NP, int MODE, bool TOP>
__global__ void __launch_bounds__(kMlThreads)
    ml_zsmooth(const float* __restrict__ R, const float* __restrict__ xv, const float* __restrict__ lf,
               const float* __restrict__ ipd, float* __restrict__ yo, MLGrid g, SolveCtl* ctl, double* partials,
               unsigned int* counter) {
    __shared__ __align__(16) unsigned char scratch_raw[sizeof(Acc32) * 32];
    Acc32* const scratch = reinterpret_cast<Acc32*>(scratch_raw);
    pdl_enter();
    if (MODE != ML_ONLY && ctl->state != ST_RUNNING) return;
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    Acc32 acc[1];
    if (c < g.plane) ml_zsmooth_column<NP, TOP && MODE != ML_ONLY>(R, xv, lf, ipd, yo, g, c, acc[0]);
    if (!TOP || MODE == ML_ONLY) return;
    Acc32 tot[1];
    if (ml_finish<1>(acc, scratch, partials, counter, tot)) {
        const double rzn = ctl->rdr + tot[0].value();
        if (MODE == ML_START) {
            ctl->rz = rzn;
        } else if (!isfinite(rzn) || ctl->rz == 0.0) {
            ctl->state = ST_BREAKDOWN;
        } else {
            ctl->beta = rzn / ctl->rz;
            ctl->rz = rzn;
            if (ctl->iterations >= ctl->max_it) ctl->state = ST_MAXIT;
        }
    }
}

// ------------------------------------------------------------ set-up (FP64)
// z-line factors of the fine operator: per node column the tridiagonal block
// with the Jacobi diagonal d and the coupling to the node above,
//     e = sum over the four elements of the slab that share the vertical edge
//         of (a_x / 18 + a_y / 18 - a_z / 9)
// (U_x[i,j] = M_z[0,1] M_y[k,k] S_x[m,m] = 1/18, U_y likewise, U_z = -1/9), zero
// when either end is fixed; LDL^T: p_0 = d_0, l_z = e_{z-1} / p_{z-1},
// p_z = d_z - l_z e_{z-1}; stored l_z and 1/p_z (-1 on fixed rows, 0 on pads).
__global__ void ml_fine_factors(float* __restrict__ zl, float* __restrict__ zi, const double* __restrict__ diag,
                                const double* __restrict__ rf, const double* __restrict__ kin,
                                const double* __restrict__ kz, const double* __restrict__ thick,
                                const double* __restrict__ px, const double* __restrict__ py, Layout lay,
                                long long pstride) {
    const long long ncol = (long long)(lay.R + 1) * lay.Xp;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long cidx = (long long)blockIdx.x * blockDim.x + threadIdx.x; cidx < ncol; cidx += stride) {
        const int y = (int)(cidx / lay.Xp);
        const int x = (int)(cidx - (long long)y * lay.Xp);
        if (x > lay.C) {
            for (int z = 0; z <= lay.S; ++z) {
                zl[z * pstride + cidx] = 0.f;
                zi[z * pstride + cidx] = 0.f;
            }
            continue;
        }
        double p_prev = 1.0, e_prev = 0.0;
        for (int z = 0; z <= lay.S; ++z) {
            const long long idx = z * pstride + cidx;
            const bool fixed = rf[idx] < 0.0;
            const double d = fixed ? 1.0 : diag[idx];
            const double l = (z == 0) ? 0.0 : e_prev / p_prev;
            const double p = d - l * e_prev;
            zl[idx] = (float)l;
            zi[idx] = fixed ? -1.0f : (float)(1.0 / p);
            double e = 0.0;
            if (z < lay.S && !fixed && !(rf[idx + pstride] < 0.0)) {
                const double hz = thick[z];
                for (int c = 0; c < 4; ++c) {
                    const int ey = y - (c >> 1), ex = x - (c & 1);
                    if (ey < 0 || ey >= lay.R || ex < 0 || ex >= lay.C) continue;
                    const long long el = ((long long)z * lay.R + ey) * lay.Xe + ex;
                    const double hy = py[ey], hx = px[ex];
                    const double ax = kin[el] * hy * hz / hx;
                    const double ay = kin[el] * hx * hz / hy;
                    const double az = kz[el] * hx * hy / hz;
                    e += ax / 18.0 + ay / 18.0 - az / 9.0;
                }
            }
            p_prev = p;
            e_prev = e;
        }
    }
}

// Level-1 Galerkin entries from one coloured operator action y = A 1_colour:
// for aggregate I, the sum of y over its free nodes is A_1(I, J) for the one
// aggregate J of that colour next to I; the upper entries are kept.
__global__ void ml_galerkin_gather(double* __restrict__ st64, const double* __restrict__ y,
                                   const double* __restrict__ rf, Layout lay, long long pstride, MLGrid g1,
                                   int colour) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long I = (long long)blockIdx.x * blockDim.x + threadIdx.x; I < g1.n; I += stride) {
        const int z = (int)(I / g1.plane);
        const long long rem = I - (long long)z * g1.plane;
        const int Y = (int)(rem / g1.nx);
        const int X = (int)(rem - (long long)Y * g1.nx);
        int o = -1;
        for (int dz = -1; dz <= 1 && o < 0; ++dz)
            for (int dy = -1; dy <= 1 && o < 0; ++dy)
                for (int dx = -1; dx <= 1 && o < 0; ++dx) {
                    const int jz = z + dz, jy = Y + dy, jx = X + dx;
                    if (jz < 0 || jz >= g1.L || jy < 0 || jy >= g1.ny || jx < 0 || jx >= g1.nx) continue;
                    if (patch_colour(jz, jy, jx) == colour) o = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
                }
        if (o < 13) continue;
        double sum = 0.0;
        for (int u = 0; u < kMlAgg; ++u) {
            const int yy = kMlAgg * Y + u;
            if (yy > lay.R) break;
            for (int v = 0; v < kMlAgg; ++v) {
                const int xx = kMlAgg * X + v;
                if (xx > lay.C) break;
                const long long idx = (long long)z * pstride + (long long)yy * lay.Xp + xx;
                if (rf[idx] >= 0.0) sum += y[idx];
            }
        }
        st64[(long long)(o - 13) * g1.n + I] = sum;
    }
}

// Empty coarse nodes (no free node below them): centre 0 -> -1 (marker).
__global__ void ml_mark_empty(double* __restrict__ st64, long long n) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        if (st64[i] == 0.0) st64[i] = -1.0;
}

// A_{l+1} = Z^T A_l Z from the stencil of level l (FP64): per coarse node I,
// the fine entries A_l(i, j) of its non-empty nodes i, summed by the offset of
// j's aggregate from I, in a fixed order; upper entries kept, empty marked.
__global__ void ml_coarsen(double* __restrict__ out, const double* __restrict__ in, MLGrid g, MLGrid gc) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long I = (long long)blockIdx.x * blockDim.x + threadIdx.x; I < gc.n; I += stride) {
        const int z = (int)(I / gc.plane);
        const long long rem = I - (long long)z * gc.plane;
        const int Y = (int)(rem / gc.nx);
        const int X = (int)(rem - (long long)Y * gc.nx);
        double acc[kMlStencil];
#pragma unroll
        for (int k = 0; k < kMlStencil; ++k) acc[k] = 0.0;
        const int b = g.b;
        for (int u = 0; u < b; ++u) {
            const int y = b * Y + u;
            if (y >= g.ny) break;
            for (int v = 0; v < b; ++v) {
                const int x = b * X + v;
                if (x >= g.nx) break;
                const long long i = ml_index(g, z, y, x);
                if (in[i] < 0.0) continue;  // empty
#pragma unroll 1
                for (int o = 0; o < 27; ++o) {
                    const int dz = o / 9 - 1, dy = (o / 3) % 3 - 1, dx = o % 3 - 1;
                    const int jz = z + dz, jy = y + dy, jx = x + dx;
                    if (jz < 0 || jz >= g.L || jy < 0 || jy >= g.ny || jx < 0 || jx >= g.nx) continue;
                    const long long j = ml_index(g, jz, jy, jx);
                    const double a = ml_coef(in, g.n, i, j, o);
                    if (a == 0.0) continue;
                    const int Dy = jy / b - Y, Dx = jx / b - X;
                    const int O = (dz + 1) * 9 + (Dy + 1) * 3 + (Dx + 1);
                    if (O >= 13) acc[O - 13] += a;
                }
            }
        }
        if (acc[0] == 0.0) acc[0] = -1.0;
#pragma unroll
        for (int k = 0; k < kMlStencil; ++k) out[(long long)k * gc.n + I] = acc[k];
    }
}

// z-line factors of a coarse level from its FP64 stencil, and the FP32
// stencil the iteration reads (empty nodes: a unit row, reciprocal -1).
__global__ void ml_level_factors(float* __restrict__ st32, float* __restrict__ lf, float* __restrict__ ipd,
                                 const double* __restrict__ st64, MLGrid g) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < g.plane; c += stride) {
        double p_prev = 1.0, e_prev = 0.0;
        for (int z = 0; z < g.L; ++z) {
            const long long i = (long long)z * g.plane + c;
            const double centre = st64[i];
            const bool empty = centre < 0.0;
            const double d = empty ? 1.0 : centre;
            const double l = (z == 0) ? 0.0 : e_prev / p_prev;
            const double p = d - l * e_prev;
            lf[i] = (float)l;
            ipd[i] = empty ? -1.0f : (float)(1.0 / p);
            st32[i] = (float)d;
#pragma unroll
            for (int k = 1; k < kMlStencil; ++k) st32[(long long)k * g.n + i] = (float)st64[(long long)k * g.n + i];
            p_prev = p;
            e_prev = (z + 1 < g.L) ? st64[9LL * g.n + i] : 0.0;  // o = 22: the node above
        }
    }
}

// Dense matrix of the coarsest level (rows zeroed before): its 27-point
// stencil, a unit row for an empty node.
__global__ void ml_dense(double* __restrict__ M, const double* __restrict__ st64, MLGrid g) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long I = (long long)blockIdx.x * blockDim.x + threadIdx.x; I < g.n; I += stride) {
        const int z = (int)(I / g.plane);
        const long long rem = I - (long long)z * g.plane;
        const int y = (int)(rem / g.nx);
        const int x = (int)(rem - (long long)y * g.nx);
        if (st64[I] < 0.0) {
            M[I * g.n + I] = 1.0;
            continue;
        }
        for (int o = 0; o < 27; ++o) {
            const int dz = o / 9 - 1, dy = (o / 3) % 3 - 1, dx = o % 3 - 1;
            const int jz = z + dz, jy = y + dy, jx = x + dx;
            if (jz < 0 || jz >= g.L || jy < 0 || jy >= g.ny || jx < 0 || jx >= g.nx) continue;
            const long long j = ml_index(g, jz, jy, jx);
            M[I * g.n + j] = ml_coef(st64, g.n, I, j, o);
        }
    }
}

}  // namespace tb
