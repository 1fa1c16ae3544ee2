// Batched MPIR: many boards of different sizes solved by the same kernels.
//
// Every board keeps its own padded fields in HBM (as a single system does)
// and one BatchInstance entry in a device table.  A BatchSchedule lists the
// live boards with prefix sums of their work items: operator tiles (FP32 and
// FP64 tile shapes) and vector chunks of kBatchChunkQuads quads.  Each batched
// kernel runs a fixed, SM-filling grid whose blocks walk the concatenated item
// range; an item looks its board up by binary search in the prefix sums, and
// boards whose phase does not call for this kernel are skipped item by item.
// This is the per-instance convergence mask: a converged board costs one
// check per item and moves no field data.
//
// Reductions are per board and deterministic: every item writes one partial
// at its index within the board, and the board's last item (an atomic ticket
// on the board's own counter) combines them in index order.  The bits of a
// board's solve therefore depend only on the board and the tile shape, never
// on which other boards share the launch: a result is identical alone and in
// any mix.
//
// The MPIR outer loop runs on the device too (reference solver.py:580-698):
// the FP64 residual kernel decides convergence in the board's last tile and
// prepares the inner solve; the start kernel scales the residual into the
// FP32 right-hand side; the finish kernel adds the FP32 correction into the
// FP64 iterate.  The host only admits boards, launches graph chunks and
// collects finished boards.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "tb_apply.cuh"
#include "tb_coarse.cuh"
#include "tb_reduce.cuh"
#include "tb_types.h"
#include "tb_vec.cuh"

namespace tb {

constexpr int kBatchMax = 256;                     // boards in one schedule
constexpr int kBatchChunkQuads = kVecThreads * 8;  // 2048 quads = 8192 nodes per vector chunk
constexpr int kBatchHist = 64;                     // outer steps recorded per board

enum BatchPhase {
    PH_IDLE = 0,    // slot empty
    PH_RESID = 1,   // FP64 residual of the current iterate wanted
    PH_START = 2,   // inner solve prepared, its right-hand side wanted
    PH_INNER = 3,   // inner FP32 PCG running (or just stopped)
    PH_DONE = 4,    // outer loop finished (converged or out of outer steps)
    PH_FAILED = 5,  // the inner PCG met a non-SPD operator (or its operator staging timed out)
    PH_PRECOND = 6, // two-level: inner solve started, its first coarse step wanted
};

// Host-visible status of one slot, copied to the host after every chunk.
struct BatchStatus {
    long long ticket;
    int phase;
    int pad;
};

// Device-managed MPIR control and result of one board.
struct BatchOuter {
    double target;     // absolute target on ||b - A x|| (atol + rtol ||b||)
    double bscale;     // ||b|| (1 when b = 0): the relative residual's scale
    double inner_tol;  // inner relative tolerance
    double rel;        // relative residual of the last outer residual
    int max_inner, max_outer;
    int outer;         // completed outer steps
    int inner_total;   // inner iterations over all outer steps
    int high, low;     // FP64 and FP32 operator applications
    int converged;
    int nhist;
    double hist[kBatchHist][3];  // high relative residual, inner iterations, inner relative residual
};

struct BatchInstance {
    ApplyParams<float> a32;   // x = p32, y = q32
    ApplyParams<double> a64;  // x = x64, y = r64, b = b64
    float *x32, *r32, *p32, *q32;
    const float* dinv32;
    double *x64, *r64;
    double* partials;       // max(tiles32, tiles64, chunks) x 4 doubles
    unsigned int* counter;  // [4]: FP32 apply, PCG update, FP64 residual, start / finish
    SolveCtl* ctl;
    BatchOuter* outer;
    BatchStatus* status;
    long long nq;
    int gx32, tiles32, gx64, tiles64, chunks, pad;
    // two-level preconditioner (twolevel != 0): coarse grid, FP32 inverse of
    // Z^T A Z (nc x nc), R = Z^T r and c = Minv R
    CoarseLayout cl;
    int twolevel, coarse_items;  // coarse_items: blocks of kCoarseRows rows of Minv
    const float* minv;
    float *rc, *cvec;
    Layout lay;
    // tensor maps of the FP32 operator fields, one set per tile height 8, 16,
    // 32 (engine device memory; null when the engine stages by cp.async)
    const ApplyMaps* maps;
};

struct BatchSchedule {
    int n;
    int slot[kBatchMax];
    int tile32[kBatchMax + 1];
    int tile64[kBatchMax + 1];
    int chunk[kBatchMax + 1];
    int patch[kBatchMax + 1];  // two-level boards: one item per patch (restriction)
    int crow[kBatchMax + 1];   // two-level boards: one item per kCoarseRows rows of Minv
    // FP32 operator tiles handed out one at a time: [0] next tile, [1] blocks
    // done; the last block of a launch sets both back to zero.  [2], [3]: the
    // same for the coarse kernel's items.
    unsigned int grab[4];
};

enum { ITEMS_TILE32 = 0, ITEMS_TILE64 = 1, ITEMS_CHUNK = 2, ITEMS_PATCH = 3, ITEMS_CROW = 4 };
constexpr int kCoarseRows = 8;  // rows of the coarse inverse per item (one warp each)

__global__ void batch_set_schedule(BatchSchedule value, BatchSchedule* dst) {
    const int* src = reinterpret_cast<const int*>(&value);
    int* out = reinterpret_cast<int*>(dst);
    for (int i = threadIdx.x; i < (int)(sizeof(BatchSchedule) / sizeof(int)); i += blockDim.x) out[i] = src[i];
}

// Admission of a board into `slot`: table entry, cleared scalars and
// counters, outer control in phase PH_RESID.
__global__ void batch_admit(BatchInstance inst, BatchOuter outer, long long ticket, BatchInstance* table, int slot) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    table[slot] = inst;
    SolveCtl c;
    memset(&c, 0, sizeof(c));
    *inst.ctl = c;
    for (int k = 0; k < 4; ++k) inst.counter[k] = 0u;
    *inst.outer = outer;
    inst.status->ticket = ticket;
    __threadfence();
    inst.status->phase = PH_RESID;
}

__global__ void batch_release(BatchStatus* status) {
    if (threadIdx.x == 0 && blockIdx.x == 0) status->phase = PH_IDLE;
}

// The schedule's slots and one prefix array in shared memory.
struct ItemMap {
    int n;
    int slot[kBatchMax];
    int prefix[kBatchMax + 1];
};

template <int WHICH>
__device__ __forceinline__ void load_items(const BatchSchedule* __restrict__ sched, ItemMap& m) {
    const int n = sched->n;
    const int* pre = WHICH == ITEMS_TILE32   ? sched->tile32
                     : WHICH == ITEMS_TILE64 ? sched->tile64
                     : WHICH == ITEMS_CHUNK  ? sched->chunk
                     : WHICH == ITEMS_PATCH  ? sched->patch
                                             : sched->crow;
    for (int i = threadIdx.x; i <= n; i += blockDim.x) {
        m.prefix[i] = pre[i];
        if (i < n) m.slot[i] = sched->slot[i];
    }
    if (threadIdx.x == 0) m.n = n;
    __syncthreads();
}

// Largest k with prefix[k] <= t (boards with no items are passed over).
__device__ __forceinline__ int find_board(const ItemMap& m, int t) {
    int lo = 0, hi = m.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (m.prefix[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int load_phase(const BatchStatus* s) { return *reinterpret_cast<const volatile int*>(&s->phase); }
__device__ __forceinline__ int load_state(const SolveCtl* c) { return *reinterpret_cast<const volatile int*>(&c->state); }

// Board ticket: true in every thread of the block that finished the board's
// last item.  Thread 0 must have stored the block's partial before the call.
__device__ __forceinline__ bool last_item(unsigned int* counter, int items, bool* flag) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) *flag = (atomicAdd(counter, 1u) == (unsigned)(items - 1));
    __syncthreads();
    const bool last = *flag;
    if (last) __threadfence();
    return last;
}

// Copy a parameter block from global into shared memory, word by word.
template <typename P>
__device__ __forceinline__ void copy_params(P* dst, const P* src) {
    static_assert(sizeof(P) % 8 == 0, "parameter blocks are 8-byte words");
    const unsigned long long* s = reinterpret_cast<const unsigned long long*>(src);
    unsigned long long* d = reinterpret_cast<unsigned long long*>(dst);
    for (int i = threadIdx.x; i < (int)(sizeof(P) / 8); i += blockDim.x) d[i] = s[i];
}

// ------------------------------------------------------------ FP32 operator
// Map set of a tile height within a board's three.
__host__ __device__ constexpr int maps_index(int rows) { return rows == 8 ? 0 : (rows == 16 ? 1 : 2); }

// q = A p over the tiles of every board in PH_INNER with a running PCG, with
// the p.Ap epilogue: the board's last tile sets pq and alpha (or NOT_SPD).
// With TMA the stages are filled by tensor copies from the board's maps; the
// block's staged-plane count runs on across the tiles it walks.
template <int ROWS, bool TMA = false>
__global__ void __launch_bounds__(16 * ROWS, ApplyOccupancy<float, ROWS>::min_blocks)
    batch_apply32(const BatchInstance* __restrict__ table, const BatchSchedule* __restrict__ sched) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ ItemMap m;
    __shared__ __align__(16) unsigned char p_raw[sizeof(ApplyParams<float>)];
    __shared__ __align__(16) unsigned char red_raw[sizeof(Acc32) * 32];
    __shared__ int s_go;
    __shared__ bool s_last;
    ApplyParams<float>* const sP = reinterpret_cast<ApplyParams<float>*>(p_raw);
    Acc32* const red = reinterpret_cast<Acc32*>(red_raw);
    __shared__ int s_t;
    load_items<ITEMS_TILE32>(sched, m);
    const int total = m.prefix[m.n];
    unsigned int* const grab = const_cast<unsigned int*>(sched->grab);
    int seq = 0;
    bool aborted = false;
    // Tiles are taken one at a time from a counter, so that blocks finish
    // together although the boards' tiles differ in cost (slab counts); the
    // schedule lists the boards with the most slabs first.  A tile's output
    // and partial do not depend on the block that computes it.
    for (;;) {
        if (threadIdx.x == 0) s_t = (int)atomicAdd(grab, 1u);
        __syncthreads();
        const int t = s_t;
        if (t >= total) break;
        const int k = find_board(m, t);
        const BatchInstance* I = table + m.slot[k];
        if (threadIdx.x == 0) s_go = load_phase(I->status) == PH_INNER && load_state(I->ctl) == ST_RUNNING;
        copy_params(sP, &I->a32);
        __syncthreads();
        if (!s_go) {
            __syncthreads();
            continue;
        }
        const int lt = t - m.prefix[k];
        const int gx = I->gx32;
        float dot = 0.f;
        double rmax = 0.0;
        // after an abandoned wait the block's mbarrier phases are out of step:
        // its remaining tiles only join the reductions, and fail their boards
        if (aborted && threadIdx.x == 0) I->ctl->state = ST_STAGE_TIMEOUT;
        if (!aborted)
            aborted = apply_tile<float, MODE_OPERATOR, EPI_DOT, ROWS, TMA>(*sP, lt % gx, lt / gx, smem_raw, dot, rmax,
                                                                          false, 0, 1 << 30,
                                                                          TMA ? I->maps + maps_index(ROWS) : nullptr,
                                                                          &seq, true) == TILE_ABORTED;
        Acc32 acc[1];
        acc[0].s = dot;
        block_merge<1>(acc, red);
        if (threadIdx.x == 0) acc_store(I->partials + (size_t)lt * 4, acc[0]);
        if (last_item(I->counter + 0, I->tiles32, &s_last)) {
            Acc32 tot[1];
            grid_merge<1>(I->partials, I->tiles32, 4, tot, red, I->counter + 0);
            if (threadIdx.x == 0) {
                SolveCtl* ctl = I->ctl;
                const double pq = tot[0].value();
                ctl->pq = pq;
                ctl->applications += 1;
                if (!(isfinite(pq) && pq > 0.0)) ctl->state = ST_NOT_SPD;
                else ctl->alpha = ctl->rz / pq;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(grab + 1, 1u) == gridDim.x - 1) {  // every block has stopped taking tiles
            grab[0] = 0u;
            grab[1] = 0u;
        }
    }
}

// ------------------------------------------------------------ FP64 residual
// r = b - A x over the tiles of every board in PH_RESID.  The board's last
// tile takes the outer step's decision (reference solver.py:640-662):
// converged, out of outer steps, or an inner solve on f32(r 2^-e) with
// max |r 2^-e| in [0.5, 1).
template <int ROWS>
__global__ void __launch_bounds__(16 * ROWS, 1)
    batch_residual64(const BatchInstance* __restrict__ table, const BatchSchedule* __restrict__ sched) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ ItemMap m;
    __shared__ __align__(16) unsigned char p_raw[sizeof(ApplyParams<double>)];
    __shared__ __align__(16) unsigned char red_raw[sizeof(Acc64) * 32];
    __shared__ double max_scratch[32];
    __shared__ int s_go;
    __shared__ bool s_last;
    ApplyParams<double>* const sP = reinterpret_cast<ApplyParams<double>*>(p_raw);
    Acc64* const red = reinterpret_cast<Acc64*>(red_raw);
    load_items<ITEMS_TILE64>(sched, m);
    const int total = m.prefix[m.n];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int k = find_board(m, t);
        const BatchInstance* I = table + m.slot[k];
        if (threadIdx.x == 0) s_go = load_phase(I->status) == PH_RESID;
        copy_params(sP, &I->a64);
        __syncthreads();
        if (!s_go) {
            __syncthreads();
            continue;
        }
        const int lt = t - m.prefix[k];
        const int gx = I->gx64;
        double dot = 0.0, rmax = 0.0;
        apply_tile<double, MODE_OPERATOR, EPI_RESIDUAL, ROWS>(*sP, lt % gx, lt / gx, smem_raw, dot, rmax, false);
        Acc64 acc[1];
        acc[0].s = dot;
        block_merge<1>(acc, red);
        const double bmax = block_max(rmax, max_scratch);
        if (threadIdx.x == 0) {
            acc_store(I->partials + (size_t)lt * 4, acc[0]);
            I->partials[(size_t)lt * 4 + 2] = bmax;
        }
        if (last_item(I->counter + 2, I->tiles64, &s_last)) {
            Acc64 tot[1];
            grid_merge<1>(I->partials, I->tiles64, 4, tot, red, I->counter + 2);
            double mx = 0.0;
            for (int b = threadIdx.x; b < I->tiles64; b += blockDim.x) mx = fmax(mx, __ldcg(I->partials + (size_t)b * 4 + 2));
            const double peak = block_max(mx, max_scratch);
            if (threadIdx.x == 0) {
                BatchOuter* o = I->outer;
                const double rnorm = sqrt(tot[0].value());
                o->high += 1;
                o->rel = rnorm / o->bscale;
                int next;
                if (rnorm <= o->target) {
                    o->converged = 1;
                    next = PH_DONE;
                } else if (o->outer >= o->max_outer) {
                    next = PH_DONE;
                } else {
                    double pscale = 1.0;
                    if (peak > 0.0 && isfinite(peak)) {
                        int e = 0;
                        frexp(peak, &e);
                        pscale = ldexp(1.0, -e);
                    }
                    SolveCtl* c = I->ctl;
                    c->tol = o->inner_tol;
                    c->max_it = o->max_inner;
                    c->scale = pscale;
                    c->inv_scale = 1.0 / pscale;
                    c->bnorm = 0.0;
                    c->state = ST_RUNNING;
                    c->iterations = 0;
                    c->applications = 0;
                    c->rel = 1.0;
                    c->rz = 1.0;
                    c->alpha = 0.0;
                    c->beta = 0.0;
                    next = PH_START;
                }
                __threadfence();
                I->status->phase = next;
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------ vector chunks
// Walks the chunks of the boards that `select` accepts (decided by thread 0
// of the block, shared with the block).  `body(I, q0, q1, acc)` works on quads
// [q0, q1) of the board; with NA > 0 its accumulators are reduced per board
// and `finish(I, tot)` runs in thread 0 of the board's last chunk.
template <int NA, class Select, class Body, class Finish>
__device__ __forceinline__ void batch_chunks(const BatchInstance* __restrict__ table,
                                             const BatchSchedule* __restrict__ sched, int counter_index,
                                             Select select, Body body, Finish finish) {
    __shared__ ItemMap m;
    __shared__ __align__(16) unsigned char red_raw[sizeof(Acc32) * (NA > 0 ? NA : 1) * 32];
    __shared__ int s_go;
    __shared__ bool s_last;
    Acc32* const red = reinterpret_cast<Acc32*>(red_raw);
    load_items<ITEMS_CHUNK>(sched, m);
    const int total = m.prefix[m.n];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int k = find_board(m, t);
        const BatchInstance* I = table + m.slot[k];
        if (threadIdx.x == 0) s_go = select(I);
        __syncthreads();
        const bool go = s_go;
        __syncthreads();
        if (!go) continue;
        const int lc = t - m.prefix[k];
        const long long q0 = (long long)lc * kBatchChunkQuads;
        const long long q1 = min(q0 + kBatchChunkQuads, I->nq);
        Acc32 acc[NA > 0 ? NA : 1];
        body(I, q0, q1, acc);
        if constexpr (NA > 0) {
            block_merge<NA>(acc, red);
            if (threadIdx.x == 0) {
#pragma unroll
                for (int a = 0; a < NA; ++a) acc_store(I->partials + (size_t)lc * 4 + 2 * a, acc[a]);
            }
            if (last_item(I->counter + counter_index, I->chunks, &s_last)) {
                Acc32 tot[NA];
                grid_merge<NA>(I->partials, I->chunks, 4, tot, red, I->counter + counter_index);
                if (threadIdx.x == 0) finish(I, tot);
            }
            __syncthreads();
        } else {
            if (last_item(I->counter + counter_index, I->chunks, &s_last)) {
                if (threadIdx.x == 0) {
                    I->counter[counter_index] = 0u;
                    Acc32 tot[1];
                    finish(I, tot);
                }
            }
            __syncthreads();
        }
    }
}

// x += alpha p; r -= alpha q; r.r and r.z with z = r / d (the single-board
// pcg_update_f32, per board).
__global__ void __launch_bounds__(kVecThreads)
    batch_update32(const BatchInstance* __restrict__ table, const BatchSchedule* __restrict__ sched) {
    batch_chunks<2>(
        table, sched, 1,
        [](const BatchInstance* I) { return load_phase(I->status) == PH_INNER && load_state(I->ctl) == ST_RUNNING; },
        [](const BatchInstance* I, long long q0, long long q1, Acc32 (&acc)[2]) {
            // the step x += alpha p is taken by the direction kernel (or the
            // outer finish), as in the single-board PCG
            const float alpha = (float)I->ctl->alpha;
            float4* const r = reinterpret_cast<float4*>(I->r32);
            const float4* const q = reinterpret_cast<const float4*>(I->q32);
            const float4* const dv = reinterpret_cast<const float4*>(I->dinv32);
            for (long long i = q0 + threadIdx.x; i < q1; i += blockDim.x) {
                float4 rv = r[i];
                const float4 qv = q[i], d = dv[i];
                rv.x = fmaf(-alpha, qv.x, rv.x);
                rv.y = fmaf(-alpha, qv.y, rv.y);
                rv.z = fmaf(-alpha, qv.z, rv.z);
                rv.w = fmaf(-alpha, qv.w, rv.w);
                r[i] = rv;
                acc[0].add_product(rv.x, rv.x);
                acc[0].add_product(rv.y, rv.y);
                acc[0].add_product(rv.z, rv.z);
                acc[0].add_product(rv.w, rv.w);
                acc[1].add_product(rv.x, rv.x * fabsf(d.x));
                acc[1].add_product(rv.y, rv.y * fabsf(d.y));
                acc[1].add_product(rv.z, rv.z * fabsf(d.z));
                acc[1].add_product(rv.w, rv.w * fabsf(d.w));
            }
        },
        [](const BatchInstance* I, Acc32 (&tot)[2]) {
            if (I->twolevel) finalize_update_2l(I->ctl, tot[0].value(), tot[1].value());
            else finalize_update(I->ctl, tot[0].value(), tot[1].value());
        });
}

// x += alpha p (the update's step, on the old p), then p = z + beta p,
// z = r / d (+ Z c for two-level boards).  A two-level board in PH_PRECOND
// takes p = z and, with its last chunk, enters PH_INNER.
__device__ __forceinline__ void x_step(float4* __restrict__ x, const float4 pv, const float alpha, const long long i) {
    float4 xv = x[i];
    xv.x = fmaf(alpha, pv.x, xv.x);
    xv.y = fmaf(alpha, pv.y, xv.y);
    xv.z = fmaf(alpha, pv.z, xv.z);
    xv.w = fmaf(alpha, pv.w, xv.w);
    x[i] = xv;
}

__global__ void __launch_bounds__(kVecThreads)
    batch_direction32(const BatchInstance* __restrict__ table, const BatchSchedule* __restrict__ sched) {
    __shared__ ItemMap m;
    __shared__ int s_go;
    __shared__ bool s_last;
    load_items<ITEMS_CHUNK>(sched, m);
    const int total = m.prefix[m.n];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int k = find_board(m, t);
        const BatchInstance* I = table + m.slot[k];
        if (threadIdx.x == 0) {
            const int ph = load_phase(I->status);
            s_go = (ph == PH_INNER && load_state(I->ctl) == ST_RUNNING) ? 1 : (ph == PH_PRECOND ? 2 : 0);
        }
        __syncthreads();
        const int go = s_go;
        __syncthreads();
        if (!go) continue;
        const long long q0 = (long long)(t - m.prefix[k]) * kBatchChunkQuads;
        const long long q1 = min(q0 + kBatchChunkQuads, I->nq);
        const bool start = go == 2;
        const float beta = start ? 0.f : (float)I->ctl->beta;
        const float alpha = start ? 0.f : (float)I->ctl->alpha;
        float4* const p = reinterpret_cast<float4*>(I->p32);
        float4* const xs = reinterpret_cast<float4*>(I->x32);
        const float4* const r = reinterpret_cast<const float4*>(I->r32);
        const float4* const dv = reinterpret_cast<const float4*>(I->dinv32);
        if (!I->twolevel) {
            for (long long i = q0 + threadIdx.x; i < q1; i += blockDim.x) {
                float4 pv = p[i];
                x_step(xs, pv, alpha, i);
                const float4 rv = r[i], d = dv[i];
                pv.x = fmaf(beta, pv.x, rv.x * fabsf(d.x));
                pv.y = fmaf(beta, pv.y, rv.y * fabsf(d.y));
                pv.z = fmaf(beta, pv.z, rv.z * fabsf(d.z));
                pv.w = fmaf(beta, pv.w, rv.w * fabsf(d.w));
                p[i] = pv;
            }
            continue;
        }
        const Layout lay = I->lay;
        const CoarseLayout cl = I->cl;
        const float* const c = I->cvec;
        const int qpl = lay.Xp / 4;
        for (long long i = q0 + threadIdx.x; i < q1; i += blockDim.x) {
            const long long line = i / qpl;
            const int x0 = 4 * (int)(i - line * qpl);
            const int z = (int)(line / (lay.R + 1));
            const int y = (int)(line - (long long)z * (lay.R + 1));
            const int rowbase = (z * cl.nby + y / cl.b) * cl.nbx;
            const float4 rv = r[i], d = dv[i];
            const float rr[4] = {rv.x, rv.y, rv.z, rv.w};
            const float dd[4] = {d.x, d.y, d.z, d.w};
            const float4 pv = start ? make_float4(0.f, 0.f, 0.f, 0.f) : p[i];
            if (!start) x_step(xs, pv, alpha, i);
            const float po[4] = {pv.x, pv.y, pv.z, pv.w};
            float out[4];
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                const int x = x0 + kk;
                float zc = rr[kk] * fabsf(dd[kk]);
                if (dd[kk] > 0.f && x <= lay.C) zc += c[rowbase + x / cl.b];
                out[kk] = start ? zc : fmaf(beta, po[kk], zc);
            }
            p[i] = make_float4(out[0], out[1], out[2], out[3]);
        }
        if (start) {
            if (last_item(I->counter + 3, I->chunks, &s_last) && threadIdx.x == 0) {
                I->counter[3] = 0u;
                __threadfence();
                I->status->phase = PH_INNER;
            }
            __syncthreads();
        }
    }
}

// R = Z^T r over the patches of every two-level board whose PCG runs (or
// starts): one warp per patch.  Lane j sums the free nodes j, j+32, ... of
// the patch (row-major) in FP32, and the warp merges the 32 sums in FP64 by a
// fixed shuffle tree, so a patch's R depends only on its own board.  Small
// boards have small patches (5 x 5 nodes at 96 x 96 cells), so a warp, not a
// block with its barriers, is the unit of work.
__global__ void __launch_bounds__(256)
    batch_restrict(const BatchInstance* __restrict__ table, const BatchSchedule* __restrict__ sched) {
    __shared__ ItemMap m;
    load_items<ITEMS_PATCH>(sched, m);
    const int total = m.prefix[m.n];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    for (int t = blockIdx.x * wpb + warp; t < total; t += gridDim.x * wpb) {
        const int k = find_board(m, t);
        const BatchInstance* I = table + m.slot[k];
        int go = 0;
        if (lane == 0) {
            const int ph = load_phase(I->status);
            go = ((ph == PH_INNER && load_state(I->ctl) == ST_RUNNING) || ph == PH_PRECOND) ? 1 : 0;
        }
        go = __shfl_sync(0xffffffffu, go, 0);
        if (!go) continue;
        const CoarseLayout cl = I->cl;
        const Layout lay = I->lay;
        const int P = t - m.prefix[k];
        const int per_layer = cl.nby * cl.nbx;
        const int l = P / per_layer;
        const int rem = P - l * per_layer;
        const int pr = rem / cl.nbx;
        const int pc = rem - pr * cl.nbx;
        const int y0 = pr * cl.b, x0 = pc * cl.b;
        const int bh = min(cl.b, lay.R + 1 - y0), bw = min(cl.b, lay.C + 1 - x0);
        const long long base = (long long)l * (lay.R + 1) * lay.Xp + (long long)y0 * lay.Xp + x0;
        const float* const r = I->r32 + base;
        const float* const d = I->dinv32 + base;
        const int count = bh * bw;
        float acc = 0.f;
#pragma unroll 4
        for (int i = lane; i < count; i += 32) {
            const int yy = i / bw;
            const int off = yy * lay.Xp + (i - yy * bw);
            const float v = r[off];
            if (d[off] >= 0.f) acc += v;
        }
        double sum = (double)acc;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
        if (lane == 0) I->rc[P] = (float)sum;
    }
}

// c = Minv R over the row blocks of every such board; the coarse part R.c of
// r.z is reduced per board and its last item finishes the scalars (start:
// rz; iteration: beta, breakdown and the iteration limit).
__global__ void __launch_bounds__(256)
    batch_coarse(const BatchInstance* __restrict__ table, const BatchSchedule* __restrict__ sched) {
    extern __shared__ float s_rc[];
    __shared__ ItemMap m;
    __shared__ __align__(16) unsigned char red_raw[sizeof(Acc32) * 32];
    __shared__ int s_go;
    __shared__ bool s_last;
    Acc32* const red = reinterpret_cast<Acc32*>(red_raw);
    __shared__ int s_t;
    load_items<ITEMS_CROW>(sched, m);
    const int total = m.prefix[m.n];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned int* const grab = const_cast<unsigned int*>(sched->grab) + 2;
    // items (rows of boards whose coarse grids differ in size) taken one at a
    // time from a counter, as the operator's tiles are
    for (;;) {
        if (threadIdx.x == 0) s_t = (int)atomicAdd(grab, 1u);
        __syncthreads();
        const int t = s_t;
        if (t >= total) break;
        const int k = find_board(m, t);
        const BatchInstance* I = table + m.slot[k];
        if (threadIdx.x == 0) {
            const int ph = load_phase(I->status);
            s_go = (ph == PH_INNER && load_state(I->ctl) == ST_RUNNING) ? 1 : (ph == PH_PRECOND ? 2 : 0);
        }
        __syncthreads();
        const int go = s_go;
        if (!go) {
            __syncthreads();
            continue;
        }
        const int nc = I->cl.nc, ld = I->cl.ld;
        for (int i = threadIdx.x; i < ld; i += blockDim.x) s_rc[i] = I->rc[i];
        __syncthreads();
        const int row = (t - m.prefix[k]) * kCoarseRows + warp;
        Acc32 acc[1];
        if (warp < kCoarseRows && row < nc) {
            const float sum = coarse_row(I->minv + (long long)row * ld, s_rc, ld, lane);
            if (lane == 0) {
                I->cvec[row] = sum;
                acc[0].add_product(s_rc[row], sum);
            }
        }
        block_merge<1>(acc, red);
        const int lt = t - m.prefix[k];
        if (threadIdx.x == 0) acc_store(I->partials + (size_t)lt * 4, acc[0]);
        if (last_item(I->counter + 1, I->coarse_items, &s_last)) {
            Acc32 tot[1];
            grid_merge<1>(I->partials, I->coarse_items, 4, tot, red, I->counter + 1);
            if (threadIdx.x == 0) {
                SolveCtl* ctl = I->ctl;
                const double rzn = ctl->rdr + tot[0].value();
                if (go == 2) {
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
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(grab + 1, 1u) == gridDim.x - 1) {  // every block has stopped taking items
            grab[0] = 0u;
            grab[1] = 0u;
        }
    }
}

// Inner start of every board in PH_START (the single-board inner_start_f32):
// r32 = f32(r64 * scale), x32 = 0, p = z = r32 / d, then r.r and r.z.
__global__ void __launch_bounds__(kVecThreads)
    batch_inner_start(const BatchInstance* __restrict__ table, const BatchSchedule* __restrict__ sched) {
    batch_chunks<2>(
        table, sched, 3, [](const BatchInstance* I) { return load_phase(I->status) == PH_START; },
        [](const BatchInstance* I, long long q0, long long q1, Acc32 (&acc)[2]) {
            const double scale = I->ctl->scale;
            const double2* const r64 = reinterpret_cast<const double2*>(I->r64);
            float4* const x = reinterpret_cast<float4*>(I->x32);
            float4* const r = reinterpret_cast<float4*>(I->r32);
            float4* const p = reinterpret_cast<float4*>(I->p32);
            const float4* const dv = reinterpret_cast<const float4*>(I->dinv32);
            for (long long i = q0 + threadIdx.x; i < q1; i += blockDim.x) {
                const double2 a = r64[2 * i], b = r64[2 * i + 1];
                const float4 d = dv[i];
                const float4 rv = make_float4((float)(a.x * scale), (float)(a.y * scale), (float)(b.x * scale),
                                              (float)(b.y * scale));
                const float4 zv = make_float4(rv.x * fabsf(d.x), rv.y * fabsf(d.y), rv.z * fabsf(d.z), rv.w * fabsf(d.w));
                r[i] = rv;
                p[i] = zv;
                x[i] = make_float4(0.f, 0.f, 0.f, 0.f);
                acc[0].add_product(rv.x, rv.x);
                acc[0].add_product(rv.y, rv.y);
                acc[0].add_product(rv.z, rv.z);
                acc[0].add_product(rv.w, rv.w);
                acc[1].add_product(rv.x, zv.x);
                acc[1].add_product(rv.y, zv.y);
                acc[1].add_product(rv.z, zv.z);
                acc[1].add_product(rv.w, zv.w);
            }
        },
        [](const BatchInstance* I, Acc32 (&tot)[2]) {
            if (I->twolevel) finalize_start_2l(I->ctl, tot[0].value(), tot[1].value());
            else finalize_start(I->ctl, tot[0].value(), tot[1].value());
            const bool precond = I->twolevel && I->ctl->state == ST_RUNNING;
            __threadfence();
            I->status->phase = precond ? PH_PRECOND : PH_INNER;
        });
}

// End of an inner solve (the PCG state left ST_RUNNING): x64 += f64(x32) /
// scale, history entry, back to PH_RESID; a non-SPD inner operator fails the
// board (reference solver.py:664-690).
__global__ void __launch_bounds__(kVecThreads)
    batch_outer_finish(const BatchInstance* __restrict__ table, const BatchSchedule* __restrict__ sched) {
    batch_chunks<0>(
        table, sched, 3,
        [](const BatchInstance* I) { return load_phase(I->status) == PH_INNER && load_state(I->ctl) != ST_RUNNING; },
        [](const BatchInstance* I, long long q0, long long q1, Acc32 (&)[1]) {
            const int st = load_state(I->ctl);
            if (st == ST_NOT_SPD || st == ST_STAGE_TIMEOUT) return;
            const double inv = I->ctl->inv_scale;
            const bool pending = x_step_pending(I->ctl);  // the last update's step, not yet taken
            const float alpha = (float)I->ctl->alpha;
            const float4* const c = reinterpret_cast<const float4*>(I->x32);
            const float4* const p = reinterpret_cast<const float4*>(I->p32);
            double2* const x = reinterpret_cast<double2*>(I->x64);
            for (long long i = q0 + threadIdx.x; i < q1; i += blockDim.x) {
                float4 cv = c[i];
                if (pending) {
                    const float4 pv = p[i];
                    cv.x = fmaf(alpha, pv.x, cv.x);
                    cv.y = fmaf(alpha, pv.y, cv.y);
                    cv.z = fmaf(alpha, pv.z, cv.z);
                    cv.w = fmaf(alpha, pv.w, cv.w);
                }
                double2 a = x[2 * i], b = x[2 * i + 1];
                a.x += (double)cv.x * inv;
                a.y += (double)cv.y * inv;
                b.x += (double)cv.z * inv;
                b.y += (double)cv.w * inv;
                x[2 * i] = a;
                x[2 * i + 1] = b;
            }
        },
        [](const BatchInstance* I, Acc32 (&)[1]) {
            const SolveCtl* c = I->ctl;
            BatchOuter* o = I->outer;
            if (c->state == ST_NOT_SPD || c->state == ST_STAGE_TIMEOUT) {
                __threadfence();
                I->status->phase = PH_FAILED;
                return;
            }
            if (o->nhist < kBatchHist) {
                o->hist[o->nhist][0] = o->rel;
                o->hist[o->nhist][1] = (double)c->iterations;
                o->hist[o->nhist][2] = (c->state == ST_ZERO_RHS) ? 0.0 : c->rel;
            }
            o->nhist += 1;
            o->inner_total += c->iterations;
            o->low += c->applications;
            o->outer += 1;
            __threadfence();
            I->status->phase = PH_RESID;
        });
}

}  // namespace tb
