// Deterministic block and grid reductions for the PCG scalars.
//
// FP32 inner products are compensated.  The vector kernels accumulate each
// thread's terms with the Dot2 scheme of Ogita, Rump and Oishi ("Accurate sum
// and dot product", SIAM J. Sci. Comput. 26(6), 2005): every product is split
// exactly with an FMA (TwoProduct) and every addition keeps its rounding error
// (Knuth's TwoSum), as if accumulated in twice the working precision.  The
// operator kernel and the multilevel fine pass (r.r, r.T^-1 r: terms of one
// sign), both close to issue-bound, sum their few terms per thread with plain
// FMAs; from there on every merge (warp, block, grid) is a TwoSum with the
// error carried.  FP64 accumulators (outer residual norm, plain FP64 PCG)
// add in double.
//
// Grid reductions are deterministic: each block writes one partial, the last
// block to finish (an atomic ticket after a fence) combines the partials in
// block-index order with a fixed tree.  The bits therefore depend only on the
// data and the grid shape, never on scheduling.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tb {

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ---------------------------------------------------------------- accumulators
struct Acc32 {  // compensated FP32 sum: value = s + c
    float s, c;
    __device__ __forceinline__ Acc32() : s(0.f), c(0.f) {}
    __device__ __forceinline__ void add_product(float a, float b) {
        const float p = a * b;
        const float pe = __fmaf_rn(a, b, -p);  // exact error of the product
        const float t = s + p;
        const float z = t - s;
        const float se = (s - (t - z)) + (p - z);  // exact error of the sum
        s = t;
        c += se + pe;
    }
    __device__ __forceinline__ void merge(const Acc32& o) {
        const float t = s + o.s;
        const float z = t - s;
        const float se = (s - (t - z)) + (o.s - z);
        s = t;
        c += (o.c + se);
    }
    __device__ __forceinline__ double value() const { return (double)s + (double)c; }
};

struct Acc64 {  // plain FP64 sum
    double s;
    __device__ __forceinline__ Acc64() : s(0.0) {}
    __device__ __forceinline__ void add_product(double a, double b) { s = __fma_rn(a, b, s); }
    __device__ __forceinline__ void merge(const Acc64& o) { s += o.s; }
    __device__ __forceinline__ double value() const { return s; }
};

template <typename T> struct AccOf;
template <> struct AccOf<float> { using type = Acc32; };
template <> struct AccOf<double> { using type = Acc64; };

// Storage of one accumulator in the global partials array (2 doubles wide).
__device__ __forceinline__ void acc_store(double* slot, const Acc32& a) {
    float2 v = make_float2(a.s, a.c);
    *reinterpret_cast<float2*>(slot) = v;
}
__device__ __forceinline__ void acc_store(double* slot, const Acc64& a) { slot[0] = a.s; }
__device__ __forceinline__ void acc_load(const double* slot, Acc32& a) {
    const float2 v = __ldcg(reinterpret_cast<const float2*>(slot));
    a.s = v.x;
    a.c = v.y;
}
__device__ __forceinline__ void acc_load(const double* slot, Acc64& a) { a.s = __ldcg(slot); }

// ------------------------------------------------------------- warp / block
__device__ __forceinline__ void warp_merge(Acc32& a) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        Acc32 o;
        o.s = __shfl_down_sync(0xffffffffu, a.s, off);
        o.c = __shfl_down_sync(0xffffffffu, a.c, off);
        a.merge(o);
    }
}
__device__ __forceinline__ void warp_merge(Acc64& a) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        Acc64 o;
        o.s = __shfl_down_sync(0xffffffffu, a.s, off);
        a.merge(o);
    }
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
    return v;
}

// Reduce NA accumulators across the block; thread 0 receives the result.
// `scratch` must hold NA * (blockDim/32) accumulators.  Fixed tree order.
template <int NA, class A>
__device__ __forceinline__ void block_merge(A (&acc)[NA], A* scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NA; ++k) warp_merge(acc[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NA; ++k) scratch[k * 32 + warp] = acc[k];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NA; ++k) {
            A v = (lane < nw) ? scratch[k * 32 + lane] : A();
            warp_merge(v);
            acc[k] = v;
        }
    }
    __syncthreads();
}

// Block max of a non-negative double, result in thread 0.
__device__ __forceinline__ double block_max(double v, double* scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = warp_max(v);
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double w = (lane < nw) ? scratch[lane] : 0.0;
        v = warp_max(w);
    }
    __syncthreads();
    return v;
}

// Ticket for the last-block pattern.  Returns true in every thread of the
// block that finished last.  Thread 0 must have written this block's partials
// before the call, and only those writes are published: thread 0 fences them
// before it takes its ticket, so that the block's other threads, whose
// vector stores the last block never reads, do not wait for theirs to drain.
__device__ __forceinline__ bool last_block(unsigned int* counter) {
    __shared__ bool is_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned int ticket = atomicAdd(counter, 1u);
        is_last = (ticket == gridDim.x * gridDim.y * gridDim.z - 1u);
    }
    __syncthreads();
    if (is_last) __threadfence();
    return is_last;
}

// In the last block: combine NA accumulators stored per block in
// partials[b * stride + 2*k] (b in block order) with a fixed tree, result in
// thread 0.  Resets the ticket counter for the next launch.
template <int NA, class A>
__device__ __forceinline__ void grid_merge(const double* partials, int nblocks, int stride, A (&acc)[NA],
                                           A* scratch, unsigned int* counter) {
#pragma unroll
    for (int k = 0; k < NA; ++k) acc[k] = A();
    // Four partials per thread are loaded before any is merged (the loads are
    // L2 round trips; the merges a dependent chain); the merge order is still
    // b, b + blockDim, b + 2 blockDim, ...
    constexpr int kBatch = 4;
    for (int b0 = threadIdx.x; b0 < nblocks; b0 += kBatch * blockDim.x) {
        A v[kBatch][NA];
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
            const int b = b0 + u * (int)blockDim.x;
#pragma unroll
            for (int k = 0; k < NA; ++k) {
                if (b < nblocks) acc_load(partials + (size_t)b * stride + 2 * k, v[u][k]);
                else v[u][k] = A();
            }
        }
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
#pragma unroll
            for (int k = 0; k < NA; ++k) {
                if (b0 + u * (int)blockDim.x < nblocks) acc[k].merge(v[u][k]);
            }
        }
    }
    block_merge<NA>(acc, scratch);
    if (threadIdx.x == 0) *counter = 0u;
}

}  // namespace tb
