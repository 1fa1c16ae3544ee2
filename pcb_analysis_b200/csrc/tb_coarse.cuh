// Two-level preconditioner on the device:
//
//     M^-1 r = D^-1 r + Z (Z^T A Z)^-1 Z^T r
//
// (reference src/electrical/matrix_free_mpir_fem/two_level.py:1-229).  A
// coarse unknown is a patch of b x b nodes of one node layer; Z^T sums a
// free-node field over a patch and Z copies a patch value onto its free nodes,
// so Z is never stored.
//
// Set-up (FP64, once per system): the Galerkin matrix Z^T A Z from 27 operator
// actions, one per colour (l mod 3, r mod 3, c mod 3) of the patches, because
// same-coloured patches share no element; patches without free nodes get a
// unit diagonal; the inverse by Gauss-Jordan elimination without pivoting
// (the matrix is SPD, so every pivot is positive and a non-positive one is
// reported), symmetrised and rounded to FP32 for the inner PCG.
//
// Per inner PCG iteration (FP32): the update kernel already sums r.r and
// sum r^2 / d; a restriction kernel forms R = Z^T r (one block per patch,
// fixed order, FP64 accumulation), the coarse kernel forms c = (Z^T A Z)^-1 R
// and r.z = sum r^2 / d + R.c, and the direction kernel builds
// p = (r / d + Z c) + beta p.  The free mask is the sign of the FP32 Jacobi
// reciprocal: -1 marks a fixed row (whose diagonal is 1).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "tb_reduce.cuh"
#include "tb_types.h"
#include "tb_vec.cuh"

namespace tb {

struct CoarseLayout {
    int b;       // patch width in nodes
    int layers;  // S + 1
    int nby;     // patches along y: ceil((R + 1) / b)
    int nbx;     // patches along x: ceil((C + 1) / b)
    int nc;      // layers * nby * nbx
    int ld;      // row stride of the FP32 inverse and length of R: nc rounded up to 4 (zero pads)
};

__device__ __forceinline__ int patch_colour(int l, int r, int c) { return (l % 3) * 9 + (r % 3) * 3 + (c % 3); }

__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// --------------------------------------------------------------- set-up
// x = 1 on the free nodes of the patches of one colour (every patch when
// colour < 0), 0 elsewhere and on the pads.
__global__ void coarse_indicator(double* __restrict__ x, const double* __restrict__ rf, Layout lay, CoarseLayout cl,
                                 int colour) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < lay.L; i += stride) {
        const long long line = i / lay.Xp;
        const int xx = (int)(i - line * lay.Xp);
        const int z = (int)(line / (lay.R + 1));
        const int y = (int)(line - (long long)z * (lay.R + 1));
        double v = 0.0;
        if (xx <= lay.C && rf[i] >= 0.0 && (colour < 0 || patch_colour(z, y / cl.b, xx / cl.b) == colour)) v = 1.0;
        x[i] = v;
    }
}

// Sum over the free nodes (mask >= 0) of one patch of a node field, in this
// thread's share: one warp per patch row, lanes along the row, four rows in
// flight per warp, in a fixed order.  The sum is kept in T: FP32 for the
// per-iteration restriction of the inner PCG (the precision the reference's
// low-precision runtime uses for it), FP64 for the set-up.
template <typename T>
__device__ __forceinline__ T patch_sum(const T* __restrict__ v, const T* __restrict__ mask, long long base, int bh,
                                       int bw, int Xp) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    T acc = T(0);
    for (int y0 = warp; y0 < bh; y0 += 4 * nw) {
        for (int xx = lane; xx < bw; xx += 32) {
            T vv[4], mm[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int yy = y0 + u * nw;
                const long long idx = base + (long long)(yy < bh ? yy : y0) * Xp + xx;
                vv[u] = v[idx];
                mm[u] = mask[idx];
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (y0 + u * nw < bh && mm[u] >= T(0)) acc += vv[u];
        }
    }
    return acc;
}

// out[I] = sum over the free nodes of patch I of v (one block per patch; the
// free mask is mask >= 0).  FP64 accumulation in a fixed order.  With a
// solve state, the whole grid returns unless the PCG is running.
template <typename T>
__global__ void __launch_bounds__(128)
    coarse_restrict(const T* __restrict__ v, const T* __restrict__ mask, T* __restrict__ out, Layout lay,
                    CoarseLayout cl, long long pstride, const SolveCtl* ctl) {
    __shared__ __align__(16) unsigned char scratch_raw[sizeof(Acc64) * 32];
    Acc64* const scratch = reinterpret_cast<Acc64*>(scratch_raw);
    pdl_enter();
    if (ctl != nullptr && ctl->state != ST_RUNNING) return;
    const int I = blockIdx.x;
    const int per_layer = cl.nby * cl.nbx;
    const int l = I / per_layer;
    const int rem = I - l * per_layer;
    const int pr = rem / cl.nbx;
    const int pc = rem - pr * cl.nbx;
    const int y0 = pr * cl.b, x0 = pc * cl.b;
    const int bh = min(cl.b, lay.R + 1 - y0), bw = min(cl.b, lay.C + 1 - x0);
    const long long base = (long long)l * pstride + (long long)y0 * lay.Xp + x0;
    Acc64 acc[1];
    acc[0].s = (double)patch_sum(v, mask, base, bh, bw, lay.Xp);
    block_merge<1>(acc, scratch);
    if (threadIdx.x == 0) out[I] = (T)acc[0].s;
}

// Row I of Z^T A Z against the patch J of `colour` next to I gets R[I].
__global__ void coarse_scatter(double* __restrict__ M, const double* __restrict__ R, CoarseLayout cl, int colour) {
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= cl.nc) return;
    const int per_layer = cl.nby * cl.nbx;
    const int l = I / per_layer;
    const int rem = I - l * per_layer;
    const int pr = rem / cl.nbx;
    const int pc = rem - pr * cl.nbx;
    for (int dl = -1; dl <= 1; ++dl) {
        const int jl = l + dl;
        if (jl < 0 || jl >= cl.layers) continue;
        for (int dr = -1; dr <= 1; ++dr) {
            const int jr = pr + dr;
            if (jr < 0 || jr >= cl.nby) continue;
            for (int dc = -1; dc <= 1; ++dc) {
                const int jc = pc + dc;
                if (jc < 0 || jc >= cl.nbx) continue;
                if (patch_colour(jl, jr, jc) != colour) continue;
                const int J = (jl * cl.nby + jr) * cl.nbx + jc;
                M[(long long)I * cl.nc + J] = R[I];
            }
        }
    }
}

// Patches with no free node: zero row and column, unit diagonal.
__global__ void coarse_fix_empty(double* __restrict__ M, const double* __restrict__ counts, int nc) {
    const long long total = (long long)nc * nc;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += stride) {
        const int i = (int)(e / nc);
        const int j = (int)(e - (long long)i * nc);
        if (counts[i] <= 0.0 || counts[j] <= 0.0) M[e] = (i == j) ? 1.0 : 0.0;
    }
}

// Gauss-Jordan step k, part 1: copy row k and column k; flag a pivot that is
// not positive and finite.
__global__ void gj_pivot(const double* __restrict__ A, double* __restrict__ rk, double* __restrict__ ck, int nc, int k,
                         int* err) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nc; j += gridDim.x * blockDim.x) {
        rk[j] = A[(long long)k * nc + j];
        ck[j] = A[(long long)j * nc + k];
        if (j == k) {
            const double piv = A[(long long)k * nc + k];
            if (!(piv > 0.0) || !isfinite(piv)) atomicOr(err, 1);
        }
    }
}

// Part 2: eliminate with pivot k in place (rows and columns k become the
// inverse's).
__global__ void gj_update(double* __restrict__ A, const double* __restrict__ rk, const double* __restrict__ ck, int nc,
                          int k) {
    const double p = 1.0 / ck[k];
    const long long total = (long long)nc * nc;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += stride) {
        const int i = (int)(e / nc);
        const int j = (int)(e - (long long)i * nc);
        double v;
        if (i == k && j == k) v = p;
        else if (i == k) v = rk[j] * p;
        else if (j == k) v = -ck[i] * p;
        else v = A[e] - ck[i] * (rk[j] * p);
        A[e] = v;
    }
}

// ---- blocked Gauss-Jordan inversion (no pivoting; the matrix is SPD).
// With A split in kGjB x kGjB blocks, block step K is
//     P = A_KK^-1,  A_KJ <- P A_KJ,  A_IJ <- A_IJ - A_IK A_KJ,  A_IK <- -A_IK P,  A_KK <- P
// (I, J != K); after every step A holds A^-1.  Four launches per block step:
// the diagonal block (one block of threads, unblocked elimination in shared
// memory, pivots checked), the row panel, the trailing update (64 x 64
// tiles, 4 x 4 outputs per thread) and the column panel.
constexpr int kGjB = 64;
constexpr int kGjLd = kGjB + 1;  // padded shared-memory row

__global__ void __launch_bounds__(256) gjb_diag(double* __restrict__ A, int nc, int K, int* err) {
    static_assert(kGjB == 64, "256 threads: a row and 16 columns each");
    __shared__ double D[kGjB * kGjLd];
    __shared__ double rowk[kGjB], colk[kGjB];
    __shared__ double s_p;
    const int k0 = K * kGjB;
    const int b = min(kGjB, nc - k0);
    const int i = threadIdx.x >> 2, j0 = (threadIdx.x & 3) * 16;  // row i, columns j0 .. j0+15 of the block
    if (i < b) {
        for (int jj = 0; jj < 16; ++jj)
            if (j0 + jj < b) D[i * kGjLd + j0 + jj] = A[(long long)(k0 + i) * nc + k0 + j0 + jj];
    }
    __syncthreads();
    for (int k = 0; k < b; ++k) {
        if (threadIdx.x < b) {
            rowk[threadIdx.x] = D[k * kGjLd + threadIdx.x];
            colk[threadIdx.x] = D[threadIdx.x * kGjLd + k];
        }
        __syncthreads();
        if (threadIdx.x == 0) {  // one reciprocal per step, shared
            const double piv = colk[k];
            if (!(piv > 0.0) || !isfinite(piv)) atomicOr(err, 1);
            s_p = 1.0 / piv;
        }
        __syncthreads();
        const double p = s_p;
        if (i < b) {
            const double ci = colk[i];
            for (int jj = 0; jj < 16; ++jj) {
                const int j = j0 + jj;
                if (j >= b) break;
                double v;
                if (i == k && j == k) v = p;
                else if (i == k) v = rowk[j] * p;
                else if (j == k) v = -ci * p;
                else v = D[i * kGjLd + j] - ci * (rowk[j] * p);
                D[i * kGjLd + j] = v;
            }
        }
        __syncthreads();
    }
    if (i < b) {
        for (int jj = 0; jj < 16; ++jj)
            if (j0 + jj < b) A[(long long)(k0 + i) * nc + k0 + j0 + jj] = D[i * kGjLd + j0 + jj];
    }
}

// Load the b_r x b_c block with corner (r0, c0) into shared memory (zero pad).
__device__ __forceinline__ void gjb_load(double* __restrict__ dst, const double* __restrict__ A, int nc, int r0,
                                         int c0, int br, int bc) {
    for (int e = threadIdx.x; e < kGjB * kGjB; e += blockDim.x) {
        const int i = e / kGjB, j = e - (e / kGjB) * kGjB;
        dst[i * kGjLd + j] = (i < br && j < bc) ? A[(long long)(r0 + i) * nc + c0 + j] : 0.0;
    }
}

// out (64 x 64 tile, 4 x 4 per thread) = X Y of two shared 64 x 64 blocks.
__device__ __forceinline__ void gjb_product(const double* __restrict__ X, const double* __restrict__ Y,
                                            double (&acc)[4][4]) {
    const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[a][c] = 0.0;
    for (int k = 0; k < kGjB; ++k) {
        double xv[4], yv[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) xv[a] = X[(ty * 4 + a) * kGjLd + k];
#pragma unroll
        for (int c = 0; c < 4; ++c) yv[c] = Y[k * kGjLd + tx * 4 + c];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[a][c] = fma(xv[a], yv[c], acc[a][c]);
    }
}

// Row panel: A_KJ <- P A_KJ for every column block J != K (grid.x = blocks).
__global__ void __launch_bounds__(256) gjb_row(double* __restrict__ A, int nc, int K) {
    extern __shared__ double sm[];
    const int J = blockIdx.x;
    if (J == K) return;
    double* const P = sm;
    double* const T = sm + kGjB * kGjLd;
    const int k0 = K * kGjB, j0 = J * kGjB;
    const int bk = min(kGjB, nc - k0), bj = min(kGjB, nc - j0);
    gjb_load(P, A, nc, k0, k0, bk, bk);
    gjb_load(T, A, nc, k0, j0, bk, bj);
    __syncthreads();
    double acc[4][4];
    gjb_product(P, T, acc);
    const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int i = ty * 4 + a, j = tx * 4 + c;
            if (i < bk && j < bj) A[(long long)(k0 + i) * nc + j0 + j] = acc[a][c];
        }
}

// Trailing update: A_IJ -= A_IK A_KJ for I, J != K (grid = blocks x blocks).
__global__ void __launch_bounds__(256) gjb_trailing(double* __restrict__ A, int nc, int K) {
    extern __shared__ double sm[];
    const int I = blockIdx.y, J = blockIdx.x;
    if (I == K || J == K) return;
    double* const L = sm;
    double* const U = sm + kGjB * kGjLd;
    const int k0 = K * kGjB, i0 = I * kGjB, j0 = J * kGjB;
    const int bk = min(kGjB, nc - k0), bi = min(kGjB, nc - i0), bj = min(kGjB, nc - j0);
    gjb_load(L, A, nc, i0, k0, bi, bk);
    gjb_load(U, A, nc, k0, j0, bk, bj);
    __syncthreads();
    double acc[4][4];
    gjb_product(L, U, acc);
    const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int i = ty * 4 + a, j = tx * 4 + c;
            if (i < bi && j < bj) {
                double* const dst = A + (long long)(i0 + i) * nc + j0 + j;
                *dst = *dst - acc[a][c];
            }
        }
}

// Column panel: A_IK <- -A_IK P for every row block I != K (grid.x = blocks).
__global__ void __launch_bounds__(256) gjb_col(double* __restrict__ A, int nc, int K) {
    extern __shared__ double sm[];
    const int I = blockIdx.x;
    if (I == K) return;
    double* const T = sm;
    double* const P = sm + kGjB * kGjLd;
    const int k0 = K * kGjB, i0 = I * kGjB;
    const int bk = min(kGjB, nc - k0), bi = min(kGjB, nc - i0);
    gjb_load(T, A, nc, i0, k0, bi, bk);
    gjb_load(P, A, nc, k0, k0, bk, bk);
    __syncthreads();
    double acc[4][4];
    gjb_product(T, P, acc);
    const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int i = ty * 4 + a, j = tx * 4 + c;
            if (i < bi && j < bk) A[(long long)(i0 + i) * nc + k0 + j] = -acc[a][c];
        }
}

// Invert the SPD matrix A (nc x nc, row-major, in place) on `stream`; a
// pivot that is not positive sets *err.
inline cudaError_t gauss_jordan_invert(double* A, int nc, int* err, cudaStream_t stream) {
    const int smem = 2 * kGjB * kGjLd * (int)sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(gjb_row, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(gjb_trailing, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(gjb_col, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    const int nb = (nc + kGjB - 1) / kGjB;
    for (int K = 0; K < nb; ++K) {
        gjb_diag<<<1, 256, 0, stream>>>(A, nc, K, err);
        if (nb > 1) {
            gjb_row<<<nb, 256, smem, stream>>>(A, nc, K);
            gjb_trailing<<<dim3(nb, nb), 256, smem, stream>>>(A, nc, K);
            gjb_col<<<nb, 256, smem, stream>>>(A, nc, K);
        }
    }
    return cudaGetLastError();
}

// inverse = (A + A^T) / 2 in FP64 (nc x nc) and FP32 (rows of ld, zero pads).
__global__ void coarse_symmetrize(const double* __restrict__ A, double* __restrict__ inv64, float* __restrict__ inv32,
                                  int nc, int ld) {
    const long long total = (long long)nc * ld;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += stride) {
        const int i = (int)(e / ld);
        const int j = (int)(e - (long long)i * ld);
        double v = 0.0;
        if (j < nc) {
            v = 0.5 * (A[(long long)i * nc + j] + A[(long long)j * nc + i]);
            inv64[(long long)i * nc + j] = v;
        }
        inv32[e] = (float)v;
    }
}

// One row of Minv times R: float4 loads along the padded row, four loads in
// flight per lane, fixed order; the full sum in every lane.
__device__ __forceinline__ float coarse_row(const float* __restrict__ row, const float* __restrict__ r, int ld,
                                            int lane) {
    const float4* m4 = reinterpret_cast<const float4*>(row);
    const float4* r4 = reinterpret_cast<const float4*>(r);
    const int n4 = ld >> 2;
    float s[4] = {0.f, 0.f, 0.f, 0.f};
    for (int j = lane; j < n4; j += 128) {
        float4 a[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) a[u] = (j + 32 * u < n4) ? __ldg(m4 + j + 32 * u) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const float4 rv = (j + 32 * u < n4) ? r4[j + 32 * u] : make_float4(0.f, 0.f, 0.f, 0.f);
            s[u] = fmaf(a[u].x, rv.x, s[u]);
            s[u] = fmaf(a[u].y, rv.y, s[u]);
            s[u] = fmaf(a[u].z, rv.z, s[u]);
            s[u] = fmaf(a[u].w, rv.w, s[u]);
        }
    }
    float t = (s[0] + s[1]) + (s[2] + s[3]);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) t += __shfl_xor_sync(0xffffffffu, t, off);
    return t;
}

// Part `part` of `parts` of one row of Minv times R: the row's float4s in
// chunks of 32 (one per lane), chunk k going to part k % parts, four chunks
// in flight per lane; the part's sum, in a fixed order, in every lane.
__device__ __forceinline__ float coarse_row_part(const float* __restrict__ row, const float* __restrict__ r, int ld,
                                                 int lane, int part, int parts) {
    const float4* m4 = reinterpret_cast<const float4*>(row);
    const float4* r4 = reinterpret_cast<const float4*>(r);
    const int n4 = ld >> 2, step = 32 * parts;
    float s[4] = {0.f, 0.f, 0.f, 0.f};
    for (int j = 32 * part + lane; j < n4; j += 4 * step) {
        float4 a[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) a[u] = (j + u * step < n4) ? __ldg(m4 + j + u * step) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const float4 rv = (j + u * step < n4) ? r4[j + u * step] : make_float4(0.f, 0.f, 0.f, 0.f);
            s[u] = fmaf(a[u].x, rv.x, s[u]);
            s[u] = fmaf(a[u].y, rv.y, s[u]);
            s[u] = fmaf(a[u].z, rv.z, s[u]);
            s[u] = fmaf(a[u].w, rv.w, s[u]);
        }
    }
    float t = (s[0] + s[1]) + (s[2] + s[3]);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) t += __shfl_xor_sync(0xffffffffu, t, off);
    return t;
}

// ------------------------------------------------------------ per iteration
enum { COARSE_ITERATE = 0, COARSE_START = 1, COARSE_ONLY = 2 };
constexpr int kCoarseSplit = 4;       // warps sharing one row of the inverse (single board)
constexpr int kCoarseThreads = 1024;  // R is staged once per block for 8 rows at a time

// c = Minv R (kCoarseSplit warps per row, their parts summed in a fixed
// order) and, unless MODE is COARSE_ONLY, the coarse part R.c of r.z; the
// last block finishes the scalars: COARSE_START sets rz; COARSE_ITERATE
// computes beta (or BREAKDOWN) and checks the iteration limit, as the Jacobi
// update does in one step.  The rows are read from L2 (the inverse persists
// there); four warps per row keep enough loads in flight to cover its latency.
template <int MODE>
__global__ void __launch_bounds__(kCoarseThreads, 2)
    coarse_apply(const float* __restrict__ minv, const float* __restrict__ rc, float* __restrict__ c, int nc, int ld,
                 SolveCtl* ctl, double* partials, unsigned int* counter) {
    extern __shared__ float s_rc[];
    __shared__ __align__(16) unsigned char scratch_raw[sizeof(Acc32) * 32];
    __shared__ float s_part[kCoarseThreads / 32];
    Acc32* const scratch = reinterpret_cast<Acc32*>(scratch_raw);
    pdl_enter();
    if (MODE != COARSE_ONLY && ctl->state != ST_RUNNING) return;
    for (int i = threadIdx.x; i < ld; i += blockDim.x) s_rc[i] = rc[i];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int slot = warp / kCoarseSplit, part = warp % kCoarseSplit;
    constexpr int kRows = kCoarseThreads / 32 / kCoarseSplit;
    Acc32 acc[1];
    for (int base = blockIdx.x * kRows; base < nc; base += gridDim.x * kRows) {  // uniform across the block
        const int row = base + slot;
        const float t = row < nc ? coarse_row_part(minv + (long long)row * ld, s_rc, ld, lane, part, kCoarseSplit) : 0.f;
        if (lane == 0) s_part[warp] = t;
        __syncthreads();
        if (part == 0 && lane == 0 && row < nc) {
            const float s = (s_part[warp] + s_part[warp + 1]) + (s_part[warp + 2] + s_part[warp + 3]);
            c[row] = s;
            acc[0].add_product(s_rc[row], s);
        }
        __syncthreads();
    }
    if (MODE == COARSE_ONLY) return;
    block_merge<1>(acc, scratch);
    if (threadIdx.x == 0) acc_store(partials + (size_t)blockIdx.x * 4, acc[0]);
    if (!last_block(counter)) return;
    Acc32 tot[1];
    grid_merge<1>(partials, gridDim.x, 4, tot, scratch, counter);
    if (threadIdx.x == 0) {
        const double rzn = ctl->rdr + tot[0].value();
        if (MODE == COARSE_START) {
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

// p = z + beta p with z = r |d^-1| + (free ? c[patch] : 0); START: p = z.
// Not START: x += alpha p first (the update's step, on the old p).
template <bool START>
__global__ void __launch_bounds__(kVecThreads)
    pcg_direction_2l(float* __restrict__ p, float* __restrict__ x, const float* __restrict__ r,
                     const float* __restrict__ dinv, const float* __restrict__ c, long long nq, Layout lay,
                     CoarseLayout cl, const SolveCtl* ctl) {
    pdl_enter();
    if (ctl != nullptr && ctl->state != ST_RUNNING) return;
    const float beta = START ? 0.f : (float)ctl->beta;
    const float alpha = START ? 0.f : (float)ctl->alpha;
    const int qpl = lay.Xp / 4, rows = lay.R + 1;
    const long long stride = (long long)gridDim.x * blockDim.x;
    // The thread's place (node plane z, node row y, quad q of the row) moves by
    // the grid stride; it is advanced by additions and carries, so the loop
    // divides only for the patch of the row and of the quad.
    const long long i0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long line0 = i0 / qpl;
    int q = (int)(i0 - line0 * qpl);
    int z = (int)(line0 / rows);
    int y = (int)(line0 - (long long)z * rows);
    const long long sline = stride / qpl;
    const int sq = (int)(stride - sline * qpl);
    const int sz = (int)(sline / rows);
    const int sy = (int)(sline - (long long)sz * rows);
    const bool wide = cl.b >= 4;  // a quad then spans at most two patches
    for (long long i = i0; i < nq; i += stride) {
        const int x0 = 4 * q;
        const int rowbase = (z * cl.nby + y / cl.b) * cl.nbx;
        const int px0 = x0 / cl.b;
        const float4 rv = reinterpret_cast<const float4*>(r)[i];
        const float4 d = reinterpret_cast<const float4*>(dinv)[i];
        const float rr[4] = {rv.x, rv.y, rv.z, rv.w};
        const float dd[4] = {d.x, d.y, d.z, d.w};
        float out[4];
        float4 pv = make_float4(0.f, 0.f, 0.f, 0.f);
        if (!START) {
            pv = reinterpret_cast<const float4*>(p)[i];
            float4 xv = reinterpret_cast<const float4*>(x)[i];
            xv.x = fmaf(alpha, pv.x, xv.x);
            xv.y = fmaf(alpha, pv.y, xv.y);
            xv.z = fmaf(alpha, pv.z, xv.z);
            xv.w = fmaf(alpha, pv.w, xv.w);
            reinterpret_cast<float4*>(x)[i] = xv;
        }
        const float po[4] = {pv.x, pv.y, pv.z, pv.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int xn = x0 + k;  // node column
            const int px = wide ? px0 + (xn >= (px0 + 1) * cl.b ? 1 : 0) : xn / cl.b;
            float zc = rr[k] * fabsf(dd[k]);
            if (dd[k] > 0.f && xn <= lay.C) zc += c[rowbase + px];
            out[k] = START ? zc : fmaf(beta, po[k], zc);
        }
        reinterpret_cast<float4*>(p)[i] = make_float4(out[0], out[1], out[2], out[3]);
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

}  // namespace tb
