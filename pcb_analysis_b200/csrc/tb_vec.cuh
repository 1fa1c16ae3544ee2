// Node-wise kernels of the solve: layout conversion, the Jacobi diagonal, the
// fused PCG vector updates and the MPIR start / finish steps.
//
// Device layout.  Node fields are stored as (S+1, R+1, Xp) with the row pitch
// Xp = round_up(C+1, 4), so every row starts on a 16-byte boundary and the
// kernels move four nodes per access; element fields are (S, R, Xe) with
// Xe = round_up(C, 4).  Pad entries are zero in every vector, which keeps them
// out of every inner product.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "tb_reduce.cuh"
#include "tb_types.h"

namespace tb {

constexpr int kVecThreads = 256;

struct Layout {
    int S, R, C, Xp, Xe;
    long long N;   // (S+1)(R+1)(C+1)
    long long L;   // (S+1)(R+1)Xp, a multiple of 4
    long long E;   // S R C
    long long LE;  // S R Xe
};

// ----------------------------------------------------------------- layout
template <typename D, typename Src>
__global__ void pack_nodes(D* __restrict__ dst, const Src* __restrict__ src, Layout lay) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    const int cols = lay.C + 1;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < lay.L; i += stride) {
        const long long line = i / lay.Xp;
        const int x = (int)(i - line * lay.Xp);
        dst[i] = (x < cols) ? (D)src[line * cols + x] : (D)0;
    }
}

template <typename D, typename Src>
__global__ void unpack_nodes(D* __restrict__ dst, const Src* __restrict__ src, Layout lay) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    const int cols = lay.C + 1;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < lay.N; n += stride) {
        const long long line = n / cols;
        const int x = (int)(n - line * cols);
        dst[n] = (D)src[line * lay.Xp + x];
    }
}

// Element conductivities: flat FP64 (S, R, C) -> padded FP64 and FP32 (S, R, Xe).
__global__ void pack_elements(double* __restrict__ d64, float* __restrict__ d32, const double* __restrict__ src,
                              Layout lay) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < lay.LE; i += stride) {
        const long long line = i / lay.Xe;
        const int c = (int)(i - line * lay.Xe);
        const double v = (c < lay.C) ? src[line * lay.C + c] : 0.0;
        d64[i] = v;
        d32[i] = (float)v;
    }
}

// rf = Robin total on free nodes, -1 on fixed ones; plane flags mark planes
// with any fixed node or non-zero Robin term.
__global__ void build_rf(double* __restrict__ rf64, float* __restrict__ rf32, int* __restrict__ plane_flags,
                         const double* __restrict__ robin, const uint8_t* __restrict__ free_nodes, Layout lay) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    const int cols = lay.C + 1;
    const long long plane = (long long)(lay.R + 1) * lay.Xp;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < lay.L; i += stride) {
        const long long line = i / lay.Xp;
        const int x = (int)(i - line * lay.Xp);
        double v = 0.0;
        if (x < cols) {
            const long long n = line * cols + x;
            v = free_nodes[n] ? robin[n] : -1.0;
        }
        rf64[i] = v;
        rf32[i] = (float)v;
        if (v != 0.0) {
            int* flag = plane_flags + (int)(i / plane);
            if (*reinterpret_cast<volatile int*>(flag) == 0) atomicOr(flag, 1);
        }
    }
}

// New Robin totals on the free nodes of a prepared system; fixed rows keep
// -1.  Plane flags must be cleared before.
__global__ void update_rf(double* __restrict__ rf64, float* __restrict__ rf32, int* __restrict__ plane_flags,
                          const double* __restrict__ robin, Layout lay) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    const int cols = lay.C + 1;
    const long long plane = (long long)(lay.R + 1) * lay.Xp;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < lay.L; i += stride) {
        const long long line = i / lay.Xp;
        const int x = (int)(i - line * lay.Xp);
        if (x >= cols) continue;
        const double v = (rf64[i] < 0.0) ? -1.0 : robin[line * cols + x];
        rf64[i] = v;
        rf32[i] = (float)v;
        if (v != 0.0) {
            int* flag = plane_flags + (int)(i / plane);
            if (*reinterpret_cast<volatile int*>(flag) == 0) atomicOr(flag, 1);
        }
    }
}

// Jacobi diagonal, bit-identical to the reference's FP64 build
// (operator.py:290-306 _build_diagonal, thermal_system.cpp:328-349): for node
// n and corner index c = 4dz+2dy+dx in order 0..7, add
// (a_x u + a_y u) + a_z u of element (z-dz, y-dy, x-dx), u = U[c,c] = (2/6)((2/6)(1)),
// with a_x = ((k_in h_y) h_z) / h_x etc.; then add the Robin total; fixed rows 1.
// Explicit _rn intrinsics keep the compiler from contracting into FMAs.
__global__ void build_diagonal(double* __restrict__ diag, double* __restrict__ dinv64, float* __restrict__ dinv32,
                               int* __restrict__ err, const double* __restrict__ kin, const double* __restrict__ kz,
                               const double* __restrict__ rf, const double* __restrict__ thick,
                               const double* __restrict__ px, const double* __restrict__ py, Layout lay) {
    const double t = 2.0 / 6.0;
    const double u = __dmul_rn(t, __dmul_rn(t, 1.0));
    const long long stride = (long long)gridDim.x * blockDim.x;
    const int cols = lay.C + 1;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < lay.L; i += stride) {
        const long long line = i / lay.Xp;
        const int x = (int)(i - line * lay.Xp);
        const int z = (int)(line / (lay.R + 1));
        const int y = (int)(line - (long long)z * (lay.R + 1));
        if (x >= cols) {
            diag[i] = 0.0;
            dinv64[i] = 0.0;
            dinv32[i] = 0.0f;
            continue;
        }
        double acc = 0.0;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int ez = z - (c >> 2), ey = y - ((c >> 1) & 1), ex = x - (c & 1);
            if (ez < 0 || ez >= lay.S || ey < 0 || ey >= lay.R || ex < 0 || ex >= lay.C) continue;
            const long long e = ((long long)ez * lay.R + ey) * lay.Xe + ex;
            const double hz = thick[ez], hy = py[ey], hx = px[ex];
            const double ax = __ddiv_rn(__dmul_rn(__dmul_rn(kin[e], hy), hz), hx);
            const double ay = __ddiv_rn(__dmul_rn(__dmul_rn(kin[e], hx), hz), hy);
            const double az = __ddiv_rn(__dmul_rn(__dmul_rn(kz[e], hx), hy), hz);
            acc = __dadd_rn(acc, __dadd_rn(__dadd_rn(__dmul_rn(ax, u), __dmul_rn(ay, u)), __dmul_rn(az, u)));
        }
        const double r = rf[i];
        double d;
        if (r < 0.0) {
            d = 1.0;
        } else {
            d = __dadd_rn(acc, r);
            if (!(d > 0.0)) atomicOr(err, 1);
        }
        diag[i] = d;
        dinv64[i] = (d > 0.0) ? 1.0 / d : 0.0;
        dinv32[i] = (r < 0.0) ? -1.0f : ((d > 0.0) ? (float)(1.0 / d) : 0.0f);  // -1 marks a fixed row (d = 1)
    }
}

// ------------------------------------------------------------ small scalars
__global__ void set_ctl(SolveCtl* ctl, double tol, int max_it, double scale, double bnorm, double beta = 0.0) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        ctl->tol = tol;
        ctl->max_it = max_it;
        ctl->scale = scale;
        ctl->inv_scale = 1.0 / scale;
        ctl->bnorm = bnorm;
        ctl->state = ST_RUNNING;
        ctl->iterations = 0;
        ctl->applications = 0;
        ctl->rel = 1.0;
        ctl->rz = 1.0;
        ctl->alpha = 0.0;
        ctl->beta = beta;
    }
}

// Shared tail of the kernels that end with a reduction.
template <int NA, class A>
__device__ __forceinline__ bool finish_partials(A (&acc)[NA], A* scratch, double* partials, unsigned int* counter,
                                                A (&tot)[NA]) {
    block_merge<NA>(acc, scratch);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NA; ++k) acc_store(partials + (size_t)blockIdx.x * 4 + 2 * k, acc[k]);
    }
    if (!last_block(counter)) return false;
    grid_merge<NA>(partials, gridDim.x, 4, tot, scratch, counter);
    return threadIdx.x == 0;
}

// ||v||^2 of an FP64 node field.
__global__ void __launch_bounds__(kVecThreads) norm2_f64(const double* __restrict__ v, long long nq, SolveCtl* ctl,
                                                         double* partials, unsigned int* counter) {
    __shared__ __align__(16) unsigned char scratch_raw[sizeof(Acc64) * (32)];
    Acc64* const scratch = reinterpret_cast<Acc64*>(scratch_raw);
    Acc64 acc[1];
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += stride) {
        const double2 a = reinterpret_cast<const double2*>(v)[2 * i];
        const double2 b = reinterpret_cast<const double2*>(v)[2 * i + 1];
        acc[0].add_product(a.x, a.x);
        acc[0].add_product(a.y, a.y);
        acc[0].add_product(b.x, b.x);
        acc[0].add_product(b.y, b.y);
    }
    Acc64 tot[1];
    if (finish_partials<1>(acc, scratch, partials, counter, tot)) ctl->norm2 = tot[0].value();
}

__device__ __forceinline__ void finalize_start(SolveCtl* ctl, double rr0, double rz) {
    ctl->rr = rr0;
    ctl->rz = rz;
    ctl->iterations = 0;
    ctl->applications = 0;
    const double r0 = sqrt(rr0);
    if (!(ctl->bnorm > 0.0)) ctl->bnorm = r0;
    if (r0 == 0.0) {
        ctl->rel = 0.0;
        ctl->state = ST_ZERO_RHS;
    } else {
        ctl->rel = r0 / ctl->bnorm;
        ctl->state = (ctl->rel <= ctl->tol) ? ST_CONVERGED : ST_RUNNING;
    }
}

// Two-level form: r.z = sum r^2 / d + R.c needs the coarse step, which
// finishes it (coarse_apply); here only the norms and the stopping test.
__device__ __forceinline__ void finalize_start_2l(SolveCtl* ctl, double rr0, double rdr) {
    ctl->rdr = rdr;
    finalize_start(ctl, rr0, 0.0);
}

// Start of the FP32 inner PCG from the FP64 outer residual (reference
// solver.py:172-196): rhs = f32(r * 2^-e) with max|r * 2^-e| in [0.5, 1),
// x = 0, r = rhs, z = r / d, p = z, rz = r.z, ||rhs||.
template <bool TL>
__global__ void __launch_bounds__(kVecThreads)
    inner_start_f32(const double* __restrict__ r64, float* __restrict__ x, float* __restrict__ r,
                    float* __restrict__ p, const float* __restrict__ dinv, long long nq, SolveCtl* ctl,
                    double* partials, unsigned int* counter) {
    __shared__ __align__(16) unsigned char scratch_raw[sizeof(Acc32) * (2 * 32)];
    Acc32* const scratch = reinterpret_cast<Acc32*>(scratch_raw);
    const double scale = ctl->scale;
    Acc32 acc[2];
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += stride) {
        const double2 a = reinterpret_cast<const double2*>(r64)[2 * i];
        const double2 b = reinterpret_cast<const double2*>(r64)[2 * i + 1];
        const float4 d = reinterpret_cast<const float4*>(dinv)[i];
        const float4 rv = make_float4((float)(a.x * scale), (float)(a.y * scale), (float)(b.x * scale),
                                      (float)(b.y * scale));
        const float4 zv = make_float4(rv.x * fabsf(d.x), rv.y * fabsf(d.y), rv.z * fabsf(d.z), rv.w * fabsf(d.w));
        reinterpret_cast<float4*>(r)[i] = rv;
        reinterpret_cast<float4*>(p)[i] = zv;
        reinterpret_cast<float4*>(x)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        acc[0].add_product(rv.x, rv.x);
        acc[0].add_product(rv.y, rv.y);
        acc[0].add_product(rv.z, rv.z);
        acc[0].add_product(rv.w, rv.w);
        acc[1].add_product(rv.x, zv.x);
        acc[1].add_product(rv.y, zv.y);
        acc[1].add_product(rv.z, zv.z);
        acc[1].add_product(rv.w, zv.w);
    }
    Acc32 tot[2];
    if (finish_partials<2>(acc, scratch, partials, counter, tot)) {
        if (TL) finalize_start_2l(ctl, tot[0].value(), tot[1].value());
        else finalize_start(ctl, tot[0].value(), tot[1].value());
    }
}

// Start of the plain FP64 PCG from r = b - A x0: z = r / d, p = z.
__global__ void __launch_bounds__(kVecThreads)
    pcg_start_f64(const double* __restrict__ r, double* __restrict__ p, const double* __restrict__ dinv, long long nq,
                  SolveCtl* ctl, double* partials, unsigned int* counter) {
    __shared__ __align__(16) unsigned char scratch_raw[sizeof(Acc64) * (2 * 32)];
    Acc64* const scratch = reinterpret_cast<Acc64*>(scratch_raw);
    Acc64 acc[2];
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < 2 * nq; i += stride) {
        const double2 rv = reinterpret_cast<const double2*>(r)[i];
        const double2 d = reinterpret_cast<const double2*>(dinv)[i];
        const double2 zv = make_double2(rv.x * d.x, rv.y * d.y);
        reinterpret_cast<double2*>(p)[i] = zv;
        acc[0].add_product(rv.x, rv.x);
        acc[0].add_product(rv.y, rv.y);
        acc[1].add_product(rv.x, zv.x);
        acc[1].add_product(rv.y, zv.y);
    }
    Acc64 tot[2];
    if (finish_partials<2>(acc, scratch, partials, counter, tot)) finalize_start(ctl, tot[0].value(), tot[1].value());
}

__device__ __forceinline__ void finalize_update(SolveCtl* ctl, double rr, double rzn) {
    const int it = ctl->iterations + 1;
    ctl->iterations = it;
    ctl->rr = rr;
    const double rel = sqrt(rr) / ctl->bnorm;
    ctl->rel = rel;
    if (rel <= ctl->tol) {
        ctl->state = ST_CONVERGED;
    } else if (!isfinite(rzn) || ctl->rz == 0.0) {
        ctl->state = ST_BREAKDOWN;
    } else {
        ctl->beta = rzn / ctl->rz;
        ctl->rz = rzn;
        if (it >= ctl->max_it) ctl->state = ST_MAXIT;
    }
}

// Two-level form of the update's scalars: beta and the iteration limit wait
// for the coarse part of r.z (coarse_apply).
__device__ __forceinline__ void finalize_update_2l(SolveCtl* ctl, double rr, double rdr) {
    ctl->iterations += 1;
    ctl->rr = rr;
    ctl->rdr = rdr;
    const double rel = sqrt(rr) / ctl->bnorm;
    ctl->rel = rel;
    if (rel <= ctl->tol) ctl->state = ST_CONVERGED;
}

// After the inner PCG stopped: the last update's x += alpha p is still to be
// added when that update ran (at least one iteration) and it stopped the PCG
// (converged), or the scalars after it did (breakdown, iteration limit), so
// that no direction step followed.  A stop at the operator (non-SPD) comes
// after a direction step, which added its x step already.
__device__ __forceinline__ bool x_step_pending(const SolveCtl* c) {
    return c->iterations > 0 && (c->state == ST_CONVERGED || c->state == ST_BREAKDOWN || c->state == ST_MAXIT);
}

// r -= alpha q; z = r / d; r.r and r.z (reference solver.py:199-216); with TL
// (two-level) the second sum is sum r^2 / d, completed by coarse_apply.  The
// step x += alpha p of the same iteration is taken by the direction kernel,
// which reads p anyway, before it overwrites p (or, when the PCG stops here,
// by mpir_finish): the same operations on the same values, 4 bytes per node
// less traffic.
template <bool TL>
__global__ void __launch_bounds__(kVecThreads)
    pcg_update_f32(float* __restrict__ r, const float* __restrict__ q, const float* __restrict__ dinv, long long nq,
                   SolveCtl* ctl, double* partials, unsigned int* counter) {
    __shared__ __align__(16) unsigned char scratch_raw[sizeof(Acc32) * (2 * 32)];
    Acc32* const scratch = reinterpret_cast<Acc32*>(scratch_raw);
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (ctl->state != ST_RUNNING) return;
    const float alpha = (float)ctl->alpha;
    Acc32 acc[2];
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += stride) {
        float4 rv = reinterpret_cast<float4*>(r)[i];
        const float4 qv = reinterpret_cast<const float4*>(q)[i];
        const float4 d = reinterpret_cast<const float4*>(dinv)[i];
        rv.x = fmaf(-alpha, qv.x, rv.x);
        rv.y = fmaf(-alpha, qv.y, rv.y);
        rv.z = fmaf(-alpha, qv.z, rv.z);
        rv.w = fmaf(-alpha, qv.w, rv.w);
        reinterpret_cast<float4*>(r)[i] = rv;
        acc[0].add_product(rv.x, rv.x);
        acc[0].add_product(rv.y, rv.y);
        acc[0].add_product(rv.z, rv.z);
        acc[0].add_product(rv.w, rv.w);
        acc[1].add_product(rv.x, rv.x * fabsf(d.x));
        acc[1].add_product(rv.y, rv.y * fabsf(d.y));
        acc[1].add_product(rv.z, rv.z * fabsf(d.z));
        acc[1].add_product(rv.w, rv.w * fabsf(d.w));
    }
    Acc32 tot[2];
    if (finish_partials<2>(acc, scratch, partials, counter, tot)) {
        if (TL) finalize_update_2l(ctl, tot[0].value(), tot[1].value());
        else finalize_update(ctl, tot[0].value(), tot[1].value());
    }
}

__global__ void __launch_bounds__(kVecThreads)
    pcg_update_f64(double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
                   const double* __restrict__ q, const double* __restrict__ dinv, long long nq, SolveCtl* ctl,
                   double* partials, unsigned int* counter) {
    __shared__ __align__(16) unsigned char scratch_raw[sizeof(Acc64) * (2 * 32)];
    Acc64* const scratch = reinterpret_cast<Acc64*>(scratch_raw);
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (ctl->state != ST_RUNNING) return;
    const double alpha = ctl->alpha;
    Acc64 acc[2];
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < 2 * nq; i += stride) {
        double2 xv = reinterpret_cast<double2*>(x)[i];
        double2 rv = reinterpret_cast<double2*>(r)[i];
        const double2 pv = reinterpret_cast<const double2*>(p)[i];
        const double2 qv = reinterpret_cast<const double2*>(q)[i];
        const double2 d = reinterpret_cast<const double2*>(dinv)[i];
        xv.x = fma(alpha, pv.x, xv.x);
        xv.y = fma(alpha, pv.y, xv.y);
        rv.x = fma(-alpha, qv.x, rv.x);
        rv.y = fma(-alpha, qv.y, rv.y);
        reinterpret_cast<double2*>(x)[i] = xv;
        reinterpret_cast<double2*>(r)[i] = rv;
        acc[0].add_product(rv.x, rv.x);
        acc[0].add_product(rv.y, rv.y);
        acc[1].add_product(rv.x, rv.x * d.x);
        acc[1].add_product(rv.y, rv.y * d.y);
    }
    Acc64 tot[2];
    if (finish_partials<2>(acc, scratch, partials, counter, tot)) finalize_update(ctl, tot[0].value(), tot[1].value());
}

// x += alpha p (the update's step, on the old p), then p = z + beta p with
// z = r / d (reference solver.py:199-224).
__global__ void __launch_bounds__(kVecThreads)
    pcg_direction_f32(float* __restrict__ p, float* __restrict__ x, const float* __restrict__ r,
                      const float* __restrict__ dinv, long long nq, const SolveCtl* ctl) {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (ctl->state != ST_RUNNING) return;
    const float beta = (float)ctl->beta;
    const float alpha = (float)ctl->alpha;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += stride) {
        float4 pv = reinterpret_cast<float4*>(p)[i];
        float4 xv = reinterpret_cast<float4*>(x)[i];
        const float4 rv = reinterpret_cast<const float4*>(r)[i];
        const float4 d = reinterpret_cast<const float4*>(dinv)[i];
        xv.x = fmaf(alpha, pv.x, xv.x);
        xv.y = fmaf(alpha, pv.y, xv.y);
        xv.z = fmaf(alpha, pv.z, xv.z);
        xv.w = fmaf(alpha, pv.w, xv.w);
        reinterpret_cast<float4*>(x)[i] = xv;
        pv.x = fmaf(beta, pv.x, rv.x * fabsf(d.x));
        pv.y = fmaf(beta, pv.y, rv.y * fabsf(d.y));
        pv.z = fmaf(beta, pv.z, rv.z * fabsf(d.z));
        pv.w = fmaf(beta, pv.w, rv.w * fabsf(d.w));
        reinterpret_cast<float4*>(p)[i] = pv;
    }
}

__global__ void __launch_bounds__(kVecThreads)
    pcg_direction_f64(double* __restrict__ p, const double* __restrict__ r, const double* __restrict__ dinv,
                      long long nq, const SolveCtl* ctl) {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (ctl->state != ST_RUNNING) return;
    const double beta = ctl->beta;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < 2 * nq; i += stride) {
        double2 pv = reinterpret_cast<double2*>(p)[i];
        const double2 rv = reinterpret_cast<const double2*>(r)[i];
        const double2 d = reinterpret_cast<const double2*>(dinv)[i];
        pv.x = fma(beta, pv.x, rv.x * d.x);
        pv.y = fma(beta, pv.y, rv.y * d.y);
        reinterpret_cast<double2*>(p)[i] = pv;
    }
}

// x64 += f64(x32) / scale (the scale is a power of two, so this is exact
// scaling; reference solver.py:226-232 and the outer update :671), x32 with
// the last update's pending step x32 + alpha p added first in FP32.
__global__ void __launch_bounds__(kVecThreads)
    mpir_finish(double* __restrict__ x64, const float* __restrict__ x32, const float* __restrict__ p, long long nq,
                const SolveCtl* ctl) {
    const double inv = ctl->inv_scale;
    const bool pending = x_step_pending(ctl);
    const float alpha = (float)ctl->alpha;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += stride) {
        float4 c = reinterpret_cast<const float4*>(x32)[i];
        if (pending) {
            const float4 pv = reinterpret_cast<const float4*>(p)[i];
            c.x = fmaf(alpha, pv.x, c.x);
            c.y = fmaf(alpha, pv.y, c.y);
            c.z = fmaf(alpha, pv.z, c.z);
            c.w = fmaf(alpha, pv.w, c.w);
        }
        double2 a = reinterpret_cast<double2*>(x64)[2 * i];
        double2 b = reinterpret_cast<double2*>(x64)[2 * i + 1];
        a.x += (double)c.x * inv;
        a.y += (double)c.y * inv;
        b.x += (double)c.z * inv;
        b.y += (double)c.w * inv;
        reinterpret_cast<double2*>(x64)[2 * i] = a;
        reinterpret_cast<double2*>(x64)[2 * i + 1] = b;
    }
}

}  // namespace tb
