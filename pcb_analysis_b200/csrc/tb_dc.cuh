// Layered DC conduction operator: bilinear (Q1) sheet elements on each copper
// layer plus resistive vias between layer nodes (reference
// src/electrical/matrix_free_mpir_fem/pcb.py:275-621; C++
// native/layered_dc_q1.cpp, cpp/src/fem/layered_dc_system.cpp).
//
//     y = where(free, K (x * free) + V (x * free), x)
//
// K_e = c_x U_x + c_y U_y per element, U_x = M (x) S and U_y = S (x) M in the
// local order 2 dy + dx, c_x = sigma t h_y / h_x, c_y = sigma t h_x / h_y
// (zero on void elements).  A via of conductance g between nodes a and b adds
// g (x_a - x_b) to row a and g (x_b - x_a) to row b.
//
// Element action in the Haar basis.  [1,1] and [1,-1] are eigenvectors of M
// (1/2, 1/6) and S (0, 2), so with u~_m = v_m . u the element action is
//     K_e u = (c_x / 4) u~_sd v_sd + (c_y / 4) u~_ds v_ds + ((c_x + c_y) / 12) u~_dd v_dd
// (pattern y, x: s = sum, d = difference; the ss pattern has eigenvalue 0).
//
// Node fields use the solver's padded layout (L, R+1, Xp) with the layers as
// node planes; the sheet conductance sigma t is an element field (L, R, Xe).
// One byte per node carries bit 0 = free and bit 1 = the node ends a via.
// A via node's list (its vias as the lower end in via order, then as the upper
// end) is found through a per-node slot, read only where the via bit is set,
// so the stencil threads pay for vias only where they sit.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "tb_apply.cuh"
#include "tb_reduce.cuh"
#include "tb_types.h"

namespace tb {

constexpr uint8_t kDcFree = 1;
constexpr uint8_t kDcVia = 2;
constexpr int kDcThreads = 256;

// Via tables of a DC system (device): the i-th node with vias owns entries
// start[i] .. start[i+1]-1 of other / g; slot[n] = i for that node (padded
// index n), read only where the node's via bit is set.
template <typename T>
struct DcVias {
    const int* slot;
    const int* start;
    const long long* other;
    const T* g;
    int count;  // nodes with vias
};

template <typename T>
struct DcParams {
    ApplyParams<T> A;      // x, y, b, kin = sigma t, reductions, geometry, layout
    const uint8_t* mask;   // (L, R+1, Xp) node bits
    const T* colh;         // (Xp) h_x per element column, zero past C
    const T* colih;        // (Xp) 1 / h_x, zero past C
    DcVias<T> vias;
};

template <typename T>
__device__ __forceinline__ T dc_masked(const T v, const uint8_t m, const bool stiffness) {
    return (stiffness || (m & kDcFree)) ? v : T(0);
}

// Sum of g (w_n - w_other) over the vias of the node in list `slot` (w = x *
// free, or x for the unconstrained action), in list order.
template <typename T, int MODE>
__device__ T dc_via_sum(const DcParams<T>& P, const int slot, const T wn) {
    T acc = T(0);
    const int end = P.vias.start[slot + 1];
    for (int e = P.vias.start[slot]; e < end; ++e) {
        const long long o = P.vias.other[e];
        const T wo = dc_masked(P.A.x[o], P.mask[o], MODE == MODE_STIFFNESS);
        acc += P.vias.g[e] * (wn - wo);
    }
    return acc;
}

// The corner outputs of one element, order (dy, dx) = (0,0) (0,1) (1,0) (1,1).
template <typename T>
__device__ __forceinline__ void dc_element(const T cxq, const T cyq, const T cdd, const T u00, const T u01, const T u10,
                                           const T u11, T (&out)[4]) {
    const T d0 = u00 - u01, d1 = u10 - u11;
    const T sd = d0 + d1;
    const T ds = (u00 + u01) - (u10 + u11);
    const T dd = d0 - d1;
    const T a = cxq * sd, b = cyq * ds, c = cdd * dd;
    out[0] = (a + b) + c;
    out[1] = (b - a) - c;
    out[2] = (a - b) - c;
    out[3] = c - (a + b);
}

// One thread per four consecutive nodes of a node row; the lanes of a warp
// hold consecutive quads, so the node and element to the left and right of a
// quad come from the neighbouring lanes by shuffles (a load where the
// neighbour sits in another row or warp).  Every load is a 16-byte quad
// (node values, sheet conductance, the padded per-column geometry) or a
// 4-byte quad of node bits.  The loop runs the same number of times in every
// lane of a warp, so the shuffles always see the whole warp.  Epilogues as
// the hex operator's: store, p.Ap, or the FP64 residual with its norm and peak.
template <typename T, int MODE, int EPI>
__global__ void __launch_bounds__(kDcThreads, sizeof(T) == 4 ? 3 : 2) dc_apply_kernel(const DcParams<T> P) {
    const ApplyParams<T>& A = P.A;
    pdl_trigger();
    pdl_wait();
    if (EPI == EPI_DOT && A.ctl->state != ST_RUNNING) return;
    if (EPI != EPI_STORE && A.clock != nullptr && threadIdx.x == 0) atomicMin(&A.clock->first, global_ns());
    constexpr bool STIFF = MODE == MODE_STIFFNESS;
    const int R = A.R, C = A.C, Xp = A.Xp, Xe = A.Xe;
    const int qrow = Xp >> 2;
    const long long nq = (long long)(A.S + 1) * (R + 1) * qrow;
    const int lane = threadIdx.x & 31;
    T dot = T(0);
    double rmax = 0.0;
    const T quarter = T(0.25), twelfth = T(1) / T(12);
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long warp_first = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31);
    for (long long qb = warp_first; qb < nq; qb += stride) {
        const long long q = qb + lane;
        const bool valid = q < nq;
        const long long qq = valid ? q : nq - 1;
        const long long line = qq / qrow;  // l * (R+1) + y
        const int x0 = 4 * (int)(qq - line * qrow);
        const int l = (int)(line / (R + 1));
        const int y = (int)(line - (long long)l * (R + 1));
        const long long n0 = line * Xp + x0;
        // neighbours in the same node row sit in lane -1 / +1 of this warp
        const long long line_lo = __shfl_up_sync(0xffffffffu, line, 1);
        const long long line_hi = __shfl_down_sync(0xffffffffu, line, 1);
        const bool left_in_warp = lane > 0 && line_lo == line;
        const bool right_in_warp = lane < 31 && line_hi == line;
        // w at node rows y-1, y, y+1 and columns x0-1 .. x0+4; raw x of row y
        T w[3][6];
        Quad<T> self = zero_quad<T>();
        uchar4 mself = make_uchar4(0, 0, 0, 0);
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            const int yy = y - 1 + r;
            const bool row_ok = yy >= 0 && yy <= R;
            const long long base = n0 + (long long)(r - 1) * Xp;
            Quad<T> xv = zero_quad<T>();
            uchar4 m = make_uchar4(0, 0, 0, 0);
            // the edge loads go out with the quad, not after the shuffle
            T xl = T(0), xr = T(0);
            uint8_t ml = 0, mr = 0;
            if (row_ok) {
                xv = ldg_quad(A.x + base);
                m = *reinterpret_cast<const uchar4*>(P.mask + base);
                if (x0 >= 1 && !left_in_warp) {
                    xl = __ldg(A.x + base - 1);
                    ml = P.mask[base - 1];
                }
                if (x0 + 4 < Xp && !right_in_warp) {
                    xr = __ldg(A.x + base + 4);
                    mr = P.mask[base + 4];
                }
            }
            if (r == 1) {
                self = xv;
                mself = m;
            }
            w[r][1] = dc_masked(xv.v[0], m.x, STIFF);
            w[r][2] = dc_masked(xv.v[1], m.y, STIFF);
            w[r][3] = dc_masked(xv.v[2], m.z, STIFF);
            w[r][4] = dc_masked(xv.v[3], m.w, STIFF);
            const T from_left = __shfl_up_sync(0xffffffffu, w[r][4], 1);
            const T from_right = __shfl_down_sync(0xffffffffu, w[r][1], 1);
            w[r][0] = T(0);
            w[r][5] = T(0);
            if (row_ok && x0 >= 1) w[r][0] = left_in_warp ? from_left : dc_masked(xl, ml, STIFF);
            if (row_ok && x0 + 4 < Xp) w[r][5] = right_in_warp ? from_right : dc_masked(xr, mr, STIFF);
        }
        // via lists of this quad's nodes, fetched now so the load overlaps the element math
        int slot[4] = {-1, -1, -1, -1};
        {
            const uint8_t mk[4] = {mself.x, mself.y, mself.z, mself.w};
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (valid && (mk[k] & kDcVia)) slot[k] = __ldg(P.vias.slot + n0 + k);
        }
        // per-column geometry of element columns x0-1 .. x0+3 (padded arrays, zero past C)
        const Quad<T> hxq = ldg_quad(P.colh + x0);
        const Quad<T> ihxq = ldg_quad(P.colih + x0);
        T hx_edge = T(0), ihx_edge = T(0);
        if (x0 >= 1 && !left_in_warp) {
            hx_edge = __ldg(P.colh + x0 - 1);
            ihx_edge = __ldg(P.colih + x0 - 1);
        }
        const T hx_left_s = __shfl_up_sync(0xffffffffu, hxq.v[3], 1);
        const T ihx_left_s = __shfl_up_sync(0xffffffffu, ihxq.v[3], 1);
        T hxs[5], ihxs[5];
        hxs[0] = x0 >= 1 ? (left_in_warp ? hx_left_s : hx_edge) : T(0);
        ihxs[0] = x0 >= 1 ? (left_in_warp ? ihx_left_s : ihx_edge) : T(0);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            hxs[k + 1] = hxq.v[k];
            ihxs[k + 1] = ihxq.v[k];
        }
        T acc[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll
        for (int er = 0; er < 2; ++er) {  // element rows y-1 (node row y is their dy = 1) and y (dy = 0)
            const int ey = y - 1 + er;
            const bool erow_ok = ey >= 0 && ey < R;
            Quad<T> sq = zero_quad<T>();
            T hy = T(0), ihy = T(0), s_edge = T(0);
            if (erow_ok) {
                const T* const srow = A.kin + ((long long)l * R + ey) * Xe;
                if (x0 < Xe) sq = ldg_quad(srow + x0);  // else all past C
                if (x0 >= 1 && !left_in_warp) s_edge = __ldg(srow + x0 - 1);
                hy = A.hy[ey];
                ihy = A.ihy[ey];
            }
            const T sl = __shfl_up_sync(0xffffffffu, sq.v[3], 1);
            T st[5];
            st[0] = (erow_ok && x0 >= 1) ? (left_in_warp ? sl : s_edge) : T(0);
#pragma unroll
            for (int k = 0; k < 4; ++k) st[k + 1] = sq.v[k];
            if (!erow_ok) continue;
            const int dy = er == 0 ? 1 : 0;
#pragma unroll
            for (int k = 0; k < 5; ++k) {  // element column x0-1+k (sheet zero past C and on voids)
                const T cx = st[k] * (hy * ihxs[k]);
                const T cy = st[k] * (hxs[k] * ihy);
                T out[4];
                dc_element(cx * quarter, cy * quarter, (cx + cy) * twelfth, w[er][k], w[er][k + 1], w[er + 1][k],
                           w[er + 1][k + 1], out);
                if (k >= 1) acc[k - 1] += out[2 * dy];  // node x0+k-1 is the element's corner dx = 0
                if (k <= 3) acc[k] += out[2 * dy + 1];  // node x0+k is its corner dx = 1
            }
        }
        if (!valid) continue;
        const uint8_t mk[4] = {mself.x, mself.y, mself.z, mself.w};
        Quad<T> yv;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            T v = acc[k];
            if (slot[k] >= 0) v += dc_via_sum<T, MODE>(P, slot[k], w[1][k + 1]);
            if (!STIFF && !(mk[k] & kDcFree)) v = self.v[k];
            if (x0 + k > C) v = T(0);
            yv.v[k] = v;
        }
        if (EPI == EPI_RESIDUAL) {
            const Quad<T> bq = ldg_quad(A.b + n0);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                yv.v[k] = (x0 + k > C) ? T(0) : bq.v[k] - yv.v[k];
                dot = fma(yv.v[k], yv.v[k], dot);
                rmax = fmax(rmax, fabs((double)yv.v[k]));
            }
        } else if (EPI == EPI_DOT) {
#pragma unroll
            for (int k = 0; k < 4; ++k) dot = fma(self.v[k], yv.v[k], dot);
        }
        st_quad(A.y + n0, yv);
    }
    if (EPI == EPI_STORE) return;
    apply_reduce<T, EPI>(A, dot, rmax, gridDim.x, blockIdx.x);
}

// Jacobi diagonal, bit-identical to the reference's FP64 build
// (pcb.py:598-617 _build_diagonal): for node n, element views 0..3 in order
// (the elements whose corner 0, 1, 2, 3 is n) add c_x u + c_y u with
// u = U[i,i] = 2/6 and c_x = ((sigma t) h_y) / h_x, c_y = ((sigma t) h_x) / h_y;
// then the via conductances in list order (as the lower end in via order, then
// as the upper end, the two np.add.at passes); fixed rows 1.  `err` is set
// when a free node's diagonal is not positive.
__global__ void dc_build_diagonal(double* __restrict__ diag, double* __restrict__ dinv64, float* __restrict__ dinv32,
                                  int* __restrict__ err, const double* __restrict__ sheet,
                                  const uint8_t* __restrict__ mask, const double* __restrict__ px,
                                  const double* __restrict__ py, const DcVias<double> vias, const int L, const int R,
                                  const int C, const int Xp, const int Xe) {
    const double u = 2.0 / 6.0;
    const long long total = (long long)L * (R + 1) * Xp;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        const long long line = i / Xp;
        const int x = (int)(i - line * Xp);
        const int l = (int)(line / (R + 1));
        const int y = (int)(line - (long long)l * (R + 1));
        if (x > C) {
            diag[i] = 0.0;
            dinv64[i] = 0.0;
            dinv32[i] = 0.0f;
            continue;
        }
        double acc = 0.0;
#pragma unroll
        for (int c = 0; c < 4; ++c) {  // view c: element (y - dy, x - dx), dy = c >> 1, dx = c & 1
            const int ey = y - (c >> 1), ex = x - (c & 1);
            if (ey < 0 || ey >= R || ex < 0 || ex >= C) continue;
            const double st = sheet[((long long)l * R + ey) * Xe + ex];
            const double cx = __ddiv_rn(__dmul_rn(st, py[ey]), px[ex]);
            const double cy = __ddiv_rn(__dmul_rn(st, px[ex]), py[ey]);
            acc = __dadd_rn(acc, __dadd_rn(__dmul_rn(cx, u), __dmul_rn(cy, u)));
        }
        if (mask[i] & kDcVia) {
            const int at = vias.slot[i];
            for (int e = vias.start[at]; e < vias.start[at + 1]; ++e) acc = __dadd_rn(acc, vias.g[e]);
        }
        const bool free_node = (mask[i] & kDcFree) != 0;
        if (free_node && !(acc > 0.0)) atomicOr(err, 1);
        const double d = free_node ? acc : 1.0;
        diag[i] = d;
        dinv64[i] = 1.0 / d;
        dinv32[i] = free_node ? (float)(1.0 / d) : -1.0f;  // the sign marks fixed rows
    }
}

// rf of a DC system: 0 on free nodes, -1 on fixed ones (no Robin term); the
// two-level set-up reads the free mask from it.
__global__ void dc_build_rf(double* __restrict__ rf64, float* __restrict__ rf32, const uint8_t* __restrict__ mask,
                            long long total) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        const double v = (mask[i] & kDcFree) ? 0.0 : -1.0;
        rf64[i] = v;
        rf32[i] = (float)v;
    }
}

}  // namespace tb
