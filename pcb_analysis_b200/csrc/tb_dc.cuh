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
// One byte per node carries bit 0 = free, bit 1 = the node ends a via and
// bit 2 = active.
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

// ------------------------------------------------------------- y-march
// The same action with every element computed once and every node row loaded
// once.  A warp owns a segment of 31 node quads of one layer (lanes 1..31;
// lane 0 holds the quad to the left as a halo) and marches down a band of node
// rows.  Per row it loads the next node row (prefetched one row ahead) and one
// row of sheet conductances, runs the four elements under its quad, and
// completes the node row above: the lower corners of the element row below
// plus the upper corners of the row above, kept from the previous step.  The
// element to the left of a quad is the left lane's last one, whose corner
// contributions arrive by a shuffle; the node to the right of a quad is the
// right lane's first.
template <typename T>
struct DcRow {
    T w[4];        // masked values (x for the unconstrained action) of the quad
    Quad<T> raw;   // x of the quad
    uchar4 m;      // node bits
    T right;       // masked value of node x0+4 (lane 31 loads it; others shuffle)
};

template <typename T, bool STIFF>
__device__ __forceinline__ DcRow<T> dc_load_row(const DcParams<T>& P, const int yy, const int R, const long long n,
                                                const bool quad_ok, const bool edge_ok) {
    DcRow<T> r;
    r.raw = zero_quad<T>();
    r.m = make_uchar4(0, 0, 0, 0);
    r.right = T(0);
    if (quad_ok && yy >= 0 && yy <= R) {
        r.raw = ldg_quad(P.A.x + n);
        r.m = *reinterpret_cast<const uchar4*>(P.mask + n);
        if (edge_ok) r.right = dc_masked(__ldg(P.A.x + n + 4), P.mask[n + 4], STIFF);
    }
    r.w[0] = dc_masked(r.raw.v[0], r.m.x, STIFF);
    r.w[1] = dc_masked(r.raw.v[1], r.m.y, STIFF);
    r.w[2] = dc_masked(r.raw.v[2], r.m.z, STIFF);
    r.w[3] = dc_masked(r.raw.v[3], r.m.w, STIFF);
    return r;
}

template <typename T, int MODE, int EPI>
__global__ void __launch_bounds__(kDcThreads, sizeof(T) == 4 ? 3 : 2)
    dc_march_kernel(const DcParams<T> P, const int nseg, const int nband, const int band) {
    const ApplyParams<T>& A = P.A;
    pdl_trigger();
    pdl_wait();
    if (EPI == EPI_DOT && A.ctl->state != ST_RUNNING) return;
    if (EPI != EPI_STORE && A.clock != nullptr && threadIdx.x == 0) atomicMin(&A.clock->first, global_ns());
    constexpr bool STIFF = MODE == MODE_STIFFNESS;
    const int R = A.R, C = A.C, Xp = A.Xp, Xe = A.Xe;
    const int qrow = Xp >> 2;
    const int lane = threadIdx.x & 31;
    const long long units = (long long)(A.S + 1) * nband * nseg;
    const long long unit = (long long)blockIdx.x * (kDcThreads / 32) + (threadIdx.x >> 5);
    T dot = T(0);
    double rmax = 0.0;
    if (unit < units) {  // uniform per warp
        const int l = (int)(unit / ((long long)nband * nseg));
        const int rem = (int)(unit - (long long)l * nband * nseg);
        const int b = rem / nseg, g = rem - b * nseg;
        const int xq = g * 31 + lane - 1;  // lane 0: the halo quad to the left
        const bool quad_ok = xq >= 0 && xq < qrow;
        const bool out_lane = lane >= 1 && quad_ok;
        const int x0 = 4 * (quad_ok ? xq : 0);
        const bool edge_ok = lane == 31 && x0 + 4 < Xp;
        const int y0 = b * band;
        const int y1 = min(y0 + band, R + 1);  // output rows y0 .. y1-1
        const long long plane = (long long)(R + 1) * Xp;
        const long long col = (long long)l * plane + x0;
        const T quarter = T(0.25), twelfth = T(1) / T(12);
        // per-column geometry of element columns x0 .. x0+3 (zero past C)
        const Quad<T> hxq = ldg_quad(P.colh + x0);
        const Quad<T> ihxq = ldg_quad(P.colih + x0);
        const T* const sheet_layer = A.kin + (long long)l * R * Xe;

        // element row e between node rows e (top) and e+1 (bottom): lower-corner
        // sums for node row e (lo) and upper-corner sums for node row e+1 (hi)
        auto element_row = [&](const int e, const DcRow<T>& top, const DcRow<T>& bot, T (&lo)[4], T (&hi)[4]) {
            const T tr = __shfl_down_sync(0xffffffffu, top.w[0], 1);
            const T br = __shfl_down_sync(0xffffffffu, bot.w[0], 1);
            const T top5 = lane == 31 ? top.right : tr;
            const T bot5 = lane == 31 ? bot.right : br;
            Quad<T> sq = zero_quad<T>();
            T hy = T(0), ihy = T(0);
            const bool erow = e >= 0 && e < R;
            if (erow && quad_ok && x0 < Xe) sq = ldg_quad(sheet_layer + (long long)e * Xe + x0);
            if (erow) {
                hy = A.hy[e];
                ihy = A.ihy[e];
            }
            const T u0[5] = {top.w[0], top.w[1], top.w[2], top.w[3], top5};
            const T u1[5] = {bot.w[0], bot.w[1], bot.w[2], bot.w[3], bot5};
            T dx0_lo[4], dx1_lo[4], dx0_hi[4], dx1_hi[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {  // element column x0+k
                const T cx = sq.v[k] * (hy * ihxq.v[k]);
                const T cy = sq.v[k] * (hxq.v[k] * ihy);
                T out[4];
                dc_element(cx * quarter, cy * quarter, (cx + cy) * twelfth, u0[k], u0[k + 1], u1[k], u1[k + 1], out);
                dx0_lo[k] = out[0];
                dx1_lo[k] = out[1];
                dx0_hi[k] = out[2];
                dx1_hi[k] = out[3];
            }
            // the element left of the quad is the left lane's element 3
            const T left_lo = __shfl_up_sync(0xffffffffu, dx1_lo[3], 1);
            const T left_hi = __shfl_up_sync(0xffffffffu, dx1_hi[3], 1);
            lo[0] = (lane >= 1 ? left_lo : T(0)) + dx0_lo[0];
            hi[0] = (lane >= 1 ? left_hi : T(0)) + dx0_hi[0];
#pragma unroll
            for (int k = 1; k < 4; ++k) {
                lo[k] = dx1_lo[k - 1] + dx0_lo[k];
                hi[k] = dx1_hi[k - 1] + dx0_hi[k];
            }
        };

        DcRow<T> cur = dc_load_row<T, STIFF>(P, y0 - 1, R, col + (long long)(y0 - 1) * Xp, quad_ok, edge_ok);
        DcRow<T> nxt = dc_load_row<T, STIFF>(P, y0, R, col + (long long)y0 * Xp, quad_ok, edge_ok);
        T top[4], lo[4], hi[4];
        element_row(y0 - 1, cur, nxt, lo, top);  // upper corners of node row y0
        if (y0 == 0) {
#pragma unroll
            for (int k = 0; k < 4; ++k) top[k] = T(0);
        }
        cur = nxt;
        nxt = dc_load_row<T, STIFF>(P, y0 + 1, R, col + (long long)(y0 + 1) * Xp, quad_ok, edge_ok);
        for (int y = y0; y < y1; ++y) {
            // prefetch the row after next while this row's elements run
            const DcRow<T> ahead = dc_load_row<T, STIFF>(P, y + 2, R, col + (long long)(y + 2) * Xp, quad_ok, edge_ok);
            element_row(y, cur, nxt, lo, hi);
            if (out_lane) {
                const long long n0 = col + (long long)y * Xp;
                const uint8_t mk[4] = {cur.m.x, cur.m.y, cur.m.z, cur.m.w};
                Quad<T> yv;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    T v = top[k] + lo[k];
                    if (mk[k] & kDcVia) v += dc_via_sum<T, MODE>(P, __ldg(P.vias.slot + n0 + k), cur.w[k]);
                    if (!STIFF && !(mk[k] & kDcFree)) v = cur.raw.v[k];
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
                    for (int k = 0; k < 4; ++k) dot = fma(cur.raw.v[k], yv.v[k], dot);
                }
                st_quad(A.y + n0, yv);
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) top[k] = hi[k];
            cur = nxt;
            nxt = ahead;
        }
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

// Post-processing of a DC solution (reference pcb.py:810-848): per element of
// layer l, row y, column x, in flat element order, with corner potentials
// v_{dy dx} read from the flat node-order field `pot`:
//   field (x, y) = -(((v01 + v11) - (v00 + v10)) / (2 h_x), ((v10 + v11) - (v00 + v01)) / (2 h_y)),
//   zero on void elements (sheet conductance sigma t == 0);
//   loss = c_x v^T U_x v + c_y v^T U_y v, c_x = (sigma t h_y) / h_x, c_y = (sigma t h_x) / h_y.
// With U_x = M (x) S the quadratic form is (d0^2 + d0 d1 + d1^2) / 3 over the
// two x-differences d0 = v00 - v01, d1 = v10 - v11 (and the y-differences for
// U_y).  One thread per element; the reads of a row of corners and the writes
// are coalesced.
__global__ void __launch_bounds__(kDcThreads)
    dc_post_kernel(const double* __restrict__ pot, const double* __restrict__ sheet, const double* __restrict__ hx,
                   const double* __restrict__ hy, const int layers, const int R, const int C, const int Xe,
                   double* __restrict__ field, double* __restrict__ loss) {
    const long long E = (long long)layers * R * C;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += stride) {
        const long long line = e / C;  // l * R + y
        const int x = (int)(e - line * C);
        const int l = (int)(line / R);
        const int y = (int)(line - (long long)l * R);
        const long long n00 = ((long long)l * (R + 1) + y) * (C + 1) + x;
        const double v00 = pot[n00], v01 = pot[n00 + 1];
        const double v10 = pot[n00 + C + 1], v11 = pot[n00 + C + 2];
        const double st = sheet[line * Xe + x];
        const double px = hx[x], py = hy[y];
        // The sheet conductance sigma t is built as sigma * t * active with
        // sigma and t required positive (check_dc rejects anything else), so
        // it is zero exactly on the void elements, whose field the reference
        // zeroes by element_active.
        const bool on = st != 0.0;
        const double fx = -(((v01 + v11) - (v00 + v10)) / (2.0 * px));
        const double fy = -(((v10 + v11) - (v00 + v01)) / (2.0 * py));
        field[2 * e] = on ? fx : 0.0;
        field[2 * e + 1] = on ? fy : 0.0;
        const double cx = (st * py) / px, cy = (st * px) / py;
        const double a0 = v00 - v01, a1 = v10 - v11;  // x-differences
        const double b0 = v00 - v10, b1 = v01 - v11;  // y-differences
        const double qx = (a0 * a0 + a0 * a1 + a1 * a1) / 3.0;
        const double qy = (b0 * b0 + b0 * b1 + b1 * b1) / 3.0;
        loss[e] = cx * qx + cy * qy;
    }
}

}  // namespace tb
