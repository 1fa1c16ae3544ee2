// FP32 conduction action for the inner PCG: warp-marching form.
//
// Same operator and the same Haar-basis element action as tb_apply.cuh (see
// there for the mathematics); this kernel moves the data differently so that
// the inner loop needs no block barrier and no shared memory.
//
// A warp owns a strip of element columns and marches along y through a band of
// element rows.  Its 32 lanes are ZW groups of CW = 32 / ZW lanes: lane c of
// group zg holds element column ex = X0 - 1 + c and the SL slabs
// [zg * SL, zg * SL + SL) of it, i.e. node planes zg * SL .. zg * SL + SL.
// Per element row ey the lane
//   * loads its node column of row ey + 1 on its SL + 1 planes (the right-hand
//     column comes from the next lane by a shuffle; the last lane of a group
//     loads it),
//   * takes the (z, x) Haar transform of each slab's face on row ey + 1,
//   * finishes each element of row ey with the y butterfly (this face and the
//     one kept from the previous row), the eigenvalue scaling and the inverse
//     y butterfly; the part on row ey + 1 stays in registers (Haar domain) for
//     the next element row, the part on row ey is added to what the previous
//     element row left there,
//   * maps that face back to its four corners, sums the corners of adjacent
//     slabs in registers, the corners of adjacent columns by a shuffle and the
//     plane shared with the next z group by a shuffle,
//   * writes node row ey (lanes c >= 1; lane 0's column is the halo, written by
//     the warp to the left).
// The kernel serves boards whose Robin terms and fixed nodes lie on the bottom
// and top node planes only (every plain board); their marks are held as two
// scalars per lane.  Other boards use the z-marching tile kernel.
// Loads for row ey + 2 are issued while row ey + 1 is computed.  The band's
// first element row (Y0 - 1) is the y halo and writes nothing.  Summation
// orders are fixed per node, so the result is deterministic and independent
// of the warp / band decomposition.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "tb_apply.cuh"
#include "tb_reduce.cuh"
#include "tb_types.h"

namespace tb {

constexpr int kWarpMaxSlabs = 32;
constexpr int kWarpBlockWarps = 4;

struct WarpApplyParams {
    const float* x;          // node field (S+1, R+1, Xp)
    float* y;                // output node field
    const float* kin;        // element fields (S, R, Xe)
    const float* kz;
    const float* rf;         // Robin total (>= 0) on free nodes, -1 on fixed ones
    const float* hx;         // (C)
    const float* ihx;
    const float* hy;         // (R)
    const float* ihy;
    double* partials;
    unsigned int* counter;
    SolveCtl* ctl;
    KernelClock* clock;
    float tz[kWarpMaxSlabs];  // h_z / 16 per slab
    float iz[kWarpMaxSlabs];  // 1 / (16 h_z) per slab
    int special_lo;          // the bottom plane holds a Robin term or a fixed node
    int special_hi;          // the top plane (z = S) does
    long long pstride;       // (R+1) Xp
    long long sstride;       // R Xe
    int S, R, C, Xp, Xe;
    int ncolw;               // warp strips across the columns
    int band;                // node rows per warp
    int nband;               // bands across the rows
};

template <int ZW, int SL, int EPI>
__global__ void __launch_bounds__(32 * kWarpBlockWarps, 4) warp_apply_kernel(const __grid_constant__ WarpApplyParams P) {
    constexpr int CW = 32 / ZW;  // lanes (element columns) per z group
    constexpr int NP = SL + 1;   // node planes per lane
    constexpr unsigned FULL = 0xffffffffu;
    using Acc = Acc32;
    __shared__ __align__(16) unsigned char red_scratch_raw[sizeof(Acc) * 32];
    Acc* const red_scratch = reinterpret_cast<Acc*>(red_scratch_raw);

    pdl_trigger();
    const int lane = threadIdx.x & 31;
    const int zg = lane / CW, c = lane % CW;
    const int unit = blockIdx.x * kWarpBlockWarps + (threadIdx.x >> 5);
    const bool unit_ok = unit < P.ncolw * P.nband;
    const int bx = unit % P.ncolw, by = unit / P.ncolw;
    const int X0 = bx * (CW - 1);
    const int Y0 = by * P.band;
    const int ex = X0 - 1 + c;  // this lane's element column = its node column
    const int S = P.S, R = P.R, Xp = P.Xp;
    const int z0 = zg * SL;
    const bool node_col_ok = unit_ok && ex >= 0 && ex < Xp;
    const bool right_col_ok = unit_ok && ex + 1 >= 0 && ex + 1 < Xp;
    const bool elem_col_ok = unit_ok && ex >= 0 && ex < P.C;
    const float third = 1.0f / 3.0f;
    const float hx = elem_col_ok ? P.hx[ex] : 0.0f;
    const float ihx = elem_col_ok ? P.ihx[ex] : 0.0f;
    bool plane_ok[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) plane_ok[k] = (z0 + k) <= S;
    // planes of this lane that carry Robin / fixed marks: its k = 0 if it is
    // the bottom plane, its k = khi if that is the top plane
    const bool has_lo = P.special_lo && zg == 0;
    const int khi = S - z0;
    const bool has_hi = P.special_hi && khi >= 0 && khi <= SL && !(khi == 0 && zg > 0);

    pdl_wait();
    if (EPI == EPI_DOT && P.ctl->state != ST_RUNNING) return;
    if (EPI == EPI_DOT && P.clock != nullptr && threadIdx.x == 0) atomicMin(&P.clock->first, global_ns());

    // Row loads: own column on the lane's planes (and the Robin/fixed marks on
    // special planes); the last lane of a group also loads the column to its right.
    float xa[NP], xra[NP];
    float ra_lo, ra_hi, rra_lo, rra_hi;  // marks of the bottom / top plane, own and right column
    float kina[SL], kza[SL];
    // Offsets inside a field are 32-bit (the host allows this kernel only for
    // fields below 2^31 elements), taken from per-lane base pointers.
    const int pstride = (int)P.pstride, sstride = (int)P.sstride;
    const int exc = ex < 0 ? 0 : ex;  // a valid column for the base pointers
    const float* const xbase = P.x + (long long)z0 * P.pstride + exc;
    const float* const rbase = P.rf + exc;
    const float* const kbase = P.kin + (long long)z0 * P.sstride + exc;
    const float* const zbase = P.kz + (long long)z0 * P.sstride + exc;
    auto load_row = [&](const int yy) {
        const bool row_ok = yy >= 0 && yy <= R;
        const int rowoff = yy * Xp;
        const bool edge = c == CW - 1;
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            const int off = k * pstride + rowoff;
            const bool ok = row_ok && plane_ok[k] && node_col_ok;
            xa[k] = ok ? __ldg(xbase + off) : 0.0f;
            const bool rok = row_ok && plane_ok[k] && right_col_ok && edge;
            xra[k] = rok ? __ldg(xbase + off + 1) : 0.0f;
        }
        const int hi = S * pstride + rowoff;
        ra_lo = (has_lo && row_ok && node_col_ok) ? __ldg(rbase + rowoff) : 0.0f;
        ra_hi = (has_hi && row_ok && node_col_ok) ? __ldg(rbase + hi) : 0.0f;
        rra_lo = (has_lo && row_ok && right_col_ok && edge) ? __ldg(rbase + rowoff + 1) : 0.0f;
        rra_hi = (has_hi && row_ok && right_col_ok && edge) ? __ldg(rbase + hi + 1) : 0.0f;
    };
    auto load_coef = [&](const int ey) {
        const bool ok = elem_col_ok && ey >= 0 && ey < R;
        const int off = ey * P.Xe;
#pragma unroll
        for (int s = 0; s < SL; ++s) {
            const bool sok = ok && (z0 + s) < S;
            kina[s] = sok ? __ldg(kbase + s * sstride + off) : 0.0f;
            kza[s] = sok ? __ldg(zbase + s * sstride + off) : 0.0f;
        }
    };

    // State carried from one element row to the next.
    float Al[NP], Dl[NP];   // x butterflies (sum, difference with the right column) of the lower face
    float xl[NP];           // node values of the row being written
    float rl_lo, rl_hi;     // its bottom / top plane marks
    float Up[SL][4];        // Haar-domain contributions to the upper face, per slab
#pragma unroll
    for (int s = 0; s < SL; ++s)
#pragma unroll
        for (int m = 0; m < 4; ++m) Up[s][m] = 0.0f;

    // Face of row yy in registers: fetch the right column, mask fixed nodes
    // (x * free: they do not enter free rows), butterfly.
    auto face = [&](float (&A)[NP], float (&D)[NP], float (&xo)[NP], float& ro_lo, float& ro_hi) {
        float rlo = __shfl_down_sync(FULL, ra_lo, 1, CW);
        float rhi = __shfl_down_sync(FULL, ra_hi, 1, CW);
        if (c == CW - 1) {
            rlo = rra_lo;
            rhi = rra_hi;
        }
        ro_lo = ra_lo;
        ro_hi = ra_hi;
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            float xv = xa[k];
            float xr = __shfl_down_sync(FULL, xv, 1, CW);
            if (c == CW - 1) xr = xra[k];
            xo[k] = xv;
            if (k == 0 && has_lo) {
                xv = (ra_lo < 0.0f) ? 0.0f : xv;
                xr = (rlo < 0.0f) ? 0.0f : xr;
            }
            if (k == khi && has_hi) {
                xv = (ra_hi < 0.0f) ? 0.0f : xv;
                xr = (rhi < 0.0f) ? 0.0f : xr;
            }
            A[k] = xv + xr;
            D[k] = xv - xr;
        }
    };

    const int ey_first = Y0 - 1;
    const int ey_last = min(Y0 + P.band - 1, R);  // element row R is a void row whose lower face is node row R
    load_row(ey_first);
    face(Al, Dl, xl, rl_lo, rl_hi);
    load_row(ey_first + 1);
    load_coef(ey_first);

    float dot = 0.0f;
    for (int ey = ey_first; ey <= ey_last; ++ey) {
        float Au[NP], Du[NP], xu[NP], ru_lo, ru_hi;
        face(Au, Du, xu, ru_lo, ru_hi);
        float kin_c[SL], kz_c[SL];
#pragma unroll
        for (int s = 0; s < SL; ++s) {
            kin_c[s] = kina[s];
            kz_c[s] = kza[s];
        }
        if (ey + 1 <= ey_last) {  // next row's loads fly while this row is computed
            load_row(ey + 2);
            load_coef(ey + 1);
        }
        const bool erow_ok = ey >= 0 && ey < R;
        float qx = 0.f, qy = 0.f, qxy = 0.f, qz = 0.f;
        if (erow_ok && elem_col_ok) {
            const float hy = P.hy[ey], ihy = P.ihy[ey];
            qx = hy * ihx;
            qy = hx * ihy;
            qxy = (qx + qy) * third;
            qz = hx * hy;
        }
        float out[NP], outr[NP];
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            out[k] = 0.0f;
            outr[k] = 0.0f;
        }
#pragma unroll
        for (int s = 0; s < SL; ++s) {
            // (z, x) modes of the lower (row ey) and upper (row ey+1) faces of slab s
            const float lSS = Al[s] + Al[s + 1], lDS = Al[s] - Al[s + 1];
            const float lSD = Dl[s] + Dl[s + 1], lDD = Dl[s] - Dl[s + 1];
            const float uSS = Au[s] + Au[s + 1], uDS = Au[s] - Au[s + 1];
            const float uSD = Du[s] + Du[s + 1], uDD = Du[s] - Du[s + 1];
            const float tz = P.tz[z0 + s < S ? z0 + s : 0], iz = P.iz[z0 + s < S ? z0 + s : 0];
            const float tk = kin_c[s] * tz;
            const float ax = tk * qx, ay = tk * qy, cxy = tk * qxy;
            const float az = (kz_c[s] * iz) * qz;
            const float az3 = az * third;
            const float cxz = fmaf(ax, third, az3);
            const float cyz = fmaf(ay, third, az3);
            const float cxyz = (cxy + az3) * third;
            // y butterfly and eigenvalue scaling; pattern (z, y, x)
            const float wSDS = ay * (lSS - uSS);
            const float wDSS = az * (lDS + uDS), wDDS = cyz * (lDS - uDS);
            const float wSSD = ax * (lSD + uSD), wSDD = cxy * (lSD - uSD);
            const float wDSD = cxz * (lDD + uDD), wDDD = cxyz * (lDD - uDD);
            // lower face (row ey) = what the previous row left + this row's part
            const float tSS = Up[s][0] + wSDS;
            const float tDS = Up[s][1] + (wDSS + wDDS);
            const float tSD = Up[s][2] + (wSSD + wSDD);
            const float tDD = Up[s][3] + (wDSD + wDDD);
            Up[s][0] = -wSDS;
            Up[s][1] = wDSS - wDDS;
            Up[s][2] = wSSD - wSDD;
            Up[s][3] = wDSD - wDDD;
            // corners (dz, dx) of the face on row ey
            const float Pp = tSS + tDS, Qq = tSS - tDS, Rr = tSD + tDD, Ww = tSD - tDD;
            out[s] += Pp + Rr;       // (z, x)
            outr[s] += Pp - Rr;      // (z, x + 1)
            out[s + 1] += Qq + Ww;   // (z + 1, x)
            outr[s + 1] += Qq - Ww;  // (z + 1, x + 1)
        }
        // the top plane of this group is the bottom plane of the next group
        {
            const float up0 = __shfl_down_sync(FULL, out[0], CW);
            const float upr0 = __shfl_down_sync(FULL, outr[0], CW);
            if (zg < ZW - 1) {
                out[SL] += up0;
                outr[SL] += upr0;
            }
        }
        // corners of the column to the left
#pragma unroll
        for (int k = 0; k < NP; ++k) out[k] += __shfl_up_sync(FULL, outr[k], 1, CW);

        if (ey >= Y0 && c >= 1 && node_col_ok) {
            float* const ybase = P.y + (long long)z0 * P.pstride + (long long)ey * Xp + ex;
#pragma unroll
            for (int k = 0; k < NP; ++k) {
                if (!plane_ok[k] || (k == 0 && zg > 0)) continue;  // a group's bottom plane belongs to the group below
                float v = out[k];
                if (k == 0 && has_lo) v = (rl_lo < 0.0f) ? xl[k] : v + rl_lo * xl[k];
                if (k == khi && has_hi) v = (rl_hi < 0.0f) ? xl[k] : v + rl_hi * xl[k];
                if (EPI == EPI_DOT) dot = fmaf(xl[k], v, dot);
                ybase[k * pstride] = v;
            }
        }
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            Al[k] = Au[k];
            Dl[k] = Du[k];
            xl[k] = xu[k];
        }
        rl_lo = ru_lo;
        rl_hi = ru_hi;
    }

    if (EPI == EPI_STORE) return;
    Acc accs[1];
    accs[0].s = dot;
    block_merge<1>(accs, red_scratch);
    const int nblocks = gridDim.x;
    if (threadIdx.x == 0) acc_store(P.partials + (size_t)blockIdx.x * 4, accs[0]);
    if (!last_block(P.counter)) return;
    Acc tot[1];
    grid_merge<1>(P.partials, nblocks, 4, tot, red_scratch, P.counter);
    if (threadIdx.x == 0) {
        SolveCtl* ctl = P.ctl;
        const double pq = tot[0].value();
        ctl->pq = pq;
        ctl->applications += 1;
        if (!(isfinite(pq) && pq > 0.0)) {
            ctl->state = ST_NOT_SPD;
        } else {
            ctl->alpha = ctl->rz / pq;
        }
        if (P.clock != nullptr) {
            KernelClock* clk = P.clock;
            const unsigned long long first = atomicExch(&clk->first, ~0ULL);
            clk->total_ns += global_ns() - first;
            clk->count += 1;
        }
    }
}

}  // namespace tb
