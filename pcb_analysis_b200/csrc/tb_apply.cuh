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
// it stages the node tile in shared memory (triple buffered, loads for the next
// plane issued one plane ahead), takes the 2D (y,x) Haar transform of each
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

#include <cuda_runtime.h>
#include <stdint.h>

#include "tb_reduce.cuh"
#include "tb_types.h"

namespace tb {

constexpr int kApplyThreads = 256;
constexpr int kOutX = 60;   // output node columns per block
constexpr int kOutY = 15;   // output node rows per block
constexpr int kTileW = 68;  // node tile width: node columns X0-4 .. X0+63
constexpr int kTileH = 17;  // node tile height: node rows Y0-1 .. Y0+15
constexpr int kTileQ = 17;  // quads (4 nodes) per tile row
constexpr int kTileQuads = kTileH * kTileQ;
constexpr int kTileSize = kTileH * kTileW;
constexpr int kXchW = 64;

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

// Dynamic shared memory of apply_kernel<T>.
template <typename T>
constexpr size_t apply_smem_bytes() {
    return (size_t)(2 * 3 * kTileSize + 16 * kXchW) * sizeof(T);
}

template <typename T, int MODE, int EPI>
__global__ void __launch_bounds__(kApplyThreads) apply_kernel(const ApplyParams<T> P) {
    using Acc = typename AccOf<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* const tile = reinterpret_cast<T*>(smem_raw);  // [3][17][68] node values
    T* const rft = tile + 3 * kTileSize;              // [3][17][68] Robin / fixed marks
    T* const xch = rft + 3 * kTileSize;               // [16][64] y-exchange
    __shared__ __align__(16) unsigned char red_scratch_raw[sizeof(Acc) * (2 * 32)];
    Acc* const red_scratch = reinterpret_cast<Acc*>(red_scratch_raw);
    __shared__ double max_scratch[32];

    if (EPI == EPI_DOT && P.ctl->state != ST_RUNNING) return;  // whole grid skips

    const int tid = threadIdx.x;
    const int g = tid & 15;   // column group: element columns exb .. exb+3
    const int j = tid >> 4;   // element row of this thread in the tile
    const int X0 = blockIdx.x * kOutX;
    const int Y0 = blockIdx.y * kOutY;
    const int S = P.S, R = P.R, C = P.C, Xp = P.Xp;
    const int ey = Y0 - 1 + j;
    const int exb = X0 - 4 + 4 * g;
    const bool erow_ok = (ey >= 0) && (ey < R);
    const bool equad_ok = erow_ok && (exb >= 0) && (exb < P.Xe);

    // Per element column geometry: a_x/16 = k_in (h_z/16) (h_y/h_x) etc.
    T qx[4], qy[4], qz[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int ex = exb + k;
        if (erow_ok && ex >= 0 && ex < C) {
            const T hx = P.hx[ex], ihx = P.ihx[ex], hy = P.hy[ey], ihy = P.ihy[ey];
            qx[k] = hy * ihx;
            qy[k] = hx * ihy;
            qz[k] = hx * hy;
        } else {
            qx[k] = T(0);
            qy[k] = T(0);
            qz[k] = T(0);
        }
    }

    // Tile quads loaded by this thread: q = tid and tid + 256.
    const int q0 = tid, q1 = tid + kApplyThreads;
    const bool has_q1 = q1 < kTileQuads;
    const int tr0 = q0 / kTileQ, tc0 = (q0 % kTileQ) * 4;
    const int tr1 = q1 / kTileQ, tc1 = (q1 % kTileQ) * 4;
    const int nr0 = Y0 - 1 + tr0, nc0 = X0 - 4 + tc0;
    const int nr1 = Y0 - 1 + tr1, nc1 = X0 - 4 + tc1;
    const bool ok0 = (nr0 >= 0) && (nr0 <= R) && (nc0 >= 0) && (nc0 < Xp);
    const bool ok1 = has_q1 && (nr1 >= 0) && (nr1 <= R) && (nc1 >= 0) && (nc1 < Xp);
    const long long off0 = (long long)nr0 * Xp + nc0;
    const long long off1 = (long long)nr1 * Xp + nc1;

    auto plane_special = [&](int p) -> bool {
        return (MODE == MODE_OPERATOR) && (P.plane_flags[p] != 0);
    };

    Quad<T> xa = zero_quad<T>(), xb = zero_quad<T>(), ra = zero_quad<T>(), rb = zero_quad<T>();
    auto load_plane = [&](int p) {
        const long long base = (long long)p * P.pstride;
        xa = ok0 ? ldg_quad(P.x + base + off0) : zero_quad<T>();
        xb = ok1 ? ldg_quad(P.x + base + off1) : zero_quad<T>();
        if (plane_special(p)) {
            ra = ok0 ? ldg_quad(P.rf + base + off0) : zero_quad<T>();
            rb = ok1 ? ldg_quad(P.rf + base + off1) : zero_quad<T>();
        }
    };
    Quad<T> kin_n = zero_quad<T>(), kz_n = zero_quad<T>();
    const long long eoff = (long long)ey * P.Xe + exb;
    auto load_slab = [&](int s) {
        if (equad_ok) {
            kin_n = ldg_quad(P.kin + (long long)s * P.sstride + eoff);
            kz_n = ldg_quad(P.kz + (long long)s * P.sstride + eoff);
        }
    };

    load_plane(0);
    load_slab(0);

    T Fl[4][4];  // face transform of the plane below (lower face of the current slab)
    T Up[4][4];  // upper-face contributions (Haar domain) waiting for the next plane
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            Fl[k][m] = T(0);
            Up[k][m] = T(0);
        }

    Acc acc_dot;
    double rmax = 0.0;

    // Sum one plane's Haar-domain contributions into nodes and write them.
    auto emit_plane = [&](const int pl, T (&tot)[4][4]) {
        const int tb = pl % 3;
        T R0[5], R1[5];
        {
            T c00[4], c01[4], c10[4], c11[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const T A = tot[k][0] + tot[k][1];
                const T B = tot[k][0] - tot[k][1];
                const T Cc = tot[k][2] + tot[k][3];
                const T D = tot[k][2] - tot[k][3];
                c00[k] = A + Cc;
                c01[k] = A - Cc;
                c10[k] = B + D;
                c11[k] = B - D;
            }
            R0[0] = c00[0];
            R1[0] = c10[0];
#pragma unroll
            for (int k = 1; k < 4; ++k) {
                R0[k] = c01[k - 1] + c00[k];
                R1[k] = c11[k - 1] + c10[k];
            }
            R0[4] = c01[3];
            R1[4] = c11[3];
        }
        const T left0 = __shfl_up_sync(0xffffffffu, R0[4], 1);
        const T left1 = __shfl_up_sync(0xffffffffu, R1[4], 1);
        R0[0] += left0;
        R1[0] += left1;
        {
            Quad<T> w = {{R0[0], R0[1], R0[2], R0[3]}};
            st_quad(xch + j * kXchW + 4 * g, w);
        }
        __syncthreads();
        if (j < kOutY && g >= 1) {
            const int yr = Y0 + j;
            const int xc = exb;  // = X0 + 4 (g - 1)
            if (yr <= R && xc < Xp) {
                const Quad<T> other = lds_quad(xch + (j + 1) * kXchW + 4 * g);
                const Quad<T> xo = lds_quad(tile + tb * kTileSize + (j + 1) * kTileW + 4 * g);
                Quad<T> out;
                if (plane_special(pl)) {
                    const Quad<T> rr = lds_quad(rft + tb * kTileSize + (j + 1) * kTileW + 4 * g);
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const T acc = R1[k] + other.v[k];
                        out.v[k] = (rr.v[k] < T(0)) ? xo.v[k] : acc + rr.v[k] * xo.v[k];
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < 4; ++k) out.v[k] = R1[k] + other.v[k];
                }
                const long long node = (long long)pl * P.pstride + (long long)yr * Xp + xc;
                if (EPI == EPI_RESIDUAL) {
                    const Quad<T> bq = ldg_quad(P.b + node);
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        out.v[k] = bq.v[k] - out.v[k];
                        acc_dot.add_product(out.v[k], out.v[k]);
                        rmax = fmax(rmax, fabs((double)out.v[k]));
                    }
                } else if (EPI == EPI_DOT) {
#pragma unroll
                    for (int k = 0; k < 4; ++k) acc_dot.add_product(xo.v[k], out.v[k]);
                }
                st_quad(P.y + node, out);
            }
        }
    };

    for (int p = 0; p <= S; ++p) {
        const int buf = p % 3;
        const bool special = plane_special(p);
        // Stage plane p (loaded during the previous step).
        st_quad(tile + buf * kTileSize + tr0 * kTileW + tc0, xa);
        if (has_q1) st_quad(tile + buf * kTileSize + tr1 * kTileW + tc1, xb);
        if (special) {
            st_quad(rft + buf * kTileSize + tr0 * kTileW + tc0, ra);
            if (has_q1) st_quad(rft + buf * kTileSize + tr1 * kTileW + tc1, rb);
        }
        const Quad<T> kin_c = kin_n, kz_c = kz_n;  // slab p-1
        if (p + 1 <= S) load_plane(p + 1);
        if (p >= 1 && p < S) load_slab(p);
        __syncthreads();

        // Face transform of plane p for the four elements.
        T F[4][4];
        {
            const T* r0 = tile + buf * kTileSize + j * kTileW + 4 * g;
            const T* r1 = r0 + kTileW;
            const Quad<T> a4 = lds_quad(r0), c4 = lds_quad(r1);
            T a[5] = {a4.v[0], a4.v[1], a4.v[2], a4.v[3], r0[4]};
            T c[5] = {c4.v[0], c4.v[1], c4.v[2], c4.v[3], r1[4]};
            if (special) {  // x * free: fixed nodes do not enter free rows
                const T* f0 = rft + buf * kTileSize + j * kTileW + 4 * g;
                const T* f1 = f0 + kTileW;
                const Quad<T> fa = lds_quad(f0), fc = lds_quad(f1);
                const T fav[5] = {fa.v[0], fa.v[1], fa.v[2], fa.v[3], f0[4]};
                const T fcv[5] = {fc.v[0], fc.v[1], fc.v[2], fc.v[3], f1[4]};
#pragma unroll
                for (int k = 0; k < 5; ++k) {
                    a[k] = (fav[k] < T(0)) ? T(0) : a[k];
                    c[k] = (fcv[k] < T(0)) ? T(0) : c[k];
                }
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const T A0 = a[k] + a[k + 1], D0 = a[k] - a[k + 1];
                const T A1 = c[k] + c[k + 1], D1 = c[k] - c[k + 1];
                F[k][0] = A0 + A1;  // SS
                F[k][1] = A0 - A1;  // DS (y difference)
                F[k][2] = D0 + D1;  // SD (x difference)
                F[k][3] = D0 - D1;  // DD
            }
        }

        if (p >= 1) {
            const int s = p - 1;
            const T tz = P.gzt[s], iz = P.gzi[s];
            const T third = T(1) / T(3), ninth = T(1) / T(9);
            T tot[4][4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const T tk = kin_c.v[k] * tz;
                const T ax = tk * qx[k];
                const T ay = tk * qy[k];
                const T az = (kz_c.v[k] * iz) * qz[k];
                const T sxy = ax + ay;
                const T cxy = sxy * third;
                const T cxz = (ax + az) * third;
                const T cyz = (ay + az) * third;
                const T cxyz = (sxy + az) * ninth;
                // z butterfly: pattern (z, face) with faces SS, DS, SD, DD
                const T sDS = Fl[k][1] + F[k][1], sSD = Fl[k][2] + F[k][2], sDD = Fl[k][3] + F[k][3];
                const T dSS = Fl[k][0] - F[k][0], dDS = Fl[k][1] - F[k][1];
                const T dSD = Fl[k][2] - F[k][2], dDD = Fl[k][3] - F[k][3];
                const T wSDS = ay * sDS, wSSD = ax * sSD, wSDD = cxy * sDD;
                const T wDSS = az * dSS, wDDS = cyz * dDS, wDSD = cxz * dSD, wDDD = cxyz * dDD;
                // lower face (plane p-1) and upper face (plane p) contributions
                tot[k][0] = Up[k][0] + wDSS;
                tot[k][1] = Up[k][1] + (wSDS + wDDS);
                tot[k][2] = Up[k][2] + (wSSD + wDSD);
                tot[k][3] = Up[k][3] + (wSDD + wDDD);
                Up[k][0] = -wDSS;
                Up[k][1] = wSDS - wDDS;
                Up[k][2] = wSSD - wDSD;
                Up[k][3] = wSDD - wDDD;
            }
            emit_plane(p - 1, tot);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int m = 0; m < 4; ++m) Fl[k][m] = F[k][m];
    }
    __syncthreads();  // the exchange buffer of plane S-1 is still being read
    emit_plane(S, Up);

    if (EPI == EPI_STORE) return;

    // Block partials, then the last block finishes the scalar.
    Acc accs[1] = {acc_dot};
    block_merge<1>(accs, red_scratch);
    double bmax = 0.0;
    if (EPI == EPI_RESIDUAL) bmax = block_max(rmax, max_scratch);
    const int nblocks = gridDim.x * gridDim.y;
    const int bid = blockIdx.y * gridDim.x + blockIdx.x;
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
        if (EPI == EPI_DOT) {
            const double pq = tot[0].value();
            ctl->pq = pq;
            ctl->applications += 1;
            if (!(isfinite(pq) && pq > 0.0)) {
                ctl->state = ST_NOT_SPD;
            } else {
                ctl->alpha = ctl->rz / pq;
            }
        } else {
            ctl->res2 = tot[0].value();
            ctl->peak = gmax;
        }
    }
}

}  // namespace tb
