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
// the conductivity tiles of the slab below in shared memory with cp.async
// (four stages, two planes in flight ahead of the one in use), takes the 2D (y,x) Haar transform of each
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

constexpr int kStages = 4;  // plane p computes, p-1 is emitted, p+1 and p+2 are in flight
static_assert((kStages & (kStages - 1)) == 0, "stage index uses a mask");

// Shared memory of one pipeline stage: node tile, Robin/fixed tile, and the
// k_in / k_z tiles of the slab below the plane.
template <typename T, int ROWS>
struct StageLayout {
    static constexpr int x_off = 0;
    static constexpr int rf_off = TileShape<ROWS>::tile_size;
    static constexpr int kin_off = 2 * TileShape<ROWS>::tile_size;
    static constexpr int kz_off = kin_off + ROWS * 64;
    static constexpr int size = kz_off + ROWS * 64;  // in T
};

// Blocks per SM the FP32 kernels are compiled for (registers capped to fit):
// 5 x 128, 3 x 256 or 1 x 512 threads, within the shared memory of their
// pipeline stages.  The FP64 kernels run once per outer step and are not capped.
template <typename T, int ROWS>
struct ApplyOccupancy {
    static constexpr int min_blocks = sizeof(T) == 4 ? (ROWS == 8 ? 5 : (ROWS == 16 ? 3 : 1)) : 1;
};

// Dynamic shared memory of apply_kernel<T, ..., ROWS> for S slabs.
template <typename T, int ROWS>
inline size_t apply_smem_bytes(int S) {
    const size_t stages = (size_t)kStages * StageLayout<T, ROWS>::size * sizeof(T);
    const size_t xch = (size_t)ROWS * kXchW * sizeof(T);
    const size_t tables = 2 * (size_t)S * sizeof(T) + (size_t)(S + 1) * sizeof(int);
    return (stages + xch + tables + 15) / 16 * 16;
}

// The work of one tile (bx, by): stage its planes, run the element actions,
// write its output nodes.  Adds this thread's share of the tile's reduction
// (p.Ap, or ||b - Ax||^2 and max |b - Ax|) to `dot` and `rmax`.  Ends with a
// barrier, so a block may call it for several tiles in a row.
//
// With `gate`, the tile first waits for the preceding launch (programmatic
// dependent launch) after loading the static tables and per-thread offsets,
// then returns false without touching anything when an inner-product launch
// finds its solve no longer running (a value uniform across the grid).
template <typename T, int MODE, int EPI, int ROWS>
__device__ __forceinline__ bool apply_tile(const ApplyParams<T>& P, const int bx, const int by,
                                           unsigned char* smem_raw, T& dot, double& rmax, const bool gate) {
    constexpr bool DOT = EPI == EPI_DOT;
    using Sh = TileShape<ROWS>;
    using St = StageLayout<T, ROWS>;
    T* const stage = reinterpret_cast<T*>(smem_raw);        // [kStages][St::size]
    T* const xch = stage + kStages * St::size;               // [ROWS][64] y-exchange
    T* const s_tz = xch + ROWS * kXchW;                      // [S] h_z / 16
    T* const s_iz = s_tz + P.S;                              // [S] 1 / (16 h_z)
    int* const s_flag = reinterpret_cast<int*>(s_iz + P.S);  // [S+1] plane holds Robin / fixed nodes
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

    if (gate) {
        pdl_wait();  // the predecessor's writes (the direction, the scalars) are visible from here on
        if (DOT && P.ctl->state != ST_RUNNING) return false;  // whole grid skips
        if (EPI != EPI_STORE && P.clock != nullptr && threadIdx.x == 0) atomicMin(&P.clock->first, global_ns());
    }
    __syncthreads();  // tables ready

    // Asynchronous staging of plane p (and of slab p-1 below it) into stage p % kStages.
    auto issue = [&](const int p) {
        T* const st = stage + (p & (kStages - 1)) * St::size;
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
        if (p >= 1) {
            const long long kb = (long long)(p - 1) * P.sstride;
            const int sk = sface - 4 * j;  // = j * 64 + 4 g
            cp_async_quad(st + St::kin_off + sk, P.kin + kb + gk, equad_ok);
            cp_async_quad(st + St::kz_off + sk, P.kz + kb + gk, equad_ok);
        }
    };

    T Fl[4][4];  // face transform of the plane below (lower face of the current slab)
    T Up[4][4];  // upper-face contributions (Haar domain) waiting for the next plane
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            Fl[k][m] = T(0);
            Up[k][m] = T(0);
        }


    // Sum one plane's Haar-domain contributions into nodes and write them.
    auto emit_plane = [&](const int pl, T (&tot)[4][4]) {
        const T* const st = stage + (pl & (kStages - 1)) * St::size;
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
        if (out_ok) {
            {
                const Quad<T> other = lds_quad(xch + (j + 1) * kXchW + 4 * g);
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
                const long long node = (long long)pl * P.pstride + gout;
                if (EPI == EPI_RESIDUAL) {
                    const Quad<T> bq = ldg_quad(P.b + node);
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        out.v[k] = bq.v[k] - out.v[k];
                        dot = fma(out.v[k], out.v[k], dot);
                        rmax = fmax(rmax, fabs((double)out.v[k]));
                    }
                } else if (DOT) {
#pragma unroll
                    for (int k = 0; k < 4; ++k) dot = fma(xo.v[k], out.v[k], dot);
                }
                st_quad(P.y + node, out);
            }
        }
    };

    issue(0);
    cp_async_commit();
    if (S >= 1) issue(1);
    cp_async_commit();

    for (int p = 0; p <= S; ++p) {
        cp_async_wait<1>();  // this thread's copies of plane p have landed
        __syncthreads();     // everybody's have, and every thread is done with plane p-2
        if (p + 2 <= S) issue(p + 2);
        cp_async_commit();

        const T* const st = stage + (p & (kStages - 1)) * St::size;
        const bool special = s_flag[p] != 0;
        // Face transform of plane p for the four elements.  The fifth column
        // comes from the next lane's first one by a shuffle; the last group of
        // a row reads it from shared memory.
        T F[4][4];
        {
            const T* r0 = st + St::x_off + sface;
            const T* r1 = r0 + kTileW;
            Quad<T> a4 = lds_quad(r0), c4 = lds_quad(r1);
            if (special) {  // x * free: fixed nodes do not enter free rows
                const Quad<T> fa = lds_quad(st + St::rf_off + sface);
                const Quad<T> fc = lds_quad(st + St::rf_off + sface + kTileW);
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    a4.v[k] = (fa.v[k] < T(0)) ? T(0) : a4.v[k];
                    c4.v[k] = (fc.v[k] < T(0)) ? T(0) : c4.v[k];
                }
            }
            T a5 = __shfl_down_sync(0xffffffffu, a4.v[0], 1);
            T c5 = __shfl_down_sync(0xffffffffu, c4.v[0], 1);
            if (g == 15) {
                a5 = r0[4];
                c5 = r1[4];
                if (special) {
                    a5 = (st[St::rf_off + j * kTileW + 64] < T(0)) ? T(0) : a5;
                    c5 = (st[St::rf_off + (j + 1) * kTileW + 64] < T(0)) ? T(0) : c5;
                }
            }
            const T a[5] = {a4.v[0], a4.v[1], a4.v[2], a4.v[3], a5};
            const T c[5] = {c4.v[0], c4.v[1], c4.v[2], c4.v[3], c5};
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
            const T tz = s_tz[s], iz = s_iz[s];
            const Quad<T> kin_c = lds_quad(st + St::kin_off + sface - 4 * j);
            const Quad<T> kz_c = lds_quad(st + St::kz_off + sface - 4 * j);
            T tot[4][4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const T tk = kin_c.v[k] * tz;
                const T ax = tk * qx[k];
                const T ay = tk * qy[k];
                const T cxy = tk * qxy[k];
                const T az = (kz_c.v[k] * iz) * qz[k];
                const T az3 = az * third;
                const T cxz = fma(ax, third, az3);
                const T cyz = fma(ay, third, az3);
                const T cxyz = (cxy + az3) * third;
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
    cp_async_wait<0>();
    __syncthreads();  // the exchange buffer of plane S-1 is still being read
    emit_plane(S, Up);
    __syncthreads();  // shared memory is free for the next tile
    return true;
}

template <typename T, int MODE, int EPI, int ROWS>
__global__ void __launch_bounds__(16 * ROWS, ApplyOccupancy<T, ROWS>::min_blocks) apply_kernel(const ApplyParams<T> P) {
    constexpr bool DOT = EPI == EPI_DOT;
    using Acc = typename AccOf<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(16) unsigned char red_scratch_raw[sizeof(Acc) * 32];
    Acc* const red_scratch = reinterpret_cast<Acc*>(red_scratch_raw);
    __shared__ double max_scratch[32];

    pdl_trigger();
    T dot = T(0);  // per-thread sum, merged with compensation across the grid
    double rmax = 0.0;
    if (!apply_tile<T, MODE, EPI, ROWS>(P, blockIdx.x, blockIdx.y, smem_raw, dot, rmax, true)) return;

    if (EPI == EPI_STORE) return;

    // Block partials, then the last block finishes the scalar.
    Acc accs[1];
    accs[0].s = dot;
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
        if (DOT) {
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
        if (P.clock != nullptr) {
            KernelClock* clk = P.clock;
            const unsigned long long first = atomicExch(&clk->first, ~0ULL);
            clk->total_ns += global_ns() - first;
            clk->count += 1;
        }
    }
}

}  // namespace tb
