// Problem preparation and post-processing on the device.
//
// The reference prepares a conduction problem on the host (NumPy,
// src/thermal/matrix_free_mpir_fem/operator.py:86-128,374-525 and
// boundaries.py:82-183; C++ cpp/src/thermal/thermal_system.cpp:146-250,
// 411-511): node masks, the lumped Robin conductance and load of every
// convection boundary, the nodal heat load, the right-hand side for a
// reference temperature, and after the solve the unconstrained residual, the
// heat removed per boundary and -k grad T at element centres.  Every one of
// those arrays is elementwise in the node or element grid, so each node (or
// element) here is one thread that adds the same terms in the same order as
// the reference: the arrays carry the reference's bits.  Explicit _rn
// intrinsics keep the compiler from contracting a product and a sum into an
// FMA, which would change the rounding.
//
// Flat arrays in this file are in the reference's node order
// (z (R+1) + y)(C+1) + x and element order (z R + y) C + x; the padded
// solver fields (rows of Xp nodes, Xe elements) are named as such.
//
// The scalar budgets (sum of the loads, heat through the fixed nodes, heat
// removed by each boundary, stored heat) are sums over the grid.  The
// reference forms them with NumPy's pairwise summation; here they are
// compensated sums (Knuth's TwoSum and an exact FMA product error, the
// accumulation of Ogita, Rump and Oishi, SIAM J. Sci. Comput. 26(6), 2005),
// reduced in a fixed order: they agree with the reference within the
// reference's own rounding error and are reproducible bit for bit.
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "tb_vec.cuh"

namespace tb {

// Node flag bits of a prepared problem.
constexpr uint8_t kNodeActive = 1;    // node of at least one active element
constexpr uint8_t kNodeFixed = 2;     // fixed: a fixed temperature or not active
constexpr uint8_t kNodeFixedT = 4;    // carries a fixed temperature (fixed mask and active)

// d_err bits of the validation kernels.
constexpr int kErrConductivity = 1;
constexpr int kErrCoefficient = 2;
constexpr int kErrAmbient = 4;
constexpr int kErrHeat = 8;
constexpr int kErrFixed = 16;
constexpr int kErrCapacity = 32;

// One convection boundary as the lumping kernels take it.
//   kind 0: one outer face of the stack (side 0 the -z face of slab 0, side 1
//           the +z face of slab S-1), coefficient / ambient fields (R, C);
//   kind 1: every exposed face of the active elements in `dirs` order
//           (0 -x, 1 +x, 2 -y, 3 +y, 4 -z, 5 +z), fields (S, R, C).
// A NULL field takes the scalar.
struct ConvectionTerm {
    int kind;
    int side;
    int ndir;
    int dirs[6];
    double coef, amb;
    const double* coef_field;
    const double* amb_field;
};

__device__ __forceinline__ bool element_active(const uint8_t* active, int z, int y, int x, const Layout& L) {
    return active == nullptr || active[((long long)z * L.R + y) * L.C + x] != 0;
}

// ------------------------------------------------------------ validation
// Conductivities finite and non-negative (the mesh zeroes them on void
// elements), heats finite, element fields of the problem.
__global__ void check_elements(const double* __restrict__ kin, const double* __restrict__ kz,
                               const double* __restrict__ element_heat, int* __restrict__ err, long long E) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    int bits = 0;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += stride) {
        const double a = kin[e], b = kz[e];
        if (!(isfinite(a) && a >= 0.0 && isfinite(b) && b >= 0.0)) bits |= kErrConductivity;
        if (element_heat && !isfinite(element_heat[e])) bits |= kErrHeat;
    }
    if (bits) atomicOr(err, bits);
}

__global__ void check_nodes(const double* __restrict__ nodal_heat, const uint8_t* __restrict__ fixed_mask,
                            const double* __restrict__ fixed_t, const double* __restrict__ capacity,
                            int* __restrict__ err, long long N) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    int bits = 0;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < N; n += stride) {
        if (nodal_heat && !isfinite(nodal_heat[n])) bits |= kErrHeat;
        if (fixed_mask && fixed_mask[n] && !isfinite(fixed_t[n])) bits |= kErrFixed;
        if (capacity && !(isfinite(capacity[n]) && capacity[n] >= 0.0)) bits |= kErrCapacity;
    }
    if (bits) atomicOr(err, bits);
}

__global__ void check_field(const double* __restrict__ field, long long n, int non_negative, int bit,
                            int* __restrict__ err) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    int bits = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double v = field[i];
        if (!isfinite(v) || (non_negative && v < 0.0)) bits |= bit;
    }
    if (bits) atomicOr(err, bits);
}

// ----------------------------------------------------------------- masks
// Node flags, the free mask the solver takes, and the fixed temperatures
// (reference operator.py:89-96, mesh.py:319-325): a node is active when one
// of its (up to eight) elements is; fixed = fixed mask or not active; the
// fixed value is kept where the mask is set on an active node, else 0.
__global__ void prep_nodes(uint8_t* __restrict__ flags, uint8_t* __restrict__ free_nodes,
                           double* __restrict__ fixed_value, const uint8_t* __restrict__ active,
                           const uint8_t* __restrict__ fixed_mask, const double* __restrict__ fixed_t, Layout L) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    const int cols = L.C + 1;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < L.N; n += stride) {
        const long long line = n / cols;
        const int x = (int)(n - line * cols);
        const int z = (int)(line / (L.R + 1));
        const int y = (int)(line - (long long)z * (L.R + 1));
        bool act = false;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int ez = z - (c >> 2), ey = y - ((c >> 1) & 1), ex = x - (c & 1);
            if (ez < 0 || ez >= L.S || ey < 0 || ey >= L.R || ex < 0 || ex >= L.C) continue;
            act = act || element_active(active, ez, ey, ex, L);
        }
        const bool mask = fixed_mask != nullptr && fixed_mask[n] != 0;
        const bool fixed = mask || !act;
        const bool carries = mask && act;
        flags[n] = (uint8_t)((act ? kNodeActive : 0) | (fixed ? kNodeFixed : 0) | (carries ? kNodeFixedT : 0));
        free_nodes[n] = fixed ? 0 : 1;
        fixed_value[n] = carries ? fixed_t[n] : 0.0;
    }
}

// ----------------------------------------------------------------- loads
// q_n = nodal heat, plus element heat / 8 from each corner element in corner
// order 0..7 (the element whose corner c is node n), reference
// operator.py:374-387 (`for target in corner_views(load): target += share`).
// Without element heat the reference still adds its zeros; one + 0.0 has the
// same effect on every value.
__global__ void prep_load(double* __restrict__ load, const double* __restrict__ nodal_heat,
                          const double* __restrict__ element_heat, Layout L) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    const int cols = L.C + 1;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < L.N; n += stride) {
        const long long line = n / cols;
        const int x = (int)(n - line * cols);
        const int z = (int)(line / (L.R + 1));
        const int y = (int)(line - (long long)z * (L.R + 1));
        double v = nodal_heat ? nodal_heat[n] : 0.0;
        if (element_heat == nullptr) {
            v = __dadd_rn(v, 0.0);
        } else {
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const int ez = z - (c >> 2), ey = y - ((c >> 1) & 1), ex = x - (c & 1);
                if (ez < 0 || ez >= L.S || ey < 0 || ey >= L.R || ex < 0 || ex >= L.C) continue;
                v = __dadd_rn(v, __ddiv_rn(element_heat[((long long)ez * L.R + ey) * L.C + ex], 8.0));
            }
        }
        load[n] = v;
    }
}

// Heat sources: entries (node, power / node count) sorted by node, stable in
// source order, so each run of equal nodes adds its values in the order the
// reference's loop does (`load.flat[node] += per_node`, operator.py:383-386).
__global__ void prep_sources(double* __restrict__ load, const long long* __restrict__ node,
                             const double* __restrict__ value, int count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const long long n = node[i];
    if (i > 0 && node[i - 1] == n) return;
    double v = load[n];
    for (int j = i; j < count && node[j] == n; ++j) v = __dadd_rn(v, value[j]);
    load[n] = v;
}

// ------------------------------------------------------------ Robin terms
// Face area normal to a direction (reference mesh.py:95-106): z faces
// h_x h_y, y faces h_x h_z, x faces h_y h_z.
__device__ __forceinline__ double face_area(int dir, int z, int y, int x, const double* thick, const double* px,
                                            const double* py) {
    const int axis = dir >> 1;  // 0 x, 1 y, 2 z
    if (axis == 2) return __dmul_rn(px[x], py[y]);
    if (axis == 1) return __dmul_rn(px[x], thick[z]);
    return __dmul_rn(py[y], thick[z]);
}

// Corner (4dz + 2dy + dx) of the k-th node of face `dir`, in the reference's
// FACE_CORNERS order (mesh.py:44-51).
__device__ __forceinline__ int face_corner(int dir, int k) {
    // -x (0,2,4,6) +x (1,3,5,7) -y (0,1,4,5) +y (2,3,6,7) -z (0,1,2,3) +z (4,5,6,7)
    const int axis = dir >> 1, plus = dir & 1;
    if (axis == 0) return 2 * k + plus;
    if (axis == 1) return (k & 1) | ((k >> 1) << 2) | (plus << 1);
    return k | (plus << 2);
}

__device__ __forceinline__ bool face_exposed(const uint8_t* active, int dir, int z, int y, int x, const Layout& L) {
    if (!element_active(active, z, y, x, L)) return false;
    const int axis = dir >> 1, step = (dir & 1) ? 1 : -1;
    int nz = z, ny = y, nx = x;
    if (axis == 0) nx += step;
    else if (axis == 1) ny += step;
    else nz += step;
    if (nz < 0 || nz >= L.S || ny < 0 || ny >= L.R || nx < 0 || nx >= L.C) return true;
    return !element_active(active, nz, ny, nx, L);
}

// One outer face (kind 0), on the node plane it touches.  The reference
// builds the element face field (h * active) * area, its load field
// face * T_amb, and spreads face / 4 onto the four corners in FACE_CORNERS
// order starting from zero (boundaries.py:82-102, mesh.py:80-92).  Writes the
// boundary's weights on the plane ((R+1)(C+1)) and adds them to the running
// totals over the boundaries, which start at zero: the reference sums the
// per-boundary arrays in boundary order (np.sum(list, axis=0)).
__global__ void lump_outer_face(double* __restrict__ w_plane, double* __restrict__ rw_plane,
                                double* __restrict__ robin_only, double* __restrict__ robin_rhs, ConvectionTerm t,
                                const uint8_t* __restrict__ active, const double* __restrict__ px,
                                const double* __restrict__ py, Layout L) {
    const long long plane = (long long)(L.R + 1) * (L.C + 1);
    const int slab = t.side ? L.S - 1 : 0;
    const int zn = t.side ? L.S : 0;  // node plane of the face
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < plane; p += stride) {
        const int y = (int)(p / (L.C + 1));
        const int x = (int)(p - (long long)y * (L.C + 1));
        double w = 0.0, rw = 0.0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {  // corners (dy, dx) = (0,0) (0,1) (1,0) (1,1)
            const int ey = y - (k >> 1), ex = x - (k & 1);
            if (ey < 0 || ey >= L.R || ex < 0 || ex >= L.C) continue;
            const long long f = (long long)ey * L.C + ex;
            const double h = t.coef_field ? t.coef_field[f] : t.coef;
            const double amb = t.amb_field ? t.amb_field[f] : t.amb;
            const double act = element_active(active, slab, ey, ex, L) ? 1.0 : 0.0;
            const double face = __dmul_rn(__dmul_rn(h, act), __dmul_rn(px[ex], py[ey]));
            w = __dadd_rn(w, __ddiv_rn(face, 4.0));
            rw = __dadd_rn(rw, __ddiv_rn(__dmul_rn(face, amb), 4.0));
        }
        w_plane[p] = w;
        rw_plane[p] = rw;
        const long long n = (long long)zn * plane + p;
        robin_only[n] = __dadd_rn(robin_only[n], w);
        robin_rhs[n] = __dadd_rn(robin_rhs[n], rw);
    }
}

// Exposed faces (kind 1) over the whole node grid.  Per direction the
// reference lumps (h * area) * exposed and ((h * area) * exposed) * T_amb onto
// a zero grid in FACE_CORNERS order and adds that grid to the boundary's
// total, directions in the boundary's order (boundaries.py:171-183).
// Faces that are not exposed add +0, which changes no partial sum here
// (every partial sum of the weights is +0 or positive, and a sum that starts
// at +0 never becomes -0), so they are skipped.
__global__ void lump_exposed_faces(double* __restrict__ w_out, double* __restrict__ rw_out,
                                   double* __restrict__ robin_only, double* __restrict__ robin_rhs, ConvectionTerm t,
                                   const uint8_t* __restrict__ active, const double* __restrict__ thick,
                                   const double* __restrict__ px, const double* __restrict__ py, Layout L) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    const int cols = L.C + 1;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < L.N; n += stride) {
        const long long line = n / cols;
        const int x = (int)(n - line * cols);
        const int z = (int)(line / (L.R + 1));
        const int y = (int)(line - (long long)z * (L.R + 1));
        double w = 0.0, rw = 0.0;
        for (int d = 0; d < t.ndir; ++d) {
            const int dir = t.dirs[d];
            double lw = 0.0, lrw = 0.0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int c = face_corner(dir, k);
                const int ez = z - (c >> 2), ey = y - ((c >> 1) & 1), ex = x - (c & 1);
                if (ez < 0 || ez >= L.S || ey < 0 || ey >= L.R || ex < 0 || ex >= L.C) continue;
                if (!face_exposed(active, dir, ez, ey, ex, L)) continue;
                const long long e = ((long long)ez * L.R + ey) * L.C + ex;
                const double h = t.coef_field ? t.coef_field[e] : t.coef;
                const double amb = t.amb_field ? t.amb_field[e] : t.amb;
                const double face = __dmul_rn(__dmul_rn(h, face_area(dir, ez, ey, ex, thick, px, py)), 1.0);
                lw = __dadd_rn(lw, __ddiv_rn(face, 4.0));
                lrw = __dadd_rn(lrw, __ddiv_rn(__dmul_rn(face, amb), 4.0));
            }
            w = __dadd_rn(w, lw);
            rw = __dadd_rn(rw, lrw);
        }
        w_out[n] = w;
        rw_out[n] = rw;
        robin_only[n] = __dadd_rn(robin_only[n], w);
        robin_rhs[n] = __dadd_rn(robin_rhs[n], rw);
    }
}

// robin_total = robin_only + capacity (reference system.py: the capacity is
// a zero array in a steady solve, which the + 0.0 reproduces).
__global__ void prep_robin_total(double* __restrict__ total, const double* __restrict__ robin_only,
                                 const double* __restrict__ capacity, long long N) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < N; n += stride)
        total[n] = __dadd_rn(robin_only[n], capacity ? capacity[n] : 0.0);
}

// ------------------------------------------------------ right-hand side
// Fixed rises T_fix - T_ref on active fixed nodes, 0 elsewhere, into a padded
// FP64 field (the operand of the unconstrained stiffness action).
__global__ void prep_shifted(double* __restrict__ shifted_padded, const double* __restrict__ fixed_value,
                             const uint8_t* __restrict__ flags, double reference, Layout L) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    const int cols = L.C + 1;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L.L; i += stride) {
        const long long line = i / L.Xp;
        const int x = (int)(i - line * L.Xp);
        double v = 0.0;
        if (x < cols) {
            const long long n = line * cols + x;
            if (flags[n] & kNodeFixedT) v = __dsub_rn(fixed_value[n], reference);
        }
        shifted_padded[i] = v;
    }
}

// Smallest and largest value of t over the active nodes (non-NaN values;
// NaN where there are none), as NumPy's nanmin / nanmax of the temperature
// with NaN on the void nodes.  Block extrema go to partials[4 b], [4 b + 1]
// (gridDim.x <= the partials' block count); the last block to finish (ticket
// after a fence by thread 0) writes the grid's into out2[0], out2[1] and
// resets the ticket.  max and min are exact: the result does not depend on
// the order.
__global__ void node_extrema(const double* __restrict__ t, const uint8_t* __restrict__ flags, long long n,
                             double* partials, unsigned int* counter, double* out2) {
    __shared__ double s_lo[32], s_hi[32];
    __shared__ bool is_last;
    double lo = CUDART_INF, hi = -CUDART_INF;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        if (flags[i] & kNodeActive) {
            const double v = t[i];
            lo = fmin(lo, v);  // fmin / fmax ignore a NaN operand
            hi = fmax(hi, v);
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int off = 16; off > 0; off >>= 1) {
        lo = fmin(lo, __shfl_down_sync(0xffffffffu, lo, off));
        hi = fmax(hi, __shfl_down_sync(0xffffffffu, hi, off));
    }
    if (lane == 0) {
        s_lo[warp] = lo;
        s_hi[warp] = hi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < nw; ++w) {
            lo = fmin(lo, s_lo[w]);
            hi = fmax(hi, s_hi[w]);
        }
        partials[4 * (size_t)blockIdx.x] = lo;
        partials[4 * (size_t)blockIdx.x + 1] = hi;
        __threadfence();
        is_last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!is_last || threadIdx.x != 0) return;
    __threadfence();
    for (unsigned b = 0; b < gridDim.x; ++b) {
        lo = fmin(lo, __ldcg(partials + 4 * (size_t)b));
        hi = fmax(hi, __ldcg(partials + 4 * (size_t)b + 1));
    }
    out2[0] = (lo == CUDART_INF) ? CUDART_NAN : lo;
    out2[1] = (hi == -CUDART_INF) ? CUDART_NAN : hi;
    *counter = 0u;
}

// dst = src + c on n flat nodes (a temperature from its rise over the
// reference temperature; the same IEEE addition the host would do).
__global__ void shift_nodes(double* __restrict__ dst, const double* __restrict__ src, double c, long long n) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) dst[i] = __dadd_rn(src[i], c);
}

// b = ((q + (R T_amb - R_total T_ref)) + C/dt T_prev) - K shifted, and the
// shifted value on fixed rows (reference operator.py:411-440).  `action` is
// the padded stiffness action of the shifted field; the previous
// temperature's non-finite entries count as 0.
__global__ void prep_rhs(double* __restrict__ rhs, const double* __restrict__ load,
                         const double* __restrict__ robin_rhs, const double* __restrict__ robin_total,
                         const double* __restrict__ capacity, const double* __restrict__ previous,
                         const double* __restrict__ fixed_value, const uint8_t* __restrict__ flags,
                         const double* __restrict__ action_padded, double reference, Layout L) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    const int cols = L.C + 1;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < L.N; n += stride) {
        const uint8_t f = flags[n];
        if (f & kNodeFixed) {
            rhs[n] = (f & kNodeFixedT) ? __dsub_rn(fixed_value[n], reference) : 0.0;
            continue;
        }
        const long long line = n / cols;
        const int x = (int)(n - line * cols);
        double cap_load = 0.0;
        if (previous) {
            const double prev = isfinite(previous[n]) ? previous[n] : 0.0;
            cap_load = __dmul_rn(capacity ? capacity[n] : 0.0, prev);
        }
        const double rr = __dsub_rn(robin_rhs[n], __dmul_rn(robin_total[n], reference));
        double b = __dadd_rn(load[n], rr);
        b = __dadd_rn(b, cap_load);
        rhs[n] = __dsub_rn(b, action_padded[line * L.Xp + x]);
    }
}

// ------------------------------------------------------ post-processing
// -k grad T at each element centre, (x, y, z) per element (reference
// operator.py:500-525): face sums of the corner temperatures in corner order,
// differences over 4 h, times -k; zero on void elements, as the reference's
// solve sets them (solve.py:255-280).
__global__ void element_flux(double* __restrict__ flux, const double* __restrict__ temperature,
                             const double* __restrict__ kin_padded, const double* __restrict__ kz_padded,
                             const double* __restrict__ thick, const double* __restrict__ px,
                             const double* __restrict__ py, const uint8_t* __restrict__ active, Layout L) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long row = L.C + 1, plane = (long long)(L.R + 1) * (L.C + 1);
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < L.E; e += stride) {
        const long long line = e / L.C;
        const int x = (int)(e - line * L.C);
        const int z = (int)(line / L.R);
        const int y = (int)(line - (long long)z * L.R);
        double fx = 0.0, fy = 0.0, fz = 0.0;
        if (element_active(active, z, y, x, L)) {
            const long long base = (long long)z * plane + (long long)y * row + x;
            double c[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) c[k] = temperature[base + (k >> 2) * plane + ((k >> 1) & 1) * row + (k & 1)];
            const double xp = __dadd_rn(__dadd_rn(__dadd_rn(c[1], c[3]), c[5]), c[7]);
            const double xm = __dadd_rn(__dadd_rn(__dadd_rn(c[0], c[2]), c[4]), c[6]);
            const double yp = __dadd_rn(__dadd_rn(__dadd_rn(c[2], c[3]), c[6]), c[7]);
            const double ym = __dadd_rn(__dadd_rn(__dadd_rn(c[0], c[1]), c[4]), c[5]);
            const double zp = __dadd_rn(__dadd_rn(__dadd_rn(c[4], c[5]), c[6]), c[7]);
            const double zm = __dadd_rn(__dadd_rn(__dadd_rn(c[0], c[1]), c[2]), c[3]);
            const double gx = __ddiv_rn(__dsub_rn(xp, xm), __dmul_rn(4.0, px[x]));
            const double gy = __ddiv_rn(__dsub_rn(yp, ym), __dmul_rn(4.0, py[y]));
            const double gz = __ddiv_rn(__dsub_rn(zp, zm), __dmul_rn(4.0, thick[z]));
            const long long ep = ((long long)z * L.R + y) * L.Xe + x;
            const double ki = kin_padded[ep], kz = kz_padded[ep];
            fx = __dmul_rn(-ki, gx);
            fy = __dmul_rn(-ki, gy);
            fz = __dmul_rn(-kz, gz);
        }
        flux[3 * e] = fx;
        flux[3 * e + 1] = fy;
        flux[3 * e + 2] = fz;
    }
}

// Compensated FP64 sum (value = s + c).
struct Acc2 {
    double s = 0.0, c = 0.0;
    __device__ __forceinline__ void add(double v) {
        const double t = __dadd_rn(s, v);
        const double z = __dsub_rn(t, s);
        c = __dadd_rn(c, __dadd_rn(__dsub_rn(s, __dsub_rn(t, z)), __dsub_rn(v, z)));
        s = t;
    }
    __device__ __forceinline__ void add_product(double a, double b) {
        const double p = __dmul_rn(a, b);
        add(p);
        c = __dadd_rn(c, __fma_rn(a, b, -p));
    }
    __device__ __forceinline__ void merge(double os, double oc) {
        add(os);
        c = __dadd_rn(c, oc);
    }
};

constexpr int kSumThreads = 256;
constexpr int kMaxSums = 4;

// Block merge of K accumulators in a fixed tree; thread 0 writes the block's
// (s, c) pairs to partials[block][K][2].
template <int K>
__device__ __forceinline__ void block_store(Acc2 (&acc)[K], double* __restrict__ partials) {
    __shared__ double sh[kMaxSums][2][kSumThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double os = __shfl_down_sync(0xffffffffu, acc[k].s, o);
            const double oc = __shfl_down_sync(0xffffffffu, acc[k].c, o);
            acc[k].merge(os, oc);
        }
        if (lane == 0) {
            sh[k][0][warp] = acc[k].s;
            sh[k][1][warp] = acc[k].c;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            Acc2 a;
            for (int w = 0; w < kSumThreads / 32; ++w) a.merge(sh[k][0][w], sh[k][1][w]);
            partials[((long long)blockIdx.x * K + k) * 2] = a.s;
            partials[((long long)blockIdx.x * K + k) * 2 + 1] = a.c;
        }
    }
}

// Sum the block partials of K quantities in block order: out[k] = s + c.
__global__ void finish_sums(const double* __restrict__ partials, int blocks, int K, double* __restrict__ out) {
    if (threadIdx.x >= K) return;
    const int k = threadIdx.x;
    Acc2 a;
    for (int b = 0; b < blocks; ++b) a.merge(partials[((long long)b * K + k) * 2], partials[((long long)b * K + k) * 2 + 1]);
    out[k] = __dadd_rn(a.s, a.c);
}

// The node pass after a solve: the unconstrained residual
// r = (((K T + R_conv T) - R T_amb) + C/dt (T - T_prev)) - q (reference
// operator.py:458-482, the stored term 0 in a steady solve and where T or
// T_prev is not finite), written out when `residual` is not NULL, and the
// sums {-sum r over fixed nodes, sum C/dt (T - T_prev)}.
__global__ void __launch_bounds__(kSumThreads)
post_nodes(double* __restrict__ residual, double* __restrict__ partials, const double* __restrict__ temperature,
           const double* __restrict__ conduction_padded, const double* __restrict__ robin_only,
           const double* __restrict__ robin_rhs, const double* __restrict__ load, const double* __restrict__ capacity,
           const double* __restrict__ previous, const uint8_t* __restrict__ flags, Layout L) {
    Acc2 acc[2];
    const long long stride = (long long)gridDim.x * blockDim.x;
    const int cols = L.C + 1;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < L.N; n += stride) {
        const long long line = n / cols;
        const int x = (int)(n - line * cols);
        const double t = temperature[n];
        double stored = 0.0;
        if (previous) {
            const double prev = previous[n];
            if (isfinite(t) && isfinite(prev)) stored = __dmul_rn(capacity ? capacity[n] : 0.0, __dsub_rn(t, prev));
        }
        double r = __dadd_rn(conduction_padded[line * L.Xp + x], __dmul_rn(robin_only[n], t));
        r = __dsub_rn(r, robin_rhs[n]);
        r = __dadd_rn(r, stored);
        r = __dsub_rn(r, load[n]);
        if (residual) residual[n] = r;
        if (flags[n] & kNodeFixed) acc[0].add(-r);
        acc[1].add(stored);
    }
    block_store<2>(acc, partials);
}

// sum w v over n entries, and optionally sum of v alone: {sum w v, sum v}.
__global__ void __launch_bounds__(kSumThreads)
dot_sums(double* __restrict__ partials, const double* __restrict__ w, const double* __restrict__ v, long long n) {
    Acc2 acc[2];
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double b = v[i];
        if (w) acc[0].add_product(w[i], b);
        acc[1].add(b);
    }
    block_store<2>(acc, partials);
}

}  // namespace tb
