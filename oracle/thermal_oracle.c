/*
 * thermal_oracle.c -- CPU restatement of pcb-analysis's steady Q1 thermal
 * operator and its Jacobi PCG / MPIR solve.  TEST INFRASTRUCTURE ONLY: this is
 * the checker the B200 kernels are compared against and the CPU baseline the
 * benchmark times; no product code path links or calls it.
 *
 * Followed, function by function (paths within the reference project):
 *   or_apply_*     HexOperatorT::gather / apply_lines,
 *                  src/thermal/matrix_free_mpir_fem/native/hex_q1.cpp:90-193
 *                  (node-owned gather: per node the <= 8 adjacent elements, per
 *                  element the 8 corner columns, weight a_x Ux + a_y Uy + a_z Uz,
 *                  fixed columns skipped, Robin on the diagonal, fixed rows copy x)
 *   or_diagonal    _build_diagonal, operator.py:290-306 / thermal_system.cpp:328-349
 *   lane_sum       cpp/include/pcbcore/lane_sum.hpp:18-40 (8 lanes by index, fixed tree)
 *   or_pcg_f64     the PCG control flow of solver.py:151-232 in FP64 throughout
 *   or_solve_mpir  solve_mpir, solver.py:580-698 / hex_q1.cpp:837-925, with the
 *                  inner FP32 Jacobi PCG of hex_q1.cpp:323-499 and the power-of-two
 *                  right-hand-side scaling of solver.py:172-185
 *
 * Parallel over node lines (z, y) with OpenMP; every inner product is one
 * lane sum per line followed by an ordered sum over lines, so the bits do not
 * depend on the thread count.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    int32_t slabs, rows, cols;
    const double* coef;         /* (3, S, R, C): a_x, a_y, a_z */
    const double* robin;        /* (N) Robin total */
    const uint8_t* free_nodes;  /* (N) 1 free */
} or_view;

typedef struct {
    int32_t converged, outer_iterations, inner_iterations, high_applications, low_applications, history_length;
    double relative_residual;
} or_mpir_result;

typedef struct {
    int32_t outer_iteration, inner_iterations;
    double high_relative_residual, inner_relative_residual;
} or_mpir_step;

/* U_x = M(x)M(x)S, U_y = M(x)S(x)M, U_z = S(x)M(x)M, local order 4dz+2dy+dx
 * (mesh.py:346-359, thermal_system.cpp:279-288), products in the same order. */
void or_unit_matrices(double* unit) {
    const double S1[2][2] = {{1.0, -1.0}, {-1.0, 1.0}};
    const double M1[2][2] = {{2.0 / 6.0, 1.0 / 6.0}, {1.0 / 6.0, 2.0 / 6.0}};
    for (int i = 0; i < 8; ++i) {
        for (int j = 0; j < 8; ++j) {
            const int zi = i >> 2, yi = (i >> 1) & 1, xi = i & 1;
            const int zj = j >> 2, yj = (j >> 1) & 1, xj = j & 1;
            unit[8 * i + j] = M1[zi][zj] * (M1[yi][yj] * S1[xi][xj]);
            unit[64 + 8 * i + j] = M1[zi][zj] * (S1[yi][yj] * M1[xi][xj]);
            unit[128 + 8 * i + j] = S1[zi][zj] * (M1[yi][yj] * M1[xi][xj]);
        }
    }
}

static int64_t node_count(const or_view* v) { return (int64_t)(v->slabs + 1) * (v->rows + 1) * (v->cols + 1); }

/* ------------------------------------------------------------- operator */
#define DEFINE_APPLY(NAME, T)                                                                                     \
    static void NAME##_lines(const or_view* v, const T* coef, const T* unit, const T* robin, const T* x, T* y,     \
                             int stiffness, int64_t lb, int64_t le) {                                             \
        const int S = v->slabs, R = v->rows, C = v->cols;                                                        \
        const int nr = R + 1, nc = C + 1;                                                                         \
        const int64_t plane = (int64_t)nr * nc;                                                                   \
        const int64_t ne = (int64_t)S * R * C;                                                                    \
        const T* ux = unit;                                                                                       \
        const T* uy = unit + 64;                                                                                  \
        const T* uz = unit + 128;                                                                                 \
        for (int64_t line = lb; line < le; ++line) {                                                              \
            const int z = (int)(line / nr), yy = (int)(line - (int64_t)z * nr);                                   \
            const int z0 = z > 0 ? z - 1 : 0, z1 = z < S ? z : S - 1;                                             \
            const int y0 = yy > 0 ? yy - 1 : 0, y1 = yy < R ? yy : R - 1;                                         \
            for (int xi = 0; xi < nc; ++xi) {                                                                     \
                const int64_t node = line * nc + xi;                                                              \
                const int fr = stiffness ? 1 : v->free_nodes[node];                                               \
                if (!fr) {                                                                                        \
                    y[node] = x[node];                                                                            \
                    continue;                                                                                     \
                }                                                                                                 \
                const int x0 = xi > 0 ? xi - 1 : 0, x1 = xi < C ? xi : C - 1;                                     \
                T acc = (T)0;                                                                                     \
                for (int ez = z0; ez <= z1; ++ez) {                                                               \
                    for (int ey = y0; ey <= y1; ++ey) {                                                           \
                        for (int ex = x0; ex <= x1; ++ex) {                                                       \
                            const int lr = 4 * (z - ez) + 2 * (yy - ey) + (xi - ex);                              \
                            const int64_t e = ((int64_t)ez * R + ey) * C + ex;                                    \
                            const T a = coef[e], b = coef[ne + e], d = coef[2 * ne + e];                          \
                            const int64_t corner = ((int64_t)ez * nr + ey) * nc + ex;                             \
                            for (int c = 0; c < 8; ++c) {                                                         \
                                const int64_t cn = corner + (int64_t)(c >> 2) * plane + (int64_t)((c >> 1) & 1) * nc + (c & 1); \
                                if (!stiffness && !v->free_nodes[cn]) continue;                                   \
                                acc += ((a * ux[8 * lr + c]) + (b * uy[8 * lr + c]) + (d * uz[8 * lr + c])) * x[cn]; \
                            }                                                                                     \
                        }                                                                                         \
                    }                                                                                             \
                }                                                                                                 \
                y[node] = stiffness ? acc : acc + robin[node] * x[node];                                          \
            }                                                                                                     \
        }                                                                                                         \
    }                                                                                                             \
    static void NAME(const or_view* v, const T* coef, const T* unit, const T* robin, const T* x, T* y,             \
                     int stiffness, int threads) {                                                                \
        const int64_t lines = (int64_t)(v->slabs + 1) * (v->rows + 1);                                            \
        _Pragma("omp parallel for schedule(static) num_threads(threads)") for (int64_t l = 0; l < lines; ++l)    \
            NAME##_lines(v, coef, unit, robin, x, y, stiffness, l, l + 1);                                        \
    }

DEFINE_APPLY(apply64, double)
DEFINE_APPLY(apply32, float)

/* Line form of the same action (hex_q1.cpp:131-193 apply_lines): the two end
 * nodes of a line by the gather above, the interior nodes with the two
 * x-neighbouring elements unrolled and the fixed columns removed by a 0/1 mask
 * multiply, which the compiler vectorises.  Used for the timed CPU baseline. */
#define DEFINE_FAST(NAME, T, GATHER)                                                                              \
    static void NAME(const or_view* v, const T* coef, const T* unit, const T* robin, const T* mask, const T* x,    \
                     T* y, int threads) {                                                                         \
        const int S = v->slabs, R = v->rows, C = v->cols, nr = R + 1, nc = C + 1;                                 \
        const int64_t plane = (int64_t)nr * nc, ne = (int64_t)S * R * C, lines = (int64_t)(S + 1) * nr;           \
        const T* ux = unit;                                                                                       \
        const T* uy = unit + 64;                                                                                  \
        const T* uz = unit + 128;                                                                                 \
        _Pragma("omp parallel for schedule(static) num_threads(threads)") for (int64_t line = 0; line < lines; ++line) { \
            const int z = (int)(line / nr), yy = (int)(line - (int64_t)z * nr);                                   \
            T* const o = y + line * nc;                                                                           \
            /* end nodes by the generic gather */                                                                 \
            GATHER##_lines(v, coef, unit, robin, x, y, 0, line, line + 1);                                        \
            if (C < 2) continue;                                                                                  \
            const T save0 = o[0], saveC = o[C];                                                                   \
            const int z0 = z > 0 ? z - 1 : 0, z1 = z < S ? z : S - 1;                                             \
            const int y0 = yy > 0 ? yy - 1 : 0, y1 = yy < R ? yy : R - 1;                                         \
            for (int xi = 1; xi < C; ++xi) o[xi] = (T)0;                                                          \
            for (int ez = z0; ez <= z1; ++ez) {                                                                   \
                for (int ey = y0; ey <= y1; ++ey) {                                                               \
                    const int lrb = 4 * (z - ez) + 2 * (yy - ey);                                                 \
                    const int64_t erow = ((int64_t)ez * R + ey) * C;                                              \
                    const T* ax = coef + erow;                                                                    \
                    const T* ay = coef + ne + erow;                                                               \
                    const T* az = coef + 2 * ne + erow;                                                           \
                    const int64_t crow = ((int64_t)ez * nr + ey) * nc;                                            \
                    for (int xi = 1; xi < C; ++xi) {                                                              \
                        T acc = (T)0;                                                                             \
                        for (int dx = 0; dx < 2; ++dx) {                                                          \
                            const int ex = xi - 1 + dx, lr = lrb + (1 - dx);                                      \
                            const T a = ax[ex], b = ay[ex], d = az[ex];                                           \
                            const int64_t corner = crow + ex;                                                     \
                            for (int c = 0; c < 8; ++c) {                                                         \
                                const int64_t cn = corner + (int64_t)(c >> 2) * plane + (int64_t)((c >> 1) & 1) * nc + (c & 1); \
                                const T w = (a * ux[8 * lr + c]) + (b * uy[8 * lr + c]) + (d * uz[8 * lr + c]);  \
                                acc += w * (x[cn] * mask[cn]);                                                    \
                            }                                                                                     \
                        }                                                                                         \
                        o[xi] += acc;                                                                             \
                    }                                                                                             \
                }                                                                                                 \
            }                                                                                                     \
            for (int xi = 1; xi < C; ++xi) {                                                                      \
                const int64_t node = line * nc + xi;                                                              \
                const T f = mask[node];                                                                           \
                o[xi] = (f * (o[xi] + robin[node] * x[node])) + (((T)1 - f) * x[node]);                           \
            }                                                                                                     \
            o[0] = save0;                                                                                         \
            o[C] = saveC;                                                                                         \
        }                                                                                                         \
    }

DEFINE_FAST(fast64, double, apply64)
DEFINE_FAST(fast32, float, apply32)

void or_apply_f64(const or_view* v, const double* x, double* y, int threads) {
    double unit[192];
    or_unit_matrices(unit);
    apply64(v, v->coef, unit, v->robin, x, y, 0, threads);
}

void or_stiffness_f64(const or_view* v, const double* x, double* y, int threads) {
    double unit[192];
    or_unit_matrices(unit);
    apply64(v, v->coef, unit, v->robin, x, y, 1, threads);
}

/* FP32 action with FP32 copies of the FP64 coefficients, unit matrices and
 * Robin term (thermal_system.cpp:352-356: cast_all<float>). */
void or_apply_f32(const or_view* v, const float* coef32, const float* robin32, const float* x, float* y, int threads) {
    double u64[192];
    float unit[192];
    or_unit_matrices(u64);
    for (int i = 0; i < 192; ++i) unit[i] = (float)u64[i];
    apply32(v, coef32, unit, robin32, x, y, 0, threads);
}

/* Jacobi diagonal in the reference's summation order. */
void or_diagonal(const or_view* v, double* diag) {
    double unit[192];
    or_unit_matrices(unit);
    const int S = v->slabs, R = v->rows, C = v->cols, nr = R + 1, nc = C + 1;
    const int64_t n = node_count(v), ne = (int64_t)S * R * C;
    memset(diag, 0, sizeof(double) * (size_t)n);
    for (int corner = 0; corner < 8; ++corner) {
        const int k = 9 * corner, dz = corner >> 2, dy = (corner >> 1) & 1, dx = corner & 1;
        for (int s = 0; s < S; ++s)
            for (int r = 0; r < R; ++r)
                for (int c = 0; c < C; ++c) {
                    const int64_t e = ((int64_t)s * R + r) * C + c;
                    const int64_t node = ((int64_t)(s + dz) * nr + (r + dy)) * nc + (c + dx);
                    diag[node] += (v->coef[e] * unit[k] + v->coef[ne + e] * unit[64 + k]) + v->coef[2 * ne + e] * unit[128 + k];
                }
    }
    for (int64_t i = 0; i < n; ++i) diag[i] = v->free_nodes[i] ? diag[i] + v->robin[i] : 1.0;
}

static double* mask64_of(const or_view* v) {
    const int64_t n = node_count(v);
    double* m = malloc(sizeof(double) * (size_t)n);
    for (int64_t i = 0; i < n; ++i) m[i] = v->free_nodes[i] ? 1.0 : 0.0;
    return m;
}

/* The line form, exported so the tests can hold it to the gather. */
void or_apply_fast_f64(const or_view* v, const double* x, double* y, int threads) {
    double unit[192];
    or_unit_matrices(unit);
    double* m = mask64_of(v);
    fast64(v, v->coef, unit, v->robin, m, x, y, threads);
    free(m);
}

void or_apply_fast_f32(const or_view* v, const float* coef32, const float* robin32, const float* x, float* y,
                       int threads) {
    double u64[192];
    float unit[192];
    or_unit_matrices(u64);
    for (int i = 0; i < 192; ++i) unit[i] = (float)u64[i];
    const int64_t n = node_count(v);
    float* m = malloc(sizeof(float) * (size_t)n);
    for (int64_t i = 0; i < n; ++i) m[i] = v->free_nodes[i] ? 1.0f : 0.0f;
    fast32(v, coef32, unit, robin32, m, x, y, threads);
    free(m);
}

/* ------------------------------------------------------------ lane sums */
static double lane_sum_prod64(const double* a, const double* b, int64_t count) {
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int64_t i = 0;
    for (; i + 8 <= count; i += 8)
        for (int k = 0; k < 8; ++k) acc[k] += a[i + k] * b[i + k];
    for (int k = 0; i < count; ++i, ++k) acc[k] += a[i] * b[i];
    return ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
}

static double lane_sum_prod32(const float* a, const float* b, int64_t count) {
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int64_t i = 0;
    for (; i + 8 <= count; i += 8)
        for (int k = 0; k < 8; ++k) acc[k] += (double)a[i + k] * (double)b[i + k];
    for (int k = 0; i < count; ++i, ++k) acc[k] += (double)a[i] * (double)b[i];
    return ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
}

/* Inner products by node line, then in line order. */
static double dot64(const or_view* v, const double* a, const double* b, double* part, int threads) {
    const int64_t lines = (int64_t)(v->slabs + 1) * (v->rows + 1), nc = v->cols + 1;
#pragma omp parallel for schedule(static) num_threads(threads)
    for (int64_t l = 0; l < lines; ++l) part[l] = lane_sum_prod64(a + l * nc, b + l * nc, nc);
    double s = 0.0;
    for (int64_t l = 0; l < lines; ++l) s += part[l];
    return s;
}

static double dot32(const or_view* v, const float* a, const float* b, double* part, int threads) {
    const int64_t lines = (int64_t)(v->slabs + 1) * (v->rows + 1), nc = v->cols + 1;
#pragma omp parallel for schedule(static) num_threads(threads)
    for (int64_t l = 0; l < lines; ++l) part[l] = lane_sum_prod32(a + l * nc, b + l * nc, nc);
    double s = 0.0;
    for (int64_t l = 0; l < lines; ++l) s += part[l];
    return s;
}

/* ----------------------------------------------------------- FP64 PCG */
/* Plain FP64 Jacobi PCG from x (in/out); stops when the recursive residual
 * reaches atol + rtol ||b||, then restarts from the iterate while the true
 * residual is still above that (at most 8 restarts), so the reported
 * solution meets the tolerance on its true residual.
 * Returns 0, or 2 when p.Ap is not positive. */
int or_pcg_f64(const or_view* v, const double* diag, const double* b, double* x, double rtol, double atol,
               int max_it, int threads, int32_t* iterations, double* relative_residual) {
    const int64_t n = node_count(v), lines = (int64_t)(v->slabs + 1) * (v->rows + 1);
    double unit[192];
    or_unit_matrices(unit);
    double* r = malloc(sizeof(double) * (size_t)n);
    double* z = malloc(sizeof(double) * (size_t)n);
    double* p = malloc(sizeof(double) * (size_t)n);
    double* q = malloc(sizeof(double) * (size_t)n);
    double* part = malloc(sizeof(double) * (size_t)lines);
    double* mask = mask64_of(v);
    int status = 0;
    const double bnorm = sqrt(dot64(v, b, b, part, threads));
    const double scale = bnorm > 0.0 ? bnorm : 1.0;
    const double target = atol + rtol * scale;
    int it = 0;
    double true_norm = 0.0;
    for (int restart = 0; restart <= 8; ++restart) {
        fast64(v, v->coef, unit, v->robin, mask, x, q, threads);
#pragma omp parallel for schedule(static) num_threads(threads)
        for (int64_t i = 0; i < n; ++i) {
            r[i] = b[i] - q[i];
            z[i] = r[i] / diag[i];
            p[i] = z[i];
        }
        true_norm = sqrt(dot64(v, r, r, part, threads));
        if (true_norm <= target || it >= max_it) break;
        double rz = dot64(v, r, z, part, threads);
        double rnorm = true_norm;
        while (rnorm > target && it < max_it) {
            fast64(v, v->coef, unit, v->robin, mask, p, q, threads);
            const double pq = dot64(v, p, q, part, threads);
            if (!(isfinite(pq) && pq > 0.0)) {
                status = 2;
                break;
            }
            const double alpha = rz / pq;
#pragma omp parallel for schedule(static) num_threads(threads)
            for (int64_t i = 0; i < n; ++i) {
                x[i] += alpha * p[i];
                r[i] -= alpha * q[i];
                z[i] = r[i] / diag[i];
            }
            ++it;
            rnorm = sqrt(dot64(v, r, r, part, threads));
            if (rnorm <= target) break;
            const double rz_next = dot64(v, r, z, part, threads);
            const double beta = rz_next / rz;
            rz = rz_next;
#pragma omp parallel for schedule(static) num_threads(threads)
            for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
        }
        if (status) break;
    }
    *relative_residual = true_norm / scale;
    *iterations = it;
    free(r);
    free(z);
    free(p);
    free(q);
    free(part);
    free(mask);
    return status;
}

/* -------------------------------------------------------- FP32 inner PCG */
typedef struct {
    const or_view* v;
    const float *coef32, *robin32, *dinv32;
    float unit[192];
    float *rhs, *x, *r, *z, *p, *q, *mask;
    double* part;
    int threads;
} inner_ws;

/* Runs at most `max_it` iterations of the FP32 Jacobi PCG on ws->rhs.
 * Returns 0, or 2 when p.Ap is not positive. */
static int inner_pcg(inner_ws* w, double tol, int max_it, int32_t* iterations, int32_t* applications, double* rel_out) {
    const or_view* v = w->v;
    const int64_t n = node_count(v);
    const int T = w->threads;
#pragma omp parallel for schedule(static) num_threads(T)
    for (int64_t i = 0; i < n; ++i) {
        w->x[i] = 0.0f;
        w->r[i] = w->rhs[i];
        w->z[i] = w->r[i] * w->dinv32[i];
        w->p[i] = w->z[i];
    }
    const double bnorm = sqrt(dot32(v, w->rhs, w->rhs, w->part, T));
    *iterations = 0;
    *applications = 0;
    *rel_out = 0.0;
    if (bnorm == 0.0) return 0;
    double rz = dot32(v, w->r, w->z, w->part, T);
    double rel = 1.0;
    int it = 0;
    while (it < max_it) {
        fast32(v, w->coef32, w->unit, w->robin32, w->mask, w->p, w->q, T);
        ++*applications;
        const double pq = dot32(v, w->p, w->q, w->part, T);
        if (!(isfinite(pq) && pq > 0.0)) return 2;
        const float alpha = (float)(rz / pq);
#pragma omp parallel for schedule(static) num_threads(T)
        for (int64_t i = 0; i < n; ++i) {
            w->x[i] += alpha * w->p[i];
            w->r[i] -= alpha * w->q[i];
        }
        ++it;
        rel = sqrt(dot32(v, w->r, w->r, w->part, T)) / bnorm;
        *iterations = it;
        *rel_out = rel;
        if (rel <= tol) break;
#pragma omp parallel for schedule(static) num_threads(T)
        for (int64_t i = 0; i < n; ++i) w->z[i] = w->r[i] * w->dinv32[i];
        const double rz_next = dot32(v, w->r, w->z, w->part, T);
        if (!isfinite(rz_next) || rz == 0.0) break;
        const float beta = (float)(rz_next / rz);
#pragma omp parallel for schedule(static) num_threads(T)
        for (int64_t i = 0; i < n; ++i) w->p[i] = w->z[i] + beta * w->p[i];
        rz = rz_next;
    }
    return 0;
}

static void inner_alloc(inner_ws* w, const or_view* v, const float* coef32, const float* robin32, const float* dinv32,
                        int threads) {
    const int64_t n = node_count(v), lines = (int64_t)(v->slabs + 1) * (v->rows + 1);
    double u64[192];
    or_unit_matrices(u64);
    for (int i = 0; i < 192; ++i) w->unit[i] = (float)u64[i];
    w->v = v;
    w->coef32 = coef32;
    w->robin32 = robin32;
    w->dinv32 = dinv32;
    w->threads = threads;
    w->rhs = malloc(sizeof(float) * (size_t)n);
    w->x = malloc(sizeof(float) * (size_t)n);
    w->r = malloc(sizeof(float) * (size_t)n);
    w->z = malloc(sizeof(float) * (size_t)n);
    w->p = malloc(sizeof(float) * (size_t)n);
    w->q = malloc(sizeof(float) * (size_t)n);
    w->part = malloc(sizeof(double) * (size_t)lines);
    w->mask = malloc(sizeof(float) * (size_t)n);
    for (int64_t i = 0; i < n; ++i) w->mask[i] = v->free_nodes[i] ? 1.0f : 0.0f;
}

static void inner_free(inner_ws* w) {
    free(w->rhs);
    free(w->x);
    free(w->r);
    free(w->z);
    free(w->p);
    free(w->q);
    free(w->part);
    free(w->mask);
}

/* MPIR: FP64 residual, norm and update; FP32 Jacobi PCG corrections.
 * Returns 0, or 2 when an inner PCG met a non-positive curvature. */
int or_solve_mpir(const or_view* v, const float* coef32, const float* robin32, const float* dinv32, const double* b,
                  double* x, double rtol, double atol, double inner_rtol, int max_outer, int max_inner, int threads,
                  or_mpir_result* res, or_mpir_step* hist, int cap) {
    const int64_t n = node_count(v), lines = (int64_t)(v->slabs + 1) * (v->rows + 1);
    double unit[192];
    or_unit_matrices(unit);
    double* ax = malloc(sizeof(double) * (size_t)n);
    double* rr = malloc(sizeof(double) * (size_t)n);
    double* part = malloc(sizeof(double) * (size_t)lines);
    double* mask = mask64_of(v);
    inner_ws w;
    inner_alloc(&w, v, coef32, robin32, dinv32, threads);
    memset(res, 0, sizeof(*res));
    const double bnorm = sqrt(dot64(v, b, b, part, threads));
    const double scale = bnorm > 0.0 ? bnorm : 1.0;
    const double target = atol + rtol * scale;
    int status = 0, outer, nh = 0;
    double rel = 1.0;
    for (outer = 0; outer <= max_outer; ++outer) {
        fast64(v, v->coef, unit, v->robin, mask, x, ax, threads);
        res->high_applications++;
        double peak = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            rr[i] = b[i] - ax[i];
            if (fabs(rr[i]) > peak) peak = fabs(rr[i]);
        }
        const double rn = sqrt(dot64(v, rr, rr, part, threads));
        rel = rn / scale;
        if (rn <= target) {
            res->converged = 1;
            break;
        }
        if (outer == max_outer) break;
        double ps = 1.0;
        if (peak > 0.0 && isfinite(peak)) {
            int e;
            frexp(peak, &e);
            ps = ldexp(1.0, -e);
        }
        for (int64_t i = 0; i < n; ++i) w.rhs[i] = (float)(rr[i] * ps);
        int32_t its = 0, apps = 0;
        double irel = 0.0;
        status = inner_pcg(&w, inner_rtol, max_inner, &its, &apps, &irel);
        if (status) break;
        for (int64_t i = 0; i < n; ++i) x[i] += (double)w.x[i] / ps;
        res->inner_iterations += its;
        res->low_applications += apps;
        if (hist && nh < cap) {
            hist[nh].outer_iteration = outer + 1;
            hist[nh].high_relative_residual = rel;
            hist[nh].inner_iterations = its;
            hist[nh].inner_relative_residual = irel;
        }
        ++nh;
    }
    res->outer_iterations = res->converged ? outer : max_outer;
    res->relative_residual = rel;
    res->history_length = nh < cap ? nh : cap;
    inner_free(&w);
    free(ax);
    free(rr);
    free(part);
    free(mask);
    return status;
}

/* Exactly `iterations` iterations of the FP32 inner PCG on `rhs` (tolerance 0),
 * for timing a bounded sample of a solve. */
int or_inner_iterations(const or_view* v, const float* coef32, const float* robin32, const float* dinv32,
                        const double* rhs, int iterations, int threads, double* rel) {
    inner_ws w;
    inner_alloc(&w, v, coef32, robin32, dinv32, threads);
    const int64_t n = node_count(v);
    for (int64_t i = 0; i < n; ++i) w.rhs[i] = (float)rhs[i];
    int32_t its = 0, apps = 0;
    const int st = inner_pcg(&w, 0.0, iterations, &its, &apps, rel);
    inner_free(&w);
    return st;
}

int or_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
