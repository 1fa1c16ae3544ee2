/*
 * thermal_b200.h -- C ABI of libthermal_b200.so: the steady Q1 heat-conduction
 * solve of pcb-analysis's thermal package (matrix-free trilinear hexahedral FEM
 * on the layered board grid, MPIR around a Jacobi-preconditioned PCG), built for
 * NVIDIA B200 (sm_100a).
 *
 * Conventions
 *   - Every function returns an int status (TB_OK == 0).  No C++ exception
 *     crosses this boundary; tb_last_error() returns the message of the last
 *     failure on the calling thread.
 *   - Host arrays are caller-owned, C-contiguous, and are copied in or out.
 *     Node arrays are flat in the reference's node order
 *     (z * (rows + 1) + y) * (cols + 1) + x, z = 0 at the bottom of the stack;
 *     element arrays are (slabs, rows, cols) in C order.
 *   - A system is device-resident: its coefficients, masks and iterates live in
 *     HBM behind the handle, and it owns one CUDA stream.  Calls on different
 *     systems may run from different threads; calls on one system must not
 *     overlap.
 *   - The *_device entry points take device pointers (flat node order) and run
 *     on the system's stream; they are the form to use when the inputs are
 *     already resident in HBM.
 */
#ifndef THERMAL_B200_H
#define THERMAL_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The Python facade maps them to ValueError, RuntimeError,
 * RuntimeError, TimeoutError, MemoryError and FloatingPointError. */
enum {
    TB_OK = 0,
    TB_EINVAL = 1,      /* invalid input (shapes, values, sizes)            */
    TB_ENOTSPD = 2,     /* inner PCG met a non-positive or non-finite pAp   */
    TB_ECUDA = 3,       /* CUDA runtime or launch failure                    */
    TB_ETIMEOUT = 4,    /* a bounded device wait ran out                     */
    TB_ENOMEM = 5,      /* device allocation or admission budget exceeded    */
    TB_ENONFINITE = 6,  /* non-finite values where finite ones are required  */
    TB_ENOTSUP = 7      /* feature not available in this library             */
};

typedef struct tb_system tb_system;

/* The prepared linear system of one board.
 *
 * Replaces the reference's prepared ThermalSystem
 * (cpp/src/thermal/thermal_system.cpp:252-363) and the non-owning
 * OperatorView it hands to the kernels
 * (cpp/include/pcbcore/fem/thermal_hex.hpp:16-30), plus the device upload of
 * make_thermal_hex (cpp/cuda/inner_pcg.cu:619-686).  Unlike OperatorView the
 * coefficients are given as conductivities and grid pitches, not as the three
 * premultiplied element factors: the device keeps 8 bytes per element in FP32
 * and recomputes a_x, a_y, a_z from per-slab, per-row and per-column geometry.
 */
typedef struct {
    int32_t slabs;                    /* element layers (z), >= 1                */
    int32_t rows;                     /* element rows (y), >= 1                  */
    int32_t cols;                     /* element columns (x), >= 1               */
    const double* slab_thickness_m;   /* (slabs) bottom to top                   */
    const double* pitch_x_m;          /* (cols)                                  */
    const double* pitch_y_m;          /* (rows)                                  */
    const double* k_in;               /* (slabs*rows*cols) in-plane W/mK, 0 void */
    const double* k_z;                /* (slabs*rows*cols) through-plane W/mK    */
    const double* robin_total;        /* (nodes) lumped Robin conductance + C/dt */
    const uint8_t* free_nodes;        /* (nodes) 1 free, 0 fixed or void-only    */
} tb_system_desc;

/* MPIRConfig (reference src/electrical/matrix_free_mpir_fem/solver.py:52-79,
 * cpp/include/pcbcore/fem/mpir.hpp:11-20). */
typedef struct {
    double relative_tolerance;
    double absolute_tolerance;
    double inner_relative_tolerance;
    int32_t max_outer_iterations;
    int32_t max_inner_iterations;
} tb_mpir_config;

/* MPIRResult without the solution and history arrays
 * (reference solver.py:90-100, mpir.hpp:22-35). */
typedef struct {
    int32_t converged;
    int32_t outer_iterations;
    int32_t inner_iterations;
    int32_t high_operator_applications;
    int32_t low_operator_applications;
    int32_t history_length;           /* entries written to the history array */
    double relative_residual;
} tb_mpir_result;

/* MPIRStep (reference solver.py:82-87). */
typedef struct {
    int32_t outer_iteration;
    int32_t inner_iterations;
    double high_relative_residual;
    double inner_relative_residual;
} tb_mpir_step;

/* Result of the plain FP64 Jacobi PCG. */
typedef struct {
    int32_t converged;
    int32_t iterations;
    double relative_residual;         /* true residual ||b - A x|| / ||b||     */
} tb_pcg_result;

/* Library version string and the compute capability it was built for. */
const char* tb_version(void);

/* Message of the last failed call on this thread ("" if none). */
const char* tb_last_error(void);

/* Number of visible CUDA devices (0 when there is no driver or device). */
int tb_device_count(int32_t* count);

/* Upload and prepare a system on `device`: packs the element conductivities
 * into FP32 and FP64 device arrays, builds the FP64 diagonal on the device
 * (bit-identical to the reference's _build_diagonal, operator.py:290-306 /
 * thermal_system.cpp:328-349) and its FP32 reciprocal for the Jacobi step.
 * Fails with TB_EINVAL when a free node has non-positive conductance. */
int tb_system_create(const tb_system_desc* desc, int32_t device, tb_system** out);
int tb_system_destroy(tb_system* system);

/* Node count (slabs+1)*(rows+1)*(cols+1) and device bytes held by the system. */
int tb_system_info(const tb_system* system, int64_t* nodes, int64_t* device_bytes);

/* y = A x, A = where(free, K (x * free) + R x, x): the FP32 low action
 * (reference apply_low, operator.py:349-361; hex_q1.cpp:503-509) and the FP64
 * high action (apply_high, operator.py:308-316; thermal_hex.hpp:32-39). */
int tb_apply_f32(tb_system* system, const float* x, float* y);
int tb_apply_f64(tb_system* system, const double* x, double* y);
int tb_apply_f32_device(tb_system* system, const float* d_x, float* d_y);
int tb_apply_f64_device(tb_system* system, const double* d_x, double* d_y);

/* y = K x, the unconstrained conduction action with every node free and no
 * Robin term (reference ThermalSystem::stiffness, thermal_system.cpp:372-374;
 * operator.py _stiffness_action:243-269), used by build_rhs and the heat
 * budget. */
int tb_stiffness_f64(tb_system* system, const double* x, double* y);

/* The FP64 Jacobi diagonal built on the device (fixed rows hold 1). */
int tb_diagonal(tb_system* system, double* diagonal);

/* Mixed-precision iterative refinement: FP64 residual, norm and update on the
 * device, FP32 Jacobi PCG for each correction with compensated dot products.
 * Replaces solve_mpir (reference solver.py:580-698; hex_q1.cpp:837-925;
 * inner_pcg.cu:688-728) and the native_solve_mpir hook (operator.py:318-347).
 * `x` holds the initial guess on entry (zeros when the caller has none) and
 * the solution on return.  `history` may be NULL; at most `history_capacity`
 * steps are written.  Returns TB_ENOTSPD when the inner PCG meets a
 * non-positive curvature, as the reference raises RuntimeError. */
int tb_solve_mpir(tb_system* system, const double* rhs, double* x, const tb_mpir_config* config,
                  tb_mpir_result* result, tb_mpir_step* history, int32_t history_capacity);
int tb_solve_mpir_device(tb_system* system, const double* d_rhs, double* d_x, const tb_mpir_config* config,
                         tb_mpir_result* result, tb_mpir_step* history, int32_t history_capacity);

/* Plain FP64 Jacobi PCG on the device (no refinement), the single-solve GPU
 * baseline: stops when the recursive residual reaches
 * absolute_tolerance + relative_tolerance * ||b|| and reports the true one. */
int tb_solve_pcg_f64(tb_system* system, const double* rhs, double* x, double relative_tolerance,
                     double absolute_tolerance, int32_t max_iterations, tb_pcg_result* result);
int tb_solve_pcg_f64_device(tb_system* system, const double* d_rhs, double* d_x, double relative_tolerance,
                            double absolute_tolerance, int32_t max_iterations, tb_pcg_result* result);
/* The same FP64 PCG preconditioned by the system's multilevel operator (kind 2
 * of tb_set_preconditioner; TB_EINVAL otherwise): FP64 vectors, inner
 * products and updates, the preconditioner applied in FP32 to f32(r) and its
 * result widened to FP64.  No reference counterpart: the like-for-like FP64
 * baseline of the multilevel MPIR solve. */
int tb_solve_pcg_f64_ml(tb_system* system, const double* rhs, double* x, double relative_tolerance,
                        double absolute_tolerance, int32_t max_iterations, tb_pcg_result* result);
int tb_solve_pcg_f64_ml_device(tb_system* system, const double* d_rhs, double* d_x, double relative_tolerance,
                               double absolute_tolerance, int32_t max_iterations, tb_pcg_result* result);

/* Test only, no reference counterpart: exercises the give-up path of the
 * tensor-copy staging without a GPU fault.  With polls > 0 the issuing thread
 * of every FP32 operator block arms each stage barrier but issues no copy,
 * and each wait gives up after `polls` polls; every block then records the
 * timeout and returns with nothing in flight, and the apply or solve fails
 * with TB_ETIMEOUT.  0 restores normal staging.  Affects launch plans with
 * tensor-copy staging only (tb_set_apply_plan). */
int tb_set_stage_test(tb_system* system, int32_t polls);

/* Launch form of the multilevel preconditioner's fine pass in the inner FP32
 * PCG iterations (no reference counterpart; the reference's preconditioners
 * are Jacobi and two-level): staged = 1 runs the persistent kernel whose
 * column boxes (32 x 8 node columns, every plane, of q, r and the z-line
 * factors) are copied by tensor copies several tiles ahead of the one
 * computed; 0 the kernel that loads its columns itself.  The same arithmetic
 * per column; the two differ only in the order in which r.r and r.T^-1 r are
 * merged.  The staged form is available where the board's boxes fit in
 * shared memory (at least two stages; elsewhere setting 1 returns
 * TB_ENOTSUP); the default is 0: the staged kernel is faster by itself
 * (c3: 0.80 of the measured copy peak against 0.69-0.76) but, holding 214 KB
 * of shared memory per SM, it slows the kernels after it more than it saves.
 * tb_get_ml_staging reports the form in use (0 also for systems without the
 * multilevel preconditioner).  tb_set_stage_test applies to the staged form
 * too. */
int tb_set_ml_staging(tb_system* system, int32_t staged);
int tb_get_ml_staging(const tb_system* system, int32_t* staged);

/* Device-time accounting, for benchmarks.  tb_set_timing(1) resets the
 * counters and switches the PCG chunks to graphs that record a CUDA event
 * around every kernel; tb_get_timing then returns the summed device time in
 * milliseconds and the number of launches that did work, by kind:
 * [0] FP32 apply (with the p.Ap epilogue), [1] FP64 apply (residual epilogue),
 * [2] PCG vector kernels (update + direction), [3] whole solve calls. */
int tb_set_timing(tb_system* system, int32_t enabled);
int tb_get_timing(const tb_system* system, double* ms4, int64_t* launches4);

/* Launch shape of the FP32 operator: plan5 = {kind, rows, zw, sl, band}.
 * kind 0: z-marching tiles of `rows` element rows (8, 16 or 32); for kinds 0
 *         and 2, plan5[2] selects how the tile stages are filled: 0 per-thread
 *         cp.async copies, 1 tensor copies (TMA) issued by one thread per
 *         block onto an mbarrier per stage (same output bits; TB_ENOTSUP where
 *         the system has no tensor maps); plan5[3] the stage count: 0 (or 4)
 *         keeps two planes in flight ahead of the one computed, 5 three (kind
 *         0 with tensor copies, 8 or 16 rows; the same output bits);
 * kind 1: warp-marching kernel, zw z groups of sl slabs per lane (zw*sl >= slabs),
 *         bands of `band` node rows; `rows` still sets the FP64 tile height;
 * kind 2: the z-marching tiles of `rows` rows launched as one wave of
 *         resident blocks that share the board's (tile, node plane) pairs
 *         evenly (same output bits as kind 0, no second partial wave).
 * Chosen at creation by timing the candidates on the board (cached per slab
 * count and board size); tb_set_apply_plan overrides the choice.
 * tb_set_tile_rows(rows) is tb_set_apply_plan({0, rows, 0, 0, 0}). */
int tb_set_apply_plan(tb_system* system, const int32_t* plan5);
int tb_get_apply_plan(const tb_system* system, int32_t* plan5);
int tb_set_tile_rows(tb_system* system, int32_t rows);
int tb_get_tile_rows(const tb_system* system, int32_t* rows);

/* Device time of the operator kernels, always on: [0] FP32 apply with the
 * p.Ap epilogue (the inner PCG), [1] FP64 apply with a reduction epilogue
 * (outer residual, FP64 PCG).  Each launch adds last-block-end minus
 * first-block-start from %globaltimer; `ns2` and `count2` are running totals
 * since creation. */
int tb_get_kernel_clock(tb_system* system, double* ns2, int64_t* count2);
/* The same for the first n (<= 3) clocks: [0] FP32 apply, [1] FP64 apply,
 * [2] the multilevel fine pass of the inner PCG (ml_update). */
int tb_get_kernel_clocks(tb_system* system, int32_t n, double* ns, int64_t* counts);

/* The CUDA stream (cudaStream_t) every kernel of this system runs on. */
int tb_system_stream(const tb_system* system, void** stream);

/* Kernels of this library launched for this system since creation
 * (graph-launched PCG chunks count every kernel node). */
int tb_get_launch_count(const tb_system* system, int64_t* count);

/* ----------------------------------------------------------- batch engine
 * Many boards resident in HBM at once, solved by MPIR in one set of batched
 * kernels (one CUDA-graph chunk = the outer-step kernels plus 16 inner PCG
 * iterations over every resident board, each board masked by its own
 * convergence state).  The outer MPIR loop of every board runs on the device
 * (reference solver.py:580-698): the host admits boards, steps the engine and
 * collects finished boards while the others keep running.  A board's result
 * depends only on the board and the tile height, not on the other boards.
 * No counterpart in the reference, which solves one board per call. */
typedef struct tb_engine tb_engine;

typedef struct {
    int32_t capacity;       /* boards resident at once, 1..256                    */
    int32_t max_slabs;      /* largest slab count admitted, 1..256                */
    int32_t tile_rows;      /* FP32 operator tile height 8, 16 or 32; 0 = timed on
                               the first boards and fixed from then on            */
    int32_t preconditioner; /* inner PCG of every board: 0 Jacobi, 1 two-level      */
    int64_t budget_bytes;   /* HBM admission budget for resident boards           */
    int32_t staging;        /* FP32 operator stages: 0 = timed with the tile height
                               when tile_rows is 0 (else cp.async), 1 = cp.async,
                               2 = tensor copies (TMA; TB_ENOTSUP without them)   */
    int32_t reserved;       /* 0                                                  */
} tb_engine_config;

int tb_engine_create(int32_t device, const tb_engine_config* config, tb_engine** out);
int tb_engine_destroy(tb_engine* engine);

/* Bytes a board holds while resident, and the extra bytes its admission
 * holds while it is prepared, in an engine with this preconditioner. */
int tb_engine_footprint(const tb_system_desc* desc, int32_t preconditioner, int64_t* resident_bytes,
                        int64_t* transient_bytes);

/* Admit a board: upload and prepare it on the engine's I/O stream (the
 * inputs are copied before the call returns), then enter it into the next
 * chunk.  `x0` may be NULL (zeros).  Fails with TB_ENOMEM, changing nothing,
 * when no slot is free or its bytes do not fit the budget: the caller keeps
 * the request and submits it again after collecting others. */
int tb_engine_submit(tb_engine* engine, const tb_system_desc* desc, const double* rhs, const double* x0,
                     const tb_mpir_config* config, int64_t* ticket);

/* Launch one graph chunk over the resident boards (two are kept in flight)
 * and read the board states of the oldest one; `finished` receives the
 * number of finished boards not yet collected. */
int tb_engine_step(tb_engine* engine, int32_t* finished);

/* Tickets of finished boards not yet collected (up to `capacity` of them);
 * `count` receives how many there are. */
int tb_engine_finished(tb_engine* engine, int64_t* tickets, int32_t capacity, int32_t* count);

/* Copy a finished board's solution (node order, may be NULL), result and
 * history out and release its slot and memory.  Returns TB_ENOTSPD for a
 * board whose inner PCG met a non-SPD operator (the slot is released too). */
int tb_engine_collect(tb_engine* engine, int64_t ticket, double* x, tb_mpir_result* result,
                      tb_mpir_step* history, int32_t history_capacity);

/* Device time (ms) of one batched FP32 operator launch over every resident
 * board not yet finished, averaged over `launches` launches after a warm-up
 * (store epilogue, between chunks); for the roofline of the batched path. */
int tb_engine_time_apply(tb_engine* engine, int32_t launches, double* ms_per_launch);

/* The CUDA stream (cudaStream_t) the engine's graph chunks run on. */
int tb_engine_stream(const tb_engine* engine, void** stream);

/* [resident boards, boards in the schedule, bytes in use, budget, chunks
 * launched, kernels launched, FP32 tile height, capacity]. */
int tb_engine_info(const tb_engine* engine, int64_t* info8);
/* Staging of the batched FP32 operator in use: 1 cp.async, 2 tensor copies. */
int tb_engine_staging(const tb_engine* engine, int32_t* staging);

/* Replace the lumped Robin totals of a prepared system (node order, the
 * free mask is kept): the backward-Euler step adds C / dt where the Robin
 * conductance sits (reference transient.py:1-24) and the radiation Newton step
 * adds its linearisation (solve.py:126-168).  The Robin/fixed field, the
 * Jacobi diagonal and, with the two-level preconditioner, the coarse operator
 * are rebuilt on the device, so a transient march keeps one resident system
 * instead of preparing a new one per step (the reference's C++ march reuses
 * its prepared system while dt repeats, thermal_solve.cpp:165-324). */
int tb_set_robin(tb_system* system, const double* robin_total);

/* Preconditioner of the inner FP32 PCG: kind 0 Jacobi (the default), kind 1
 * the reference's default two-level preconditioner D^-1 r + Z (Z^T A Z)^-1 Z^T r
 * with patch-constant coarse functions on b x b node patches of each node
 * layer (reference two_level.py:62-229, hex_q1.cpp:388-432,703-835,
 * inner_pcg.cu:352-407).  `coarse_block_nodes` 0 picks the smallest patch
 * width >= 4 whose coarse grid has at most 2048 patches (two_level.py:36-50).
 * Z^T A Z is assembled on the device from 27 coloured FP64 actions and
 * inverted there; fails with TB_EINVAL when it is not positive definite. */
int tb_set_preconditioner(tb_system* system, int32_t kind, int32_t coarse_block_nodes);
/* Kind 2, the multilevel preconditioner, has no reference counterpart; it
 * takes the place of kind 1 on boards whose two-level patches would be too
 * wide (the reference's own note for boards beyond a few hundred thousand
 * nodes, docs/THERMAL_MPIR_FEM.md:619-621):
 *     M^-1 r = T^-1 r + Z_1 V_1(Z_1^T r),
 * T the z-line block (each node column's tridiagonal coupling along z,
 * solved exactly), Z_1 the patch-constant functions of kind 1 at a patch
 * width of 4, and V_1 one symmetric V-cycle over Galerkin coarse grids of
 * 2 x 2 aggregates of the level above (damped z-line smoothing, the last grid
 * of at most 2048 unknowns inverted densely).  Thermal systems of at most 32
 * slabs;
 * `coarse_block_nodes` is ignored. */
/* {kind, patch width, node layers, patches along y, patches along x}; for
 * kind 2 the grid is the coarsest (densely inverted) one. */
int tb_get_preconditioner(const tb_system* system, int32_t* info5);
/* Kind 2 only: *count coarse grids, and up to `cap` of their shapes
 * {node layers, rows, columns} into dims (3 per grid, level 1 first). */
int tb_get_multilevel(const tb_system* system, int32_t* dims, int32_t cap, int32_t* count);
/* Kind 2 only: the FP32 stencil of coarse grid `level` (1 .. count - 1; the
 * last grid is held as a dense inverse), 14 arrays of the grid's node count:
 * array k holds A(i, i + d(o)) for o = 13 + k, o = 9 (dz+1) + 3 (dy+1) + (dx+1),
 * node i = (layer * rows + row) * columns + column. */
int tb_get_multilevel_stencil(tb_system* system, int32_t level, float* stencil);
/* Z^T A Z and its symmetrised inverse (row-major, n x n with n the patch
 * count), either pointer may be NULL; kind 1, or the coarsest grid of kind 2. */
int tb_get_coarse(tb_system* system, double* matrix, double* inverse);
/* y = M^-1 x with the FP32 two-level preconditioner (the reference's
 * precondition_low, operator.py:366-371), or the multilevel one (kind 2). */
int tb_precondition_f32(tb_system* system, const float* x, float* y);

/* ------------------------------------------------------------ problems
 * A board given as its conduction problem instead of prepared arrays.  The
 * device builds what the reference's host code prepares
 * (src/thermal/matrix_free_mpir_fem/operator.py:86-128,374-440 and
 * boundaries.py:82-183; cpp/src/thermal/thermal_system.cpp:146-250,411-436):
 * node masks, the lumped Robin conductance and R T_amb of every convection
 * boundary, the nodal heat load and the right-hand side, each with the
 * reference's operation order, so the arrays carry the reference's bits; and
 * after a solve its post-processing (operator.py:443-525, solve.py:255-280). */

enum { TB_CONVECTION_FACE = 0, TB_CONVECTION_EXPOSED = 1 };
#define TB_MAX_CONVECTION 64

/* One convection boundary (reference boundaries.py:35-183).
 * TB_CONVECTION_FACE: ConvectionBoundary, one outer face of the stack (side 0
 *   bottom, 1 top); fields are (rows, cols).
 * TB_CONVECTION_EXPOSED: ExposedFaceConvection, every face of an active
 *   element whose neighbour is void or outside, for the listed directions in
 *   order (0 -x, 1 +x, 2 -y, 3 +y, 4 -z, 5 +z); fields are (slabs, rows, cols).
 * A NULL field takes the scalar beside it. */
typedef struct {
    int32_t kind;
    int32_t side;
    int32_t direction_count;
    int32_t directions[6];
    double coefficient_w_per_m2_k;
    double ambient_temperature_k;
    const double* coefficient_field;
    const double* ambient_field;
} tb_convection_desc;

/* ThermalConductionProblem (reference solve.py / problem model) with its
 * mesh (mesh.py:127-343).  Optional arrays may be NULL. */
typedef struct {
    int32_t slabs, rows, cols;
    const double* slab_thickness_m;     /* (slabs)                                  */
    const double* pitch_x_m;            /* (cols)                                   */
    const double* pitch_y_m;            /* (rows)                                   */
    const double* k_in;                 /* (slabs*rows*cols), 0 on void elements    */
    const double* k_z;                  /* (slabs*rows*cols)                        */
    const uint8_t* active;              /* (slabs*rows*cols) or NULL: all exist     */
    const uint8_t* fixed_mask;          /* (nodes) or NULL                          */
    const double* fixed_temperature_k;  /* (nodes), read where fixed_mask is set    */
    const double* nodal_heat_w;         /* (nodes) or NULL                          */
    const double* element_heat_w;       /* (slabs*rows*cols) or NULL                */
    int32_t source_entries;             /* heat sources: one entry per source node, */
    const int64_t* source_nodes;        /*   flat node index, in source order       */
    const double* source_node_w;        /*   power / node count of its source       */
    int32_t convection_count;           /* <= TB_MAX_CONVECTION                     */
    const tb_convection_desc* convection;
    const double* capacity_per_s;       /* (nodes) C / dt of a backward-Euler step, */
                                        /*   or NULL for a steady solve             */
} tb_problem_desc;

/* Prepare a problem on the device and make its system (as tb_system_create
 * with the Robin totals and free mask the device computed). */
int tb_system_create_problem(const tb_problem_desc* desc, int32_t device, tb_system** out);
/* Replace the convection boundaries (the radiation Newton step's
 * linearisation, reference solve.py:126-168) or the C / dt term (a new
 * transient step size, transient.py:196-212) of a problem system; the Robin
 * totals, diagonal and coarse operator are rebuilt on the device.
 * tb_set_robin is refused on a problem system. */
int tb_set_convection(tb_system* system, const tb_convection_desc* convection, int32_t count);
int tb_set_capacity(tb_system* system, const double* capacity_per_s);
/* The prepared arrays (nodes each; any pointer may be NULL): Robin
 * conductance, Robin total (conductance + C / dt), sum of R T_amb, nodal load,
 * free mask (not fixed and active) and active-node mask. */
int tb_get_prepared(tb_system* system, double* robin_only, double* robin_total, double* robin_rhs, double* load,
                    uint8_t* free_nodes, uint8_t* active_nodes);
/* One boundary's lumped conductance and R T_amb over all nodes. */
int tb_get_boundary_weights(tb_system* system, int32_t index, double* weights, double* rhs_weights);
/* Right-hand side of the solve for the rise above the reference temperature
 * (reference operator.py:411-440): q + R T_amb - R_total T_ref + C/dt T_prev
 * - K (fixed rise) on free rows, the fixed rise on fixed rows.
 * previous_temperature_k (nodes) is required when C / dt is positive. */
int tb_build_rhs(tb_system* system, double reference_temperature_k, const double* previous_temperature_k,
                 double* rhs);
/* Post-processing of a temperature field (nodes, K; reference operator.py:
 * 443-525 and solve.py:255-280):
 *   heat_flux (slabs*rows*cols*3): -k grad T at element centres, 0 on void;
 *   convective_heat (one per boundary): heat each boundary removes, W;
 *   budget3: {total heat input, heat through fixed nodes, stored heat}, W;
 *   residual (nodes): the unconstrained residual K T + R (T - T_amb)
 *     + C/dt (T - T_prev) - q.
 * Any output may be NULL.  Flux and residual carry the reference's bits for
 * the same temperature; the sums are compensated and agree with the
 * reference's NumPy sums within their rounding error. */
int tb_postprocess(tb_system* system, const double* temperature_k, const double* previous_temperature_k,
                   double* heat_flux, double* convective_heat, double* budget3, double* residual);

/* Device-resident forms of the two calls above (no reference counterpart:
 * the reference's operator takes and returns host arrays).  A solve that
 * keeps its right-hand side and its solution in HBM calls them with flat
 * (nodes) device arrays of the system's device:
 *   tb_build_rhs_device writes the right-hand side of tb_build_rhs into
 *     `rhs` (device); previous_temperature_k is a device array or NULL;
 *   tb_postprocess_rise_device post-processes T = rise + reference, `rise`
 *     being the device solution of tb_solve_mpir_device for that reference;
 *     previous_temperature_k and the outputs are host arrays as in
 *     tb_postprocess, plus temperature_k (nodes; may be NULL): T itself,
 *     and extrema2 (may be NULL): {min, max} of T over the active nodes
 *     (NumPy's nanmin / nanmax of T with NaN on void nodes);
 *   tb_download copies `bytes` of a device array of the system's device to
 *     a host array, after the work queued on the system's stream.
 * The first two give the bits of the host-array calls for the same data. */
int tb_build_rhs_device(tb_system* system, double reference_temperature_k, const double* previous_temperature_k,
                        double* rhs);
int tb_postprocess_rise_device(tb_system* system, const double* rise, double reference_temperature_k,
                               const double* previous_temperature_k, double* heat_flux, double* convective_heat,
                               double* budget3, double* residual, double* temperature_k, double* extrema2);
int tb_download(tb_system* system, void* host, const void* device_array, size_t bytes);

/* ------------------------------------------------------- layered DC
 * DC conduction in layered PCB copper (reference
 * src/electrical/matrix_free_mpir_fem/pcb.py:105-621; C++ LayeredDCSystem,
 * cpp/src/fem/layered_dc_system.cpp and native/layered_dc_q1.cpp): bilinear
 * sheet elements of conductance sigma t on each layer plus resistive vias
 * between layer nodes, on the same solver as the thermal operator.  Node n of
 * layer l, row y, column x is (l * (rows + 1) + y) * (cols + 1) + x.
 *
 * The system answers tb_apply_*, tb_stiffness_f64 (the unconstrained
 * conductance action K v, the reference's apply_full_high), tb_diagonal,
 * tb_solve_mpir*, tb_solve_pcg_f64*, tb_set_preconditioner (the same
 * patch-constant two-level preconditioner on the (layers, rows+1, cols+1)
 * node grid) and the timing calls.  The thermal-only entry points refuse it. */
typedef struct {
    int32_t layers, rows, cols;             /* element grid, >= 1 each              */
    const double* layer_thickness_m;        /* (layers)                             */
    const double* pitch_x_m;                /* (cols)                               */
    const double* pitch_y_m;                /* (rows)                               */
    const double* conductivity_s_per_m;     /* (layers*rows*cols), > 0              */
    const uint8_t* element_active;          /* (layers*rows*cols)                   */
    int32_t via_count;
    const int64_t* via_lower;               /* flat node of each via's lower end    */
    const int64_t* via_upper;               /* flat node of its upper end           */
    const double* via_conductance_s;        /* 1 / resistance                       */
    int64_t reference_node;                 /* flat node fixing the gauge, or -1    */
    int32_t dirichlet_count;
    const int64_t* dirichlet_nodes;         /* nodes held at a fixed potential      */
} tb_dc_desc;

/* Prepare a layered DC system: active nodes (corners of active elements and
 * via ends), fixed nodes (inactive, the reference node, the Dirichlet nodes),
 * the diagonal bit-identical to the reference's _build_diagonal
 * (pcb.py:598-617).  TB_EINVAL with the reference's messages for a reference
 * or Dirichlet node off the copper and for a free node without conductance. */
int tb_dc_system_create(const tb_dc_desc* desc, int32_t device, tb_system** out);
/* Active and free node masks (nodes each, 0/1; either may be NULL). */
int tb_dc_get_masks(tb_system* system, uint8_t* active_nodes, uint8_t* free_nodes);
/* Post-processing of a DC potential (reference pcb.py:810-848,
 * MatrixFreePCBOperator.element_electric_field and element_joule_loss): from
 * the potential (nodes, node order) it writes the element-centre field
 * (layers*rows*cols*2, x then y, V/m, zero on void elements) and each
 * element's Joule loss c_x v^T U_x v + c_y v^T U_y v (layers*rows*cols, W). */
int tb_dc_post(tb_system* system, const double* potential, double* field, double* element_loss);

/* Allocation-free FP64 residual; it has no counterpart in the reference.
 * For callers that may not allocate device memory while they run: a host
 * program whose device memory is owned by another allocator (a framework's
 * caching allocator, or an arena sized once at start-up that must not be
 * bypassed), and latency-critical loops where cudaMalloc / cudaFree would
 * stall on an implicit device synchronisation.  It computes
 * r = b - A x with the FP64 high action (device pointers, node order) and
 * returns norms2 = {||r||^2, max |r|} on the host, with the same kernel as the
 * outer MPIR step; the kernel's block partials, ticket counter and result
 * scalars sit in one statically allocated device array of 256.5 KiB that
 * every GPU which loads this library holds until the process exits, instead
 * of scratch owned by the system.  The call allocates nothing.
 * - The array holds partials for at most 8192 operator tiles (at 16-row
 *   tiles, about 7.3 million nodes per plane); larger boards fail with
 *   TB_EINVAL before anything is launched.
 * - The first call on a device looks the array's device address up
 *   (cudaGetSymbolAddress, with that device current); make that first call
 *   before any stream capture on the device.
 * - The array keeps what the last call left; every call zeroes the ticket
 *   counter on the system's stream before its launch and waits for the
 *   stream before returning.
 * - All calls share the one array: calls that overlap on the GPU (from other
 *   threads or other systems on the same device) race; serialise them.
 * - The call also works in the system's own FP64 vectors (it copies x and b
 *   into them and computes r there), so a solve or another call on the same
 *   system that runs at the same time races with it too.
 * - The cached address belongs to the device's primary context; do not use
 *   the entry point after cudaDeviceReset on that device in this process. */
int tb_residual_f64_device_static(tb_system* system, const double* d_x, const double* d_b, double* d_r,
                                  double* norms2);

#ifdef __cplusplus
}
#endif

#endif /* THERMAL_B200_H */
