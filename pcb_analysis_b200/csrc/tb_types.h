// Types shared by the device kernels and the host orchestration.
#pragma once

#include <stdint.h>

namespace tb {

// State of a running PCG (the inner solve of MPIR, or the plain FP64 PCG).
enum InnerState : int {
    ST_RUNNING = 0,
    ST_CONVERGED = 1,   // recursive residual met the tolerance
    ST_NOT_SPD = 2,     // p.Ap non-positive or non-finite
    ST_BREAKDOWN = 3,   // r.z non-finite or previous r.z zero: stop as the reference does
    ST_MAXIT = 4,       // iteration limit reached
    ST_ZERO_RHS = 5,    // right-hand side is zero: correction is zero
    ST_STAGE_TIMEOUT = 6,  // an operator block gave up waiting for its staged tiles
};

// Scalars of one solve, resident in device memory.  Written only by the last
// block of a reduction kernel and read by the kernels that follow on the same
// stream, so the host never has to take part in an iteration.
struct SolveCtl {
    // PCG
    double rz;          // r . z of the current residual
    double pq;          // p . Ap of the current direction
    double rr;          // r . r after the last update
    double bnorm;       // ||b|| the relative residual is taken against (0: use ||r0||)
    double rel;         // ||r|| / bnorm after the last update
    double alpha;
    double beta;
    double tol;         // stop when rel <= tol
    int iterations;
    int applications;
    int state;
    int max_it;
    // outer FP64 residual
    double res2;        // ||b - A x||^2
    double peak;        // max |b - A x|
    double scale;       // power-of-two scale of the current inner right-hand side
    double inv_scale;
    double norm2;       // result of a plain norm kernel
    double rdr;         // sum r^2 / d of the current residual (two-level PCG)
    double pad[2];
};

// Device-side duration of one kernel kind, from %globaltimer: the first block
// to start lowers `first`, the last block to finish adds now - first to
// `total_ns` and resets `first`.  Costs one atomic per block, so it stays on.
struct KernelClock {
    unsigned long long first;     // ~0 between launches
    unsigned long long total_ns;
    unsigned long long count;
    unsigned long long pad;
};

}  // namespace tb
