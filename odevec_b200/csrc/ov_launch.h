/* Launch arguments shared by the kernels and the C-ABI layer. */
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ov {

struct LaunchArgs {
    int64_t ncells;
    /* row stride of y and ws in cells (>= ncells): the full arrays' cell
       count when a launch covers a range of their cells */
    int64_t stride;
    double* y;             /* [neq][stride] */
    double* t;             /* [ncells] */
    double* dt;            /* [ncells] */
    const double* t_stop;  /* [ncells] */
    const uint8_t* mask;   /* [ncells] or null */
    int32_t* status;       /* [ncells] or null */
    int32_t* stats;        /* [ncells][OV_NSTATS] or null */
    unsigned long long* queue; /* work counter, zero at launch */
    double rtol, atol, dt_min;
    int32_t check_neg;
    int32_t max_attempts;
    /* per-cell control (G = 1) on staging 1: the Jacobian+LU and the
       step-size selection run for all waiting lanes of a warp at once when at
       least this many lanes wait, when no lane of the warp can progress
       otherwise, or when a lane has waited max_wait trips (the other
       stagings run them on fixed trips, StageCfg::PERIOD) */
    int32_t jac_batch;
    int32_t ss_batch;
    int32_t max_wait;
    int32_t fix_restart; /* undo the prediction before an order-1 restart */
    /* resident integrator state (continuation across calls): ws = null for
       none; otherwise ws holds ws_doubles(ND) doubles per cell, [field][cell],
       written at the end of every successful solve and, with resume = 1,
       read at the start instead of a fresh start; with resume = 2 the start
       is fresh but takes en_old (the previous call's last correction) from
       it, as the reference's solver object keeps this%en_old between calls */
    double* ws;
    int32_t resume;
    /* if non-null, the kernel returns at once unless *run_if != 0 (a count
       written by an earlier kernel on the same stream) */
    const unsigned long long* run_if;
    /* if non-null, every cell's inputs y (all species), t and dt are copied
       here as the cell is loaded ([neq][ncells], [ncells], [ncells], packed):
       the FP32-LU form's escalation restores failed cells from them, without
       a separate copy of the inputs (which may be host memory) */
    double* save_y;
    double* save_t;
    double* save_dt;
    /* if non-null and nonzero when a warp (or lane group) is about to take
       new cells -- on any refill trip after its first -- it takes none:
       the launch ends once its running cells are done, the cells not
       started stay untouched, and a later launch on the same work counter
       continues with them (read with a volatile load: device memory or
       pinned, mapped host memory) */
    const int32_t* yield;
    /* per-cell control only: if non-null, the q-th cell taken from the work
       counter is cell order[q] (a permutation of 0..ncells-1), so cells are
       visited in that order; results do not depend on it */
    const int32_t* order;
};

/* Several solves of different networks in one launch (the multi-network
   kernel): job j's launch arguments, the index of its network in the
   kernel's network list, and its first block; a block starts with the job
   whose block range holds it and then drains the other jobs' work counters
   in turn, so blocks whose job is done help the others. */
constexpr int MULTI_MAX_JOBS = 8;
struct MultiArgs {
    LaunchArgs job[MULTI_MAX_JOBS];
    int32_t net[MULTI_MAX_JOBS];
    int32_t block_start[MULTI_MAX_JOBS + 1];
    int32_t njobs;
};
typedef cudaError_t (*multi_fn)(MultiArgs& P, int lu, cudaStream_t stream);

/* doubles per cell of the resident workspace: history y_NS(0:5), en_old,
   error weights, and 12 scalars (internal time, step, control state) */
__host__ __device__ constexpr int ws_doubles(int nd) { return 6 * nd + 2 * nd + 12; }

/* one launcher per network variant and arithmetic mode; returns the CUDA
   error of the launch.  G: 1 or 32; lu: 0 = FP64 LU, 1 = FP32 LU;
   stage: 1 = thread-local arrays, 2 = shared-memory arrays (per-cell
   control only; cudaErrorNotSupported where the arrays do not fit).
   block/grid 0: default (persistent grid from the occupancy). */
typedef cudaError_t (*launch_fn)(const LaunchArgs& a, int G, int lu, int stage, int block,
                                 int grid, cudaStream_t stream);

}  // namespace ov
