/* odevec_b200: C ABI of the B200 OdeVec solve path.
 *
 * This is the boundary a Fortran, C or Python caller binds in place of the
 * reference's solver module src/odevec.F90.  Plain pointers and sizes only.
 *
 *   reference (src/odevec.F90)                     this ABI
 *   InitOdevec(this)                  :94-154      odevec_init
 *   this%RelativeTolerance, %AbsoluteTolerance,
 *   %MinimalTimestep, %CheckNegatives  :48-52       odevec_opts
 *   SolveODE(this,time,dt,t_stop,y,
 *            GetRHS,GetJac,GetLU,Mask) :158-214     odevec_solve (device arrays)
 *                                                  odevec_solve_host (host arrays)
 *   CloseOdevec(this)                 :1058-1074   odevec_close
 *   print + stop on failure   :114-124,272-287,380-390,585-597
 *                                                  per-cell status codes below
 *
 * The network routines GetRHS/GetJac/GetLU are compiled into the library by
 * the preprocessor (one "variant" per network, packaging and ordering) and
 * chosen by name at odevec_init.
 *
 * Layout: y holds neq species of ncells cells, species-major ("structure of
 * arrays"): y[s * ncells + c] -- the reference's y(nvector, neq) in Fortran
 * column-major order.  t, dt, t_stop, mask and status have one entry per
 * cell; stats has OV_NSTATS int32 entries per cell (cell-major).
 *
 * Cells are solved independently (group_size 1) or in lockstep groups of 32
 * consecutive cells sharing time, step size, order and Jacobian decisions
 * through max-norms over the group (group_size 32), which is the
 * reference's semantics with nvector = 32.  A lockstep group needs equal t,
 * dt and t_stop in all its cells. */
#ifndef ODEVEC_B200_H
#define ODEVEC_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- per-cell status (replaces the reference's `stop`) ---- */
#define OV_OK 0
#define OV_ERR_DTMIN_PREDICTOR 1 /* step below dt_min after a negative prediction, :272-275 :284-287 */
#define OV_ERR_CONV_FAILURES 2   /* more than 10 Newton failures in one step, :380-383 */
#define OV_ERR_DTMIN_CONV 3      /* step below dt_min after a Newton failure, :387-390 */
#define OV_ERR_MAX_STEPS 4       /* predictor attempts exceeded opts.max_attempts (no reference counterpart) */
#define OV_ERR_ORDER 5           /* impossible order change, :585-586 :596-597 */
#define OV_ERR_GROUP_MISMATCH 6  /* lockstep group with differing t, dt or t_stop */

/* ---- API return codes ---- */
#define OV_API_OK 0
#define OV_API_EINVAL (-1)      /* bad argument */
#define OV_API_ENONET (-2)      /* unknown network variant */
#define OV_API_ECUDA (-3)       /* CUDA runtime error (see odevec_last_error) */
#define OV_API_ENOMEM (-4)      /* allocation failed */
#define OV_API_EUNSUPPORTED (-5) /* option combination not compiled in */
#define OV_API_ETOOBIG (-6)     /* more cells than the solver was created for */

/* stats per cell: accepted steps, predictor attempts, error-test failures,
   Newton failures, Newton iterations (right-hand-side evaluations in the
   corrector), Jacobian+LU evaluations, final order, and the number of
   Nordsieck vector passes of the Pascal-triangle predictor and its undo
   (sum of q(q+1)/2 over PredictSolution and ResetSystem calls) */
#define OV_NSTATS 8

/* precision forms */
#define OV_PREC_FP64 0     /* FP64 throughout, no fused multiply-add: same bits as the CPU oracle */
#define OV_PREC_FP64_FMA 1 /* FP64 throughout with fused multiply-add */
#define OV_PREC_FP32_LU 2  /* Jacobian LU and triangular solves in FP32 on the error-weight-scaled
                              matrix; state, residual, norms and control in FP64 */

typedef struct odevec_opts {
    double rtol;              /* RelativeTolerance */
    double atol;              /* AbsoluteTolerance */
    double dt_min;            /* MinimalTimestep; negative: the variant's --dt_min */
    int32_t check_negatives;  /* CheckNegatives */
    int32_t group_size;       /* 1 or 32; 0: the variant's --nvector (1 if not 32) */
    int32_t precision;        /* OV_PREC_* */
    int32_t max_attempts;     /* cap on predictor attempts per cell or group; 0: 1000000 */
    /* scheduling of per-cell control (group_size 1) on staging 1, no effect
       on results: the Jacobian+LU and the step-size selection run for the
       waiting cells of a warp together once jac_batch / ss_batch of its 32
       cells wait, no other cell can progress, or a cell has waited max_wait
       iterations.  0: defaults (24, 24, 8); 1, 1, -1 runs each cell's block
       at once.  Stagings 2-21 ignore them: they run the two blocks on fixed
       trips (every 4th trip each, the same trips in all warps of a block). */
    int32_t jac_batch;
    int32_t ss_batch;
    int32_t max_wait;
    /* launch shape, no effect on results.  staging: 0 = automatic (the
       library's tuning table for this GPU where it has the variant, else 3
       for per-cell control up to 32 species, 1 above and for lockstep); 1 = per-cell arrays in registers /
       local memory, 2 blocks of 128 threads per SM; 2 = history and LU in
       shared memory, 1 block of 128 (where they fit); 3, 4 = as 1 with 3 or 4
       blocks per SM (fewer registers, more warps); 5 = as 2 with 192-thread
       blocks (FP32 LU); 6 = as 3 in one block of 384 threads per SM; 7 = one
       warp per cell (lanes share a cell's species; constant-coefficient
       networks in CSC packaging); 8 = as 6 with the block's warps held in
       soft lockstep at the top of every trip (bounded polling, no barrier);
       9, 10 = soft lockstep in one block of 256 or 320 threads per SM with the
       history in shared memory (where it fits); 11 = soft lockstep in one
       block of 192 with history and LU in shared memory (where they fit,
       typically with FP32 factors); 12 = as 9 in one block of 384; 13, 14 =
       as 7 with 16 or 8 lanes per cell (2 or 4 cells per warp); 15, 16 = as
       8 in one block of 256 or 512 threads (networks above 32 solver
       species); 17 = as 12 refilling on every 32nd trip; 18, 19 = as 8 in
       one block of 256 or 384 threads with the state vector in shared
       memory, 20 = as 3 with the state vector in shared memory (18-20:
       networks above 32 solver species); 21 = as 3 with the history in
       shared memory and each block in soft lockstep (up to 12 solver
       species) (2-21: per-cell control only).  In 2-6 and 8-16 idle lanes take new cells on every
       16th trip of the cell loop (17: every 32nd), so cells are set up
       several at a time (in 8-12 and 15-17 in all warps of a block at
       once); staging 1 refills on every trip.  block_threads (a multiple of 32 up to
       the block of the staging) and grid_blocks: 0 = automatic (persistent
       grid filling every SM) */
    int32_t staging;
    int32_t block_threads;
    int32_t grid_blocks;
    /* 0: reproduce the reference exactly.  1: after three consecutive
       error-test failures, undo the prediction (ResetSystem) before the
       restart at order 1; the reference restarts from the predicted state
       with the time reset (src/odevec.F90:404-421), which costs accuracy at
       tight tolerances. */
    int32_t fix_restart;
    /* OV_PREC_FP32_LU only: cells whose solve fails with FP32 factors (a
       badly conditioned iteration matrix) are solved again from their inputs
       with FP64 factors, in a second launch on the same stream that exits at
       once when no cell failed.  1 disables this escalation.  Their
       statistics are those of the FP32 attempt. */
    int32_t no_escalation;
} odevec_opts;

typedef struct odevec_solver odevec_solver;

/* network variants compiled into the library */
int32_t odevec_num_networks(void);
const char* odevec_network_tag(int32_t i);
/* info: neq, nnz, nrea, dense, idx_tgas, default group size */
int32_t odevec_network_info(const char* tag, int32_t* info);

/* InitOdevec: create a solver for up to max_cells cells of one network variant
   on the current CUDA device.  Allocates the device work counter and, for
   odevec_solve_host, staging buffers for max_cells cells. */
int32_t odevec_init(const char* network, int64_t max_cells, const odevec_opts* opts,
                    odevec_solver** out);
int32_t odevec_set_options(odevec_solver* s, const odevec_opts* opts);

/* SolveODE on device arrays, asynchronous on `stream` (a cudaStream_t, NULL =
   default stream).  y, t, dt are read and overwritten: on return t[c] =
   t_stop[c], dt[c] = the last internal step, y = the solution at t_stop.
   mask (nullable): cells with mask 0 are left untouched except t = t_stop.
   status, stats: nullable outputs.  With per-cell control and at least
   32,768 cells the cells are visited longest t_stop - t first (a device
   sort on the stream); results do not depend on the order. */
int32_t odevec_solve(odevec_solver* s, int64_t ncells, double* y, double* t, double* dt,
                     const double* t_stop, const uint8_t* mask, int32_t* status, int32_t* stats,
                     void* stream);

/* SolveODE on host arrays: copies the inputs to the solver's device buffers,
   solves, copies y, t, dt, status and stats back, and synchronises.  This is
   the drop-in for a CPU caller such as the reference's Fortran drivers.  An
   array in pinned host memory that is mapped into the device's address space
   (cudaHostAlloc / cudaMallocHost, or cudaHostRegister with mapping) is not
   copied: the kernel reads a cell's inputs from it when it sets the cell up
   and writes the cell's results when it finishes, so the transfers overlap
   the solve.  Results are the same either way. */
int32_t odevec_solve_host(odevec_solver* s, int64_t ncells, double* y, double* t, double* dt,
                          const double* t_stop, const uint8_t* mask, int32_t* status,
                          int32_t* stats);

/* Continuation across calls (no counterpart in the reference, which
   restarts from y at order 1 on every SolveODE): the integrator state of
   every cell -- Nordsieck history, order, step size, error weights and
   control counters -- stays in a device workspace owned by the caller.
   odevec_workspace_doubles gives its size in doubles per cell.  A call with
   resume = 0 starts fresh (exactly as odevec_solve) and saves the state of
   every successfully finished cell; resume = 1 continues each cell from its
   saved state to the new t_stop (the Jacobian and rate coefficients are
   recomputed, so the caller may change the temperature between calls; it
   must not change the dynamic species).  resume = 2 starts fresh exactly as
   odevec_solve, except that each cell's last Newton correction of the
   previous call (en_old) is taken from the workspace: the reference's
   solver object never resets this%en_old (src/odevec.F90:170-182, 464), and
   a call whose first step restarts at order 1 after three error-test
   failures reads it in CalcStepSizeOrder (:571).  A caller that makes its
   first call with resume = 0 and every later call with resume = 2
   reproduces a reference driver's repeated SolveODE calls on one solver
   object (tests/rober.f90:57-62) bit for bit.  Other arguments as
   odevec_solve. */
int32_t odevec_workspace_doubles(const char* network, int64_t* per_cell);
int32_t odevec_solve_resident(odevec_solver* s, int64_t ncells, double* y, double* t, double* dt,
                              const double* t_stop, const uint8_t* mask, int32_t* status,
                              int32_t* stats, double* workspace, int32_t resume, void* stream);

/* odevec_solve_resident on a range of cells of larger arrays, no
   counterpart in the reference: the caller passes y + c0, t + c0, dt + c0,
   t_stop + c0, mask + c0, status + c0, stats + c0 * OV_NSTATS and
   workspace + c0 (workspace may be null with resume = 0) for cells
   [c0, c0 + ncells), and stride = the arrays' full cell count (the row
   stride of y and of the workspace, >= ncells).  Lets a caller cut one large
   solve into several shorter launches, e.g. a serving loop that keeps short
   requests from waiting behind one long launch; results are those of the
   whole solve. */
int32_t odevec_solve_range(odevec_solver* s, int64_t ncells, int64_t stride, double* y, double* t,
                           double* dt, const double* t_stop, const uint8_t* mask, int32_t* status,
                           int32_t* stats, double* workspace, int32_t resume, void* stream);

/* Interruptible solves, no counterpart in the reference: a serving loop
   lets a short request start while a long launch runs.
   odevec_set_yield(s, flag): the kernels of s's later solves read *flag
   (int32 in device memory -- set it with a small cudaMemcpyAsync on another
   stream, which the copy engine runs while the kernel holds the SMs; pinned
   host memory mapped into the device works too but made a PRIMORDIAL solve
   3x slower; NULL: none) whenever idle cells would take new work, except on
   a launch's first such occasion.  While it is nonzero they start no new cell, and the
   launch ends once the cells it runs are done; the others are untouched.
   odevec_cells_started(s, stream, &n) synchronises `stream` and reads how
   many cells the solve has started (n >= ncells: all of them; n may exceed
   ncells).  odevec_solve_continue takes odevec_solve_range's arguments
   (the same arrays as the solve it continues) and starts the cells not yet
   started.  With OV_PREC_FP32_LU the escalation of failed cells runs after
   the launch that completes the solve.  Results are those of one
   uninterrupted solve: every cell runs once, on its own. */
int32_t odevec_set_yield(odevec_solver* s, const int32_t* flag);
int32_t odevec_solve_continue(odevec_solver* s, int64_t ncells, int64_t stride, double* y, double* t,
                              double* dt, const double* t_stop, const uint8_t* mask, int32_t* status,
                              int32_t* stats, double* workspace, int32_t resume, void* stream);
int32_t odevec_cells_started(odevec_solver* s, void* stream, int64_t* started);

/* The operator-split caller's format (tests/primordial.f90:79-87, 113-140):
   the hydro code keeps mass fractions x and the gas density rho (g/cm^3) per
   cell; the network integrates number densities n (1/cm^3).  direction
   OV_X2N: n_j = (rho * x_j) * imass_j; OV_N2X: x_j = (n_j * mass_j) / rho,
   with the network's species masses (g) and inverse masses (1/g)
   (krome_x2n / krome_n2x).  Entries without a mass (temperature, counters)
   are copied unchanged.  in and out: species-major [neq][ncells] device
   arrays, may be the same array; rho: [ncells].  Asynchronous on stream;
   allocates nothing.  OV_API_EUNSUPPORTED for a network without masses. */
#define OV_X2N 0
#define OV_N2X 1
int32_t odevec_convert(const char* network, int64_t ncells, int32_t direction, const double* in,
                       double* out, const double* rho, void* stream);

/* CloseOdevec */
int32_t odevec_close(odevec_solver* s);

/* message of the last failed call on this thread */
const char* odevec_last_error(void);

/* Several solves of different network variants in one kernel launch; no
   counterpart in the reference, which integrates one network per SolveODE.
   Each job is one odevec_solve_resident call (workspace and resume as
   there; workspace may be null with resume = 0): its own solver (distinct
   across jobs), cells and arrays.  All jobs must use the same precision
   form and per-cell control (group_size 1); the launch uses one compiled
   multi-network kernel whose set of variants holds every job's network
   (OV_API_EUNSUPPORTED if none does).  The kernel gives each job a share of
   the blocks in proportion to its cells, and a block whose job has no cells
   left takes cells of the others, so the networks share the device for the
   whole launch; each job's cells are visited longest t_stop - t first, as
   in odevec_solve.  Failed FP32-LU cells are not solved again (see
   no_escalation).  Asynchronous on stream. */
#define OV_MULTI_MAX_JOBS 8
typedef struct odevec_job {
    odevec_solver* solver;
    int64_t ncells;
    double* y;
    double* t;
    double* dt;
    const double* t_stop;
    const uint8_t* mask;
    int32_t* status;
    int32_t* stats;
    double* workspace;
    int32_t resume;
} odevec_job;
int32_t odevec_solve_many(const odevec_job* jobs, int32_t njobs, void* stream);

/* SolveODE on device arrays without allocating anything.  No counterpart in
   the reference.  For callers that cannot call cudaMalloc -- a host code
   that passes its own device arrays from a region where device allocation
   is forbidden or would break its memory-pool budget.  Same arguments as
   odevec_solve, with the network and options given directly instead of a
   solver created by odevec_init.  The solve kernel's scratch (the counter
   that hands out cells) lives in a static device array of
   OV_NOALLOC_SCRATCH_BYTES, which every GPU that loads the library holds
   until the process exits; at most OV_NOALLOC_MAX_CELLS cells per call
   (larger calls fail with OV_API_ETOOBIG).  The array has its own address in
   every CUDA context (each device's primary context, and any context a
   driver-API caller creates); the first call in a context looks that address
   up (cudaGetSymbolAddress) and caches it under the context's unique ID
   (cuCtxGetId), so a context destroyed by cudaDeviceReset or cuCtxDestroy
   and made again gets a fresh lookup.  Make the first call in each context
   before any stream capture.  Every
   call resets the counter to zero on `stream` before the launch; all calls
   share the one counter, so calls that overlap on the GPU (different
   streams, or different host threads) race and must be serialised by the
   caller.  The FP32-LU escalation of odevec_solve (see no_escalation) and
   its longest-span-first visit order need buffers and are not done here:
   cells are visited in the given order (results are the same). */
#define OV_NOALLOC_SCRATCH_BYTES 256
#define OV_NOALLOC_MAX_CELLS (1LL << 40)
int32_t odevec_solve_noalloc(const char* network, const odevec_opts* opts, int64_t ncells,
                             double* y, double* t, double* dt, const double* t_stop,
                             const uint8_t* mask, int32_t* status, int32_t* stats, void* stream);

/* Measurement utility, no counterpart in the reference: times `blocks` x
   `threads` threads each running 8 independent FMA chains of `iters` steps
   (FP64 if fp64 != 0, else FP32) on `stream`; scratch: >= blocks*8 bytes of
   device memory (never written in practice).  Returns the duration in *ms
   and the FLOPs executed in *flops. */
int32_t odevec_probe_fma(int32_t fp64, int32_t blocks, int32_t threads, int32_t iters,
                         void* scratch, void* stream, float* ms, double* flops);

#ifdef __cplusplus
}
#endif

#endif /* ODEVEC_B200_H */
