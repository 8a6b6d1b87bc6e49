/* The OdeVec BDF integrator as one persistent CUDA kernel (sm_100a).
 *
 * One thread integrates one cell.  A warp is either 32 independent cells
 * (G = 1: per-cell time, step, order and Jacobian decisions) or one lockstep
 * group of 32 cells that share them through max-norms over the warp
 * (G = 32: the reference's semantics with nvector = 32, reductions with
 * __shfl_xor_sync).  The grid is persistent: idle lanes take the next cells
 * from a global counter (warp-aggregated atomicAdd), so a warp keeps its
 * lanes busy while cells of very different stiffness finish at different
 * times.
 *
 * The reference's nested loops (src/odevec.F90: step loop :207, predictor
 * retry loop :259, corrector loop :321) are flattened into a per-lane state
 * machine.  Each trip of the main loop performs for every lane at most one
 * predictor, one right-hand-side evaluation and one Newton update, so lanes
 * in different phases still run the right-hand side and the solve together.
 * The two expensive and rarely needed blocks -- Jacobian + LU factorisation
 * and step-size/order selection -- exist once in the code; a lane that needs
 * one waits, and all waiting lanes run it together: on staging 1 once enough
 * lanes of its warp need it (jac_batch / ss_batch), no lane can progress
 * otherwise, or it has waited max_wait trips; on the other stagings on fixed
 * trips (StageCfg::PERIOD), the same trips in every warp of the block, so a
 * trip runs at most one of the two and all warps run the same code.  Waiting
 * changes only the interleaving
 * across lanes, never a cell's own sequence of operations: the arithmetic
 * per cell is that of src/odevec.F90 operation by operation, and with
 * --fmad=false it is bit-identical to the CPU oracle.
 *
 * Species whose right-hand side is identically zero and on which nothing
 * depends (the network header's frozen(); PRIMORDIAL's CR, g, Tgas, dummy)
 * are not part of the solver state: their corrections are exact zeros in
 * the reference, so leaving them out changes no result.  Norms still divide
 * by the full neq.
 *
 * Per-cell state: en, en_old, error weights, the state and the packed LU in
 * thread-local arrays with compile-time indices (the LU in shared memory for
 * stagings 2, 5 and 11); the Nordsieck history y_NS(0:5), which loops over
 * the runtime order index, in a thread-local array or, for stagings 2, 5 and
 * 9-11, in shared memory laid out [entry][lane].  The staging (StageCfg) also
 * fixes the block size, the blocks per SM, whether the block's warps run in
 * soft lockstep and how often idle lanes take new cells.
 *
 * Every loop is bounded: at most max_attempts predictor attempts per cell
 * (status OV_ERR_MAX_STEPS), at most 4 Newton iterations per attempt and 10
 * consecutive Newton failures (OV_ERR_CONV_FAILURES), so a stiff or broken
 * cell ends with a status code instead of holding the GPU. */
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "../../include/odevec_b200.h"
#include "ov_common.h"
#include "ov_launch.h"
#include "rates_primordial.h"

#ifndef OV_MODE_NS
#error "OV_MODE_NS (the arithmetic-mode namespace) must be defined"
#endif

namespace ov {
namespace OV_MODE_NS {

constexpr int MAXQ = 5; /* maxorder, pre_odevec.py:83 */
constexpr unsigned FULL = 0xffffffffu;

enum Phase : int {
    PH_IDLE = 0,      /* no cell */
    PH_START = 1,     /* cell loaded: initial right-hand side pending */
    PH_PRED = 2,      /* next: predictor attempt */
    PH_JACWAIT = 3,   /* predicted; waits for the Jacobian + LU block */
    PH_NEWTON = 4,    /* next: right-hand side + Newton update */
    PH_RESTART = 5,   /* next: right-hand side at the predicted state (3 error-test failures) */
    PH_SSWAIT = 6,    /* waits for the step-size/order selection block */
    PH_DONE = 7,      /* finished (status says how) */
    PH_EXHAUSTED = 8  /* no cells left */
};

/* why a lane waits for the step-size selection */
enum SsMode : int { SS_REJECT = 1, SS_RESTART = 2, SS_ACCEPT = 3 };

/* Nordsieck l-vectors l(q, 0:q), q = 1..6 (src/odevec.F90:127-134) */
static __constant__ double c_lcoef[7][7] = {
    {0, 0, 0, 0, 0, 0, 0},
    {1.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0},
    {2.0 / 3.0, 1.0, 1.0 / 3.0, 0.0, 0.0, 0.0, 0.0},
    {6.0 / 11.0, 1.0, 6.0 / 11.0, 1.0 / 11.0, 0.0, 0.0, 0.0},
    {12.0 / 25.0, 1.0, 7.0 / 10.0, 1.0 / 5.0, 1.0 / 50.0, 0.0, 0.0},
    {60.0 / 137.0, 1.0, 225.0 / 274.0, 85.0 / 274.0, 15.0 / 274.0, 1.0 / 274.0, 0.0},
    {20.0 / 49.0, 1.0, 58.0 / 63.0, 5.0 / 12.0, 25.0 / 252.0, 1.0 / 84.0, 1.0 / 1764.0}};

__device__ __forceinline__ double lcoef(int q, int k) { return c_lcoef[q][k]; }

/* 1/k for k = 1..7, correctly rounded at compile time: the same bits as the
   division 1.0 / k the reference evaluates (1/order, 1/(order+1), ...) */
static __constant__ double c_inv[8] = {0.0, 1.0, 1.0 / 2.0, 1.0 / 3.0, 1.0 / 4.0, 1.0 / 5.0, 1.0 / 6.0, 1.0 / 7.0};

/* tau (src/odevec.F90:1034-1054), evaluated at compile time with the same
   IEEE operations: q! by repeated multiplication, then one division */
constexpr double kL[7] = {0.0, 1.0, 1.0 / 3.0, 1.0 / 11.0, 1.0 / 50.0, 1.0 / 274.0, 1.0 / 1764.0};
constexpr double tau_c(int order, int order2)
{
    double faculty = 1.0;
    for (int i = 1; i <= order; ++i)
        faculty = faculty * i;
    if (order - 1 == order2)
        return (order2 + 1.0) / faculty;
    return (order2 + 1.0) / (faculty * kL[order]);
}
/* per order q = 1..5: tau(q,q-1), tau(q,q), tau(q,q+1) and the
   convergence-test divisor tau(q,q) / (2 (q+2)) (src/odevec.F90:640-641) */
static __constant__ double c_tau[6][4] = {
    {0, 0, 0, 0},
#define OV_TAU_ROW(q) {tau_c(q, q - 1), tau_c(q, q), tau_c(q, q + 1), tau_c(q, q) / (2.0 * (q + 2.0))}
    OV_TAU_ROW(1), OV_TAU_ROW(2), OV_TAU_ROW(3), OV_TAU_ROW(4), OV_TAU_ROW(5)
#undef OV_TAU_ROW
};
__device__ __forceinline__ double tau(int order, int order2) { return c_tau[order][order2 - order + 1]; }
__device__ __forceinline__ double conv_divisor(int order) { return c_tau[order][3]; }

/* NaN and masked-out values never win a max (as the oracle's comparison loop) */
__device__ __forceinline__ double max_operand(double v) { return v > -HUGE_VAL ? v : -HUGE_VAL; }

template <int G>
__device__ __forceinline__ double group_max(double v)
{
    v = max_operand(v);
    if (G == 32) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            v = fmax(v, __shfl_xor_sync(FULL, v, o));
    }
    return v;
}

template <int G>
__device__ __forceinline__ bool group_any(bool b)
{
    if (G == 32)
        return __any_sync(FULL, b);
    return b;
}

/* Shared-memory staging: per-lane arrays laid out [entry][lane] with a
   stride of the block size, so a warp's 32 lanes touch 32 consecutive
   words (no bank conflicts). */
template <class T, int BS>
struct LaneCol {
    T* base; /* &array[0][threadIdx.x] */
    __device__ __forceinline__ T& operator[](int i) const { return base[i * BS]; }
};

template <int ND, int BS>
struct LaneHist {
    double* base;
    __device__ __forceinline__ LaneCol<double, BS> operator[](int k) const
    {
        return LaneCol<double, BS>{base + k * ND * BS};
    }
};

/* Kernel configurations ("stagings"): where the per-cell arrays live and the
   launch shape.  BS threads per block, MINB blocks per SM for the register
   budget; SHM places the Nordsieck history and the LU in shared memory. */
template <int STAGE>
struct StageCfg;
/* SHM: 0 = history and LU in thread-local arrays, 1 = both in shared memory,
   2 = the history in shared memory and the LU thread-local.  REFILL: idle
   lanes take new cells on every REFILL-th trip of the cell loop only (the
   first trip included), so a warp sets up several cells at once instead of
   one every few trips, and the lockstep stagings set up cells in all their
   warps in the same trip.  PERIOD > 1: the Jacobian + LU block runs on the
   trips t with t % PERIOD == 1 and the step-size block on those with
   t % PERIOD == 0 (or at once when no lane of the warp can progress
   otherwise), the same trips in every warp; jac_batch / ss_batch / max_wait
   apply with PERIOD = 1 only. */
/* staging 1 keeps the straight port's refill on every trip */
template <> struct StageCfg<1> { static constexpr int SHM = 0; static constexpr bool SOFT = false; static constexpr int BS = 128, MINB = 2, REFILL = 1, PERIOD = 1; };
template <> struct StageCfg<2> { static constexpr int SHM = 1; static constexpr bool SOFT = false; static constexpr int BS = 128, MINB = 1, REFILL = 16, PERIOD = 4; };
template <> struct StageCfg<3> { static constexpr int SHM = 0; static constexpr bool SOFT = false; static constexpr int BS = 128, MINB = 3, REFILL = 16, PERIOD = 4; };
template <> struct StageCfg<4> { static constexpr int SHM = 0; static constexpr bool SOFT = false; static constexpr int BS = 128, MINB = 4, REFILL = 16, PERIOD = 4; };
template <> struct StageCfg<5> { static constexpr int SHM = 1; static constexpr bool SOFT = false; static constexpr int BS = 192, MINB = 1, REFILL = 16, PERIOD = 4; };
/* as 3, the same register budget, in one block of 384 threads per SM */
template <> struct StageCfg<6> { static constexpr int SHM = 0; static constexpr bool SOFT = false; static constexpr int BS = 384, MINB = 1, REFILL = 16, PERIOD = 4; };
/* as 6, with the block's warps held in soft lockstep (SoftSync) */
template <> struct StageCfg<8> { static constexpr int SHM = 0; static constexpr bool SOFT = true;  static constexpr int BS = 384, MINB = 1, REFILL = 16, PERIOD = 4; };
/* soft lockstep, one block of 256 threads per SM, the history in shared
   memory (the rest of L1 for the other per-cell arrays) */
template <> struct StageCfg<9> { static constexpr int SHM = 2; static constexpr bool SOFT = true;  static constexpr int BS = 256, MINB = 1, REFILL = 16, PERIOD = 4; };
/* as 9 with 320 threads (10 warps) per SM */
template <> struct StageCfg<10> { static constexpr int SHM = 2; static constexpr bool SOFT = true;  static constexpr int BS = 320, MINB = 1, REFILL = 16, PERIOD = 4; };
/* soft lockstep, one block of 192 threads per SM with history and LU in
   shared memory (fits with FP32 factors) */
template <> struct StageCfg<11> { static constexpr int SHM = 1; static constexpr bool SOFT = true;  static constexpr int BS = 192, MINB = 1, REFILL = 16, PERIOD = 4; };
/* as 9 with 384 threads (12 warps) per SM: the history of 384 cells fills
   the shared memory (221 KB for 12 species) */
template <> struct StageCfg<12> { static constexpr int SHM = 2; static constexpr bool SOFT = true;  static constexpr int BS = 384, MINB = 1, REFILL = 16, PERIOD = 4; };
/* as 8 (thread-local arrays, soft lockstep) in one block of 256 threads per
   SM (255 registers) or of 512 (128 registers): for networks above 32
   solver species, whose arrays live in local memory either way */
template <> struct StageCfg<15> { static constexpr int SHM = 0; static constexpr bool SOFT = true;  static constexpr int BS = 256, MINB = 1, REFILL = 16, PERIOD = 4; };
template <> struct StageCfg<16> { static constexpr int SHM = 0; static constexpr bool SOFT = true;  static constexpr int BS = 512, MINB = 1, REFILL = 16, PERIOD = 4; };
/* as 12, idle lanes refilled on every 32nd trip only (fewer, larger cell
   set-ups; measured on PRIMORDIAL's long solves: 1.6 % faster with FP32
   factors, 4.5 % slower in FP64; slower on short operator-split solves,
   whose lanes then wait longer for new cells) */
template <> struct StageCfg<17> { static constexpr int SHM = 2; static constexpr bool SOFT = true;  static constexpr int BS = 384, MINB = 1, REFILL = 32, PERIOD = 4; };
/* as 15 and 8 (soft lockstep, 256 or 384 threads) with the state vector y
   in shared memory (networks above 32 solver species) */
template <> struct StageCfg<18> { static constexpr int SHM = 4; static constexpr bool SOFT = true;  static constexpr int BS = 256, MINB = 1, REFILL = 16, PERIOD = 4; };
template <> struct StageCfg<19> { static constexpr int SHM = 4; static constexpr bool SOFT = true;  static constexpr int BS = 384, MINB = 1, REFILL = 16, PERIOD = 4; };
/* staging 3's shape (three 128-thread blocks per SM, so that blocks of
   several solves share an SM) with the state vector in shared memory
   (networks above 32 solver species) */
template <> struct StageCfg<20> { static constexpr int SHM = 4; static constexpr bool SOFT = false; static constexpr int BS = 128, MINB = 3, REFILL = 16, PERIOD = 4; };
/* staging 3's shape with the history in shared memory and the block's four
   warps in soft lockstep (where three blocks' histories fit an SM: up to 12
   solver species) */
template <> struct StageCfg<21> { static constexpr int SHM = 2; static constexpr bool SOFT = true;  static constexpr int BS = 128, MINB = 3, REFILL = 16, PERIOD = 4; };

/* Soft lockstep.  The warps of a block wait for each other at the top of
   every trip of the cell loop, so they run the same phase code at the same
   time and share instruction fetches.  No barrier instruction is used: lane
   0 of a warp counts itself in with a shared-memory atomic and polls a
   generation word, sleeping between polls, at most SOFT_SPIN_LIMIT times;
   after that it goes on alone.  Nothing a cell computes depends on the
   lockstep (every decision stays per lane or per warp), so a late, lost or
   early arrival costs time and never changes a result, and no wait is
   unbounded. */
struct SoftSync {
    unsigned arrive; /* warps counted in for the current generation */
    unsigned gen;    /* generation, bumped by the warp that completes it */
    unsigned active; /* warps still in the cell loop */
};
constexpr int SOFT_SPIN_LIMIT = 4096; /* polls of >= 64 ns: about 0.3 ms at most */

/* completes the current generation */
__device__ __forceinline__ void soft_release(SoftSync* s)
{
    atomicExch(&s->arrive, 0u);
    __threadfence_block();
    atomicAdd(&s->gen, 1u);
}

__device__ __forceinline__ void soft_sync(SoftSync* s, int lane)
{
    __syncwarp();
    if (lane == 0) {
        const unsigned g = *(volatile unsigned*)&s->gen;
        const unsigned n = atomicAdd(&s->arrive, 1u) + 1u;
        if (n >= *(volatile unsigned*)&s->active) {
            soft_release(s);
        } else {
            for (int i = 0; i < SOFT_SPIN_LIMIT; ++i) {
                if (*(volatile unsigned*)&s->gen != g)
                    break;
                __nanosleep(64);
            }
        }
    }
    __syncwarp();
}

/* a warp leaves the cell loop: if the others already wait for it, release them */
__device__ __forceinline__ void soft_leave(SoftSync* s, int lane)
{
    if (lane == 0) {
        const unsigned left = atomicSub(&s->active, 1u) - 1u;
        if (left > 0 && *(volatile unsigned*)&s->arrive >= left)
            soft_release(s);
    }
}


template <class Net, class LUT, int SHM, int BS>
struct Staging;

template <class Net, class LUT, int BS>
struct Staging<Net, LUT, 0, BS> { /* thread-local arrays (registers / local memory) */
    using Hist = double (*)[Net::ND];
    using LU = LUT*;
    static constexpr size_t smem_bytes = 0;
};

template <class Net, class LUT, int BS>
struct Staging<Net, LUT, 1, BS> { /* shared memory, [entry][lane] */
    using Hist = LaneHist<Net::ND, BS>;
    using LU = LaneCol<LUT, BS>;
    static constexpr size_t hist_bytes = sizeof(double) * (MAXQ + 1) * Net::ND * BS;
    static constexpr size_t smem_bytes = hist_bytes + sizeof(LUT) * Net::NNZ * BS;
};

template <class Net, class LUT, int BS>
struct Staging<Net, LUT, 4, BS> { /* the state vector y in shared memory, history and LU thread-local */
    using Hist = double (*)[Net::ND];
    using LU = LUT*;
    /* one row of NEQ + 1 doubles per thread: the odd row length spreads a
       warp's accesses to one species over the banks */
    static constexpr int YROW = Net::NEQ + 1;
    static constexpr size_t smem_bytes = sizeof(double) * YROW * BS;
};

template <class Net, class LUT, int BS>
struct Staging<Net, LUT, 2, BS> { /* history in shared memory, LU thread-local */
    using Hist = LaneHist<Net::ND, BS>;
    using LU = LUT*;
    static constexpr size_t hist_bytes = sizeof(double) * (MAXQ + 1) * Net::ND * BS;
    static constexpr size_t smem_bytes = hist_bytes;
};

template <class Net, int G, class LUT, int SHM = 0, int BS = 128>
struct Cell {
    static constexpr int N = Net::NEQ;  /* full state */
    static constexpr int ND = Net::ND;  /* solver state */
    static constexpr int NF = Net::NF;
    static constexpr int NNZ = Net::NNZ;
    static constexpr int NR = Net::NREA > 0 ? Net::NREA : 1;
    static constexpr bool SCALED = sizeof(LUT) == 4;

    typename Staging<Net, LUT, SHM, BS>::Hist yns; /* Nordsieck history y_NS(0:5) */
    /* 16-byte aligned, so that neighbouring entries can move in one 128-bit
       access when the arrays live in local memory */
    alignas(16) double en[ND];
    alignas(16) double eno[ND];
    alignas(16) double w2[ND];
    /* the full state: a thread-local array, or (SHM 4) this thread's row in
       shared memory, which the network code reloads instead of spilling */
    alignas(16) std::conditional_t<SHM == 4, double*, double[N]> y;
    typename Staging<Net, LUT, SHM, BS>::LU a; /* packed LU of the iteration matrix */
    alignas(16) double rT[NR];
    /* FP32 LU: the scale of species j is 2^sce[j] (kept as an exponent, the
       factors are formed only while the Jacobian and the solve run) */
    short sce[SCALED ? ND : 1];

    double t, h, told, tstop, crate, jchg, cerr, tint;
    double fz_add; /* 0, or NaN when a frozen species has a non-finite error weight */
    int q, swu, lju, fet, fc, it, ss_mode, wait;
    bool ujac, nuo, first, msk, fz_neg;
    int status, attempts, steps, ltef, convf, newt, jacs, ppass;

    /* x / N for the full species count: for a power of two N the product
       by 2^-k, which rounds exactly as the division does (one rounding of
       the same exact value), without the division's instruction sequence */
    __device__ __forceinline__ static double div_n(double x)
    {
        if constexpr ((N & (N - 1)) == 0)
            return x * (1.0 / N);
        else
            return x / N;
    }

    /* WeightedNorm1 (src/odevec.F90:669-684) over the solver state; the
       lane's own sum of squares is left in s_lane */
    __device__ __forceinline__ double wnorm(const double* e, double& s_lane) const
    {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < ND; ++j)
            s = s + e[j] * e[j] * w2[j];
        s = s + fz_add;
        s_lane = s;
        double v = msk ? sqrt(div_n(s)) : -HUGE_VAL;
        return group_max<G>(v);
    }
    __device__ __forceinline__ double wnorm(const double* e) const
    {
        double s;
        return wnorm(e, s);
    }

    /* WeightedNorm2 of y_NS(:,:,col) for a runtime column */
    __device__ __forceinline__ double wnorm_ns(int col) const
    {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < ND; ++j) {
            const double e = yns[col][j];
            s = s + e * e * w2[j];
        }
        s = s + fz_add;
        double v = msk ? sqrt(div_n(s)) : -HUGE_VAL;
        return group_max<G>(v);
    }

    /* CalcErrorWeightInvSquared (src/odevec.F90:706-716) */
    __device__ __forceinline__ void weights(double rtol, double atol)
    {
#pragma unroll
        for (int j = 0; j < ND; ++j) {
            /* correctly rounded reciprocal: the same bits as 1.0 / x */
            double w = __drcp_rn(rtol * fabs(y[Net::dyn(j)]) + atol);
            w2[j] = w * w;
        }
    }

    /* frozen species: constant state, so their weights and signs are fixed */
    __device__ __forceinline__ void frozen_flags(double rtol, double atol)
    {
        bool bad = false, neg = false;
#pragma unroll
        for (int j = 0; j < NF; ++j) {
            const double v = y[Net::frozen(j)];
            double w = 1.0 / (rtol * fabs(v) + atol);
            w = w * w;
            bad |= !(w - w == 0.0); /* inf or NaN */
            neg |= v < 0.0;
        }
        fz_add = bad ? __longlong_as_double(0x7ff8000000000000LL) : 0.0;
        fz_neg = neg;
    }

    /* PredictSolution (src/odevec.F90:769-793): per species, the Pascal
       triangle y_NS(k-1) += y_NS(k) for l = 0..q-1, k = q..l+1, in the
       reference's order, on register copies of the history.  The history is
       indexed by runtime order only; species indices stay compile-time so
       en, w2 and y remain in registers. */
    __device__ __forceinline__ void predict()
    {
        ppass += q * (q + 1) / 2;
#pragma unroll 4
        for (int j = 0; j < ND; ++j) {
            double v[MAXQ + 1];
#pragma unroll
            for (int k = 0; k <= MAXQ; ++k)
                v[k] = yns[k][j];
#pragma unroll
            for (int l = 0; l < MAXQ; ++l)
#pragma unroll
                for (int k = MAXQ; k >= 1; --k)
                    if (l <= q - 1 && k <= q && k >= l + 1)
                        v[k - 1] = v[k] + v[k - 1];
#pragma unroll
            for (int k = 0; k < MAXQ; ++k)
                yns[k][j] = v[k];
        }
#pragma unroll
        for (int j = 0; j < ND; ++j)
            en[j] = 0.0;
    }

    /* ResetSystem (src/odevec.F90:526-544) */
    __device__ __forceinline__ void reset()
    {
        ppass += q * (q + 1) / 2;
#pragma unroll 4
        for (int j = 0; j < ND; ++j) {
            double v[MAXQ + 1];
#pragma unroll
            for (int k = 0; k <= MAXQ; ++k)
                v[k] = yns[k][j];
#pragma unroll
            for (int k = 0; k < MAXQ; ++k)
#pragma unroll
                for (int jj = MAXQ; jj >= 1; --jj)
                    if (k <= q - 1 && jj <= q && jj >= k + 1)
                        v[jj - 1] = v[jj - 1] - v[jj];
#pragma unroll
            for (int k = 0; k < MAXQ; ++k)
                yns[k][j] = v[k];
        }
    }

    /* SetStepSize (src/odevec.F90:720-743) */
    __device__ __forceinline__ void set_step(double dt_scale)
    {
        double dtt = 1.0;
#pragma unroll 1
        for (int k = 1; k <= q; ++k) {
            dtt = dt_scale * dtt;
#pragma unroll
            for (int j = 0; j < ND; ++j)
                yns[k][j] = yns[k][j] * dtt;
        }
        h = h * dt_scale;
        jchg = jchg * dt_scale;
    }

    /* UpdateNordsieck (src/odevec.F90:747-765) */
    __device__ __forceinline__ void update_nordsieck()
    {
#pragma unroll 1
        for (int k = 0; k <= q; ++k) {
            const double c = lcoef(q, k);
#pragma unroll
            for (int j = 0; j < ND; ++j)
                yns[k][j] = yns[k][j] + en[j] * c;
        }
    }

    /* CalcStepSizeOrder (src/odevec.F90:547-618); returns dt_scale.  The
       literals 1.3, 1.2, 1.4 and 1.1 are single precision in the reference.
       The three candidate factors are independent: with per-cell control all
       three are evaluated (the unused ones are discarded) with the
       branch-free power, so their dependency chains interleave instead of
       running one after another; a lockstep group (whose order is uniform)
       skips the unused norms and their shuffle reductions.  Each kept value
       is the same IEEE expression as in the reference. */
    __device__ __forceinline__ double step_size_order()
    {
        const int order = q;
        const bool want_down = G == 1 || order != 1;
        const bool want_up = G == 1 || !(order == MAXQ || nuo);
        double d[ND];
#pragma unroll
        for (int j = 0; j < ND; ++j)
            d[j] = en[j] - eno[j];
        const double n_down = want_down ? wnorm_ns(order) / tau(order, order - 1) : 0.0;
        const double n_same = wnorm(en) / tau(order, order);
        const double n_up = want_up ? wnorm(d) / tau(order, order + 1) : 0.0;
        const double p_down = ov_pow_sel(n_down, c_inv[order]);
        const double p_same = ov_pow_sel(n_same, c_inv[order + 1]);
        const double p_up = ov_pow_sel(n_up, c_inv[order + 2]);
        const double down = order == 1 ? 0.0 : 1.0 / ((double)1.3f * p_down + 1e-6);
        const double same = 1.0 / ((double)1.2f * p_same + 1e-6);
        const double up = (order == MAXQ || nuo) ? 0.0 : 1.0 / ((double)1.4f * p_up + 1e-6);
        int loc = 1;
        double mx = down;
        if (same > mx) { mx = same; loc = 2; }
        if (up > mx) { mx = up; loc = 3; }
        double s = mx;
        if (s >= (double)1.1f) {
            if (loc == 1) {
                if (order != 1)
                    q = order - 1;
                else
                    status = OV_ERR_ORDER;
            } else if (loc == 2) {
                s = same;
            } else {
                if (order != MAXQ) {
                    const double c = lcoef(order, order);
#pragma unroll
                    for (int j = 0; j < ND; ++j)
                        yns[order + 1][j] = c * en[j] / (order + 1.0);
                    q = order + 1;
                } else
                    status = OV_ERR_ORDER;
            }
        } else {
            s = same;
        }
        double upper;
        if (first) {
            upper = 1e4;
            first = false;
        } else
            upper = 10.0;
        s = upper < s ? upper : s;
        jchg = jchg * s;
        swu = 0;
        nuo = false;
        return s;
    }

    /* CheckConvergence (src/odevec.F90:622-665), den in d */
    __device__ __forceinline__ void check_convergence(const double* d, bool& failed, bool& converged)
    {
        double s_lane;
        const double err = wnorm(d, s_lane);
        double rate_tmp = 0.0;
        if (it != 0) {
            rate_tmp = err / cerr;
            crate = fmax(0.2 * crate, rate_tmp);
        }
        const double r15 = 1.5 * crate;
        const double crit = err * (1.0 < r15 ? 1.0 : r15) / conv_divisor(q);
        /* a NaN in den or in the weights (src/odevec.F90:645) makes its
           term and so the lane's sum of squares NaN: the entries are only
           scanned when that sum is NaN */
        bool nan = false;
        if (s_lane != s_lane) {
            nan = fz_add != fz_add;
#pragma unroll
            for (int j = 0; j < ND; ++j)
                nan |= (d[j] != d[j]) | (w2[j] != w2[j]);
        }
        if (group_any<G>(nan)) {
            failed = true;
            return;
        }
        if (crit < 1.0) {
            converged = true;
            return;
        }
        if (it >= 2 && crate > 2.0 * rate_tmp)
            failed = true;
        else if (it == 3)
            failed = true;
        else {
            failed = false;
            cerr = err;
            it = it + 1;
        }
    }

    __device__ __forceinline__ bool any_negative_yns0() const
    {
        bool neg = fz_neg;
#pragma unroll
        for (int j = 0; j < ND; ++j)
            neg |= yns[0][j] < 0.0;
        return group_any<G>(msk && neg);
    }

    __device__ __forceinline__ bool any_negative_y() const
    {
        bool neg = fz_neg;
#pragma unroll
        for (int j = 0; j < ND; ++j)
            neg |= y[Net::dyn(j)] < 0.0;
        return group_any<G>(msk && neg);
    }

    /* GetJac + LUDecompose (src/odevec.F90:301-315) */
    __device__ __forceinline__ void jacobian_lu()
    {
        double sc[SCALED ? ND : 1], isc[SCALED ? ND : 1];
        if constexpr (SCALED) {
            /* scale by powers of two close to the error weights (exact in
               FP64), then round to FP32 */
#pragma unroll
            for (int j = 0; j < ND; ++j) {
                int e = (int)((ov_d2bits(w2[j]) >> 52) & 0x7ff) - 1023;
                int hexp = e >= 0 ? e / 2 : -((-e + 1) / 2);
                hexp = hexp > 480 ? 480 : (hexp < -480 ? -480 : hexp);
                sce[j] = (short)hexp;
                sc[j] = ov_pow2i(hexp);
                isc[j] = ov_pow2i(-hexp);
            }
        }
        if constexpr (Net::LU_METHOD == 3) {
            fd_jacobian(sc, isc);
        } else {
            double k[NR];
            Net::rates_k(y, rT, k);
            if constexpr (!SCALED)
                Net::template jac<LUT>(y, k, lcoef(q, 0), h, a);
            else
                Net::template jac_scaled<LUT>(y, k, lcoef(q, 0), h, a, sc, isc);
        }
        /* empty for LUmethod 2: jac() wrote the symbolic factors */
        Net::template lu_factor<LUT>(a);
    }

    /* CalcJac_dense (src/odevec.F90:469-506), the DRPEPJ difference
       quotients: P(:,k) = -(dt*beta/r) * (f(y + r e_k) - f(y)), then 1 is
       added on the diagonal.  Only the solver-state columns are formed:
       the rows and columns of frozen species are those of the identity
       whatever their off-diagonal values, so they never reach a solution.
       Every array index is a compile-time constant (the perturbed column
       is selected, not indexed), so the state stays in registers. */
    __device__ __forceinline__ void fd_jacobian(const double* sc, const double* isc)
    {
        const double uround = 2.2204460492503131e-16;  /* 2^-52 */
        const double srur = 1.4901161193847656e-08;    /* 2^-26 */
        const double beta = lcoef(q, 0);
        double k[NR], f0[N];
        Net::rates_k(y, rT, k);
        Net::rhs(y, k, f0);
        double e[ND];
#pragma unroll
        for (int j = 0; j < ND; ++j)
            e[j] = f0[Net::dyn(j)];
        const double fac = wnorm(e);
        double r0 = 1e3 * fabs(h) * uround * (double)N * fac;
        if (r0 == 0.0)
            r0 = 1.0;
#pragma unroll 1
        for (int col = 0; col < ND; ++col) {
            double yy[N];
            double yk = 0.0, wk = 0.0;
#pragma unroll
            for (int j = 0; j < N; ++j)
                yy[j] = y[j];
#pragma unroll
            for (int j = 0; j < ND; ++j) {
                if (j == col) {
                    yk = y[Net::dyn(j)];
                    wk = w2[j];
                }
            }
            const double a1 = srur * fabs(yk), a2 = r0 / sqrt(wk);
            const double r = a1 >= a2 ? a1 : a2;
            const double fk = -(h * beta / r);
#pragma unroll
            for (int j = 0; j < ND; ++j)
                if (j == col)
                    yy[Net::dyn(j)] = yk + r;
            double k1[NR], f1[N];
            Net::rates_k(yy, rT, k1);
            Net::rhs(yy, k1, f1);
#pragma unroll
            for (int c = 0; c < ND; ++c) {
                if (c == col) {
#pragma unroll
                    for (int i = 0; i < ND; ++i) {
                        double v = (f1[Net::dyn(i)] - f0[Net::dyn(i)]) * fk;
                        if (i == c)
                            v = 1.0 + v;
                        if constexpr (SCALED)
                            a[Net::pidx(i, c)] = (LUT)(v * sc[i] * isc[c]);
                        else
                            a[Net::pidx(i, c)] = v;
                    }
                }
            }
        }
    }

    /* residual, solve, Newton update (src/odevec.F90:323-352) */
    __device__ __forceinline__ void newton_update(const double* f, double* den)
    {
        double res[ND];
#pragma unroll
        for (int j = 0; j < ND; ++j)
            res[j] = h * f[Net::dyn(j)] - (yns[1][j] + en[j]);
        if constexpr (SCALED) {
            double sc[ND], isc[ND];
#pragma unroll
            for (int j = 0; j < ND; ++j) {
                sc[j] = ov_pow2i(sce[j]);
                isc[j] = ov_pow2i(-sce[j]);
            }
            Net::template lu_solve<LUT>(a, res, den, sc, isc);
        } else {
            Net::template lu_solve<LUT>(a, res, den, nullptr, nullptr);
        }
        const double l0 = lcoef(q, 0);
#pragma unroll
        for (int j = 0; j < ND; ++j) {
            en[j] = en[j] + den[j];
            if (msk)
                y[Net::dyn(j)] = yns[0][j] + l0 * en[j];
        }
    }

    /* CalcInitialStepSize (src/odevec.F90:216-238), f holds f(y) */
    __device__ __forceinline__ double initial_step(const double* f, double rtol, double atol)
    {
        weights(rtol, atol);
        const double tol = rtol;
        const double W0 = fabs(t) > fabs(tstop) ? fabs(t) : fabs(tstop);
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < ND; ++j) {
            const double fj = f[Net::dyn(j)];
            s = s + fj * fj * (w2[j] * tol * tol);
        }
        s = s + fz_add;
        const double mx = group_max<G>(msk ? s : -HUGE_VAL);
        /* W0**(-2.0): a real exponent other than -1, 0, 1 or 2 is a pow() call
           in the reference's compiled Fortran, not 1/(W0*W0) */
        const double d = sqrt(tol / (ov_pow(W0, -2.0) + div_n(mx)));
        const double span = fabs(tstop - t);
        return d < span ? d : span;
    }

    /* InterpolateSolution (src/odevec.F90:998-1030) */
    __device__ __forceinline__ void interpolate()
    {
        const double rel_t = (tstop - t) / h;
#pragma unroll
        for (int j = 0; j < ND; ++j) {
            double acc = yns[q][j];
#pragma unroll 1
            for (int k = q - 1; k >= 0; --k)
                acc = yns[k][j] + rel_t * acc;
            if (msk)
                y[Net::dyn(j)] = acc;
        }
    }

    /* end of an accepted step (src/odevec.F90:452-464, loop test :207) */
    __device__ __forceinline__ int finish_step(bool& write_y)
    {
        fet = 0;
        steps++;
        if (lju >= 20)
            ujac = true;
        else if (fabs(jchg - (double)1.0f) > (double)0.3f) /* 1.0 and 0.3 are single precision */
            ujac = true;
#pragma unroll
        for (int j = 0; j < ND; ++j)
            eno[j] = en[j];
        if (t < tstop) {
            told = t;
            return PH_PRED;
        }
        write_y = true;
        interpolate();
        tint = t;
        t = tstop;
        return PH_DONE;
    }

    /* resident workspace: [field][cell] with the launch's row stride */
    __device__ __forceinline__ void save_state(double* ws, int64_t n, int64_t cell) const
    {
        int f = 0;
#pragma unroll 1
        for (int k = 0; k <= MAXQ; ++k)
#pragma unroll
            for (int j = 0; j < ND; ++j)
                ws[(f + k * ND + j) * n + cell] = yns[k][j];
        f += (MAXQ + 1) * ND;
#pragma unroll
        for (int j = 0; j < ND; ++j) {
            ws[(f + j) * n + cell] = eno[j];
            ws[(f + ND + j) * n + cell] = w2[j];
        }
        f += 2 * ND;
        const double sc[12] = {tint, h, crate, jchg, (double)q, (double)swu, (double)lju, (double)fet,
                               (double)fc, ujac ? 1.0 : 0.0, nuo ? 1.0 : 0.0, first ? 1.0 : 0.0};
#pragma unroll
        for (int i = 0; i < 12; ++i)
            ws[(f + i) * n + cell] = sc[i];
    }

    __device__ __forceinline__ void load_state(const double* ws, int64_t n, int64_t cell)
    {
        int f = 0;
#pragma unroll 1
        for (int k = 0; k <= MAXQ; ++k)
#pragma unroll
            for (int j = 0; j < ND; ++j)
                yns[k][j] = ws[(f + k * ND + j) * n + cell];
        f += (MAXQ + 1) * ND;
#pragma unroll
        for (int j = 0; j < ND; ++j) {
            eno[j] = ws[(f + j) * n + cell];
            w2[j] = ws[(f + ND + j) * n + cell];
        }
        f += 2 * ND;
        t = ws[(f + 0) * n + cell];
        h = ws[(f + 1) * n + cell];
        crate = ws[(f + 2) * n + cell];
        jchg = ws[(f + 3) * n + cell];
        q = (int)ws[(f + 4) * n + cell];
        swu = (int)ws[(f + 5) * n + cell];
        lju = (int)ws[(f + 6) * n + cell];
        fet = (int)ws[(f + 7) * n + cell];
        fc = (int)ws[(f + 8) * n + cell];
        ujac = ws[(f + 9) * n + cell] != 0.0;
        nuo = ws[(f + 10) * n + cell] != 0.0;
        first = ws[(f + 11) * n + cell] != 0.0;
    }
};

/* number of lanes of the warp for which b holds */
__device__ __forceinline__ int warp_count(bool b) { return __popc(__ballot_sync(FULL, b)); }


/* The persistent cell loop of one network variant: the body of bdf_kernel,
   also run by the multi-network kernel for each of its jobs in turn.  A
   warp leaves it once the job's work counter has no cells left for it. */
template <class Net, int G, class LUT, int STAGE>
__device__ __forceinline__ void bdf_run(const LaunchArgs& A)
{
    constexpr int SHM = StageCfg<STAGE>::SHM;
    constexpr int BS = StageCfg<STAGE>::BS;
    using C = Cell<Net, G, LUT, SHM, BS>;
    constexpr int N = C::N;
    constexpr int ND = C::ND;
    const int lane = threadIdx.x & 31;
    const int64_t ncells = A.ncells;
    const int64_t stride = A.stride;
    if (A.run_if && *A.run_if == 0)
        return;

    C c;
    if constexpr (SHM == 4) {
        extern __shared__ __align__(16) unsigned char ov_smem[];
        c.y = reinterpret_cast<double*>(ov_smem) + (size_t)threadIdx.x * Staging<Net, LUT, 4, BS>::YROW;
    } else if constexpr (SHM != 0) {
        extern __shared__ __align__(16) unsigned char ov_smem[];
        c.yns = LaneHist<ND, BS>{reinterpret_cast<double*>(ov_smem) + threadIdx.x};
        if constexpr (SHM == 1)
            c.a = LaneCol<LUT, BS>{reinterpret_cast<LUT*>(ov_smem + Staging<Net, LUT, 1, BS>::hist_bytes)
                                   + threadIdx.x};
    }
    alignas(16) double history[(SHM == 0 || SHM == 4) ? MAXQ + 1 : 1][ND];
    alignas(16) LUT lu_local[SHM == 1 ? 1 : C::NNZ];
    if constexpr (SHM == 0 || SHM == 4)
        c.yns = history;
    if constexpr (SHM != 1)
        c.a = lu_local;
    int ph = PH_IDLE;
    int64_t cell = -1;
    bool write_y = false;
    __shared__ SoftSync soft;
    if constexpr (StageCfg<STAGE>::SOFT) {
        if (threadIdx.x == 0) {
            soft.arrive = 0u;
            soft.gen = 0u;
            soft.active = blockDim.x / 32u;
        }
        __syncthreads(); /* once, at entry, with every thread converged */
    }

    unsigned trip = 0;
    for (;;) {
        /* ---- 1. idle lanes take new cells ---------------------------- */
        if (G == 1) {
            if constexpr (StageCfg<STAGE>::SOFT)
                soft_sync(&soft, lane);
            /* with REFILL > 1, idle lanes wait for every REFILL-th trip (the
               same trip in every warp of a lockstep block), so the costly
               cell set-up (loads, temperature rates, first right-hand side)
               runs for several lanes and warps at once instead of stretching
               trip after trip for one lane */
            const bool refill = StageCfg<STAGE>::REFILL <= 1 || trip % StageCfg<STAGE>::REFILL == 0u;
            /* a yield request, seen on a refill trip after the first (so
               that every launch starts cells), turns the idle lanes into
               exhausted ones: the warp leaves once its running cells end */
            int stop = 0;
            if (refill && trip > 0u && A.yield) {
                if (lane == 0)
                    stop = *(volatile const int32_t*)A.yield;
                stop = __shfl_sync(FULL, stop, 0);
            }
            ++trip;
            if (stop && ph == PH_IDLE)
                ph = PH_EXHAUSTED;
            const unsigned need = refill && !stop ? __ballot_sync(FULL, ph == PH_IDLE) : 0u;
            if (need) {
                const int leader = __ffs(need) - 1;
                unsigned long long base = 0;
                if (lane == leader)
                    base = atomicAdd(A.queue, (unsigned long long)__popc(need));
                base = __shfl_sync(FULL, base, leader);
                if (ph == PH_IDLE) {
                    const int64_t q = (int64_t)(base + __popc(need & ((1u << lane) - 1u)));
                    if (q < ncells) {
                        cell = A.order ? (int64_t)A.order[q] : q;
                        ph = PH_START;
                    } else {
                        ph = PH_EXHAUSTED;
                    }
                }
            }
            if (__all_sync(FULL, ph == PH_EXHAUSTED)) {
                if constexpr (StageCfg<STAGE>::SOFT)
                    soft_leave(&soft, lane);
                break;
            }
        } else {
            if (ph == PH_IDLE) { /* warp-uniform */
                int stop = 0;
                if (trip > 0u && A.yield) { /* yield requests as above */
                    if (lane == 0)
                        stop = *(volatile const int32_t*)A.yield;
                    stop = __shfl_sync(FULL, stop, 0);
                }
                ++trip;
                if (stop) {
                    ph = PH_EXHAUSTED;
                } else {
                    unsigned long long g = 0;
                    if (lane == 0)
                        g = atomicAdd(A.queue, 1ull);
                    g = __shfl_sync(FULL, g, 0);
                    cell = (int64_t)g * 32 + lane;
                    ph = (int64_t)g * 32 < ncells ? PH_START : PH_EXHAUSTED;
                }
            }
            if (ph == PH_EXHAUSTED)
                break;
        }

        /* ---- load + SolveODE set-up (src/odevec.F90:169-198) --------- */
        if (ph == PH_START) {
#pragma unroll
            for (int j = 0; j < N; ++j)
                c.y[j] = A.y[(int64_t)j * stride + cell];
            c.t = A.t[cell];
            c.h = A.dt[cell];
            if (A.save_y) {
                /* the inputs, for the FP32-LU form's escalation */
#pragma unroll
                for (int j = 0; j < N; ++j)
                    A.save_y[(int64_t)j * ncells + cell] = c.y[j];
                A.save_t[cell] = c.t;
                A.save_dt[cell] = c.h;
            }
            c.tstop = A.t_stop[cell];
            c.msk = A.mask ? (A.mask[cell] != 0) : true;
            c.status = OV_OK;
            c.attempts = c.steps = c.ltef = c.convf = c.newt = c.jacs = c.ppass = 0;
            c.first = true;
            c.q = 1;
            c.swu = 0;
            c.crate = 0.7;
            c.jchg = 0.0;
            c.nuo = false;
            c.fet = 0;
            c.fc = 0;
            c.ujac = true;
            c.lju = 0;
            c.cerr = 0.0;
            c.it = 0;
            c.wait = 0;
            c.ss_mode = 0;
#pragma unroll
            for (int k = 0; k <= MAXQ; ++k)
#pragma unroll
                for (int j = 0; j < ND; ++j)
                    c.yns[k][j] = 0.0;
#pragma unroll
            for (int j = 0; j < ND; ++j)
                c.eno[j] = 0.0;
            if constexpr (Net::HC_FD) {
                /* the heating/cooling Jacobian leaves entries of cells with a
                   non-positive species as the storage holds them: zero at
                   the start, as the reference's InitOdevec leaves its LU */
#pragma unroll
                for (int kk = 0; kk < C::NNZ; ++kk)
                    c.a[kk] = (LUT)0;
            }
            write_y = false;
            bool skip = !group_any<G>(c.msk);
            if (G == 32) {
                const bool bad = c.t != __shfl_sync(FULL, c.t, 0) || c.h != __shfl_sync(FULL, c.h, 0)
                                 || c.tstop != __shfl_sync(FULL, c.tstop, 0);
                if (__any_sync(FULL, bad)) {
                    c.status = OV_ERR_GROUP_MISMATCH;
                    ph = PH_DONE;
                }
            }
            if (ph == PH_START) {
                c.weights(A.rtol, A.atol);
                c.frozen_flags(A.rtol, A.atol);
                if (skip) {
                    c.t = c.tstop; /* src/odevec.F90:187-191 */
                    ph = PH_DONE;
                } else if (A.resume == 1) {
                    /* continuation: the saved history, step, order and
                       weights; the state is the saved y_NS(0); rates and
                       Jacobian are recomputed (the caller may have changed
                       the temperature) */
                    c.load_state(A.ws, stride, cell);
#pragma unroll
                    for (int j = 0; j < ND; ++j)
                        if (c.msk)
                            c.y[Net::dyn(j)] = c.yns[0][j];
                    if (Net::NREA > 0)
                        Net::rates_T(c.y, c.rT);
                    c.ujac = true;
                    if (c.t < c.tstop) {
                        c.told = c.t;
                        ph = PH_PRED;
                    } else {
                        write_y = true;
                        c.interpolate();
                        c.tint = c.t;
                        c.t = c.tstop;
                        ph = PH_DONE;
                    }
                } else {
                    if (A.resume == 2) {
                        /* a fresh SolveODE that keeps the previous call's
                           last correction vector, as the reference's solver
                           object does (this%en_old is never reset) */
#pragma unroll
                        for (int j = 0; j < ND; ++j)
                            c.eno[j] = A.ws[((int64_t)(MAXQ + 1) * ND + j) * stride + cell];
                    }
                    if (Net::NREA > 0)
                        Net::rates_T(c.y, c.rT);
#pragma unroll
                    for (int j = 0; j < ND; ++j)
                        c.yns[0][j] = c.y[Net::dyn(j)];
                }
            }
        }

        /* ---- 2. predictor attempt (src/odevec.F90:259-299) ----------- */
        if (ph == PH_PRED) {
            if (++c.attempts > A.max_attempts) {
                c.status = OV_ERR_MAX_STEPS;
                ph = PH_DONE;
            } else {
                c.t = c.t + c.h;
                c.predict();
                if (A.check_neg && c.any_negative_yns0()) {
                    c.t = c.told;
                    c.reset();
                    c.set_step(0.25);
                    if (c.h <= A.dt_min) {
                        c.status = OV_ERR_DTMIN_PREDICTOR;
                        ph = PH_DONE;
                    }
                    /* else: another predictor attempt on the next trip */
                } else {
                    if (c.msk) {
#pragma unroll
                        for (int j = 0; j < ND; ++j)
                            c.y[Net::dyn(j)] = c.yns[0][j];
                    }
                    c.it = 0;
                    ph = c.ujac ? PH_JACWAIT : PH_NEWTON;
                    c.wait = 0;
                }
            }
        }

        /* ---- 3. Jacobian + LU for the waiting lanes (:301-315) ------- */
        {
            bool run;
            if (G == 1) {
                const int waiting = warp_count(ph == PH_JACWAIT);
                const int moving = warp_count(ph == PH_NEWTON || ph == PH_START || ph == PH_RESTART);
                if constexpr (StageCfg<STAGE>::PERIOD > 1) {
                    /* trip was counted up at the top of this trip */
                    constexpr unsigned P = StageCfg<STAGE>::PERIOD;
                    run = waiting > 0 && (trip % P == 1u % P || moving == 0);
                } else {
                    const bool aged = __any_sync(FULL, ph == PH_JACWAIT && c.wait >= A.max_wait);
                    run = waiting > 0 && (waiting >= A.jac_batch || moving == 0 || aged);
                }
            } else {
                run = ph == PH_JACWAIT;
            }
            if (run && ph == PH_JACWAIT) {
                c.jacobian_lu();
                c.jacs++;
                c.ujac = false;
                c.lju = 0;
                c.crate = 0.7;
                c.jchg = 1.0;
                ph = PH_NEWTON;
            } else if (ph == PH_JACWAIT) {
                c.wait++;
            }
        }

        /* ---- 4. right-hand side ------------------------------------- */
        double f[N];
        if (ph == PH_START || ph == PH_NEWTON || ph == PH_RESTART) {
            double k[C::NR];
            Net::rates_k(c.y, c.rT, k);
            Net::rhs(c.y, k, f);
        }

        /* ---- 5. consume it ------------------------------------------ */
        if (ph == PH_START) {
            /* src/odevec.F90:201-210 */
#pragma unroll
            for (int j = 0; j < ND; ++j)
                c.yns[1][j] = c.h * f[Net::dyn(j)];
            c.h = c.initial_step(f, A.rtol, A.atol);
            if (c.t < c.tstop) {
                c.told = c.t;
                ph = PH_PRED;
            } else {
                write_y = true;
                c.interpolate();
                c.tint = c.t;
                c.t = c.tstop;
                ph = PH_DONE;
            }
        } else if (ph == PH_RESTART) {
            /* src/odevec.F90:417-421 */
#pragma unroll
            for (int j = 0; j < ND; ++j)
                c.yns[1][j] = c.h * f[Net::dyn(j)];
            c.ujac = true;
            c.ss_mode = SS_RESTART;
            c.wait = 0;
            ph = PH_SSWAIT;
        } else if (ph == PH_NEWTON) {
            c.newt++;
            double den[ND];
            c.newton_update(f, den);
            bool failed = false, converged = false;
            c.check_convergence(den, failed, converged);
            if (A.check_neg && c.any_negative_y()) {
                failed = true;
                converged = false;
            }
            if (failed && !converged) {
                /* src/odevec.F90:375-393 */
                c.t = c.told;
                c.fc++;
                c.convf++;
                if (c.fc > 10) {
                    c.status = OV_ERR_CONV_FAILURES;
                    ph = PH_DONE;
                } else {
                    c.it = 0;
                    c.reset();
                    c.set_step(0.25);
                    if (c.h < A.dt_min) {
                        c.status = OV_ERR_DTMIN_CONV;
                        ph = PH_DONE;
                    } else {
                        c.ujac = true;
                        ph = PH_PRED;
                    }
                }
            } else if (converged) {
                c.fc = 0;
                /* local truncation error test (src/odevec.F90:400-455) */
                const double error = c.wnorm(c.en) / tau(c.q, c.q);
                c.weights(A.rtol, A.atol);
                if (error > 1.0) {
                    c.ltef++;
                    c.t = c.told;
                    if (c.fet >= 3) {
                        if (A.fix_restart)
                            c.reset();
                        c.q = 1;
                        if (c.msk) {
#pragma unroll
                            for (int j = 0; j < ND; ++j)
                                c.y[Net::dyn(j)] = c.yns[0][j];
                        }
                        ph = PH_RESTART;
                    } else {
                        c.reset();
                        c.ujac = true;
                        c.swu = 0;
                        c.nuo = true;
                        c.ss_mode = SS_REJECT;
                        c.wait = 0;
                        ph = PH_SSWAIT;
                    }
                } else {
                    c.swu++;
                    c.lju++;
                    c.update_nordsieck();
                    if (c.swu == c.q + 1) {
                        c.ss_mode = SS_ACCEPT;
                        c.wait = 0;
                        ph = PH_SSWAIT;
                    } else {
                        ph = c.finish_step(write_y);
                    }
                }
            }
            /* else: next Newton iteration on the next trip */
        }

        /* ---- 6. step-size / order selection for the waiting lanes --- */
        {
            bool run;
            if (G == 1) {
                const int waiting = warp_count(ph == PH_SSWAIT);
                const int moving = warp_count(ph == PH_PRED || ph == PH_NEWTON || ph == PH_RESTART);
                if constexpr (StageCfg<STAGE>::PERIOD > 1) {
                    run = waiting > 0 && (trip % StageCfg<STAGE>::PERIOD == 0u || moving == 0);
                } else {
                    const bool aged = __any_sync(FULL, ph == PH_SSWAIT && c.wait >= A.max_wait);
                    run = waiting > 0 && (waiting >= A.ss_batch || moving == 0 || aged);
                }
            } else {
                run = ph == PH_SSWAIT;
            }
            if (run && ph == PH_SSWAIT) {
                const double s = c.step_size_order();
                if (c.status) {
                    ph = PH_DONE;
                } else {
                    c.set_step(s);
                    if (c.ss_mode == SS_ACCEPT) {
                        ph = c.finish_step(write_y);
                    } else {
                        c.fet++; /* src/odevec.F90:434-439 */
                        ph = PH_PRED;
                    }
                }
            } else if (ph == PH_SSWAIT) {
                c.wait++;
            }
        }

        /* ---- 7. store finished cells -------------------------------- */
        if (ph == PH_DONE) {
            const bool ok = c.status == OV_OK;
            if (A.ws && ok && write_y)
                c.save_state(A.ws, stride, cell);
            if ((!ok || write_y) && c.msk) {
#pragma unroll
                for (int j = 0; j < ND; ++j)
                    A.y[(int64_t)Net::dyn(j) * stride + cell] = c.y[Net::dyn(j)];
            }
            A.t[cell] = c.t;
            if (c.status != OV_ERR_GROUP_MISMATCH)
                A.dt[cell] = c.h;
            if (A.status)
                A.status[cell] = c.status;
            if (A.stats) {
                int32_t* s = A.stats + cell * OV_NSTATS;
                s[0] = c.steps;
                s[1] = c.attempts;
                s[2] = c.ltef;
                s[3] = c.convf;
                s[4] = c.newt;
                s[5] = c.jacs;
                s[6] = c.q;
                s[7] = c.ppass;
            }
            ph = PH_IDLE;
        }
    }
}

template <class Net, int G, class LUT, int STAGE>
__global__ void __launch_bounds__(StageCfg<STAGE>::BS, StageCfg<STAGE>::MINB)
    bdf_kernel(const __grid_constant__ LaunchArgs A)
{
    bdf_run<Net, G, LUT, STAGE>(A);
}

/* ---- several networks in one launch ---------------------------------- */
/* one 384-thread block per SM in soft lockstep, each thread's state vector
   in shared memory (rows sized for the largest network of the set): the
   register budget of staging 3, without the instruction-fetch stalls of a
   large network's code, and with the large network's state reloaded from
   shared memory instead of spilled (SYN64: 1.49x over staging 1); every
   warp of a block runs the same job at a time, so the lockstep keeps them
   on the same code */
constexpr int MULTI_STAGE = 19;

template <class LUT, class... Nets>
constexpr size_t multi_smem_bytes()
{
    size_t m = 0;
    ((m = Staging<Nets, LUT, StageCfg<MULTI_STAGE>::SHM, StageCfg<MULTI_STAGE>::BS>::smem_bytes > m
              ? Staging<Nets, LUT, StageCfg<MULTI_STAGE>::SHM, StageCfg<MULTI_STAGE>::BS>::smem_bytes
              : m),
     ...);
    return m;
}

template <class LUT, class... Nets>
struct MultiDispatch {
    __device__ __forceinline__ static void run(int, const LaunchArgs&) {}
};
template <class LUT, class Net0, class... Rest>
struct MultiDispatch<LUT, Net0, Rest...> {
    __device__ __forceinline__ static void run(int idx, const LaunchArgs& A)
    {
        if (idx == 0)
            bdf_run<Net0, 1, LUT, MULTI_STAGE>(A);
        else
            MultiDispatch<LUT, Rest...>::run(idx - 1, A);
    }
};

template <class LUT, class... Nets>
__global__ void __launch_bounds__(StageCfg<MULTI_STAGE>::BS, StageCfg<MULTI_STAGE>::MINB)
    bdf_multi_kernel(const __grid_constant__ MultiArgs P)
{
    int first = 0;
    while (first + 1 < P.njobs && (int)blockIdx.x >= P.block_start[first + 1])
        ++first;
    for (int k = 0; k < P.njobs; ++k) {
        const int j = (first + k) % P.njobs;
        MultiDispatch<LUT, Nets...>::run(P.net[j], P.job[j]);
    }
}

/* Launches the multi-network kernel on P (block ranges filled in here in
   proportion to the jobs' cells, at least one block per job). */
template <class LUT, class... Nets>
cudaError_t launch_multi(MultiArgs& P, cudaStream_t stream)
{
    using Cfg = StageCfg<MULTI_STAGE>;
    auto kern = bdf_multi_kernel<LUT, Nets...>;
    constexpr size_t smem = multi_smem_bytes<LUT, Nets...>();
    static_assert(smem <= 226 * 1024, "the set's largest state vectors exceed a block's shared memory");
    static int cached_grid = 0;
    if (cached_grid == 0) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        if (smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess)
                return e;
        }
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, Cfg::BS, smem);
        cached_grid = sms * (per_sm > 0 ? per_sm : 1);
    }
    int64_t total = 0;
    for (int j = 0; j < P.njobs; ++j)
        total += P.job[j].ncells;
    int grid = cached_grid;
    if (grid < P.njobs)
        grid = P.njobs;
    int start = 0;
    for (int j = 0; j < P.njobs; ++j) {
        P.block_start[j] = start;
        int nb = total > 0 ? (int)((double)grid * (double)P.job[j].ncells / (double)total) : 0;
        if (nb < 1)
            nb = 1;
        start += nb;
    }
    P.block_start[P.njobs] = start;
    kern<<<start, Cfg::BS, smem, stream>>>(P);
    return cudaGetLastError();
}
template <class Net, int G, class LUT, int STAGE>
cudaError_t launch(const LaunchArgs& a, int block, int grid, cudaStream_t stream)
{
    using Cfg = StageCfg<STAGE>;
    auto kern = bdf_kernel<Net, G, LUT, STAGE>;
    constexpr size_t smem = Staging<Net, LUT, Cfg::SHM, Cfg::BS>::smem_bytes;
    if (Cfg::SHM || block <= 0 || block > Cfg::BS)
        block = Cfg::BS;
    static int cached_grid[2] = {0, 0};
    if (cached_grid[0] == 0 || cached_grid[1] != block) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        if (smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess)
                return e;
        }
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, block, smem);
        cached_grid[0] = sms * (per_sm > 0 ? per_sm : 1);
        cached_grid[1] = block;
    }
    if (grid <= 0) {
        grid = cached_grid[0];
        const int64_t warps_needed = (a.ncells + 31) / 32;
        const int64_t blocks_needed = (warps_needed * 32 + block - 1) / block;
        if (blocks_needed < grid)
            grid = (int)blocks_needed;
        if (grid < 1)
            grid = 1;
    }
    kern<<<grid, block, smem, stream>>>(a);
    return cudaGetLastError();
}

/* shared-memory staging is compiled for per-cell control when the per-lane
   arrays of a block fit in 200 KB */
template <class Net, class LUT, int BS>
constexpr bool shm_fits()
{
    return Staging<Net, LUT, 1, BS>::smem_bytes <= 200 * 1024;
}

/* the same for the history alone */
template <class Net, int BS>
constexpr bool hist_fits()
{
    return Staging<Net, double, 2, BS>::smem_bytes <= 200 * 1024;
}

/* the histories of three blocks of 128 within an SM's shared memory */
template <class Net>
constexpr bool hist_fits_3x128()
{
    return 3 * (Staging<Net, double, 2, 128>::smem_bytes + 1024) <= 228 * 1024;
}

/* the state vectors of a block within the 227 KB a block may hold */
template <class Net, int BS>
constexpr bool y_fits()
{
    return Staging<Net, double, 4, BS>::smem_bytes <= 226 * 1024;
}

/* the history alone within the 227 KB a block may hold (less the soft
   lockstep words) */
template <class Net, int BS>
constexpr bool hist_fits_max()
{
    return Staging<Net, double, 2, BS>::smem_bytes <= 226 * 1024;
}

}  // namespace OV_MODE_NS
}  // namespace ov

#include "wpc_kernel.cuh"

/* Defines the launcher of one network variant in the current mode.
   stage: 1 = thread-local arrays, 2 blocks of 128 per SM; 2 = history and
   LU in shared memory, 1 block of 128; 3, 4 = thread-local, 3 or 4 blocks of
   128 (fewer registers, more warps); 5 = shared memory, 1 block of 192;
   6 = thread-local, 1 block of 384; 7 = one warp per cell (wpc_kernel.cuh;
   constant-coefficient CSC variants); 8 = as 6 in soft lockstep; 9, 10 =
   soft lockstep in one block of 256 or 320 with the history in shared
   memory; 11 = soft lockstep in one block of 192 with history and LU in
   shared memory (where they fit); 12 = as 9 in one block of 384; 13, 14 =
   16 or 8 lanes per cell (wpc_kernel.cuh, as 7); 15, 16 = as 8 in one block
   of 256 or 512 (networks above 32 solver species); 17 = as 12 refilling on
   every 32nd trip; 18, 19 = as 8 in one block of 256 or 384 with the state
   vector in shared memory, 20 = as 3 with the state vector in shared memory
   (18-20: networks above 32 solver species); 21 = as 3 with the history in
   shared memory and the block in soft lockstep (up to 12 solver species).  With per-cell control stagings 2-6 and 8-16 refill idle
   lanes on every 16th trip, 17 on every 32nd, staging 1 on every trip.
   Stages 2-21 exist for per-cell control (G = 1). */
#define OV_STAGE_CASE(NET, LU, ST)                                                               \
    if (stage == ST)                                                                             \
        return launch<NET, 1, LU, ST>(a, block, grid, s);

/* Defines the multi-network launcher of one set of variants in the current
   mode: launch_multi_<sid>(P, lu, stream), lu 0 = FP64 LU, 1 = FP32 LU (fma
   mode only). */
#define OV_DEFINE_MULTI(sid, FP32, ...)                                                          \
    namespace ov {                                                                               \
    namespace OV_MODE_NS {                                                                       \
    cudaError_t launch_multi_##sid(MultiArgs& P, int lu, cudaStream_t s)                          \
    {                                                                                            \
        if (lu == 0)                                                                             \
            return launch_multi<double, __VA_ARGS__>(P, s);                                      \
        if constexpr (FP32) {                                                                    \
            if (lu == 1)                                                                         \
                return launch_multi<float, __VA_ARGS__>(P, s);                                   \
        }                                                                                        \
        return cudaErrorNotSupported;                                                            \
    }                                                                                            \
    }                                                                                            \
    }

#define OV_DEFINE_LAUNCHER(cid, FP32)                                                            \
    namespace ov {                                                                               \
    namespace OV_MODE_NS {                                                                       \
    cudaError_t launch_##cid(const LaunchArgs& a, int G, int lu, int stage, int block, int grid,  \
                             cudaStream_t s)                                                     \
    {                                                                                            \
        using NET = ov_net_##cid;                                                                \
        if (G == 1 && lu == 0) {                                                                 \
            OV_STAGE_CASE(NET, double, 1)                                                        \
            OV_STAGE_CASE(NET, double, 3)                                                        \
            OV_STAGE_CASE(NET, double, 4)                                                        \
            OV_STAGE_CASE(NET, double, 6)                                                        \
            OV_STAGE_CASE(NET, double, 8)                                                        \
            if constexpr (NET::ND > 32) {                                                    \
                OV_STAGE_CASE(NET, double, 15)                                               \
                OV_STAGE_CASE(NET, double, 16)                                               \
                if constexpr (y_fits<NET, 256>()) {                                          \
                    OV_STAGE_CASE(NET, double, 18)                                           \
                }                                                                            \
                if constexpr (y_fits<NET, 128>()) {                                          \
                    OV_STAGE_CASE(NET, double, 20)                                           \
                }                                                                            \
                if constexpr (y_fits<NET, 384>()) {                                          \
                    OV_STAGE_CASE(NET, double, 19)                                           \
                }                                                                            \
            }                                                                                \
            if constexpr (hist_fits_3x128<NET>()) {                                          \
                OV_STAGE_CASE(NET, double, 21)                                               \
            }                                                                                \
            if constexpr (hist_fits<NET, 256>()) {                                               \
                OV_STAGE_CASE(NET, double, 9)                                                    \
            }                                                                                    \
            if constexpr (hist_fits<NET, 320>()) {                                               \
                OV_STAGE_CASE(NET, double, 10)                                                   \
            }                                                                                    \
            if constexpr (hist_fits_max<NET, 384>()) {                                           \
                OV_STAGE_CASE(NET, double, 12)                                                   \
                OV_STAGE_CASE(NET, double, 17)                                               \
            }                                                                                    \
            if constexpr (shm_fits<NET, double, 192>()) {                                        \
                OV_STAGE_CASE(NET, double, 11)                                                   \
            }                                                                                    \
            if constexpr (wpc_ok<NET, double, 32>()) {                                       \
                if (stage == 7)                                                              \
                    return launch_wpc<NET, double, 32>(a, grid, s);                          \
            }                                                                                \
            if constexpr (wpc_ok<NET, double, 16>()) {                                       \
                if (stage == 13)                                                             \
                    return launch_wpc<NET, double, 16>(a, grid, s);                          \
            }                                                                                \
            if constexpr (wpc_ok<NET, double, 8>()) {                                        \
                if (stage == 14)                                                             \
                    return launch_wpc<NET, double, 8>(a, grid, s);                           \
            }                                                                                \
            if constexpr (shm_fits<NET, double, 128>()) {                                        \
                OV_STAGE_CASE(NET, double, 2)                                                    \
            }                                                                                    \
            return cudaErrorNotSupported;                                                        \
        }                                                                                        \
        if constexpr (FP32) {                                                                    \
            if (G == 1 && lu == 1) {                                                             \
                OV_STAGE_CASE(NET, float, 1)                                                     \
                OV_STAGE_CASE(NET, float, 3)                                                     \
                OV_STAGE_CASE(NET, float, 4)                                                     \
                OV_STAGE_CASE(NET, float, 6)                                                     \
                OV_STAGE_CASE(NET, float, 8)                                                     \
                if constexpr (NET::ND > 32) {                                                \
                    OV_STAGE_CASE(NET, float, 15)                                            \
                    OV_STAGE_CASE(NET, float, 16)                                            \
                    if constexpr (y_fits<NET, 256>()) {                                      \
                        OV_STAGE_CASE(NET, float, 18)                                        \
                    }                                                                        \
                    if constexpr (y_fits<NET, 128>()) {                                      \
                        OV_STAGE_CASE(NET, float, 20)                                        \
                    }                                                                        \
                    if constexpr (y_fits<NET, 384>()) {                                      \
                        OV_STAGE_CASE(NET, float, 19)                                        \
                    }                                                                        \
                }                                                                            \
                if constexpr (hist_fits_3x128<NET>()) {                                      \
                    OV_STAGE_CASE(NET, float, 21)                                            \
                }                                                                            \
                if constexpr (hist_fits<NET, 256>()) {                                           \
                    OV_STAGE_CASE(NET, float, 9)                                                 \
                }                                                                                \
                if constexpr (hist_fits<NET, 320>()) {                                           \
                    OV_STAGE_CASE(NET, float, 10)                                                \
                }                                                                                \
                if constexpr (hist_fits_max<NET, 384>()) {                                       \
                    OV_STAGE_CASE(NET, float, 12)                                                \
                    OV_STAGE_CASE(NET, float, 17)                                            \
                }                                                                                \
                if constexpr (shm_fits<NET, float, 192>()) {                                     \
                    OV_STAGE_CASE(NET, float, 11)                                                \
                }                                                                                \
                if constexpr (wpc_ok<NET, float, 32>()) {                                    \
                    if (stage == 7)                                                          \
                        return launch_wpc<NET, float, 32>(a, grid, s);                       \
                }                                                                            \
                if constexpr (wpc_ok<NET, float, 16>()) {                                    \
                    if (stage == 13)                                                         \
                        return launch_wpc<NET, float, 16>(a, grid, s);                       \
                }                                                                            \
                if constexpr (wpc_ok<NET, float, 8>()) {                                     \
                    if (stage == 14)                                                         \
                        return launch_wpc<NET, float, 8>(a, grid, s);                        \
                }                                                                            \
                if constexpr (shm_fits<NET, float, 128>()) {                                     \
                    OV_STAGE_CASE(NET, float, 2)                                                 \
                }                                                                                \
                if constexpr (shm_fits<NET, float, 192>()) {                                     \
                    OV_STAGE_CASE(NET, float, 5)                                                 \
                }                                                                                \
                return cudaErrorNotSupported;                                                    \
            }                                                                                    \
            if (G == 32 && lu == 1)                                                              \
                return launch<NET, 32, float, 1>(a, block, grid, s);                             \
        }                                                                                        \
        if (G == 32 && lu == 0)                                                                  \
            return launch<NET, 32, double, 1>(a, block, grid, s);                                \
        return cudaErrorNotSupported;                                                            \
    }                                                                                            \
    }                                                                                            \
    }
