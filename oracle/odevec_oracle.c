/* CPU oracle of the OdeVec BDF solve path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker, not the product: only tests/, the smoke test and
 * bench.py's CPU-baseline leg load it.  It restates the reference solver
 * src/odevec.F90 routine by routine (each function cites the lines it
 * follows) for one "vector" of G cells that share time, step size, order and
 * Jacobian decisions, exactly as the reference's nvector cells do.  G = 1 is
 * per-cell control.  Arrays are structure-of-arrays over the G cells of a
 * group, as the reference's (nvector, neq, ...) arrays.
 *
 * Parity status: the reference is Fortran and no Fortran compiler exists on
 * the build or GPU machines, so the solver loop below is pinned only by
 * restatement (PARITY UNPINNED against a reference binary).  The network
 * pieces it calls are pinned against the reference's own output: the
 * emitted right-hand sides and iteration matrices against values of the
 * reference's generated Fortran expressions, the permutations and CSC
 * patterns against the reference preprocessor, and the PRIMORDIAL rate laws
 * against the reference's coe() source (tests/golden/make_golden.py).
 *
 * Build: oracle/build.py (gcc -O2 -ffp-contract=off -fopenmp).  Without
 * floating-point contraction the per-cell arithmetic is the same sequence
 * of IEEE operations the CUDA kernel performs with --fmad=false, so the two
 * agree bit for bit.
 *
 * Rate coefficients and elementary functions come from the shared headers
 * (rates_primordial.h, ov_common.h) and the emitted network headers; the
 * LU factorisations and solves here are the reference's loops over runtime
 * pattern arrays, independent of the emitted straight-line versions. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../odevec_b200/csrc/ov_common.h"
#include "../odevec_b200/csrc/gen/includes_c.inc"
#include "../include/odevec_b200.h"

/* ------------------------------------------------------------ networks */
typedef void (*rhs_fn)(const double*, const double*, double*);
typedef void (*jac_fn)(const double*, const double*, double, double, double*);

typedef struct {
    const char* tag;
    int neq, nnz, nrea, dense, idx_tgas;
    int lu_method; /* 1 GetJac + LUDecompose, 2 GetLU, 3 CalcJac + LUDecompose */
    const int *perm, *row_index, *u_col_start, *l_col_start;
    rhs_fn rhs;
    jac_fn jac;
} net_desc;

/* one entry per emitted variant; sizes[] = {neq, nnz, nrea, dense, idx_tgas,
   solver-state species, LUmethod} */
typedef struct {
    const char* tag;
    const int *sizes, *perm, *row_index, *u_col_start, *l_col_start;
    rhs_fn rhs;
    jac_fn jac;
    const double *mass, *imass;
} net_entry;
#define OV_NET(cid, TAG)                                                                   \
    {TAG, ov_##cid##_sizes, ov_##cid##_perm, ov_##cid##_row_index, ov_##cid##_u_col_start, \
     ov_##cid##_l_col_start, ov_##cid##_rhs, ov_##cid##_jac, ov_##cid##_mass, ov_##cid##_imass},
static const net_entry g_entries[] = {
#include "../odevec_b200/csrc/gen/registry.inc"
};
#undef OV_NET
#define NNETS ((int)(sizeof g_entries / sizeof g_entries[0]))
static net_desc g_nets[NNETS];
static const int g_nnets = NNETS;

static const net_desc* net_find(const char* tag)
{
    static int ready = 0;
    if (!ready) {
        for (int i = 0; i < NNETS; ++i) {
            const net_entry* e = &g_entries[i];
            net_desc d = {e->tag, e->sizes[0], e->sizes[1], e->sizes[2], e->sizes[3], e->sizes[4],
                          e->sizes[6], e->perm, e->row_index, e->u_col_start, e->l_col_start, e->rhs,
                          e->jac};
            g_nets[i] = d;
        }
        ready = 1;
    }
    for (int i = 0; i < g_nnets; ++i)
        if (strcmp(g_nets[i].tag, tag) == 0)
            return &g_nets[i];
    return NULL;
}

/* ------------------------------------------------------------- solver */
#define MAXORDER 5
#define NNS (MAXORDER + 2) /* y_NS(:,:,0:maxorder+1) */

typedef struct {
    const net_desc* net;
    int G, neq;
    double rtol, atol, dt_min;
    int check_neg, fix_restart;
    int64_t max_attempts;
    /* control, src/odevec.F90:39-56 */
    int order, SuccessesWithoutUpdate, LastJacobianUpdate, FailedErrorTests, FailedCorrections;
    int UpdateJac, NeglectUpperOrder, FirstStep, DoPermute;
    double ConvergenceRate, JacobianChange, ConvergenceError;
    double coeff[7][7]; /* coeff(1:6, 0:6), row 0 unused */
    /* arrays, index [j*G + i] or [(k*neq + j)*G + i] */
    double *y_NS, *en, *en_old, *den, *den_tmp, *w2, *rhs, *res, *LU, *rT, *kk, *ytmp, *col;
    const uint8_t* mask; /* group mask or NULL */
    int status;
    int64_t attempts;
    int32_t steps, lte_fails, conv_fails, newton, jacs, ppass;
} ode_t;

static inline double* NS(ode_t* o, int k) { return o->y_NS + (size_t)k * o->neq * o->G; }
static inline int M(const ode_t* o, int i) { return o->mask ? (o->mask[i] != 0) : 1; }

/* InitOdevec: Nordsieck l-coefficients (src/odevec.F90:127-134) */
static void init_coeff(ode_t* o)
{
    static const double c[6][7] = {
        {1.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0},
        {2.0 / 3.0, 1.0, 1.0 / 3.0, 0.0, 0.0, 0.0, 0.0},
        {6.0 / 11.0, 1.0, 6.0 / 11.0, 1.0 / 11.0, 0.0, 0.0, 0.0},
        {12.0 / 25.0, 1.0, 7.0 / 10.0, 1.0 / 5.0, 1.0 / 50.0, 0.0, 0.0},
        {60.0 / 137.0, 1.0, 225.0 / 274.0, 85.0 / 274.0, 15.0 / 274.0, 1.0 / 274.0, 0.0},
        {20.0 / 49.0, 1.0, 58.0 / 63.0, 5.0 / 12.0, 25.0 / 252.0, 1.0 / 84.0, 1.0 / 1764.0}};
    for (int q = 1; q <= 6; ++q)
        for (int k = 0; k <= 6; ++k)
            o->coeff[q][k] = c[q - 1][k];
}

/* tau (src/odevec.F90:1034-1054) */
static double tau(const ode_t* o, int order, int order2)
{
    double faculty = 1.0;
    for (int i = 1; i <= order; ++i)
        faculty = faculty * i;
    if (order - 1 == order2)
        return (order2 + 1.0) / faculty;
    return (order2 + 1.0) / (faculty * o->coeff[order][order]);
}

/* GetRHS: f(y) per cell (generated routine, src/odevec_commons.F90:78-95) */
static void get_rhs(ode_t* o, const double* y, double* f)
{
    const int G = o->G, n = o->neq, nr = o->net->nrea;
    double yc[128], fc[128], kc[64];
    for (int i = 0; i < G; ++i) {
        for (int j = 0; j < n; ++j)
            yc[j] = y[j * G + i];
        if (nr)
            ov_rates_primordial_k(yc, n, o->rT + (size_t)i * nr, kc);
        o->net->rhs(yc, kc, fc);
        for (int j = 0; j < n; ++j)
            f[j * G + i] = fc[j];
    }
}

/* GetJac: P = I - dt*beta*J (src/odevec_commons.F90:32-51).  Dense: full
   n x n, zeros included; CSC: sdata in CSC order. */
static void get_jac(ode_t* o, double beta, const double* y, double dt)
{
    const int G = o->G, n = o->neq, nr = o->net->nrea, nnz = o->net->nnz;
    double yc[128], kc[64];
    double* a = (double*)malloc(sizeof(double) * nnz);
    for (int i = 0; i < G; ++i) {
        for (int j = 0; j < n; ++j)
            yc[j] = y[j * G + i];
        if (nr)
            ov_rates_primordial_k(yc, n, o->rT + (size_t)i * nr, kc);
        if (o->net->dense) {
            /* entries the generated routine leaves unwritten (the heating/
               cooling difference quotients of a species <= 0) keep what the
               matrix holds, as the reference's GetJac writes into this%LU */
            for (int c = 0; c < n; ++c)
                for (int kk = o->net->u_col_start[c]; kk < o->net->u_col_start[c + 1]; ++kk)
                    a[kk] = o->LU[((size_t)o->net->row_index[kk] * n + c) * G + i];
        }
        o->net->jac(yc, kc, beta, dt, a);
        if (o->net->dense) {
            for (int r = 0; r < n; ++r)
                for (int c = 0; c < n; ++c)
                    o->LU[((size_t)r * n + c) * G + i] = 0.0;
            for (int c = 0; c < n; ++c)
                for (int kk = o->net->u_col_start[c]; kk < o->net->u_col_start[c + 1]; ++kk)
                    o->LU[((size_t)o->net->row_index[kk] * n + c) * G + i] = a[kk];
        } else {
            for (int kk = 0; kk < nnz; ++kk)
                o->LU[(size_t)kk * G + i] = a[kk];
        }
    }
    free(a);
}

static double wnorm(const ode_t* o, const double* e, const double* w2);

/* CalcJac_dense (src/odevec.F90:469-506): P = I - dt*beta*J from the
   DRPEPJ difference quotients, column by column, in the dense n x n layout
   (LUmethod 3).  y is perturbed one species at a time and restored. */
static void calc_jac_fd(ode_t* o, double beta, const double* y_in, double dt)
{
    const int G = o->G, n = o->neq;
    const size_t N = (size_t)n * G;
    const double uround = 2.2204460492503131E-016;
    const double srur = 1.4901161193847656E-008;
    double* y = (double*)malloc(sizeof(double) * N);
    double* drhs = (double*)malloc(sizeof(double) * N);
    double* r0 = (double*)malloc(sizeof(double) * G);
    double* r = (double*)malloc(sizeof(double) * G);
    double* fac = (double*)malloc(sizeof(double) * G);
    double* ytmp = (double*)malloc(sizeof(double) * G);
    memcpy(y, y_in, sizeof(double) * N);
#define AD(row, c, i) o->LU[((size_t)(row) * n + (c)) * G + (i)]
    get_rhs(o, y, o->rhs);
    const double f = wnorm(o, o->rhs, o->w2); /* one value for the vector */
    for (int i = 0; i < G; ++i) {
        r0[i] = 1e3 * fabs(dt) * uround * (double)n * f;
        if (r0[i] == 0.0)
            r0[i] = 1.0;
    }
    for (int k = 0; k < n; ++k) {
        for (int i = 0; i < G; ++i) {
            ytmp[i] = y[(size_t)k * G + i];
            const double a1 = srur * fabs(y[(size_t)k * G + i]);
            const double a2 = r0[i] / sqrt(o->w2[(size_t)k * G + i]);
            r[i] = a1 >= a2 ? a1 : a2;
            y[(size_t)k * G + i] = y[(size_t)k * G + i] + r[i];
            fac[i] = -(dt * beta / r[i]);
        }
        get_rhs(o, y, drhs);
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < G; ++i)
                AD(j, k, i) = (drhs[(size_t)j * G + i] - o->rhs[(size_t)j * G + i]) * fac[i];
        for (int i = 0; i < G; ++i)
            y[(size_t)k * G + i] = ytmp[i];
    }
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < G; ++i)
            AD(j, j, i) = 1 + AD(j, j, i);
#undef AD
    free(y); free(drhs); free(r0); free(r); free(fac); free(ytmp);
}

/* WeightedNorm1 (src/odevec.F90:669-684): max over cells of sqrt(sum e^2 w / n) */
static double wnorm(const ode_t* o, const double* e, const double* w2)
{
    const int G = o->G, n = o->neq;
    double mx = -HUGE_VAL;
    for (int i = 0; i < G; ++i) {
        if (!M(o, i))
            continue;
        double s = 0.0;
        for (int j = 0; j < n; ++j)
            s = s + e[j * G + i] * e[j * G + i] * w2[j * G + i];
        double v = sqrt(s / n);
        if (v > mx)
            mx = v;
    }
    return mx;
}

/* CalcErrorWeightInvSquared (src/odevec.F90:706-716) */
static void calc_weights(ode_t* o, const double* y)
{
    const size_t N = (size_t)o->neq * o->G;
    for (size_t m = 0; m < N; ++m) {
        double w = 1.0 / (o->rtol * fabs(y[m]) + o->atol);
        o->w2[m] = w * w;
    }
}

/* PredictSolution: Pascal triangle (src/odevec.F90:769-793) */
static void predict(ode_t* o)
{
    const size_t N = (size_t)o->neq * o->G;
    o->ppass += o->order * (o->order + 1) / 2;
    for (int l = 0; l <= o->order - 1; ++l)
        for (int k = o->order; k >= l + 1; --k) {
            double *a = NS(o, k), *b = NS(o, k - 1);
            for (size_t m = 0; m < N; ++m)
                b[m] = a[m] + b[m];
        }
    for (size_t m = 0; m < N; ++m)
        o->en[m] = 0.0;
}

/* ResetSystem (src/odevec.F90:526-544) */
static void reset_system(ode_t* o)
{
    const size_t N = (size_t)o->neq * o->G;
    o->ppass += o->order * (o->order + 1) / 2;
    for (int k = 0; k <= o->order - 1; ++k)
        for (int j = o->order; j >= k + 1; --j) {
            double *a = NS(o, j), *b = NS(o, j - 1);
            for (size_t m = 0; m < N; ++m)
                b[m] = b[m] - a[m];
        }
}

/* SetStepSize (src/odevec.F90:720-743) */
static void set_step_size(ode_t* o, double dt_scale, double* dt)
{
    const size_t N = (size_t)o->neq * o->G;
    double dtt_scale = 1.0;
    for (int k = 1; k <= o->order; ++k) {
        dtt_scale = dt_scale * dtt_scale;
        double* a = NS(o, k);
        for (size_t m = 0; m < N; ++m)
            a[m] = a[m] * dtt_scale;
    }
    *dt = *dt * dt_scale;
    o->JacobianChange = o->JacobianChange * dt_scale;
}

/* UpdateNordsieck (src/odevec.F90:747-765) */
static void update_nordsieck(ode_t* o)
{
    const size_t N = (size_t)o->neq * o->G;
    for (int k = 0; k <= o->order; ++k) {
        double* a = NS(o, k);
        const double c = o->coeff[o->order][k];
        for (size_t m = 0; m < N; ++m)
            a[m] = a[m] + o->en[m] * c;
    }
}

/* CalcStepSizeOrder (src/odevec.F90:547-618).  The literals 1.3, 1.2, 1.4
   and 1.1 are single precision in the reference. */
static void calc_step_size_order(ode_t* o, double* dt_scale)
{
    const int G = o->G, n = o->neq;
    const size_t N = (size_t)n * G;
    int order = o->order;
    double down, same, up;
    if (order == 1)
        down = 0.0;
    else
        down = 1.0 / ((double)1.3f * ov_pow(wnorm(o, NS(o, order), o->w2) / tau(o, order, order - 1),
                                            1.0 / order) + 1e-6);
    same = 1.0 / ((double)1.2f * ov_pow(wnorm(o, o->en, o->w2) / tau(o, order, order),
                                        1.0 / (order + 1.0)) + 1e-6);
    if (order == MAXORDER || o->NeglectUpperOrder)
        up = 0.0;
    else {
        for (size_t m = 0; m < N; ++m)
            o->den_tmp[m] = o->en[m] - o->en_old[m];
        up = 1.0 / ((double)1.4f * ov_pow(wnorm(o, o->den_tmp, o->w2) / tau(o, order, order + 1),
                                          1.0 / (order + 2.0)) + 1e-6);
    }
    /* maxloc / maxval: first maximum wins */
    int loc = 1;
    double mx = down;
    if (same > mx) { mx = same; loc = 2; }
    if (up > mx) { mx = up; loc = 3; }
    double s = mx;
    if (s >= (double)1.1f) {
        if (loc == 1) {
            if (order != 1)
                order = order - 1;
            else
                o->status = OV_ERR_ORDER;
        } else if (loc == 2) {
            s = same;
        } else {
            if (order != MAXORDER) {
                double* a = NS(o, order + 1);
                const double c = o->coeff[order][order];
                for (size_t m = 0; m < N; ++m)
                    a[m] = c * o->en[m] / (order + 1.0);
                order = order + 1;
            } else
                o->status = OV_ERR_ORDER;
        }
    } else {
        s = same;
    }
    o->order = order;
    double upper;
    if (o->FirstStep) {
        upper = 1e4;
        o->FirstStep = 0;
    } else
        upper = 10.0;
    s = upper < s ? upper : s; /* min(dt_upper_limit, dt_scale) */
    o->JacobianChange = o->JacobianChange * s;
    o->SuccessesWithoutUpdate = 0;
    o->NeglectUpperOrder = 0;
    *dt_scale = s;
}

/* CheckConvergence (src/odevec.F90:622-665) */
static void check_convergence(ode_t* o, int* it, int* failed, int* converged)
{
    const size_t N = (size_t)o->neq * o->G;
    double err = wnorm(o, o->den, o->w2);
    double rate_tmp = 0.0;
    if (*it != 0) {
        rate_tmp = err / o->ConvergenceError;
        o->ConvergenceRate = fmax(0.2 * o->ConvergenceRate, rate_tmp); /* NaN-ignoring max */
    }
    double r15 = 1.5 * o->ConvergenceRate;
    double crit = err * (1.0 < r15 ? 1.0 : r15) / (tau(o, o->order, o->order) / (2.0 * (o->order + 2.0)));
    for (size_t m = 0; m < N; ++m)
        if (o->den[m] != o->den[m] || o->w2[m] != o->w2[m]) {
            *failed = 1;
            return;
        }
    if (crit < 1.0) {
        *converged = 1;
        return;
    }
    if (*it >= 2 && o->ConvergenceRate > 2.0 * rate_tmp)
        *failed = 1;
    else if (*it == 3)
        *failed = 1;
    else {
        *failed = 0;
        o->ConvergenceError = err;
        *it = *it + 1;
    }
}

/* LUDecompose_dense: right-looking Doolittle, no pivoting (src/odevec.F90:898-922) */
static void lu_dense(ode_t* o)
{
    const int G = o->G, n = o->neq;
    double* A = o->LU;
#define AD(r, c, i) A[((size_t)(r) * n + (c)) * G + (i)]
    for (int k = 0; k < n - 1; ++k) {
        for (int j = k + 1; j < n; ++j)
            for (int i = 0; i < G; ++i)
                AD(j, k, i) = AD(j, k, i) / AD(k, k, i);
        for (int j = k + 1; j < n; ++j)
            for (int m = k + 1; m < n; ++m)
                for (int i = 0; i < G; ++i)
                    AD(m, j, i) = AD(m, j, i) - AD(m, k, i) * AD(k, j, i);
    }
#undef AD
}

/* LUDecompose_sparse: left-looking Crout on the CSC pattern (src/odevec.F90:929-971) */
static void lu_sparse(ode_t* o)
{
    const int G = o->G;
    const int *ri = o->net->row_index, *ucs = o->net->u_col_start, *lcs = o->net->l_col_start;
    double* A = o->LU;
    double* w = o->col; /* w(nvector, neq), never cleared, as in the reference */
    for (int k = 0; k < o->neq; ++k) {
        for (int kk = ucs[k]; kk < ucs[k + 1]; ++kk)
            for (int i = 0; i < G; ++i)
                w[(size_t)ri[kk] * G + i] = A[(size_t)kk * G + i];
        for (int kk = ucs[k]; kk < lcs[k]; ++kk) {
            int j = ri[kk];
            for (int i = 0; i < G; ++i) {
                double alpha = w[(size_t)j * G + i] / A[(size_t)lcs[j] * G + i];
                w[(size_t)j * G + i] = alpha;
                for (int jj = lcs[j] + 1; jj < ucs[j + 1]; ++jj)
                    w[(size_t)ri[jj] * G + i] = w[(size_t)ri[jj] * G + i] - alpha * A[(size_t)jj * G + i];
            }
        }
        for (int kk = ucs[k]; kk < ucs[k + 1]; ++kk)
            for (int i = 0; i < G; ++i)
                A[(size_t)kk * G + i] = w[(size_t)ri[kk] * G + i];
    }
}

/* SolveLU_dense (src/odevec.F90:797-849): res -> den */
static void solve_dense(ode_t* o, const double* res, double* den)
{
    const int G = o->G, n = o->neq;
    const double* A = o->LU;
    double* t = o->den_tmp;
#define AD(r, c, i) A[((size_t)(r) * n + (c)) * G + (i)]
    for (size_t m = 0; m < (size_t)n * G; ++m)
        t[m] = 0.0;
    for (int k = 0; k < n; ++k) {
        for (int j = 0; j < k; ++j)
            for (int i = 0; i < G; ++i)
                t[k * G + i] = t[k * G + i] + AD(k, j, i) * t[j * G + i];
        for (int i = 0; i < G; ++i)
            t[k * G + i] = res[k * G + i] - t[k * G + i];
    }
    for (size_t m = 0; m < (size_t)n * G; ++m)
        den[m] = 0.0;
    for (int k = n - 1; k >= 0; --k) {
        for (int j = k + 1; j < n; ++j)
            for (int i = 0; i < G; ++i)
                den[k * G + i] = den[k * G + i] + AD(k, j, i) * den[j * G + i];
        for (int i = 0; i < G; ++i) {
            den[k * G + i] = t[k * G + i] - den[k * G + i];
            den[k * G + i] = den[k * G + i] / AD(k, k, i);
        }
    }
#undef AD
}

/* SolveLU_sparse (src/odevec.F90:853-891): res -> den */
static void solve_sparse(ode_t* o, const double* res, double* den)
{
    const int G = o->G, n = o->neq;
    const int *ri = o->net->row_index, *ucs = o->net->u_col_start, *lcs = o->net->l_col_start;
    const double* A = o->LU;
    memcpy(den, res, sizeof(double) * (size_t)n * G);
    for (int k = 0; k < n; ++k)
        for (int i = 0; i < G; ++i) {
            double mult = den[k * G + i] / A[(size_t)lcs[k] * G + i];
            den[k * G + i] = mult;
            for (int kk = lcs[k] + 1; kk < ucs[k + 1]; ++kk)
                den[ri[kk] * G + i] = den[ri[kk] * G + i] - mult * A[(size_t)kk * G + i];
        }
    for (int k = n - 1; k >= 0; --k)
        for (int i = 0; i < G; ++i) {
            double mult = den[k * G + i];
            for (int kk = ucs[k]; kk < lcs[k]; ++kk)
                den[ri[kk] * G + i] = den[ri[kk] * G + i] - mult * A[(size_t)kk * G + i];
        }
}

static int any_negative(const ode_t* o, const double* v)
{
    for (int j = 0; j < o->neq; ++j)
        for (int i = 0; i < o->G; ++i)
            if (M(o, i) && v[j * o->G + i] < 0.0)
                return 1;
    return 0;
}

/* y = src where Mask */
static void masked_copy(ode_t* o, double* y, const double* src)
{
    for (int j = 0; j < o->neq; ++j)
        for (int i = 0; i < o->G; ++i)
            if (M(o, i))
                y[j * o->G + i] = src[j * o->G + i];
}

/* SolveLinearSystem: one accepted step (src/odevec.F90:242-465) */
static void solve_linear_system(ode_t* o, double* t, double* dt, double* y)
{
    const int G = o->G, n = o->neq;
    const size_t N = (size_t)n * G;
    const double told = *t;
    double dt_scale;
    int success = 0;
    while (!success) { /* predictor */
        if (++o->attempts > o->max_attempts) {
            o->status = OV_ERR_MAX_STEPS;
            return;
        }
        *t = *t + *dt;
        predict(o);
        if (o->check_neg && any_negative(o, NS(o, 0))) { /* :265-291 */
            dt_scale = 0.25;
            *t = told;
            reset_system(o);
            set_step_size(o, dt_scale, dt);
            if (*dt <= o->dt_min) {
                o->status = OV_ERR_DTMIN_PREDICTOR;
                return;
            }
            continue;
        }
        masked_copy(o, y, NS(o, 0)); /* :293-299 */
        if (o->UpdateJac) { /* :301-315 */
            if (o->net->lu_method == 3) {
                calc_jac_fd(o, o->coeff[o->order][0], y, *dt);
                lu_dense(o);
            } else {
                /* LUmethod 1: P, then its factors; LUmethod 2: the factors */
                get_jac(o, o->coeff[o->order][0], y, *dt);
                if (o->net->lu_method == 1) {
                    if (o->net->dense)
                        lu_dense(o);
                    else
                        lu_sparse(o);
                }
            }
            o->jacs++;
            o->UpdateJac = 0;
            o->LastJacobianUpdate = 0;
            o->ConvergenceRate = 0.7;
            o->JacobianChange = 1.0;
        }
        /* corrector :318-394 */
        int failed = 0, converged = 0, it = 0;
        while (!converged) {
            get_rhs(o, y, o->rhs);
            o->newton++;
            /* CalcResiduum :975-990 */
            double* ns1 = NS(o, 1);
            for (size_t m = 0; m < N; ++m)
                o->res[m] = *dt * o->rhs[m] - (ns1[m] + o->en[m]);
            if (o->DoPermute) { /* :328-333 */
                for (int i = 0; i < n; ++i)
                    memcpy(o->den + (size_t)i * G, o->res + (size_t)o->net->perm[i] * G, sizeof(double) * G);
                memcpy(o->res, o->den, sizeof(double) * N);
            }
            if (o->net->dense)
                solve_dense(o, o->res, o->den);
            else
                solve_sparse(o, o->res, o->den);
            if (o->DoPermute) { /* :337-342 */
                for (int i = 0; i < n; ++i)
                    memcpy(o->res + (size_t)o->net->perm[i] * G, o->den + (size_t)i * G, sizeof(double) * G);
                memcpy(o->den, o->res, sizeof(double) * N);
            }
            const double l0 = o->coeff[o->order][0];
            double* ns0 = NS(o, 0);
            for (size_t m = 0; m < N; ++m)
                o->en[m] = o->en[m] + o->den[m];
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < G; ++i)
                    if (M(o, i))
                        y[j * G + i] = ns0[j * G + i] + l0 * o->en[j * G + i];
            check_convergence(o, &it, &failed, &converged);
            if (o->check_neg && any_negative(o, y)) { /* :361-373 */
                failed = 1;
                converged = 0;
            }
            if (failed && !converged) { /* :375-393 */
                dt_scale = 0.25;
                *t = told;
                o->FailedCorrections++;
                o->conv_fails++;
                if (o->FailedCorrections > 10) {
                    o->status = OV_ERR_CONV_FAILURES;
                    return;
                }
                it = 0;
                reset_system(o);
                set_step_size(o, dt_scale, dt);
                if (*dt < o->dt_min) {
                    o->status = OV_ERR_DTMIN_CONV;
                    return;
                }
                o->UpdateJac = 1;
                break;
            }
        }
        if (!converged)
            continue; /* cycle predictor */
        o->FailedCorrections = 0;
        /* local truncation error test :397-455 */
        double error = wnorm(o, o->en, o->w2) / tau(o, o->order, o->order);
        calc_weights(o, y);
        if (error > 1.0) {
            o->lte_fails++;
            if (o->FailedErrorTests >= 3) {
                *t = told;
                if (o->fix_restart) /* optional correction, not in the reference */
                    reset_system(o);
                o->order = 1;
                masked_copy(o, y, NS(o, 0));
                get_rhs(o, y, o->rhs);
                double* ns1 = NS(o, 1);
                for (size_t m = 0; m < N; ++m)
                    ns1[m] = *dt * o->rhs[m];
                o->UpdateJac = 1;
            } else {
                *t = told;
                reset_system(o);
                o->UpdateJac = 1;
                o->SuccessesWithoutUpdate = 0;
                o->NeglectUpperOrder = 1;
            }
            calc_step_size_order(o, &dt_scale);
            if (o->status)
                return;
            set_step_size(o, dt_scale, dt);
            o->FailedErrorTests++;
            continue;
        }
        o->SuccessesWithoutUpdate++;
        o->LastJacobianUpdate++;
        update_nordsieck(o);
        if (o->SuccessesWithoutUpdate == o->order + 1) {
            calc_step_size_order(o, &dt_scale);
            if (o->status)
                return;
            set_step_size(o, dt_scale, dt);
        }
        o->FailedErrorTests = 0;
        success = 1;
    }
    o->steps++;
    /* Jacobian age / change (:458-462); 1.0 and 0.3 are single precision */
    if (o->LastJacobianUpdate >= 20)
        o->UpdateJac = 1;
    else if (fabs(o->JacobianChange - (double)1.0f) > (double)0.3f)
        o->UpdateJac = 1;
    memcpy(o->en_old, o->en, sizeof(double) * N);
}

/* CalcInitialStepSize (src/odevec.F90:216-238) */
static double initial_step_size(ode_t* o, double time, double t_stop, const double* y)
{
    const int G = o->G, n = o->neq;
    calc_weights(o, y);
    const double tol = o->rtol;
    const double W0 = fabs(time) > fabs(t_stop) ? fabs(time) : fabs(t_stop);
    double mx = -HUGE_VAL;
    for (int i = 0; i < G; ++i) {
        if (!M(o, i))
            continue;
        double s = 0.0;
        for (int j = 0; j < n; ++j) {
            const double f = o->rhs[j * G + i];
            s = s + f * f * (o->w2[j * G + i] * tol * tol);
        }
        if (s > mx)
            mx = s;
    }
    /* W0**(-2.0) (:231, :233): gfortran keeps a real exponent other than -1,
       0, 1 or 2 as a pow() call, which is not 1/(W0*W0) in the last bit */
    double dt = sqrt(tol / (ov_pow(W0, -2.0) + mx / n));
    const double span = fabs(t_stop - time);
    return dt < span ? dt : span;
}

/* InterpolateSolution: Horner's rule back to t_out (src/odevec.F90:998-1030) */
static void interpolate(ode_t* o, double t, double dt, double t_out, double* y)
{
    const int G = o->G, n = o->neq;
    masked_copy(o, y, NS(o, o->order));
    const double rel_t = (t_out - t) / dt;
    for (int k = 1; k <= o->order; ++k) {
        const double* a = NS(o, o->order - k);
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < G; ++i)
                if (M(o, i))
                    y[j * G + i] = a[j * G + i] + rel_t * y[j * G + i];
    }
}

/* resident state of a group (continuation across calls, no counterpart in
   the reference): y_NS(0:5), en_old, weights, then 12 scalars */
static size_t ws_group_doubles(int neq, int G) { return (size_t)8 * neq * G + 12; }

static void save_state(ode_t* o, double t_int, double dt, double* w)
{
    const size_t N = (size_t)o->neq * o->G;
    memcpy(w, o->y_NS, sizeof(double) * N * (MAXORDER + 1));
    memcpy(w + N * (MAXORDER + 1), o->en_old, sizeof(double) * N);
    memcpy(w + N * (MAXORDER + 2), o->w2, sizeof(double) * N);
    double* s = w + N * (MAXORDER + 3);
    s[0] = t_int;
    s[1] = dt;
    s[2] = o->ConvergenceRate;
    s[3] = o->JacobianChange;
    s[4] = o->order;
    s[5] = o->SuccessesWithoutUpdate;
    s[6] = o->LastJacobianUpdate;
    s[7] = o->FailedErrorTests;
    s[8] = o->FailedCorrections;
    s[9] = o->UpdateJac;
    s[10] = o->NeglectUpperOrder;
    s[11] = o->FirstStep;
}

static void load_state(ode_t* o, double* t_int, double* dt, const double* w)
{
    const size_t N = (size_t)o->neq * o->G;
    memcpy(o->y_NS, w, sizeof(double) * N * (MAXORDER + 1));
    memcpy(o->en_old, w + N * (MAXORDER + 1), sizeof(double) * N);
    memcpy(o->w2, w + N * (MAXORDER + 2), sizeof(double) * N);
    const double* s = w + N * (MAXORDER + 3);
    *t_int = s[0];
    *dt = s[1];
    o->ConvergenceRate = s[2];
    o->JacobianChange = s[3];
    o->order = (int)s[4];
    o->SuccessesWithoutUpdate = (int)s[5];
    o->LastJacobianUpdate = (int)s[6];
    o->FailedErrorTests = (int)s[7];
    o->FailedCorrections = (int)s[8];
    o->UpdateJac = s[9] != 0.0;
    o->NeglectUpperOrder = s[10] != 0.0;
    o->FirstStep = s[11] != 0.0;
}

/* continuation: from the saved state to t_stop, the state saved again */
static void resume_group(ode_t* o, double* time, double* dt, double t_stop, double* y, double* w)
{
    if (o->mask) {
        int any = 0;
        for (int i = 0; i < o->G; ++i)
            any |= o->mask[i] != 0;
        if (!any) {
            *time = t_stop;
            return;
        }
    }
    double t_int;
    load_state(o, &t_int, dt, w);
    masked_copy(o, y, NS(o, 0));
    if (o->net->nrea) {
        for (int i = 0; i < o->G; ++i)
            ov_rates_primordial_T(y[(size_t)o->net->idx_tgas * o->G + i], o->rT + (size_t)i * o->net->nrea);
    }
    o->UpdateJac = 1;
    *time = t_int;
    while (*time < t_stop) {
        solve_linear_system(o, time, dt, y);
        if (o->status)
            return;
    }
    interpolate(o, *time, *dt, t_stop, y);
    save_state(o, *time, *dt, w);
    *time = t_stop;
}

/* SolveODE for one group (src/odevec.F90:158-214) */
static void solve_group(ode_t* o, double* time, double* dt, double t_stop, double* y, double* w)
{
    const size_t N = (size_t)o->neq * o->G;
    o->FirstStep = 1;
    o->order = 1;
    o->SuccessesWithoutUpdate = 0;
    o->ConvergenceRate = 0.7;
    o->JacobianChange = 0.0;
    o->NeglectUpperOrder = 0;
    memset(o->den, 0, sizeof(double) * N);
    o->FailedErrorTests = 0;
    o->FailedCorrections = 0;
    o->UpdateJac = 1;
    o->LastJacobianUpdate = 0;
    calc_weights(o, y);
    if (o->mask) {
        int any = 0;
        for (int i = 0; i < o->G; ++i)
            any |= o->mask[i] != 0;
        if (!any) {
            *time = t_stop;
            return;
        }
    }
    /* rate coefficients: temperature part once per solve */
    if (o->net->nrea) {
        for (int i = 0; i < o->G; ++i)
            ov_rates_primordial_T(y[(size_t)o->net->idx_tgas * o->G + i], o->rT + (size_t)i * o->net->nrea);
    }
    memcpy(NS(o, 0), y, sizeof(double) * N);
    get_rhs(o, y, o->rhs);
    double* ns1 = NS(o, 1);
    for (size_t m = 0; m < N; ++m)
        ns1[m] = *dt * o->rhs[m];
    *dt = initial_step_size(o, *time, t_stop, y);
    while (*time < t_stop) {
        solve_linear_system(o, time, dt, y);
        if (o->status)
            return;
    }
    interpolate(o, *time, *dt, t_stop, y);
    if (w)
        save_state(o, *time, *dt, w);
    *time = t_stop;
}

/* --------------------------------------------------------------- C ABI */
int ov_oracle_solve(const char* tag, int64_t ncells, int G, double rtol, double atol,
                    double dt_min, int check_negatives, int fix_restart, int64_t max_attempts, double* y, double* t,
                    double* dt, const double* t_stop, const uint8_t* mask, int32_t* status,
                    int32_t* stats, int nthreads, double* ws, int resume)
{
    const net_desc* net = net_find(tag);
    if (!net)
        return -1;
    if (G < 1 || ncells % G)
        return -2;
    const int n = net->neq;
    const int64_t ngroups = ncells / G;
#ifdef _OPENMP
    if (nthreads > 0)
        omp_set_num_threads(nthreads);
#pragma omp parallel
#endif
    {
        ode_t o;
        memset(&o, 0, sizeof o);
        o.net = net;
        o.G = G;
        o.neq = n;
        o.rtol = rtol;
        o.atol = atol;
        o.dt_min = dt_min;
        o.check_neg = check_negatives;
        o.fix_restart = fix_restart;
        o.max_attempts = max_attempts;
        init_coeff(&o);
        o.DoPermute = 0;
        for (int i = 0; i < n; ++i)
            o.DoPermute |= net->perm[i] != i;
        const size_t N = (size_t)n * G;
        o.y_NS = (double*)calloc(N * NNS, sizeof(double));
        o.en = (double*)calloc(N, sizeof(double));
        o.en_old = (double*)calloc(N, sizeof(double));
        o.den = (double*)calloc(N, sizeof(double));
        o.den_tmp = (double*)calloc(N, sizeof(double));
        o.w2 = (double*)calloc(N, sizeof(double));
        o.rhs = (double*)calloc(N, sizeof(double));
        o.res = (double*)calloc(N, sizeof(double));
        o.col = (double*)calloc(N, sizeof(double));
        o.ytmp = (double*)calloc(N, sizeof(double));
        o.LU = (double*)calloc((size_t)(net->dense ? n * n : net->nnz) * G, sizeof(double));
        o.rT = (double*)calloc((size_t)(net->nrea ? net->nrea : 1) * G, sizeof(double));
        uint8_t* gm = (uint8_t*)malloc(G);
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
        for (int64_t g = 0; g < ngroups; ++g) {
            const int64_t c0 = g * G;
            int bad = 0;
            for (int i = 1; i < G; ++i)
                bad |= t[c0 + i] != t[c0] || t_stop[c0 + i] != t_stop[c0] || dt[c0 + i] != dt[c0];
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < G; ++i)
                    o.ytmp[j * G + i] = y[(size_t)j * ncells + c0 + i];
            if (mask) {
                for (int i = 0; i < G; ++i)
                    gm[i] = mask[c0 + i];
                o.mask = gm;
            } else
                o.mask = NULL;
            o.status = 0;
            o.order = 1; /* SolveODE starts at order 1 (src/odevec.F90:171) */
            o.attempts = 0;
            o.steps = o.lte_fails = o.conv_fails = o.newton = o.jacs = o.ppass = 0;
            memset(o.y_NS, 0, sizeof(double) * N * NNS);
            memset(o.en_old, 0, sizeof(double) * N);
            double time = t[c0], h = dt[c0];
            double* w = ws ? ws + (size_t)g * ws_group_doubles(n, G) : NULL;
            if (resume == 2 && w) /* the reference keeps this%en_old between calls */
                memcpy(o.en_old, w + N * (MAXORDER + 1), sizeof(double) * N);
            if (bad)
                o.status = OV_ERR_GROUP_MISMATCH;
            else if (resume == 1 && w)
                resume_group(&o, &time, &h, t_stop[c0], o.ytmp, w);
            else
                solve_group(&o, &time, &h, t_stop[c0], o.ytmp, w);
            for (int i = 0; i < G; ++i) {
                const int64_t c = c0 + i;
                for (int j = 0; j < n; ++j)
                    y[(size_t)j * ncells + c] = o.ytmp[j * G + i];
                if (!bad) { /* a mismatched lockstep group keeps its inputs */
                    t[c] = time;
                    dt[c] = h;
                }
                if (status)
                    status[c] = o.status;
                if (stats) {
                    int32_t* s = stats + c * OV_NSTATS;
                    s[0] = o.steps;
                    s[1] = (int32_t)o.attempts;
                    s[2] = o.lte_fails;
                    s[3] = o.conv_fails;
                    s[4] = o.newton;
                    s[5] = o.jacs;
                    s[6] = o.order;
                    s[7] = o.ppass;
                }
            }
        }
        free(o.y_NS); free(o.en); free(o.en_old); free(o.den); free(o.den_tmp); free(o.w2);
        free(o.rhs); free(o.res); free(o.col); free(o.ytmp); free(o.LU); free(o.rT); free(gm);
    }
    return 0;
}

/* network evaluation for the golden tests: f = rhs(y, k); a = P (packed) */
int ov_oracle_eval(const char* tag, const double* y, const double* k, double beta, double dt,
                   double* f, double* a)
{
    const net_desc* net = net_find(tag);
    if (!net)
        return -1;
    net->rhs(y, k, f);
    net->jac(y, k, beta, dt, a);
    return 0;
}

int ov_oracle_rates(double T, double* r)
{
    ov_rates_primordial_T(T, r);
    return 0;
}

/* k_j = small(y) + r_j for one PRIMORDIAL state (the per-call rate floor) */
int ov_oracle_rates_k(const double* y, int neq, const double* r, double* k)
{
    ov_rates_primordial_k(y, neq, r, k);
    return 0;
}

int ov_oracle_netinfo(const char* tag, int* info /* neq nnz nrea dense idx_tgas */, int* perm,
                      int* row_index, int* u_col_start, int* l_col_start)
{
    const net_desc* net = net_find(tag);
    if (!net)
        return -1;
    info[0] = net->neq;
    info[1] = net->nnz;
    info[2] = net->nrea;
    info[3] = net->dense;
    info[4] = net->idx_tgas;
    if (perm) memcpy(perm, net->perm, sizeof(int) * net->neq);
    if (row_index) memcpy(row_index, net->row_index, sizeof(int) * net->nnz);
    if (u_col_start) memcpy(u_col_start, net->u_col_start, sizeof(int) * (net->neq + 1));
    if (l_col_start) memcpy(l_col_start, net->l_col_start, sizeof(int) * net->neq);
    return 0;
}

int64_t ov_oracle_ws_doubles(const char* tag, int64_t ncells, int G)
{
    const net_desc* net = net_find(tag);
    if (!net || G < 1 || ncells % G)
        return -1;
    return (ncells / G) * (int64_t)ws_group_doubles(net->neq, G);
}

int ov_oracle_num_nets(void) { return g_nnets; }
const char* ov_oracle_net_tag(int i) { return (i >= 0 && i < g_nnets) ? g_entries[i].tag : NULL; }

/* exposed for the elementary-function tests */
double ov_oracle_exp(double x) { return ov_exp(x); }
double ov_oracle_log(double x) { return ov_log(x); }
double ov_oracle_pow(double x, double y) { return ov_pow(x, y); }
double ov_oracle_pow_sel(double x, double y) { return ov_pow_sel(x, y); }
double ov_oracle_exp_sel(double x) { return ov_exp_sel(x); }
double ov_oracle_log_sel(double x) { return ov_log_sel(x); }

/* krome_x2n / krome_n2x of the reference's PRIMORDIAL driver
   (tests/primordial.f90:117-140): direction 0, n = rhogas * x * imass;
   direction 1, x = n * mass / rhogas; entries without a mass are copied.
   Returns -1 for an unknown network, -5 for one without masses. */
int ov_oracle_convert(const char* tag, int64_t ncells, int direction, const double* in, double* out,
                      const double* rho)
{
    if (!net_find(tag))
        return -1;
    const net_entry* e = NULL;
    for (int i = 0; i < NNETS; ++i)
        if (strcmp(g_entries[i].tag, tag) == 0)
            e = &g_entries[i];
    const int n = e->sizes[0];
    int any = 0;
    for (int j = 0; j < n; ++j)
        any |= e->mass[j] != 0.0;
    if (!any)
        return -5;
    for (int j = 0; j < n; ++j)
        for (int64_t c = 0; c < ncells; ++c) {
            const double v = in[(size_t)j * ncells + c];
            double o = v;
            if (e->mass[j] != 0.0)
                o = direction == 0 ? rho[c] * v * e->imass[j] : v * e->mass[j] / rho[c];
            out[(size_t)j * ncells + c] = o;
        }
    return 0;
}
