/* Lanes-per-cell BDF kernel for networks too large for one thread per cell.
 *
 * K lanes of a warp (K = 32, 16 or 8; 32/K cells per warp) integrate one
 * cell at a time (per-cell control, G = 1); each group of K lanes takes
 * cells from the global counter on its own.  Lane k of a group holds the
 * solver-state species k, k+K, ...: their Nordsieck history, correction,
 * previous correction, error weights and FP32 scale factors in registers.
 * The cell's full state vector, the packed LU and the solve vector live in
 * the group's slice of shared memory.  Control is uniform across a group,
 * so the reference's nested loops (src/odevec.F90: step loop :207,
 * predictor :259, corrector :321) are written as loops; every exchange
 * inside a group (__syncwarp, shuffles, votes) names the group's lanes only,
 * so the groups of one warp may be at different points of those loops.
 *
 * The network code comes from tables generated from the same emitted
 * straight-line C that the thread-per-cell kernel and the CPU oracle
 * compile (odevec_b200/wpc.py): right-hand-side terms per species, postfix
 * programs for the entries of P = I - dt*beta*J, and the LU factorisation
 * and triangular-solve statements grouped in dependency levels, one row of
 * K slots per level.  Norms are summed in species order by the group's
 * first lane.  Every value is therefore produced by the same IEEE
 * operations in the same order as in the thread kernel, and the FP64 form
 * without fused multiply-add is bit-identical to the oracle.
 *
 * All loops are bounded as in the thread kernel (max_attempts, 4 Newton
 * iterations, 10 consecutive Newton failures); no group waits on another. */
#pragma once

namespace ov {
namespace OV_MODE_NS {

/* x^y out of line: the step-size selection calls it three times */
static __device__ __noinline__ double pow_dev(double x, double y) { return ov_pow(x, y); }

/* Shared memory of one cell's group and the block shape for K lanes per
   cell: 8 warps per block; K = 32 three blocks per SM (80 registers),
   K = 16 two (128 registers), K = 8 one (255 registers: 8 species' history
   per lane) */
template <class Net, class LUT, int K>
struct WpcLayout {
    static constexpr int N = Net::NEQ, ND = Net::ND, NNZ = Net::NNZ;
    /* doubles: state y[N], reduction scratch[ND], scale[ND], inverse scale[ND];
       then LUT: packed LU[NNZ], solve vector[N] */
    static constexpr size_t dbl_bytes = (size_t)(N + 3 * ND) * 8;
    static constexpr size_t group_bytes = (dbl_bytes + (size_t)(NNZ + N) * sizeof(LUT) + 15) / 16 * 16;
    static constexpr int WARPS = 8;
    static constexpr int GROUPS = WARPS * (32 / K); /* cells in flight per block */
    static constexpr int MINB = K == 32 ? 3 : (K == 16 ? 2 : 1);
    static constexpr size_t block_bytes = group_bytes * GROUPS;
};

/* the level rows laid out for K lanes */
template <class W, int K>
struct WpcLevels;
template <class W>
struct WpcLevels<W, 32> {
    static constexpr int NFL = W::NFL, NSL = W::NSL;
    __device__ static const long long* fac() { return W::fac_op(); }
    __device__ static const long long* sol() { return W::sol_op(); }
};
template <class W>
struct WpcLevels<W, 16> {
    static constexpr int NFL = W::NFL16, NSL = W::NSL16;
    __device__ static const long long* fac() { return W::fac_op16(); }
    __device__ static const long long* sol() { return W::sol_op16(); }
};
template <class W>
struct WpcLevels<W, 8> {
    static constexpr int NFL = W::NFL8, NSL = W::NSL8;
    __device__ static const long long* fac() { return W::fac_op8(); }
    __device__ static const long long* sol() { return W::sol_op8(); }
};

template <class Net, class LUT, int K>
struct WCell {
    using W = typename Net::Wpc;
    using Lv = WpcLevels<W, K>;
    static constexpr int N = Net::NEQ, ND = Net::ND, NF = Net::NF, NNZ = Net::NNZ;
    static constexpr int NS = (ND + K - 1) / K; /* solver species per lane */
    static constexpr bool SCALED = sizeof(LUT) == 4;

    int sub;        /* lane within the cell's group, 0..K-1 */
    int glead;      /* warp lane of the group's first lane */
    unsigned gmask; /* the group's lanes */
    double* yv;   /* [N] full state */
    double* red;  /* [ND] */
    double* scv;  /* [ND] */
    double* iscv; /* [ND] */
    LUT* a;       /* [NNZ] */
    LUT* dv;      /* [N] by storage row */

    double yns[MAXQ + 1][NS], en[NS], eno[NS], w2[NS], sc[NS], isc[NS];
    int sp[NS];   /* species of the owned solver indices (-1: none) */
    double t, h, told, tstop, crate, jchg, cerr, tint, fz_add;
    int q, swu, lju, fet, fc, it;
    bool ujac, nuo, first, msk, fz_neg;
    int status, attempts, steps, ltef, convf, newt, jacs, ppass;

    __device__ __forceinline__ bool own(int m) const { return sp[m] >= 0; }

    /* sum over solver indices 0..ND-1 in order of the per-index values p */
    __device__ __forceinline__ double ordered_sum(const double (&p)[NS])
    {
        __syncwarp(gmask);
#pragma unroll
        for (int m = 0; m < NS; ++m)
            if (own(m))
                red[sub + K * m] = p[m];
        __syncwarp(gmask);
        double s = 0.0;
        if (sub == 0)
            for (int j = 0; j < ND; ++j)
                s = s + red[j];
        s = __shfl_sync(gmask, s, glead);
        return s;
    }

    __device__ __forceinline__ double wnorm(const double (&e)[NS])
    {
        double p[NS];
#pragma unroll
        for (int m = 0; m < NS; ++m)
            p[m] = own(m) ? e[m] * e[m] * w2[m] : 0.0;
        double s = ordered_sum(p);
        s = s + fz_add;
        const double v = msk ? sqrt(s / N) : -HUGE_VAL;
        return group_max<1>(v);
    }

    __device__ __forceinline__ void weights(double rtol, double atol)
    {
#pragma unroll
        for (int m = 0; m < NS; ++m)
            if (own(m)) {
                const double w = __drcp_rn(rtol * fabs(yv[sp[m]]) + atol);
                w2[m] = w * w;
            }
    }

    __device__ __forceinline__ void frozen_flags(double rtol, double atol)
    {
        bool bad = false, neg = false;
#pragma unroll
        for (int j = 0; j < NF; ++j) {
            const double v = yv[Net::frozen(j)];
            double w = 1.0 / (rtol * fabs(v) + atol);
            w = w * w;
            bad |= !(w - w == 0.0);
            neg |= v < 0.0;
        }
        fz_add = bad ? __longlong_as_double(0x7ff8000000000000LL) : 0.0;
        fz_neg = neg;
    }

    /* f for the owned species from the term tables */
    __device__ __forceinline__ void rhs(double (&f)[NS]) const
    {
        const int* ptr = W::rhs_ptr();
        const double* coef = W::rhs_coef();
        const int* fac = W::rhs_fac();
#pragma unroll
        for (int m = 0; m < NS; ++m) {
            if (!own(m)) {
                f[m] = 0.0;
                continue;
            }
            const int j = sub + K * m;
            const int p0 = ptr[j], p1 = ptr[j + 1];
            double acc = 0.0;
            for (int tt = p0; tt < p1; ++tt) {
                double v = coef[tt];
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const int code = fac[3 * tt + k];
                    if (code >= 0) {
                        const double yy = yv[code >> 1];
                        v = v * ((code & 1) ? yy * yy : yy);
                    }
                }
                acc = tt == p0 ? v : acc + v;
            }
            f[m] = acc;
        }
    }

    /* Loops over the runtime order run to MAXQ with predicates (the same
       operations in the same order), so the history stays in registers. */
    __device__ __forceinline__ void predict()
    {
        ppass += q * (q + 1) / 2;
#pragma unroll
        for (int m = 0; m < NS; ++m) {
#pragma unroll
            for (int l = 0; l < MAXQ; ++l)
#pragma unroll
                for (int k = MAXQ; k >= 1; --k)
                    if (l <= q - 1 && k <= q && k >= l + 1)
                        yns[k - 1][m] = yns[k][m] + yns[k - 1][m];
            en[m] = 0.0;
        }
    }

    __device__ __forceinline__ void reset()
    {
        ppass += q * (q + 1) / 2;
#pragma unroll
        for (int m = 0; m < NS; ++m)
#pragma unroll
            for (int k = 0; k < MAXQ; ++k)
#pragma unroll
                for (int jj = MAXQ; jj >= 1; --jj)
                    if (k <= q - 1 && jj <= q && jj >= k + 1)
                        yns[jj - 1][m] = yns[jj - 1][m] - yns[jj][m];
    }

    __device__ __forceinline__ void set_step(double dt_scale)
    {
        double dtt = 1.0;
#pragma unroll
        for (int k = 1; k <= MAXQ; ++k) {
            if (k <= q) {
                dtt = dt_scale * dtt;
#pragma unroll
                for (int m = 0; m < NS; ++m)
                    yns[k][m] = yns[k][m] * dtt;
            }
        }
        h = h * dt_scale;
        jchg = jchg * dt_scale;
    }

    __device__ __forceinline__ void update_nordsieck()
    {
#pragma unroll
        for (int k = 0; k <= MAXQ; ++k) {
            if (k <= q) {
                const double c = lcoef(q, k);
#pragma unroll
                for (int m = 0; m < NS; ++m)
                    yns[k][m] = yns[k][m] + en[m] * c;
            }
        }
    }

    /* yns[k] for a runtime k, selected with compile-time indices */
    __device__ __forceinline__ double hist(int k, int m) const
    {
        double v = 0.0;
#pragma unroll
        for (int kk = 0; kk <= MAXQ; ++kk)
            if (kk == k)
                v = yns[kk][m];
        return v;
    }

    __device__ __forceinline__ void set_y_from(const double (&v)[NS])
    {
        __syncwarp(gmask);
#pragma unroll
        for (int m = 0; m < NS; ++m)
            if (own(m) && msk)
                yv[sp[m]] = v[m];
        __syncwarp(gmask);
    }

    __device__ __forceinline__ void interpolate()
    {
        const double rel_t = (tstop - t) / h;
        double v[NS];
#pragma unroll
        for (int m = 0; m < NS; ++m) {
            double acc = hist(q, m);
#pragma unroll
            for (int k = MAXQ - 1; k >= 0; --k)
                if (k <= q - 1)
                    acc = yns[k][m] + rel_t * acc;
            v[m] = acc;
        }
        set_y_from(v);
    }

    __device__ __forceinline__ double step_size_order()
    {
        const int order = q;
        double down, same, up;
        if (order == 1) {
            down = 0.0;
        } else {
            double e[NS];
#pragma unroll
            for (int m = 0; m < NS; ++m)
                e[m] = hist(order, m);
            down = 1.0 / ((double)1.3f * pow_dev(wnorm(e) / tau(order, order - 1), 1.0 / order) + 1e-6);
        }
        same = 1.0 / ((double)1.2f * pow_dev(wnorm(en) / tau(order, order), 1.0 / (order + 1.0)) + 1e-6);
        if (order == MAXQ || nuo) {
            up = 0.0;
        } else {
            double d[NS];
#pragma unroll
            for (int m = 0; m < NS; ++m)
                d[m] = en[m] - eno[m];
            up = 1.0 / ((double)1.4f * pow_dev(wnorm(d) / tau(order, order + 1), 1.0 / (order + 2.0)) + 1e-6);
        }
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
                    for (int kk = 1; kk <= MAXQ; ++kk)
                        if (kk == order + 1)
#pragma unroll
                            for (int m = 0; m < NS; ++m)
                                yns[kk][m] = c * en[m] / (order + 1.0);
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

    __device__ __forceinline__ bool any_negative_yns0() const
    {
        bool neg = fz_neg;
#pragma unroll
        for (int m = 0; m < NS; ++m)
            neg |= own(m) && yns[0][m] < 0.0;
        return __any_sync(gmask, msk && neg);
    }

    __device__ __forceinline__ bool any_negative_y() const
    {
        bool neg = fz_neg;
#pragma unroll
        for (int m = 0; m < NS; ++m)
            neg |= own(m) && yv[sp[m]] < 0.0;
        return __any_sync(gmask, msk && neg);
    }

    /* GetJac + LUDecompose (src/odevec.F90:301-315) from the tables */
    __device__ void jacobian_lu()
    {
        if constexpr (SCALED) {
#pragma unroll
            for (int m = 0; m < NS; ++m)
                if (own(m)) {
                    int e = (int)((ov_d2bits(w2[m]) >> 52) & 0x7ff) - 1023;
                    int hexp = e >= 0 ? e / 2 : -((-e + 1) / 2);
                    hexp = hexp > 480 ? 480 : (hexp < -480 ? -480 : hexp);
                    sc[m] = ov_pow2i(hexp);
                    isc[m] = ov_pow2i(-hexp);
                    scv[sub + K * m] = sc[m];
                    iscv[sub + K * m] = isc[m];
                }
        }
        __syncwarp(gmask);
        const double beta = lcoef(q, 0);
        const int* ptr = W::jac_ptr();
        const int* code = W::jac_code();
        const double* cst = W::jac_const();
        for (int e = sub; e < NNZ; e += K) {
            double st[W::DEPTH];
            int top = 0;
            for (int pc = ptr[e]; pc < ptr[e + 1]; ++pc) {
                const int c = code[pc];
                const int op = c & 15, arg = c >> 4;
                switch (op) {
                case 0: st[top++] = cst[arg]; break;
                case 1: st[top++] = yv[arg]; break;
                case 2: st[top++] = beta; break;
                case 3: st[top++] = h; break;
                case 4: st[top - 1] = -st[top - 1]; break;
                case 5: st[top - 2] = st[top - 2] + st[top - 1]; --top; break;
                case 6: st[top - 2] = st[top - 2] - st[top - 1]; --top; break;
                case 7: st[top - 2] = st[top - 2] * st[top - 1]; --top; break;
                default: st[top - 2] = st[top - 2] / st[top - 1]; --top; break;
                }
            }
            if constexpr (SCALED) {
                const int rc = W::jac_rc()[e];
                a[e] = (LUT)(st[0] * scv[rc & 0xffff] * iscv[rc >> 16]);
            } else {
                a[e] = (LUT)(st[0]);
            }
        }
        __syncwarp(gmask);
        /* one row of K statement slots per level (a negative slot is
           empty); the rows run in order with the cell's lanes synchronised
           between */
        const long long* ops = Lv::fac();
#pragma unroll 4
        for (int l = 0; l < Lv::NFL; ++l) {
            const long long o = ops[l * K + sub];
            if (o >= 0) {
                const int x = (int)((o >> 1) & 0xfffff), y = (int)((o >> 21) & 0xfffff);
                if ((o & 1) == 0)
                    a[x] = a[x] / a[y];
                else
                    a[x] = a[x] - a[y] * a[(int)((o >> 41) & 0xfffff)];
            }
            __syncwarp(gmask);
        }
    }

    /* residual, solve, Newton update (src/odevec.F90:323-352) */
    __device__ void newton_update(const double (&f)[NS], double (&den)[NS])
    {
        const int* srow = W::srow();
#pragma unroll
        for (int m = 0; m < NS; ++m)
            if (own(m)) {
                const double res = h * f[m] - (yns[1][m] + en[m]);
                if constexpr (SCALED)
                    dv[srow[sub + K * m]] = (LUT)(res * sc[m]);
                else
                    dv[srow[sub + K * m]] = (LUT)(res * 1.0);
            }
        __syncwarp(gmask);
        const long long* ops = Lv::sol();
#pragma unroll 4
        for (int l = 0; l < Lv::NSL; ++l) {
            const long long o = ops[l * K + sub];
            if (o >= 0) {
                const int x = (int)((o >> 1) & 0xfffff), k = (int)((o >> 41) & 0xfffff);
                if ((o & 1) == 0)
                    dv[x] = dv[x] / a[k];
                else
                    dv[x] = dv[x] - dv[(int)((o >> 21) & 0xfffff)] * a[k];
            }
            __syncwarp(gmask);
        }
        const double l0 = lcoef(q, 0);
        double v[NS];
#pragma unroll
        for (int m = 0; m < NS; ++m) {
            if (own(m)) {
                if constexpr (SCALED)
                    den[m] = (double)dv[srow[sub + K * m]] * isc[m];
                else
                    den[m] = (double)dv[srow[sub + K * m]] * 1.0;
                en[m] = en[m] + den[m];
                v[m] = yns[0][m] + l0 * en[m];
            } else {
                den[m] = 0.0;
                v[m] = 0.0;
            }
        }
        set_y_from(v);
    }

    __device__ __forceinline__ void check_convergence(const double (&d)[NS], bool& failed, bool& converged)
    {
        const double err = wnorm(d);
        double rate_tmp = 0.0;
        if (it != 0) {
            rate_tmp = err / cerr;
            crate = fmax(0.2 * crate, rate_tmp);
        }
        const double r15 = 1.5 * crate;
        const double crit = err * (1.0 < r15 ? 1.0 : r15) / conv_divisor(q);
        bool nan = fz_add != fz_add;
#pragma unroll
        for (int m = 0; m < NS; ++m)
            nan |= own(m) && ((d[m] != d[m]) | (w2[m] != w2[m]));
        if (__any_sync(gmask, nan)) {
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

    __device__ __forceinline__ double initial_step(const double (&f)[NS], double rtol, double atol)
    {
        weights(rtol, atol);
        const double tol = rtol;
        const double W0 = fabs(t) > fabs(tstop) ? fabs(t) : fabs(tstop);
        double p[NS];
#pragma unroll
        for (int m = 0; m < NS; ++m)
            p[m] = own(m) ? f[m] * f[m] * (w2[m] * tol * tol) : 0.0;
        double s = ordered_sum(p);
        s = s + fz_add;
        const double mx = group_max<1>(msk ? s : -HUGE_VAL);
        /* W0**(-2.0): a real exponent other than -1, 0, 1 or 2 is a pow() call
           in the reference's compiled Fortran, not 1/(W0*W0) */
        const double d = sqrt(tol / (ov_pow(W0, -2.0) + mx / N));
        const double span = fabs(tstop - t);
        return d < span ? d : span;
    }

    __device__ void save_state(double* ws, int64_t n, int64_t cell) const
    {
#pragma unroll
        for (int k = 0; k <= MAXQ; ++k)
#pragma unroll
            for (int m = 0; m < NS; ++m)
                if (own(m))
                    ws[((int64_t)k * ND + sub + K * m) * n + cell] = yns[k][m];
        const int f = (MAXQ + 1) * ND;
#pragma unroll
        for (int m = 0; m < NS; ++m)
            if (own(m)) {
                ws[((int64_t)f + sub + K * m) * n + cell] = eno[m];
                ws[((int64_t)f + ND + sub + K * m) * n + cell] = w2[m];
            }
        if (sub == 0) {
            const int g = f + 2 * ND;
            const double scl[12] = {tint, h, crate, jchg, (double)q, (double)swu, (double)lju, (double)fet,
                                    (double)fc, ujac ? 1.0 : 0.0, nuo ? 1.0 : 0.0, first ? 1.0 : 0.0};
            for (int i = 0; i < 12; ++i)
                ws[((int64_t)g + i) * n + cell] = scl[i];
        }
    }

    __device__ void load_state(const double* ws, int64_t n, int64_t cell)
    {
#pragma unroll
        for (int k = 0; k <= MAXQ; ++k)
#pragma unroll
            for (int m = 0; m < NS; ++m)
                yns[k][m] = own(m) ? ws[((int64_t)k * ND + sub + K * m) * n + cell] : 0.0;
        const int f = (MAXQ + 1) * ND;
#pragma unroll
        for (int m = 0; m < NS; ++m)
            if (own(m)) {
                eno[m] = ws[((int64_t)f + sub + K * m) * n + cell];
                w2[m] = ws[((int64_t)f + ND + sub + K * m) * n + cell];
            }
        const int g = f + 2 * ND;
        t = ws[((int64_t)g + 0) * n + cell];
        h = ws[((int64_t)g + 1) * n + cell];
        crate = ws[((int64_t)g + 2) * n + cell];
        jchg = ws[((int64_t)g + 3) * n + cell];
        q = (int)ws[((int64_t)g + 4) * n + cell];
        swu = (int)ws[((int64_t)g + 5) * n + cell];
        lju = (int)ws[((int64_t)g + 6) * n + cell];
        fet = (int)ws[((int64_t)g + 7) * n + cell];
        fc = (int)ws[((int64_t)g + 8) * n + cell];
        ujac = ws[((int64_t)g + 9) * n + cell] != 0.0;
        nuo = ws[((int64_t)g + 10) * n + cell] != 0.0;
        first = ws[((int64_t)g + 11) * n + cell] != 0.0;
    }

    /* SolveODE for one cell (src/odevec.F90:158-214 with :242-465), in the
       thread kernel's phase order: returns with status set; write_y tells
       whether the state holds the interpolated result */
    __device__ void solve(const LaunchArgs& A, int64_t ncells, int64_t cell, bool& write_y)
    {
        write_y = false;
        if (!msk) {
            t = tstop; /* src/odevec.F90:187-191 */
            return;
        }
        double f[NS], den[NS];
        if (A.resume == 1) {
            load_state(A.ws, A.stride, cell);
            double v[NS];
#pragma unroll
            for (int m = 0; m < NS; ++m)
                v[m] = yns[0][m];
            set_y_from(v);
            ujac = true;
            if (!(t < tstop)) {
                write_y = true;
                interpolate();
                tint = t;
                t = tstop;
                return;
            }
            told = t;
        } else {
            if (A.resume == 2) {
                /* the previous call's last correction vector (this%en_old) */
                const int f0 = (MAXQ + 1) * ND;
#pragma unroll
                for (int m = 0; m < NS; ++m)
                    if (own(m))
                        eno[m] = A.ws[((int64_t)f0 + sub + K * m) * A.stride + cell];
            }
#pragma unroll
            for (int m = 0; m < NS; ++m)
                yns[0][m] = own(m) ? yv[sp[m]] : 0.0;
            rhs(f);
#pragma unroll
            for (int m = 0; m < NS; ++m)
                yns[1][m] = h * f[m];
            h = initial_step(f, A.rtol, A.atol);
            if (!(t < tstop)) {
                write_y = true;
                interpolate();
                tint = t;
                t = tstop;
                return;
            }
            told = t;
        }
        for (;;) {
            /* predictor attempt (src/odevec.F90:259-299) */
            if (++attempts > A.max_attempts) {
                status = OV_ERR_MAX_STEPS;
                return;
            }
            t = t + h;
            predict();
            if (A.check_neg && any_negative_yns0()) {
                t = told;
                reset();
                set_step(0.25);
                if (h <= A.dt_min) {
                    status = OV_ERR_DTMIN_PREDICTOR;
                    return;
                }
                continue;
            }
            {
                double v[NS];
#pragma unroll
                for (int m = 0; m < NS; ++m)
                    v[m] = yns[0][m];
                set_y_from(v);
            }
            it = 0;
            if (ujac) {
                jacobian_lu();
                jacs++;
                ujac = false;
                lju = 0;
                crate = 0.7;
                jchg = 1.0;
            }
            /* corrector (src/odevec.F90:318-394) */
            int ss_mode = 0;
            for (;;) {
                rhs(f);
                newt++;
                newton_update(f, den);
                bool failed = false, converged = false;
                check_convergence(den, failed, converged);
                if (A.check_neg && any_negative_y()) {
                    failed = true;
                    converged = false;
                }
                if (failed && !converged) {
                    t = told;
                    fc++;
                    convf++;
                    if (fc > 10) {
                        status = OV_ERR_CONV_FAILURES;
                        return;
                    }
                    it = 0;
                    reset();
                    set_step(0.25);
                    if (h < A.dt_min) {
                        status = OV_ERR_DTMIN_CONV;
                        return;
                    }
                    ujac = true;
                    ss_mode = -1; /* another predictor attempt */
                    break;
                }
                if (converged)
                    break;
            }
            if (ss_mode == -1)
                continue;
            fc = 0;
            /* local truncation error test (src/odevec.F90:400-455) */
            const double error = wnorm(en) / tau(q, q);
            weights(A.rtol, A.atol);
            if (error > 1.0) {
                ltef++;
                t = told;
                if (fet >= 3) {
                    if (A.fix_restart)
                        reset();
                    q = 1;
                    double v[NS];
#pragma unroll
                    for (int m = 0; m < NS; ++m)
                        v[m] = yns[0][m];
                    set_y_from(v);
                    /* src/odevec.F90:417-421 */
                    rhs(f);
#pragma unroll
                    for (int m = 0; m < NS; ++m)
                        yns[1][m] = h * f[m];
                    ujac = true;
                } else {
                    reset();
                    ujac = true;
                    swu = 0;
                    nuo = true;
                }
                const double s = step_size_order();
                if (status)
                    return;
                set_step(s);
                fet++; /* src/odevec.F90:434-439 */
                continue;
            }
            swu++;
            lju++;
            update_nordsieck();
            if (swu == q + 1) {
                const double s = step_size_order();
                if (status)
                    return;
                set_step(s);
            }
            /* end of an accepted step (src/odevec.F90:452-464) */
            fet = 0;
            steps++;
            if (lju >= 20)
                ujac = true;
            else if (fabs(jchg - (double)1.0f) > (double)0.3f)
                ujac = true;
#pragma unroll
            for (int m = 0; m < NS; ++m)
                eno[m] = en[m];
            if (t < tstop) {
                told = t;
                continue;
            }
            write_y = true;
            interpolate();
            tint = t;
            t = tstop;
            return;
        }
    }
};

template <class Net, class LUT, int K>
__global__ void __launch_bounds__(256, (WpcLayout<Net, LUT, K>::MINB)) wpc_kernel(const LaunchArgs A)
{
    using L = WpcLayout<Net, LUT, K>;
    using C = WCell<Net, LUT, K>;
    constexpr int N = Net::NEQ, ND = Net::ND, NNZ = Net::NNZ, NS = C::NS;
    static_assert(K == 8 || K == 16 || K == 32, "8, 16 or 32 lanes per cell");
    if (A.run_if && *A.run_if == 0)
        return;
    extern __shared__ __align__(16) unsigned char ov_wsmem[];
    const int lane = threadIdx.x & 31;
    const int sub = lane % K;
    const int group = threadIdx.x / K; /* the cell slot of this block */
    unsigned char* base = ov_wsmem + (size_t)group * L::group_bytes;
    C c;
    c.sub = sub;
    c.glead = lane - sub;
    c.gmask = K == 32 ? FULL : (((1u << K) - 1u) << (lane - sub));
    c.yv = reinterpret_cast<double*>(base);
    c.red = c.yv + N;
    c.scv = c.red + ND;
    c.iscv = c.scv + ND;
    c.a = reinterpret_cast<LUT*>(base + L::dbl_bytes);
    c.dv = c.a + NNZ;
    const int* dyn = Net::Wpc::dyn();
#pragma unroll
    for (int m = 0; m < NS; ++m) {
        const int j = sub + K * m;
        c.sp[m] = j < ND ? dyn[j] : -1;
        c.sc[m] = 1.0;
        c.isc[m] = 1.0;
    }
    const int64_t ncells = A.ncells;
    for (bool first_cell = true;; first_cell = false) {
        /* a yield request (LaunchArgs::yield), seen before any cell but the
           group's first of this launch, ends the group's work */
        int stop = 0;
        if (!first_cell && A.yield) {
            if (sub == 0)
                stop = *(volatile const int32_t*)A.yield;
            stop = __shfl_sync(c.gmask, stop, c.glead);
        }
        if (stop)
            break;
        unsigned long long g = 0;
        if (sub == 0)
            g = atomicAdd(A.queue, 1ull);
        const int64_t q = (int64_t)__shfl_sync(c.gmask, g, c.glead);
        if (q >= ncells)
            break;
        const int64_t cell = A.order ? (int64_t)A.order[q] : q;
        __syncwarp(c.gmask);
        for (int s = sub; s < N; s += K) {
            c.yv[s] = A.y[(int64_t)s * A.stride + cell];
            if (A.save_y) /* the inputs, for the FP32-LU form's escalation */
                A.save_y[(int64_t)s * ncells + cell] = c.yv[s];
        }
        __syncwarp(c.gmask);
        c.t = A.t[cell];
        c.h = A.dt[cell];
        if (A.save_y && sub == 0) {
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
#pragma unroll
        for (int m = 0; m < NS; ++m) {
#pragma unroll
            for (int k = 0; k <= MAXQ; ++k)
                c.yns[k][m] = 0.0;
            c.eno[m] = 0.0;
            c.en[m] = 0.0;
        }
        c.weights(A.rtol, A.atol);
        c.frozen_flags(A.rtol, A.atol);
        bool write_y = false;
        c.solve(A, ncells, cell, write_y);
        /* store (the thread kernel's phase DONE) */
        const bool ok = c.status == OV_OK;
        if (A.ws && ok && write_y)
            c.save_state(A.ws, A.stride, cell);
        __syncwarp(c.gmask);
        if ((!ok || write_y) && c.msk) {
#pragma unroll
            for (int m = 0; m < NS; ++m)
                if (c.own(m))
                    A.y[(int64_t)c.sp[m] * A.stride + cell] = c.yv[c.sp[m]];
        }
        if (sub == 0) {
            A.t[cell] = c.t;
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
        }
    }
}

template <class Net, class LUT, int K>
cudaError_t launch_wpc(const LaunchArgs& a, int grid, cudaStream_t stream)
{
    using L = WpcLayout<Net, LUT, K>;
    auto kern = wpc_kernel<Net, LUT, K>;
    constexpr int block = 32 * L::WARPS;
    static int cached = 0;
    if (cached == 0) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        if (L::block_bytes > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)L::block_bytes);
            if (e != cudaSuccess)
                return e;
        }
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, block, L::block_bytes);
        cached = sms * (per_sm > 0 ? per_sm : 1);
    }
    if (grid <= 0) {
        grid = cached;
        const int64_t blocks_needed = (a.ncells + L::GROUPS - 1) / L::GROUPS;
        if (blocks_needed < grid)
            grid = (int)blocks_needed;
        if (grid < 1)
            grid = 1;
    }
    kern<<<grid, block, L::block_bytes, stream>>>(a);
    return cudaGetLastError();
}

/* lanes-per-cell tables exist for this variant (constant-coefficient
   network, CSC packaging, LUmethod 1) and its shared memory fits the SM
   with the layout's blocks per SM */
template <class Net, class LUT, int K>
constexpr bool wpc_ok()
{
    if constexpr (!Net::HAS_WPC)
        return false;
    else
        return WpcLayout<Net, LUT, K>::block_bytes * WpcLayout<Net, LUT, K>::MINB <= 226 * 1024;
}

}  // namespace OV_MODE_NS
}  // namespace ov
