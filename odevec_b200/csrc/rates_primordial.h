/* Rate coefficients of the 16-species primordial network.
 *
 * Restates the reference's coe() (src/odevec_commons.F90:101-384), a KROME
 * rate-coefficient function, with two changes of structure and none of value:
 *
 *  1. The gas temperature is read per cell from the state vector
 *     (y[14], species "Tgas", whose right-hand side is 0) instead of the
 *     constant 1000 K the reference hard-codes (src/odevec_commons.F90:120-124).
 *     Setting y[14] = 1000 for every cell reproduces the reference.
 *  2. coe() is evaluated by the reference on every right-hand-side and
 *     Jacobian call.  Its value is small + r_j(Tgas), where only
 *     small = 1e-40 / max(max_j y_j, 1)^3 depends on the current state
 *     (src/odevec_commons.F90:127-130).  Tgas is constant during a solve, so
 *     ov_rates_primordial_T() computes the temperature part r_j once per
 *     solve and ov_rates_primordial_k() adds the state-dependent floor on
 *     every call: k_j = small + r_j, exactly the reference's value (an
 *     inactive temperature branch has r_j = 0 and k_j = small, as the
 *     reference initialises vec_k = small, src/odevec_commons.F90:139-141).
 *
 * The exponentials, logarithms and powers are the branch-free forms of
 * ov_common.h (the same bits as ov_exp, ov_log, ov_pow), so the compiler can
 * interleave the independent rate laws.
 *
 * Fortran literal kinds are kept: a real literal written without a d
 * exponent is single precision in the reference (e.g. 0.396 in reaction 31,
 * the constants of reactions 32 and 34, and the 1/300 of T32), so it appears
 * here as a float literal converted to double.  Integer powers are expanded
 * as gfortran expands them (x^3 = x*x^2, x^5 = x^2*x^3, x^7 = x^3*x^4,
 * x^9 = x^3*x^6); real powers use ov_pow. */
#ifndef OV_RATES_PRIMORDIAL_H
#define OV_RATES_PRIMORDIAL_H

#include "ov_common.h"

#define OV_PRIMORDIAL_NREA 38

OV_HD static OV_INLINE void ov_rates_primordial_T(double Tgas, double* OV_RESTRICT r)
{
    const double Te = Tgas * 8.617343e-5;                 /* eV */
    const double lnTe = ov_log_sel(Te);
    const double T32 = Tgas * (double)0.0033333333333333335f; /* Tgas/300 K, single-precision literal */
    const double invT = 1.0 / Tgas;
    const double invTe = 1.0 / Te;
    const double sqrTgas = sqrt(Tgas);
    /* powers of ln Te as x^n = x^(n-t) * x^t */
    const double l1 = lnTe;
    const double l2 = l1 * l1;
    const double l3 = l1 * l2;
    const double l4 = l2 * l2;
    const double l5 = l2 * l3;
    const double l6 = l3 * l3;
    const double l7 = l3 * l4;
    const double l8 = l4 * l4;
    const double l9 = l3 * l6;

    for (int i = 0; i < OV_PRIMORDIAL_NREA; ++i)
        r[i] = 0.0;

    /* 1: H + E -> H+ + E + E */
    r[0] = ov_exp_sel(-32.71396786 + 13.5365560 * l1 - 5.73932875 * l2 + 1.56315498 * l3
                  - 0.28770560 * l4 + 3.48255977e-2 * l5 - 2.63197617e-3 * l6
                  + 1.11954395e-4 * l7 - 2.03914985e-6 * l8);
    /* 2, 3: H+ + E -> H */
    if (Tgas <= 5.5e3)
        r[1] = 3.92e-13 * ov_pow_sel(invTe, 0.6353);
    if (Tgas > 5.5e3)
        r[2] = ov_exp_sel(-28.61303380689232 - 0.7241125657826851 * l1 - 0.02026044731984691 * l2
                      - 0.002380861877349834 * l3 - 0.0003212605213188796 * l4
                      - 0.00001421502914054107 * l5 + 4.989108920299513e-6 * l6
                      + 5.755614137575758e-7 * l7 - 1.856767039775261e-8 * l8
                      - 3.071135243196595e-9 * l9);
    /* 4: HE + E -> HE+ + E + E */
    r[3] = ov_exp_sel(-44.09864886 + 23.91596563 * l1 - 10.7532302 * l2 + 3.05803875 * l3
                  - 0.56851189 * l4 + 6.79539123e-2 * l5 - 5.00905610e-3 * l6
                  + 2.06723616e-4 * l7 - 3.64916141e-6 * l8);
    /* 5, 6: HE+ + E -> HE */
    if (Tgas <= 9.28e3)
        r[4] = 3.92e-13 * ov_pow_sel(invTe, 0.6353);
    if (Tgas > 9.28e3)
        r[5] = 1.54e-9 * (1.0 + 0.3 / ov_exp_sel(8.099328789667 * invTe))
                   / (ov_exp_sel(40.49664394833662 * invTe) * ov_pow_sel(Te, 1.5))
               + 3.92e-13 / ov_pow_sel(Te, 0.6353);
    /* 7: HE+ + E -> HE++ + E + E */
    r[6] = ov_exp_sel(-68.71040990212001 + 43.93347632635 * l1 - 18.48066993568 * l2
                  + 4.701626486759002 * l3 - 0.7692466334492 * l4 + 0.08113042097303 * l5
                  - 0.005324020628287001 * l6 + 0.0001975705312221 * l7
                  - 3.165581065665e-6 * l8);
    /* 8: HE++ + E -> HE+ */
    r[7] = 3.36e-10 / sqrTgas / ov_pow_sel(Tgas / 1.e3, 0.2) / (1.0 + ov_pow_sel(Tgas / 1.e6, 0.7));
    /* 9: H + E -> H- */
    r[8] = 6.77e-15 * ov_pow_sel(Te, 0.8779);
    /* 10, 11: H- + H -> H2 + E (neither branch at exactly 1160 K) */
    if (Tgas < 1160.0)
        r[9] = 1.43e-9;
    if (Tgas > 1160.0)
        r[10] = ov_exp_sel(-20.06913897587003 + 0.2289800603272916 * l1 + 0.03599837721023835 * l2
                       - 0.004555120027032095 * l3 - 0.0003105115447124016 * l4
                       + 0.0001073294010367247 * l5 - 8.36671960467864e-6 * l6
                       + 2.238306228891639e-7 * l7);
    /* 12, 13: H + H+ -> H2+ */
    if (Tgas <= 6.7e3)
        r[11] = 1.85e-23 * ov_pow_sel(Tgas, 1.8);
    if (Tgas > 6.7e3)
        r[12] = 5.81e-16 * ov_pow_sel(Tgas / 5.62e4, -0.6657 * ov_log10_sel(Tgas / 5.62e4));
    /* 14: H2+ + H -> H2 + H+ */
    r[13] = 6.0e-10;
    /* 15: H2 + H+ -> H2+ + H */
    if (Tgas > 3.48e3)
        r[14] = ov_exp_sel(-24.24914687731536 + 3.400824447095291 * l1 - 3.898003964650152 * l2
                       + 2.045587822403071 * l3 - 0.5416182856220388 * l4
                       + 0.0841077503763412 * l5 - 0.007879026154483455 * l6
                       + 0.0004138398421504563 * l7 - 9.36345888928611e-6 * l8);
    /* 16: H2 + E -> H + H + E */
    r[15] = 5.6e-11 * ov_exp_sel(-102124.0 * invT) * sqrt(Tgas);
    /* 17: H2 + H -> H + H + H */
    r[16] = 1.0670825e-10 * ov_pow_sel(Te, 2.012) * ov_exp_sel(-4.463 * invTe)
            / ov_pow_sel(1.0 + 0.2472 * Te, 3.512);
    /* 18: H- + E -> H + E + E */
    r[17] = ov_exp_sel(-18.01849334273 + 2.360852208681 * l1 - 0.2827443061704 * l2
                   + 0.01623316639567 * l3 - 0.03365012031362999 * l4 + 0.01178329782711 * l5
                   - 0.001656194699504 * l6 + 0.0001068275202678 * l7 - 2.631285809207e-6 * l8);
    /* 19, 20: H- + H -> H + H + E */
    if (Tgas <= 1.16e3)
        r[18] = 2.56e-9 * ov_pow_sel(Te, 1.78186);
    if (Tgas > 1.16e3)
        r[19] = ov_exp_sel(-20.37260896533324 + 1.139449335841631 * l1 - 0.1421013521554148 * l2
                       + 0.00846445538663 * l3 - 0.0014327641212992 * l4
                       + 0.0002012250284791 * l5 + 0.0000866396324309 * l6
                       - 0.00002585009680264 * l7 + 2.4555011970392e-6 * l8
                       - 8.06838246118e-8 * l9);
    /* 21: H- + H+ -> H + H */
    r[20] = 6.5e-9 / sqrt(Te);
    /* 22: H- + H+ -> H2+ + E */
    r[21] = 1.e-8 * ov_pow_sel(Tgas, -0.4);
    /* 23, 24: H2+ + E -> H + H */
    if (Tgas <= 6.17e2)
        r[22] = 1.e-8;
    if (Tgas > 6.17e2)
        r[23] = 1.32e-6 * ov_pow_sel(Tgas, -0.76);
    /* 25: H2+ + H- -> H + H2 */
    r[24] = 5.e-7 * sqrt(1.e2 * invT);
    /* 26, 27: H + H + H -> H2 + H */
    if (Tgas <= 3e2)
        r[25] = 1.3e-32 * ov_pow_sel(T32, -0.38);
    if (Tgas > 3e2)
        r[26] = 1.3e-32 * ov_pow_sel(T32, -1.00);
    /* 28, 29: H2 + H + H -> H2 + H2 */
    if (Tgas <= 3e2)
        r[27] = 1.3e-32 * ov_pow_sel(T32, -0.38) / 8.0;
    if (Tgas > 3e2)
        r[28] = 1.3e-32 * ov_pow_sel(T32, -1.00) / 8.0;
    /* 30: H+ + D -> H + D+ */
    if (Tgas >= 5e1)
        r[29] = 2.00e-10 * ov_pow_sel(Tgas, 0.402) * ov_exp_sel(-37.1 * invT)
                - 3.31e-17 * ov_pow_sel(Tgas, 1.48);
    /* 31: H + D+ -> H+ + D  (0.396 and -0.332 are single-precision literals) */
    if (Tgas >= 5e1)
        r[30] = 2.06e-10 * ov_pow_sel(Tgas, (double)0.396f) * ov_exp_sel(-33.0 * invT)
                + 2.03e-9 * ov_pow_sel(Tgas, (double)-0.332f);
    /* 32: H2 + D+ -> HD + H+  (single-precision constants) */
    {
        const double L = ov_log10_sel(Tgas);
        r[31] = 1.e-9 * ((double)0.417f + (double)0.846f * L - (double)0.137f * (L * L));
    }
    /* 33: HD + H+ -> H2 + D+ */
    r[32] = 1.0e-9 * ov_exp_sel(-4.57e2 * invT);
    /* 34, 35: H2 + D -> HD + H  (34: single-precision constants) */
    if (Tgas <= 2.e3) {
        const double L = ov_log10_sel(Tgas);
        const double L2 = L * L, L3 = L * L2, L4 = L2 * L2, L5 = L2 * L3;
        r[33] = ov_pow_sel(10.0, (double)-56.4737f + (double)5.88886f * L + (double)7.19692f * L2
                                 + (double)2.25069f * L3 - (double)2.16903f * L4
                                 + (double)0.317887f * L5);
    }
    if (Tgas > 2e3)
        r[34] = 3.17e-10 * ov_exp_sel(-5207.0 * invT);
    /* 36: HD + H -> H2 + D */
    if (Tgas > 2e2)
        r[35] = 5.25e-11 * ov_exp_sel(-4430.0 * invT + 1.739e5 * (invT * invT));
    /* 37: D + H- -> HD + E */
    r[36] = 1.5e-9 * ov_pow_sel(T32, -0.1);
    /* 38: D+ + E -> D */
    r[37] = 3.6e-12 * ov_pow_sel(Tgas / 300.0, -0.75);
}

/* k_j = small + r_j with small = 1e-40 / nmax^3, nmax = max(max_j y_j, 1). */
OV_HD static OV_INLINE void ov_rates_primordial_k(const double* OV_RESTRICT y, int neq,
                                               const double* OV_RESTRICT r, double* OV_RESTRICT k)
{
    double nmax = y[0];
    for (int j = 1; j < neq; ++j)
        nmax = y[j] > nmax ? y[j] : nmax;
    nmax = nmax > 1.0 ? nmax : 1.0;
    const double small = 1e-40 / (nmax * nmax * nmax);
    for (int i = 0; i < OV_PRIMORDIAL_NREA; ++i)
        k[i] = small + r[i];
}

#endif /* OV_RATES_PRIMORDIAL_H */
