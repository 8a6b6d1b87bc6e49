/* Heating and cooling of the HCTOY heat/cool test network: the functions the
 * preprocessor's --heatcool=1 term calls for the gas-temperature row,
 *
 *   dTgas/dt = ((heating(y, Tgas) - cooling(y, Tgas)) * (gamma(y) - 1))
 *              / k_B / sum_{j < nmols} y_j
 *
 * (pre_odevec.py:556-561 with KROME's heating, cooling, krome_gamma and
 * boltzmann_erg).  A network built with --heatcool=1 --heatcool_header=<file>
 * includes a header like this one; it defines
 *   OV_HC_NMOLS                 number of chemical species (the first entries)
 *   ov_hc_heating(y, Tgas)      erg cm^-3 s^-1
 *   ov_hc_cooling(y, Tgas)      erg cm^-3 s^-1
 *   ov_hc_gamma(y)              adiabatic index
 *   OV_HC_BOLTZMANN             erg/K
 * as host+device functions.  The toy laws here (a constant heating per
 * particle; recombination and H2 line cooling) use only products and sqrt,
 * so CPU and GPU evaluate them to the same bits.  Species: E, H+, H, H2, HE,
 * CR, g, Tgas, dummy. */
#ifndef OV_HEATCOOL_HCTOY_H
#define OV_HEATCOOL_HCTOY_H
#include "ov_common.h"

#define OV_HC_NMOLS 5
#define OV_HC_BOLTZMANN 1.380648e-16

OV_HD static OV_INLINE double ov_hc_heating(const double* y, double Tgas)
{
    (void)Tgas;
    return 1.0e-25 * (y[2] + y[3] + y[4]);
}

OV_HD static OV_INLINE double ov_hc_cooling(const double* y, double Tgas)
{
    return 1.0e-23 * y[0] * y[1] * sqrt(Tgas) + 2.0e-24 * y[3] * Tgas;
}

OV_HD static OV_INLINE double ov_hc_gamma(const double* y)
{
    (void)y;
    return 5.0 / 3.0;
}

#endif /* OV_HEATCOOL_HCTOY_H */
