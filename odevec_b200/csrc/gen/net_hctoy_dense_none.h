/* Generated by odevec_b200.pre_odevec -- do not edit.
 * network HCTOY, packaging DENSE, ordering None, neq 9, LU nnz 30 (P nnz 30).
 * rhs(): f = dy/dt in species order (rate array k as in the reference).
 * jac(): P = I - dt*beta*J at the LU pattern positions, CSC storage order
 *        of the permuted matrix; fill-in positions are 0.  */
#ifndef OV_NET_HCTOY_DENSE_NONE_H
#define OV_NET_HCTOY_DENSE_NONE_H
#include "../ov_common.h"
#include "../heatcool_hctoy.h"

#define OV_HCTOY_DENSE_NONE_NEQ 9
#define OV_HCTOY_DENSE_NONE_NNZ 30
#define OV_HCTOY_DENSE_NONE_NREA 0
#define OV_HCTOY_DENSE_NONE_DENSE 1
#define OV_HCTOY_DENSE_NONE_NVECTOR 1
#define OV_HCTOY_DENSE_NONE_DT_MIN 1e-20
#define OV_HCTOY_DENSE_NONE_IDX_TGAS 7
static const int ov_hctoy_dense_none_sizes[8] = {9, 30, 0, 1, 7, 6, 1, 0};
static const double ov_hctoy_dense_none_defaults[2] = {1.0, 1e-20}; /* nvector, dt_min */
static const double ov_hctoy_dense_none_mass[9] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
static const double ov_hctoy_dense_none_imass[9] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
static const int ov_hctoy_dense_none_perm[9] = {0, 1, 2, 3, 4, 5, 6, 7, 8};
static const int ov_hctoy_dense_none_row_index[30] = {0, 1, 2, 7, 0, 1, 2, 7, 0, 1, 2, 3, 7, 2, 3, 7, 4, 7, 5, 6, 0, 1, 2, 3, 4, 5, 6, 7, 8, 8};
static const int ov_hctoy_dense_none_u_col_start[10] = {0, 4, 8, 13, 16, 18, 19, 20, 29, 30};
static const int ov_hctoy_dense_none_l_col_start[9] = {0, 5, 10, 14, 16, 18, 19, 27, 29};

/* dTgas/dt: heating/cooling term of the temperature row; yv is the state
   heating and cooling see, Tgas their temperature, ys the state whose
   chemical species are summed and whose gamma is taken */
OV_HD static OV_INLINE double ov_hctoy_dense_none_hc(const double* OV_RESTRICT yv, double Tgas, const double* OV_RESTRICT ys)
{
  double s = 0.0;
  s = s + ys[0];
  s = s + ys[1];
  s = s + ys[2];
  s = s + ys[3];
  s = s + ys[4];
  return (ov_hc_heating(yv, Tgas) - ov_hc_cooling(yv, Tgas)) * (ov_hc_gamma(ys) - 1.0) / OV_HC_BOLTZMANN / s;
}

OV_HD static OV_INLINE void ov_hctoy_dense_none_rhs(const double* OV_RESTRICT y, const double* OV_RESTRICT k, double* OV_RESTRICT f)
{
  (void)k;
  f[0] = -2.0e-13*y[0]*y[1] + 1.0e-15*y[0]*y[2];
  f[1] = -2.0e-13*y[0]*y[1] + 1.0e-15*y[0]*y[2];
  f[2] = 2.0e-13*y[0]*y[1] - 1.0e-15*y[0]*y[2] - 2.0e-17*((y[2])*(y[2])) + 2.0e-10*y[3];
  f[3] = 1.0e-17*((y[2])*(y[2])) - 1.0e-10*y[3];
  f[4] = 0.0;
  f[5] = 0.0;
  f[6] = 0.0;
  f[7] = ov_hctoy_dense_none_hc(y, y[7], y);  /* heating/cooling */
  f[8] = 0.0;
}

/* P at the pattern positions, CSC storage order. With heating/cooling difference quotients, entries the reference leaves unwritten keep a[]'s content. */
OV_HD static OV_INLINE void ov_hctoy_dense_none_jac(const double* OV_RESTRICT y, const double* OV_RESTRICT k, double beta, double dt, double* OV_RESTRICT a)
{
  (void)y; (void)k; (void)beta; (void)dt; (void)a;
  const double hc_dy0 = ov_hctoy_dense_none_hc(y, y[7], y);
  double hc_yy[9];
  a[0] = -beta*dt*(-2.0e-13*y[1] + 1.0e-15*y[2]) + 1.0;  /* (0,0) */
  a[1] = -beta*dt*(-2.0e-13*y[1] + 1.0e-15*y[2]);  /* (1,0) */
  a[2] = -beta*dt*(2.0e-13*y[1] - 1.0e-15*y[2]);  /* (2,0) */
  { /* Tgas row, column 0 */
    for (int m = 0; m < 9; ++m) hc_yy[m] = y[m];
    const double dyy = y[0]*1e-2;
    hc_yy[0] = y[0] + dyy;
    const double dy1 = ov_hctoy_dense_none_hc(hc_yy, y[7], y);
    if (dyy > 0.0) a[3] = -(beta*dt*(dy1 - hc_dy0)/dyy);  /* (7,0) */
  }
  a[4] = 2.0e-13*beta*dt*y[0];  /* (0,1) */
  a[5] = 2.0e-13*beta*dt*y[0] + 1.0;  /* (1,1) */
  a[6] = -2.0e-13*beta*dt*y[0];  /* (2,1) */
  { /* Tgas row, column 1 */
    for (int m = 0; m < 9; ++m) hc_yy[m] = y[m];
    const double dyy = y[1]*1e-2;
    hc_yy[1] = y[1] + dyy;
    const double dy1 = ov_hctoy_dense_none_hc(hc_yy, y[7], y);
    if (dyy > 0.0) a[7] = -(beta*dt*(dy1 - hc_dy0)/dyy);  /* (7,1) */
  }
  a[8] = -1.0e-15*beta*dt*y[0];  /* (0,2) */
  a[9] = -1.0e-15*beta*dt*y[0];  /* (1,2) */
  a[10] = -beta*dt*(-1.0e-15*y[0] - 4.0e-17*y[2]) + 1.0;  /* (2,2) */
  a[11] = -2.0e-17*beta*dt*y[2];  /* (3,2) */
  { /* Tgas row, column 2 */
    for (int m = 0; m < 9; ++m) hc_yy[m] = y[m];
    const double dyy = y[2]*1e-2;
    hc_yy[2] = y[2] + dyy;
    const double dy1 = ov_hctoy_dense_none_hc(hc_yy, y[7], y);
    if (dyy > 0.0) a[12] = -(beta*dt*(dy1 - hc_dy0)/dyy);  /* (7,2) */
  }
  a[13] = -2.0e-10*beta*dt;  /* (2,3) */
  a[14] = 1.0e-10*beta*dt + 1.0;  /* (3,3) */
  { /* Tgas row, column 3 */
    for (int m = 0; m < 9; ++m) hc_yy[m] = y[m];
    const double dyy = y[3]*1e-2;
    hc_yy[3] = y[3] + dyy;
    const double dy1 = ov_hctoy_dense_none_hc(hc_yy, y[7], y);
    if (dyy > 0.0) a[15] = -(beta*dt*(dy1 - hc_dy0)/dyy);  /* (7,3) */
  }
  a[16] = 1.0;  /* (4,4) */
  { /* Tgas row, column 4 */
    for (int m = 0; m < 9; ++m) hc_yy[m] = y[m];
    const double dyy = y[4]*1e-2;
    hc_yy[4] = y[4] + dyy;
    const double dy1 = ov_hctoy_dense_none_hc(hc_yy, y[7], y);
    if (dyy > 0.0) a[17] = -(beta*dt*(dy1 - hc_dy0)/dyy);  /* (7,4) */
  }
  a[18] = 1.0;  /* (5,5) */
  a[19] = 1.0;  /* (6,6) */
  { /* Tgas column */
    const double dyy = y[7]*1e-2;
    hc_yy[7] = y[7] + dyy;
    double dy[9];
    ov_hctoy_dense_none_rhs(hc_yy, k, dy);
    a[20] = -(beta*dt*(dy[0]/dyy));  /* (0,7) */
    a[21] = -(beta*dt*(dy[1]/dyy));  /* (1,7) */
    a[22] = -(beta*dt*(dy[2]/dyy));  /* (2,7) */
    a[23] = -(beta*dt*(dy[3]/dyy));  /* (3,7) */
    a[24] = -(beta*dt*(dy[4]/dyy));  /* (4,7) */
    a[25] = -(beta*dt*(dy[5]/dyy));  /* (5,7) */
    a[26] = -(beta*dt*(dy[6]/dyy));  /* (6,7) */
    a[27] = 1.0 + (-(beta*dt*(dy[7]/dyy)));  /* (7,7) */
    a[28] = -(beta*dt*(dy[8]/dyy));  /* (8,7) */
  }
  a[29] = 1.0;  /* (8,8) */
}

#endif
