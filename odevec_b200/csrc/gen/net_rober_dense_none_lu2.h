/* Generated by odevec_b200.pre_odevec -- do not edit.
 * network ROBER, packaging DENSE, ordering None, neq 3, LU nnz 8 (P nnz 8).
 * rhs(): f = dy/dt in species order (rate array k as in the reference).
 * jac(): LUmethod 2, the symbolic factors L\U of P (unit L) at the
 *        pattern positions, CSC storage order; no numeric factorisation.  */
#ifndef OV_NET_ROBER_DENSE_NONE_LU2_H
#define OV_NET_ROBER_DENSE_NONE_LU2_H
#include "../ov_common.h"

#define OV_ROBER_DENSE_NONE_LU2_NEQ 3
#define OV_ROBER_DENSE_NONE_LU2_NNZ 8
#define OV_ROBER_DENSE_NONE_LU2_NREA 0
#define OV_ROBER_DENSE_NONE_LU2_DENSE 1
#define OV_ROBER_DENSE_NONE_LU2_NVECTOR 32
#define OV_ROBER_DENSE_NONE_LU2_DT_MIN 1e-20
#define OV_ROBER_DENSE_NONE_LU2_IDX_TGAS -1
static const int ov_rober_dense_none_lu2_sizes[8] = {3, 8, 0, 1, -1, 3, 2, 0};
static const double ov_rober_dense_none_lu2_defaults[2] = {32.0, 1e-20}; /* nvector, dt_min */
static const double ov_rober_dense_none_lu2_mass[3] = {0.0, 0.0, 0.0};
static const double ov_rober_dense_none_lu2_imass[3] = {0.0, 0.0, 0.0};
static const int ov_rober_dense_none_lu2_perm[3] = {0, 1, 2};
static const int ov_rober_dense_none_lu2_row_index[8] = {0, 1, 0, 1, 2, 0, 1, 2};
static const int ov_rober_dense_none_lu2_u_col_start[4] = {0, 2, 5, 8};
static const int ov_rober_dense_none_lu2_l_col_start[3] = {0, 3, 7};

OV_HD static OV_INLINE void ov_rober_dense_none_lu2_rhs(const double* OV_RESTRICT y, const double* OV_RESTRICT k, double* OV_RESTRICT f)
{
  (void)k;
  f[0] = -0.04*y[0] + 10000.0*y[1]*y[2];
  f[1] = 0.04*y[0] - 30000000.0*((y[1])*(y[1])) - 10000.0*y[1]*y[2];
  f[2] = 30000000.0*((y[1])*(y[1]));
}

/* P at the pattern positions, CSC storage order. */
OV_HD static OV_INLINE void ov_rober_dense_none_lu2_jac(const double* OV_RESTRICT y, const double* OV_RESTRICT k, double beta, double dt, double* OV_RESTRICT a)
{
  (void)y; (void)k; (void)beta; (void)dt; (void)a;
  a[0] = 0.04*beta*dt + 1.0;  /* (0,0) */
  a[1] = -0.04*beta*dt/(0.04*beta*dt + 1.0);  /* (1,0) */
  a[2] = -10000.0*beta*dt*y[2];  /* (0,1) */
  a[3] = -400.0*((beta)*(beta))*((dt)*(dt))*y[2]/(0.04*beta*dt + 1.0) - beta*dt*(-60000000.0*y[1] - 10000.0*y[2]) + 1.0;  /* (1,1) */
  a[4] = -60000000.0*beta*dt*y[1]/(-400.0*((beta)*(beta))*((dt)*(dt))*y[2]/(0.04*beta*dt + 1.0) - beta*dt*(-60000000.0*y[1] - 10000.0*y[2]) + 1.0);  /* (2,1) */
  a[5] = -10000.0*beta*dt*y[1];  /* (0,2) */
  a[6] = -400.0*((beta)*(beta))*((dt)*(dt))*y[1]/(0.04*beta*dt + 1.0) + 10000.0*beta*dt*y[1];  /* (1,2) */
  a[7] = 60000000.0*beta*dt*y[1]*(-400.0*((beta)*(beta))*((dt)*(dt))*y[1]/(0.04*beta*dt + 1.0) + 10000.0*beta*dt*y[1])/(-400.0*((beta)*(beta))*((dt)*(dt))*y[2]/(0.04*beta*dt + 1.0) - beta*dt*(-60000000.0*y[1] - 10000.0*y[2]) + 1.0) + 1.0;  /* (2,2) */
}

#endif
