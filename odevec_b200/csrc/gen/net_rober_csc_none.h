/* Generated by odevec_b200.pre_odevec -- do not edit.
 * network ROBER, packaging CSC, ordering None, neq 3, LU nnz 8 (P nnz 8).
 * rhs(): f = dy/dt in species order (rate array k as in the reference).
 * jac(): P = I - dt*beta*J at the LU pattern positions, CSC storage order
 *        of the permuted matrix; fill-in positions are 0.  */
#ifndef OV_NET_ROBER_CSC_NONE_H
#define OV_NET_ROBER_CSC_NONE_H
#include "../ov_common.h"

#define OV_ROBER_CSC_NONE_NEQ 3
#define OV_ROBER_CSC_NONE_NNZ 8
#define OV_ROBER_CSC_NONE_NREA 0
#define OV_ROBER_CSC_NONE_DENSE 0
#define OV_ROBER_CSC_NONE_NVECTOR 32
#define OV_ROBER_CSC_NONE_DT_MIN 1e-20
#define OV_ROBER_CSC_NONE_IDX_TGAS -1
static const int ov_rober_csc_none_sizes[8] = {3, 8, 0, 0, -1, 3, 1, 1};
static const double ov_rober_csc_none_defaults[2] = {32.0, 1e-20}; /* nvector, dt_min */
static const double ov_rober_csc_none_mass[3] = {0.0, 0.0, 0.0};
static const double ov_rober_csc_none_imass[3] = {0.0, 0.0, 0.0};
static const int ov_rober_csc_none_perm[3] = {0, 1, 2};
static const int ov_rober_csc_none_row_index[8] = {0, 1, 0, 1, 2, 0, 1, 2};
static const int ov_rober_csc_none_u_col_start[4] = {0, 2, 5, 8};
static const int ov_rober_csc_none_l_col_start[3] = {0, 3, 7};

OV_HD static OV_INLINE void ov_rober_csc_none_rhs(const double* OV_RESTRICT y, const double* OV_RESTRICT k, double* OV_RESTRICT f)
{
  (void)k;
  f[0] = -0.04*y[0] + 10000.0*y[1]*y[2];
  f[1] = 0.04*y[0] - 30000000.0*((y[1])*(y[1])) - 10000.0*y[1]*y[2];
  f[2] = 30000000.0*((y[1])*(y[1]));
}

/* P at the pattern positions, CSC storage order. */
OV_HD static OV_INLINE void ov_rober_csc_none_jac(const double* OV_RESTRICT y, const double* OV_RESTRICT k, double beta, double dt, double* OV_RESTRICT a)
{
  (void)y; (void)k; (void)beta; (void)dt; (void)a;
  a[0] = 0.04*beta*dt + 1.0;  /* (0,0) */
  a[1] = -0.04*beta*dt;  /* (1,0) */
  a[2] = -10000.0*beta*dt*y[2];  /* (0,1) */
  a[3] = -beta*dt*(-60000000.0*y[1] - 10000.0*y[2]) + 1.0;  /* (1,1) */
  a[4] = -60000000.0*beta*dt*y[1];  /* (2,1) */
  a[5] = -10000.0*beta*dt*y[1];  /* (0,2) */
  a[6] = 10000.0*beta*dt*y[1];  /* (1,2) */
  a[7] = 1.0;  /* (2,2) */
}

#endif
