/* Generated by odevec_b200.pre_odevec -- do not edit.
 * network ROBER, packaging DENSE, ordering None, neq 3, LU nnz 9 (P nnz 9).
 * rhs(): f = dy/dt in species order (rate array k as in the reference).
 * jac(): LUmethod 3, empty: P comes from difference quotients of rhs().  */
#ifndef OV_NET_ROBER_DENSE_NONE_LU3_H
#define OV_NET_ROBER_DENSE_NONE_LU3_H
#include "../ov_common.h"

#define OV_ROBER_DENSE_NONE_LU3_NEQ 3
#define OV_ROBER_DENSE_NONE_LU3_NNZ 9
#define OV_ROBER_DENSE_NONE_LU3_NREA 0
#define OV_ROBER_DENSE_NONE_LU3_DENSE 1
#define OV_ROBER_DENSE_NONE_LU3_NVECTOR 32
#define OV_ROBER_DENSE_NONE_LU3_DT_MIN 1e-20
#define OV_ROBER_DENSE_NONE_LU3_IDX_TGAS -1
static const int ov_rober_dense_none_lu3_sizes[8] = {3, 9, 0, 1, -1, 3, 3, 0};
static const double ov_rober_dense_none_lu3_defaults[2] = {32.0, 1e-20}; /* nvector, dt_min */
static const double ov_rober_dense_none_lu3_mass[3] = {0.0, 0.0, 0.0};
static const double ov_rober_dense_none_lu3_imass[3] = {0.0, 0.0, 0.0};
static const int ov_rober_dense_none_lu3_perm[3] = {0, 1, 2};
static const int ov_rober_dense_none_lu3_row_index[9] = {0, 1, 2, 0, 1, 2, 0, 1, 2};
static const int ov_rober_dense_none_lu3_u_col_start[4] = {0, 3, 6, 9};
static const int ov_rober_dense_none_lu3_l_col_start[3] = {0, 4, 8};

OV_HD static OV_INLINE void ov_rober_dense_none_lu3_rhs(const double* OV_RESTRICT y, const double* OV_RESTRICT k, double* OV_RESTRICT f)
{
  (void)k;
  f[0] = -0.04*y[0] + 10000.0*y[1]*y[2];
  f[1] = 0.04*y[0] - 30000000.0*((y[1])*(y[1])) - 10000.0*y[1]*y[2];
  f[2] = 30000000.0*((y[1])*(y[1]));
}

/* P at the pattern positions, CSC storage order. */
OV_HD static OV_INLINE void ov_rober_dense_none_lu3_jac(const double* OV_RESTRICT y, const double* OV_RESTRICT k, double beta, double dt, double* OV_RESTRICT a)
{
  (void)y; (void)k; (void)beta; (void)dt; (void)a;
}

#endif
