/* Generated by odevec_b200.pre_odevec -- do not edit.
 * network OREGO, packaging DENSE, ordering None, neq 3, LU nnz 8 (P nnz 7).
 * rhs(): f = dy/dt in species order (rate array k as in the reference).
 * jac(): P = I - dt*beta*J at the LU pattern positions, CSC storage order
 *        of the permuted matrix; fill-in positions are 0.  */
#ifndef OV_NET_OREGO_DENSE_NONE_H
#define OV_NET_OREGO_DENSE_NONE_H
#include "../ov_common.h"

#define OV_OREGO_DENSE_NONE_NEQ 3
#define OV_OREGO_DENSE_NONE_NNZ 8
#define OV_OREGO_DENSE_NONE_NREA 0
#define OV_OREGO_DENSE_NONE_DENSE 1
#define OV_OREGO_DENSE_NONE_NVECTOR 1
#define OV_OREGO_DENSE_NONE_DT_MIN 1e-10
#define OV_OREGO_DENSE_NONE_IDX_TGAS -1
static const int ov_orego_dense_none_sizes[8] = {3, 8, 0, 1, -1, 3, 1, 0};
static const double ov_orego_dense_none_defaults[2] = {1.0, 1e-10}; /* nvector, dt_min */
static const double ov_orego_dense_none_mass[3] = {0.0, 0.0, 0.0};
static const double ov_orego_dense_none_imass[3] = {0.0, 0.0, 0.0};
static const int ov_orego_dense_none_perm[3] = {0, 1, 2};
static const int ov_orego_dense_none_row_index[8] = {0, 1, 2, 0, 1, 2, 1, 2};
static const int ov_orego_dense_none_u_col_start[4] = {0, 3, 6, 8};
static const int ov_orego_dense_none_l_col_start[3] = {0, 4, 7};

OV_HD static OV_INLINE void ov_orego_dense_none_rhs(const double* OV_RESTRICT y, const double* OV_RESTRICT k, double* OV_RESTRICT f)
{
  (void)k;
  f[0] = -0.00064713625*((y[0])*(y[0])) - 77.27*y[0]*y[1] + 77.27*y[0] + 77.27*y[1];
  f[1] = -0.0129416332341141*y[0]*y[1] - 0.0129416332341141*y[1] + 0.0129416332341141*y[2];
  f[2] = 0.161*y[0] - 0.161*y[2];
}

/* P at the pattern positions, CSC storage order. */
OV_HD static OV_INLINE void ov_orego_dense_none_jac(const double* OV_RESTRICT y, const double* OV_RESTRICT k, double beta, double dt, double* OV_RESTRICT a)
{
  (void)y; (void)k; (void)beta; (void)dt; (void)a;
  a[0] = -beta*dt*(-0.0012942725*y[0] - 77.27*y[1] + 77.27) + 1.0;  /* (0,0) */
  a[1] = 0.0129416332341141*beta*dt*y[1];  /* (1,0) */
  a[2] = -0.161*beta*dt;  /* (2,0) */
  a[3] = -beta*dt*(77.27 - 77.27*y[0]);  /* (0,1) */
  a[4] = -beta*dt*(-0.0129416332341141*y[0] - 0.0129416332341141) + 1.0;  /* (1,1) */
  a[5] = 0.0;  /* (2,1) */
  a[6] = -0.0129416332341141*beta*dt;  /* (1,2) */
  a[7] = 0.161*beta*dt + 1.0;  /* (2,2) */
}

#endif
