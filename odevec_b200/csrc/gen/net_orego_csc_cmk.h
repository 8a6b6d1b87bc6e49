/* Generated by odevec_b200.pre_odevec -- do not edit.
 * network OREGO, packaging CSC, ordering CMK, neq 3, LU nnz 7 (P nnz 7).
 * rhs(): f = dy/dt in species order (rate array k as in the reference).
 * jac(): P = I - dt*beta*J at the LU pattern positions, CSC storage order
 *        of the permuted matrix; fill-in positions are 0.  */
#ifndef OV_NET_OREGO_CSC_CMK_H
#define OV_NET_OREGO_CSC_CMK_H
#include "../ov_common.h"

#define OV_OREGO_CSC_CMK_NEQ 3
#define OV_OREGO_CSC_CMK_NNZ 7
#define OV_OREGO_CSC_CMK_NREA 0
#define OV_OREGO_CSC_CMK_DENSE 0
#define OV_OREGO_CSC_CMK_NVECTOR 1
#define OV_OREGO_CSC_CMK_DT_MIN 1e-10
#define OV_OREGO_CSC_CMK_IDX_TGAS -1
static const int ov_orego_csc_cmk_sizes[8] = {3, 7, 0, 0, -1, 3, 1, 1};
static const double ov_orego_csc_cmk_defaults[2] = {1.0, 1e-10}; /* nvector, dt_min */
static const double ov_orego_csc_cmk_mass[3] = {0.0, 0.0, 0.0};
static const double ov_orego_csc_cmk_imass[3] = {0.0, 0.0, 0.0};
static const int ov_orego_csc_cmk_perm[3] = {2, 1, 0};
static const int ov_orego_csc_cmk_row_index[7] = {0, 1, 1, 2, 0, 1, 2};
static const int ov_orego_csc_cmk_u_col_start[4] = {0, 2, 4, 7};
static const int ov_orego_csc_cmk_l_col_start[3] = {0, 2, 6};

OV_HD static OV_INLINE void ov_orego_csc_cmk_rhs(const double* OV_RESTRICT y, const double* OV_RESTRICT k, double* OV_RESTRICT f)
{
  (void)k;
  f[0] = -0.00064713625*((y[0])*(y[0])) - 77.27*y[0]*y[1] + 77.27*y[0] + 77.27*y[1];
  f[1] = -0.0129416332341141*y[0]*y[1] - 0.0129416332341141*y[1] + 0.0129416332341141*y[2];
  f[2] = 0.161*y[0] - 0.161*y[2];
}

/* P at the pattern positions, CSC storage order. */
OV_HD static OV_INLINE void ov_orego_csc_cmk_jac(const double* OV_RESTRICT y, const double* OV_RESTRICT k, double beta, double dt, double* OV_RESTRICT a)
{
  (void)y; (void)k; (void)beta; (void)dt; (void)a;
  a[0] = 0.161*beta*dt + 1.0;  /* (0,0) */
  a[1] = -0.0129416332341141*beta*dt;  /* (1,0) */
  a[2] = -beta*dt*(-0.0129416332341141*y[0] - 0.0129416332341141) + 1.0;  /* (1,1) */
  a[3] = -beta*dt*(77.27 - 77.27*y[0]);  /* (2,1) */
  a[4] = -0.161*beta*dt;  /* (0,2) */
  a[5] = 0.0129416332341141*beta*dt*y[1];  /* (1,2) */
  a[6] = -beta*dt*(-0.0012942725*y[0] - 77.27*y[1] + 77.27) + 1.0;  /* (2,2) */
}

#endif
