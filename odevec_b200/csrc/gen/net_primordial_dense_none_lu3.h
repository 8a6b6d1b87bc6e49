/* Generated by odevec_b200.pre_odevec -- do not edit.
 * network PRIMORDIAL, packaging DENSE, ordering None, neq 16, LU nnz 148 (P nnz 148).
 * rhs(): f = dy/dt in species order (rate array k as in the reference).
 * jac(): LUmethod 3, empty: P comes from difference quotients of rhs().  */
#ifndef OV_NET_PRIMORDIAL_DENSE_NONE_LU3_H
#define OV_NET_PRIMORDIAL_DENSE_NONE_LU3_H
#include "../ov_common.h"
#include "../rates_primordial.h"

#define OV_PRIMORDIAL_DENSE_NONE_LU3_NEQ 16
#define OV_PRIMORDIAL_DENSE_NONE_LU3_NNZ 148
#define OV_PRIMORDIAL_DENSE_NONE_LU3_NREA 38
#define OV_PRIMORDIAL_DENSE_NONE_LU3_DENSE 1
#define OV_PRIMORDIAL_DENSE_NONE_LU3_NVECTOR 1
#define OV_PRIMORDIAL_DENSE_NONE_LU3_DT_MIN 1e-20
#define OV_PRIMORDIAL_DENSE_NONE_LU3_IDX_TGAS 14
static const int ov_primordial_dense_none_lu3_sizes[8] = {16, 148, 38, 1, 14, 12, 3, 0};
static const double ov_primordial_dense_none_lu3_defaults[2] = {1.0, 1e-20}; /* nvector, dt_min */
static const double ov_primordial_dense_none_lu3_mass[16] = {9.10938188e-28, 1.67444345638e-24, 1.67353251819e-24, 6.69206503638e-24, 3.34706503638e-24, 3.34603251819e-24, 5.01956503638e-24, 1.67262158e-24, 6.69115409819e-24, 3.34615409819e-24, 3.34512158e-24, 6.69024316e-24, 0.0, 0.0, 0.0, 0.0};
static const double ov_primordial_dense_none_lu3_imass[16] = {1.09776932527e+27, 5.9721335838e+23, 5.97538433901e+23, 1.49430705554e+23, 2.9876921695e+23, 2.98861411108e+23, 1.99220448934e+23, 5.97863863505e+23, 1.4945104915e+23, 2.98850552203e+23, 2.98942796572e+23, 1.49471398286e+23, 0.0, 0.0, 0.0, 0.0};
static const int ov_primordial_dense_none_lu3_perm[16] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15};
static const int ov_primordial_dense_none_lu3_row_index[148] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15};
static const int ov_primordial_dense_none_lu3_u_col_start[17] = {0, 12, 24, 36, 48, 60, 72, 84, 96, 108, 120, 132, 144, 145, 146, 147, 148};
static const int ov_primordial_dense_none_lu3_l_col_start[16] = {0, 13, 26, 39, 52, 65, 78, 91, 104, 117, 130, 143, 144, 145, 146, 147};

OV_HD static OV_INLINE void ov_primordial_dense_none_lu3_rhs(const double* OV_RESTRICT y, const double* OV_RESTRICT k, double* OV_RESTRICT f)
{
  (void)k;
  f[0] = k[0]*y[0]*y[2] + k[9]*y[1]*y[2] + k[10]*y[1]*y[2] + k[17]*y[0]*y[1] + k[18]*y[1]*y[2] - k[1]*y[0]*y[7] + k[19]*y[1]*y[2] + k[21]*y[1]*y[7] - k[22]*y[0]*y[9] - k[23]*y[0]*y[9] - k[2]*y[0]*y[7] + k[36]*y[1]*y[5] - k[37]*y[0]*y[10] + k[3]*y[0]*y[3] - k[4]*y[0]*y[8] - k[5]*y[0]*y[8] + k[6]*y[0]*y[8] - k[7]*y[0]*y[11] - k[8]*y[0]*y[2];
  f[1] = -k[9]*y[1]*y[2] - k[10]*y[1]*y[2] - k[17]*y[0]*y[1] - k[18]*y[1]*y[2] - k[19]*y[1]*y[2] - k[20]*y[1]*y[7] - k[21]*y[1]*y[7] - k[24]*y[9]*y[1] - k[36]*y[1]*y[5] + k[8]*y[0]*y[2];
  f[2] = -k[0]*y[0]*y[2] - k[9]*y[1]*y[2] - k[10]*y[1]*y[2] - k[11]*y[2]*y[7] - k[12]*y[2]*y[7] - k[13]*y[9]*y[2] + k[14]*y[4]*y[7] + 2.0*k[15]*y[0]*y[4] + 2.0*k[16]*y[2]*y[4] + k[17]*y[0]*y[1] + k[18]*y[1]*y[2] + k[1]*y[0]*y[7] + k[19]*y[1]*y[2] + 2.0*k[20]*y[1]*y[7] + 2.0*k[22]*y[0]*y[9] + 2.0*k[23]*y[0]*y[9] + k[24]*y[9]*y[1] - 2.0*k[25]*((y[2])*((y[2])*(y[2]))) - 2.0*k[26]*((y[2])*((y[2])*(y[2]))) - 2.0*k[27]*((y[2])*(y[2]))*y[4] - 2.0*k[28]*((y[2])*(y[2]))*y[4] + k[2]*y[0]*y[7] + k[29]*y[5]*y[7] - k[30]*y[10]*y[2] + k[33]*y[4]*y[5] + k[34]*y[4]*y[5] - k[35]*y[2]*y[6] - k[8]*y[0]*y[2];
  f[3] = -k[3]*y[0]*y[3] + k[4]*y[0]*y[8] + k[5]*y[0]*y[8];
  f[4] = k[9]*y[1]*y[2] + k[10]*y[1]*y[2] + k[13]*y[9]*y[2] - k[14]*y[4]*y[7] - k[15]*y[0]*y[4] - k[16]*y[2]*y[4] + k[24]*y[9]*y[1] + k[25]*((y[2])*((y[2])*(y[2]))) + k[26]*((y[2])*((y[2])*(y[2]))) + k[27]*((y[2])*(y[2]))*y[4] + k[28]*((y[2])*(y[2]))*y[4] - k[31]*y[10]*y[4] + k[32]*y[6]*y[7] - k[33]*y[4]*y[5] - k[34]*y[4]*y[5] + k[35]*y[2]*y[6];
  f[5] = -k[29]*y[5]*y[7] + k[30]*y[10]*y[2] - k[33]*y[4]*y[5] - k[34]*y[4]*y[5] + k[35]*y[2]*y[6] - k[36]*y[1]*y[5] + k[37]*y[0]*y[10];
  f[6] = k[31]*y[10]*y[4] - k[32]*y[6]*y[7] + k[33]*y[4]*y[5] + k[34]*y[4]*y[5] - k[35]*y[2]*y[6] + k[36]*y[1]*y[5];
  f[7] = k[0]*y[0]*y[2] - k[11]*y[2]*y[7] - k[12]*y[2]*y[7] + k[13]*y[9]*y[2] - k[14]*y[4]*y[7] - k[1]*y[0]*y[7] - k[20]*y[1]*y[7] - k[21]*y[1]*y[7] - k[2]*y[0]*y[7] - k[29]*y[5]*y[7] + k[30]*y[10]*y[2] + k[31]*y[10]*y[4] - k[32]*y[6]*y[7];
  f[8] = k[3]*y[0]*y[3] - k[4]*y[0]*y[8] - k[5]*y[0]*y[8] - k[6]*y[0]*y[8] + k[7]*y[0]*y[11];
  f[9] = k[11]*y[2]*y[7] + k[12]*y[2]*y[7] - k[13]*y[9]*y[2] + k[14]*y[4]*y[7] + k[21]*y[1]*y[7] - k[22]*y[0]*y[9] - k[23]*y[0]*y[9] - k[24]*y[9]*y[1];
  f[10] = k[29]*y[5]*y[7] - k[30]*y[10]*y[2] - k[31]*y[10]*y[4] + k[32]*y[6]*y[7] - k[37]*y[0]*y[10];
  f[11] = k[6]*y[0]*y[8] - k[7]*y[0]*y[11];
  f[12] = 0.0;
  f[13] = 0.0;
  f[14] = 0.0;
  f[15] = 0.0;
}

/* P at the pattern positions, CSC storage order. */
OV_HD static OV_INLINE void ov_primordial_dense_none_lu3_jac(const double* OV_RESTRICT y, const double* OV_RESTRICT k, double beta, double dt, double* OV_RESTRICT a)
{
  (void)y; (void)k; (void)beta; (void)dt; (void)a;
}

#endif
