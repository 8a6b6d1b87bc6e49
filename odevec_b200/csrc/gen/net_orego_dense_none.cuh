/* Generated by odevec_b200.pre_odevec -- do not edit.
 * CUDA traits of network variant OREGO_DENSE_NONE for the BDF kernel: straight-line
 * LU factorisation and solve over the fill pattern (right-looking Doolittle). */
#pragma once
#include "net_orego_dense_none.h"

struct ov_net_orego_dense_none {
  static constexpr int NEQ = 3;
  static constexpr int NNZ = 8;
  static constexpr int NREA = 0;
  static constexpr int IDX_TGAS = -1;
  static constexpr bool DENSE = true;
  static constexpr const char* TAG = "OREGO_DENSE_NONE";
  OV_HD static OV_INLINE void rhs(const double* y, const double* k, double* f) { ov_orego_dense_none_rhs(y, k, f); }
  OV_HD static OV_INLINE void jac(const double* y, const double* k, double beta, double dt, double* a) { ov_orego_dense_none_jac(y, k, beta, dt, a); }
  OV_HD static OV_INLINE void rates_T(const double*, double*) {}
  OV_HD static OV_INLINE void rates_k(const double*, const double*, double*) {}
  /* a = D P D^-1 rounded to T, D = diag(sc) in species order (isc = 1/sc) */
  template <class T> OV_HD static OV_INLINE void store_scaled(const double* OV_RESTRICT P, T* OV_RESTRICT a, const double* OV_RESTRICT sc, const double* OV_RESTRICT isc) {
    a[0] = (T)(P[0]*sc[0]*isc[0]);
    a[1] = (T)(P[1]*sc[1]*isc[0]);
    a[2] = (T)(P[2]*sc[2]*isc[0]);
    a[3] = (T)(P[3]*sc[0]*isc[1]);
    a[4] = (T)(P[4]*sc[1]*isc[1]);
    a[5] = (T)(P[5]*sc[2]*isc[1]);
    a[6] = (T)(P[6]*sc[1]*isc[2]);
    a[7] = (T)(P[7]*sc[2]*isc[2]);
  }
  /* in-place numeric LU of the packed matrix a[NNZ] */
  template <class T> OV_HD static OV_INLINE void lu_factor(T* OV_RESTRICT a) {
    a[1] = a[1] / a[0];
    a[2] = a[2] / a[0];
    a[4] = a[4] - a[1]*a[3];
    a[5] = a[5] - a[2]*a[3];
    a[5] = a[5] / a[4];
    a[7] = a[7] - a[5]*a[6];
  }
  /* x = P^-1 r with P = LU in a[]; r and x in species order.  sc/isc scale
     species i by sc[i] on the way in and isc[i] on the way out (pass
     nullptr for none); T is the precision of the solve. */
  template <class T> OV_HD static OV_INLINE void lu_solve(const T* OV_RESTRICT a, const double* OV_RESTRICT r, double* OV_RESTRICT x, const double* OV_RESTRICT sc, const double* OV_RESTRICT isc) {
#define OV_SC(i) (sc ? sc[i] : 1.0)
#define OV_ISC(i) (isc ? isc[i] : 1.0)
    T d0 = (T)(r[0]*OV_SC(0));
    T d1 = (T)(r[1]*OV_SC(1));
    T d2 = (T)(r[2]*OV_SC(2));
    d1 = d1 - a[1]*d0;
    d2 = d2 - (a[2]*d0 + a[5]*d1);
    d2 = d2 / a[7];
    d1 = (d1 - a[6]*d2) / a[4];
    d0 = (d0 - a[3]*d1) / a[0];
    x[0] = (double)d0*OV_ISC(0);
    x[1] = (double)d1*OV_ISC(1);
    x[2] = (double)d2*OV_ISC(2);
#undef OV_SC
#undef OV_ISC
  }
  static constexpr int perm[3] = {0, 1, 2};
};
