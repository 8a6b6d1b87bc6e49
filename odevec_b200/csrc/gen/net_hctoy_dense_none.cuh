/* Generated by odevec_b200.pre_odevec -- do not edit.
 * CUDA traits of network variant HCTOY_DENSE_NONE for the BDF kernel: straight-line
 * LU factorisation and solve over the fill pattern (right-looking Doolittle). */
#pragma once
#include "net_hctoy_dense_none.h"

struct ov_net_hctoy_dense_none {
  static constexpr bool HAS_WPC = false;
  using Wpc = void;
  static constexpr int NEQ = 9;   /* all species (state vector) */
  static constexpr int ND = 6;    /* species in the solver state */
  static constexpr int NNZ = 24;   /* packed LU entries of the dynamic block */
  static constexpr int NREA = 0;
  static constexpr int IDX_TGAS = 7;
  static constexpr bool DENSE = true;
  /* 1: symbolic Jacobian + numeric LU, 2: symbolic LU, 3: difference quotients */
  static constexpr int LU_METHOD = 1;
  /* the Tgas row is the heating/cooling term (--heatcool=1); HC_FD: GetJac writes
     its difference quotients and leaves some entries as the storage holds them */
  static constexpr bool HEATCOOL = true;
  static constexpr bool HC_FD = true;
  static constexpr const char* TAG = "HCTOY_DENSE_NONE";
  /* dynamic species (solver state index -> species) and frozen ones */
  OV_HD static constexpr int dyn(int i) { return i == 0 ? 0 : (i == 1 ? 1 : (i == 2 ? 2 : (i == 3 ? 3 : (i == 4 ? 4 : (7))))); }
  static constexpr int NF = 3;
  OV_HD static constexpr int frozen(int i) { return i == 0 ? 5 : (i == 1 ? 6 : (8)); }
  OV_HD static OV_INLINE void rhs(const double* y, const double* k, double* f) { ov_hctoy_dense_none_rhs(y, k, f); }
  static OV_INLINE __device__ void rates_k(const double*, const double*, double*) {}
  static OV_INLINE __device__ void rates_T(const double*, double*) {}
  /* P = I - dt*beta*J on the dynamic block, packed CSC order */
  template <class T, class A> OV_HD static OV_INLINE void jac(const double* OV_RESTRICT y, const double* OV_RESTRICT k, double beta, double dt, A a) {
    (void)y; (void)k; (void)beta; (void)dt; (void)a;
    const double hc_dy0 = ov_hctoy_dense_none_hc(y, y[7], y);
    double hc_yy[9];
    a[0] = (T)(-beta*dt*(-2.0e-13*y[1] + 1.0e-15*y[2]) + 1.0);
    a[1] = (T)(-beta*dt*(-2.0e-13*y[1] + 1.0e-15*y[2]));
    a[2] = (T)(-beta*dt*(2.0e-13*y[1] - 1.0e-15*y[2]));
    { /* Tgas row, column 0 */
      for (int m = 0; m < 9; ++m) hc_yy[m] = y[m];
      const double dyy = y[0]*1e-2;
      hc_yy[0] = y[0] + dyy;
      const double dy1 = ov_hctoy_dense_none_hc(hc_yy, y[7], y);
      if (dyy > 0.0) a[3] = (T)(-(beta*dt*(dy1 - hc_dy0)/dyy));
    }
    a[4] = (T)(2.0e-13*beta*dt*y[0]);
    a[5] = (T)(2.0e-13*beta*dt*y[0] + 1.0);
    a[6] = (T)(-2.0e-13*beta*dt*y[0]);
    { /* Tgas row, column 1 */
      for (int m = 0; m < 9; ++m) hc_yy[m] = y[m];
      const double dyy = y[1]*1e-2;
      hc_yy[1] = y[1] + dyy;
      const double dy1 = ov_hctoy_dense_none_hc(hc_yy, y[7], y);
      if (dyy > 0.0) a[7] = (T)(-(beta*dt*(dy1 - hc_dy0)/dyy));
    }
    a[8] = (T)(-1.0e-15*beta*dt*y[0]);
    a[9] = (T)(-1.0e-15*beta*dt*y[0]);
    a[10] = (T)(-beta*dt*(-1.0e-15*y[0] - 4.0e-17*y[2]) + 1.0);
    a[11] = (T)(-2.0e-17*beta*dt*y[2]);
    { /* Tgas row, column 2 */
      for (int m = 0; m < 9; ++m) hc_yy[m] = y[m];
      const double dyy = y[2]*1e-2;
      hc_yy[2] = y[2] + dyy;
      const double dy1 = ov_hctoy_dense_none_hc(hc_yy, y[7], y);
      if (dyy > 0.0) a[12] = (T)(-(beta*dt*(dy1 - hc_dy0)/dyy));
    }
    a[13] = (T)(-2.0e-10*beta*dt);
    a[14] = (T)(1.0e-10*beta*dt + 1.0);
    { /* Tgas row, column 3 */
      for (int m = 0; m < 9; ++m) hc_yy[m] = y[m];
      const double dyy = y[3]*1e-2;
      hc_yy[3] = y[3] + dyy;
      const double dy1 = ov_hctoy_dense_none_hc(hc_yy, y[7], y);
      if (dyy > 0.0) a[15] = (T)(-(beta*dt*(dy1 - hc_dy0)/dyy));
    }
    a[16] = (T)(1.0);
    { /* Tgas row, column 4 */
      for (int m = 0; m < 9; ++m) hc_yy[m] = y[m];
      const double dyy = y[4]*1e-2;
      hc_yy[4] = y[4] + dyy;
      const double dy1 = ov_hctoy_dense_none_hc(hc_yy, y[7], y);
      if (dyy > 0.0) a[17] = (T)(-(beta*dt*(dy1 - hc_dy0)/dyy));
    }
    { /* Tgas column */
      const double dyy = y[7]*1e-2;
      hc_yy[7] = y[7] + dyy;
      double dy[9];
      ov_hctoy_dense_none_rhs(hc_yy, k, dy);
      a[18] = (T)(-(beta*dt*(dy[0]/dyy)));
      a[19] = (T)(-(beta*dt*(dy[1]/dyy)));
      a[20] = (T)(-(beta*dt*(dy[2]/dyy)));
      a[21] = (T)(-(beta*dt*(dy[3]/dyy)));
      a[22] = (T)(-(beta*dt*(dy[4]/dyy)));
      a[23] = (T)(1.0 + (-(beta*dt*(dy[7]/dyy))));
    }
  }
  /* a = D P D^-1 rounded to T, D = diag(sc) over solver-state indices */
  template <class T, class A> OV_HD static OV_INLINE void store_scaled(const double* OV_RESTRICT P, A a, const double* OV_RESTRICT sc, const double* OV_RESTRICT isc) {
    a[0] = (T)(P[0]*sc[0]*isc[0]);
    a[1] = (T)(P[1]*sc[1]*isc[0]);
    a[2] = (T)(P[2]*sc[2]*isc[0]);
    a[3] = (T)(P[3]*sc[5]*isc[0]);
    a[4] = (T)(P[4]*sc[0]*isc[1]);
    a[5] = (T)(P[5]*sc[1]*isc[1]);
    a[6] = (T)(P[6]*sc[2]*isc[1]);
    a[7] = (T)(P[7]*sc[5]*isc[1]);
    a[8] = (T)(P[8]*sc[0]*isc[2]);
    a[9] = (T)(P[9]*sc[1]*isc[2]);
    a[10] = (T)(P[10]*sc[2]*isc[2]);
    a[11] = (T)(P[11]*sc[3]*isc[2]);
    a[12] = (T)(P[12]*sc[5]*isc[2]);
    a[13] = (T)(P[13]*sc[2]*isc[3]);
    a[14] = (T)(P[14]*sc[3]*isc[3]);
    a[15] = (T)(P[15]*sc[5]*isc[3]);
    a[16] = (T)(P[16]*sc[4]*isc[4]);
    a[17] = (T)(P[17]*sc[5]*isc[4]);
    a[18] = (T)(P[18]*sc[0]*isc[5]);
    a[19] = (T)(P[19]*sc[1]*isc[5]);
    a[20] = (T)(P[20]*sc[2]*isc[5]);
    a[21] = (T)(P[21]*sc[3]*isc[5]);
    a[22] = (T)(P[22]*sc[4]*isc[5]);
    a[23] = (T)(P[23]*sc[5]*isc[5]);
  }
  /* the same, each entry evaluated in FP64, scaled by powers of two and
     rounded to T on the fly */
  template <class T, class A> OV_HD static OV_INLINE void jac_scaled(const double* OV_RESTRICT y, const double* OV_RESTRICT k, double beta, double dt, A a, const double* OV_RESTRICT sc, const double* OV_RESTRICT isc) {
    (void)y; (void)k; (void)beta; (void)dt; (void)a; (void)sc; (void)isc;
    const double hc_dy0 = ov_hctoy_dense_none_hc(y, y[7], y);
    double hc_yy[9];
    a[0] = (T)((-beta*dt*(-2.0e-13*y[1] + 1.0e-15*y[2]) + 1.0)*sc[0]*isc[0]);
    a[1] = (T)((-beta*dt*(-2.0e-13*y[1] + 1.0e-15*y[2]))*sc[1]*isc[0]);
    a[2] = (T)((-beta*dt*(2.0e-13*y[1] - 1.0e-15*y[2]))*sc[2]*isc[0]);
    { /* Tgas row, column 0 */
      for (int m = 0; m < 9; ++m) hc_yy[m] = y[m];
      const double dyy = y[0]*1e-2;
      hc_yy[0] = y[0] + dyy;
      const double dy1 = ov_hctoy_dense_none_hc(hc_yy, y[7], y);
      if (dyy > 0.0) a[3] = (T)((-(beta*dt*(dy1 - hc_dy0)/dyy))*sc[5]*isc[0]);
    }
    a[4] = (T)((2.0e-13*beta*dt*y[0])*sc[0]*isc[1]);
    a[5] = (T)((2.0e-13*beta*dt*y[0] + 1.0)*sc[1]*isc[1]);
    a[6] = (T)((-2.0e-13*beta*dt*y[0])*sc[2]*isc[1]);
    { /* Tgas row, column 1 */
      for (int m = 0; m < 9; ++m) hc_yy[m] = y[m];
      const double dyy = y[1]*1e-2;
      hc_yy[1] = y[1] + dyy;
      const double dy1 = ov_hctoy_dense_none_hc(hc_yy, y[7], y);
      if (dyy > 0.0) a[7] = (T)((-(beta*dt*(dy1 - hc_dy0)/dyy))*sc[5]*isc[1]);
    }
    a[8] = (T)((-1.0e-15*beta*dt*y[0])*sc[0]*isc[2]);
    a[9] = (T)((-1.0e-15*beta*dt*y[0])*sc[1]*isc[2]);
    a[10] = (T)((-beta*dt*(-1.0e-15*y[0] - 4.0e-17*y[2]) + 1.0)*sc[2]*isc[2]);
    a[11] = (T)((-2.0e-17*beta*dt*y[2])*sc[3]*isc[2]);
    { /* Tgas row, column 2 */
      for (int m = 0; m < 9; ++m) hc_yy[m] = y[m];
      const double dyy = y[2]*1e-2;
      hc_yy[2] = y[2] + dyy;
      const double dy1 = ov_hctoy_dense_none_hc(hc_yy, y[7], y);
      if (dyy > 0.0) a[12] = (T)((-(beta*dt*(dy1 - hc_dy0)/dyy))*sc[5]*isc[2]);
    }
    a[13] = (T)((-2.0e-10*beta*dt)*sc[2]*isc[3]);
    a[14] = (T)((1.0e-10*beta*dt + 1.0)*sc[3]*isc[3]);
    { /* Tgas row, column 3 */
      for (int m = 0; m < 9; ++m) hc_yy[m] = y[m];
      const double dyy = y[3]*1e-2;
      hc_yy[3] = y[3] + dyy;
      const double dy1 = ov_hctoy_dense_none_hc(hc_yy, y[7], y);
      if (dyy > 0.0) a[15] = (T)((-(beta*dt*(dy1 - hc_dy0)/dyy))*sc[5]*isc[3]);
    }
    a[16] = (T)((1.0)*sc[4]*isc[4]);
    { /* Tgas row, column 4 */
      for (int m = 0; m < 9; ++m) hc_yy[m] = y[m];
      const double dyy = y[4]*1e-2;
      hc_yy[4] = y[4] + dyy;
      const double dy1 = ov_hctoy_dense_none_hc(hc_yy, y[7], y);
      if (dyy > 0.0) a[17] = (T)((-(beta*dt*(dy1 - hc_dy0)/dyy))*sc[5]*isc[4]);
    }
    { /* Tgas column */
      const double dyy = y[7]*1e-2;
      hc_yy[7] = y[7] + dyy;
      double dy[9];
      ov_hctoy_dense_none_rhs(hc_yy, k, dy);
      a[18] = (T)((-(beta*dt*(dy[0]/dyy)))*sc[0]*isc[5]);
      a[19] = (T)((-(beta*dt*(dy[1]/dyy)))*sc[1]*isc[5]);
      a[20] = (T)((-(beta*dt*(dy[2]/dyy)))*sc[2]*isc[5]);
      a[21] = (T)((-(beta*dt*(dy[3]/dyy)))*sc[3]*isc[5]);
      a[22] = (T)((-(beta*dt*(dy[4]/dyy)))*sc[4]*isc[5]);
      a[23] = (T)((1.0 + (-(beta*dt*(dy[7]/dyy))))*sc[5]*isc[5]);
    }
  }
  /* in-place numeric LU of the packed dynamic block a[0..NNZ-1]; A is a
     pointer or an accessor whose operator[] yields T& */
  template <class T, class A> OV_HD static OV_INLINE void lu_factor(A a) {
    (void)a;
    a[0] = ov_pivot<T>(a[0]);
    a[1] = ov_divp<T>(a[1], a[0]);
    a[2] = ov_divp<T>(a[2], a[0]);
    a[3] = ov_divp<T>(a[3], a[0]);
    a[5] = a[5] - a[1]*a[4];
    a[6] = a[6] - a[2]*a[4];
    a[7] = a[7] - a[3]*a[4];
    a[9] = a[9] - a[1]*a[8];
    a[10] = a[10] - a[2]*a[8];
    a[12] = a[12] - a[3]*a[8];
    a[19] = a[19] - a[1]*a[18];
    a[20] = a[20] - a[2]*a[18];
    a[23] = a[23] - a[3]*a[18];
    a[5] = ov_pivot<T>(a[5]);
    a[6] = ov_divp<T>(a[6], a[5]);
    a[7] = ov_divp<T>(a[7], a[5]);
    a[10] = a[10] - a[6]*a[9];
    a[12] = a[12] - a[7]*a[9];
    a[20] = a[20] - a[6]*a[19];
    a[23] = a[23] - a[7]*a[19];
    a[10] = ov_pivot<T>(a[10]);
    a[11] = ov_divp<T>(a[11], a[10]);
    a[12] = ov_divp<T>(a[12], a[10]);
    a[14] = a[14] - a[11]*a[13];
    a[15] = a[15] - a[12]*a[13];
    a[21] = a[21] - a[11]*a[20];
    a[23] = a[23] - a[12]*a[20];
    a[14] = ov_pivot<T>(a[14]);
    a[15] = ov_divp<T>(a[15], a[14]);
    a[23] = a[23] - a[15]*a[21];
    a[16] = ov_pivot<T>(a[16]);
    a[17] = ov_divp<T>(a[17], a[16]);
    a[23] = a[23] - a[17]*a[22];
    a[23] = ov_pivot<T>(a[23]);
  }
  /* x = P^-1 r on the dynamic block; r, x over solver-state indices.  sc/isc
     scale entry i by sc[i] on the way in and isc[i] on the way out (pass
     nullptr for none); T is the precision of the solve. */
  template <class T, class A> OV_HD static OV_INLINE void lu_solve(A a, const double* OV_RESTRICT r, double* OV_RESTRICT x, const double* OV_RESTRICT sc, const double* OV_RESTRICT isc) {
#define OV_SC(i) (sc ? sc[i] : 1.0)
#define OV_ISC(i) (isc ? isc[i] : 1.0)
    T d0 = (T)(r[0]*OV_SC(0));
    T d1 = (T)(r[1]*OV_SC(1));
    T d2 = (T)(r[2]*OV_SC(2));
    T d3 = (T)(r[3]*OV_SC(3));
    T d4 = (T)(r[4]*OV_SC(4));
    T d7 = (T)(r[5]*OV_SC(5));
    d1 = d1 - a[1]*d0;
    d2 = d2 - (a[2]*d0 + a[6]*d1);
    d3 = d3 - a[11]*d2;
    d7 = d7 - ((((a[3]*d0 + a[7]*d1) + a[12]*d2) + a[15]*d3) + a[17]*d4);
    d7 = ov_divp<T>(d7, a[23]);
    d4 = ov_divp<T>((d4 - a[22]*d7), a[16]);
    d3 = ov_divp<T>((d3 - a[21]*d7), a[14]);
    d2 = ov_divp<T>((d2 - (a[13]*d3 + a[20]*d7)), a[10]);
    d1 = ov_divp<T>((d1 - (a[9]*d2 + a[19]*d7)), a[5]);
    d0 = ov_divp<T>((d0 - ((a[4]*d1 + a[8]*d2) + a[18]*d7)), a[0]);
    x[0] = (double)d0*OV_ISC(0);
    x[1] = (double)d1*OV_ISC(1);
    x[2] = (double)d2*OV_ISC(2);
    x[3] = (double)d3*OV_ISC(3);
    x[4] = (double)d4*OV_ISC(4);
    x[5] = (double)d7*OV_ISC(5);
#undef OV_SC
#undef OV_ISC
  }
};
