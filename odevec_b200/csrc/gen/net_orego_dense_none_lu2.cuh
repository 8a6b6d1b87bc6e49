/* Generated by odevec_b200.pre_odevec -- do not edit.
 * CUDA traits of network variant OREGO_DENSE_NONE_LU2 for the BDF kernel: straight-line
 * LU factorisation and solve over the fill pattern (right-looking Doolittle). */
#pragma once
#include "net_orego_dense_none_lu2.h"

struct ov_net_orego_dense_none_lu2 {
  static constexpr bool HAS_WPC = false;
  using Wpc = void;
  static constexpr int NEQ = 3;   /* all species (state vector) */
  static constexpr int ND = 3;    /* species in the solver state */
  static constexpr int NNZ = 8;   /* packed LU entries of the dynamic block */
  static constexpr int NREA = 0;
  static constexpr int IDX_TGAS = -1;
  static constexpr bool DENSE = true;
  /* 1: symbolic Jacobian + numeric LU, 2: symbolic LU, 3: difference quotients */
  static constexpr int LU_METHOD = 2;
  /* the Tgas row is the heating/cooling term (--heatcool=1); HC_FD: GetJac writes
     its difference quotients and leaves some entries as the storage holds them */
  static constexpr bool HEATCOOL = false;
  static constexpr bool HC_FD = false;
  static constexpr const char* TAG = "OREGO_DENSE_NONE_LU2";
  /* dynamic species (solver state index -> species) and frozen ones */
  OV_HD static constexpr int dyn(int i) { return i == 0 ? 0 : (i == 1 ? 1 : (2)); }
  static constexpr int NF = 0;
  OV_HD static constexpr int frozen(int i) { return 0; }
  OV_HD static OV_INLINE void rhs(const double* y, const double* k, double* f) { ov_orego_dense_none_lu2_rhs(y, k, f); }
  static OV_INLINE __device__ void rates_k(const double*, const double*, double*) {}
  static OV_INLINE __device__ void rates_T(const double*, double*) {}
  /* P = I - dt*beta*J on the dynamic block, packed CSC order */
  template <class T, class A> OV_HD static OV_INLINE void jac(const double* OV_RESTRICT y, const double* OV_RESTRICT k, double beta, double dt, A a) {
    (void)y; (void)k; (void)beta; (void)dt; (void)a;
    a[0] = (T)(-beta*dt*(-0.0012942725*y[0] - 77.27*y[1] + 77.27) + 1.0);
    a[1] = (T)(0.0129416332341141*beta*dt*y[1]/(-beta*dt*(-0.0012942725*y[0] - 77.27*y[1] + 77.27) + 1.0));
    a[2] = (T)(-0.161*beta*dt/(-beta*dt*(-0.0012942725*y[0] - 77.27*y[1] + 77.27) + 1.0));
    a[3] = (T)(-beta*dt*(77.27 - 77.27*y[0]));
    a[4] = (T)(0.0129416332341141*((beta)*(beta))*((dt)*(dt))*y[1]*(77.27 - 77.27*y[0])/(-beta*dt*(-0.0012942725*y[0] - 77.27*y[1] + 77.27) + 1.0) - beta*dt*(-0.0129416332341141*y[0] - 0.0129416332341141) + 1.0);
    a[5] = (T)(-0.161*((beta)*(beta))*((dt)*(dt))*(77.27 - 77.27*y[0])/((-beta*dt*(-0.0012942725*y[0] - 77.27*y[1] + 77.27) + 1.0)*(0.0129416332341141*((beta)*(beta))*((dt)*(dt))*y[1]*(77.27 - 77.27*y[0])/(-beta*dt*(-0.0012942725*y[0] - 77.27*y[1] + 77.27) + 1.0) - beta*dt*(-0.0129416332341141*y[0] - 0.0129416332341141) + 1.0)));
    a[6] = (T)(-0.0129416332341141*beta*dt);
    a[7] = (T)(-0.00208360295069238*((beta)*((beta)*(beta)))*((dt)*((dt)*(dt)))*(77.27 - 77.27*y[0])/((-beta*dt*(-0.0012942725*y[0] - 77.27*y[1] + 77.27) + 1.0)*(0.0129416332341141*((beta)*(beta))*((dt)*(dt))*y[1]*(77.27 - 77.27*y[0])/(-beta*dt*(-0.0012942725*y[0] - 77.27*y[1] + 77.27) + 1.0) - beta*dt*(-0.0129416332341141*y[0] - 0.0129416332341141) + 1.0)) + 0.161*beta*dt + 1.0);
  }
  /* a = D P D^-1 rounded to T, D = diag(sc) over solver-state indices */
  template <class T, class A> OV_HD static OV_INLINE void store_scaled(const double* OV_RESTRICT P, A a, const double* OV_RESTRICT sc, const double* OV_RESTRICT isc) {
    a[0] = (T)(P[0]*sc[0]*isc[0]);
    a[1] = (T)(P[1]*sc[1]*isc[0]);
    a[2] = (T)(P[2]*sc[2]*isc[0]);
    a[3] = (T)(P[3]*sc[0]*isc[1]);
    a[4] = (T)(P[4]*sc[1]*isc[1]);
    a[5] = (T)(P[5]*sc[2]*isc[1]);
    a[6] = (T)(P[6]*sc[1]*isc[2]);
    a[7] = (T)(P[7]*sc[2]*isc[2]);
  }
  /* the same, each entry evaluated in FP64, scaled by powers of two and
     rounded to T on the fly */
  template <class T, class A> OV_HD static OV_INLINE void jac_scaled(const double* OV_RESTRICT y, const double* OV_RESTRICT k, double beta, double dt, A a, const double* OV_RESTRICT sc, const double* OV_RESTRICT isc) {
    (void)y; (void)k; (void)beta; (void)dt; (void)a; (void)sc; (void)isc;
    a[0] = (T)((-beta*dt*(-0.0012942725*y[0] - 77.27*y[1] + 77.27) + 1.0)*sc[0]*isc[0]);
    a[1] = (T)((0.0129416332341141*beta*dt*y[1]/(-beta*dt*(-0.0012942725*y[0] - 77.27*y[1] + 77.27) + 1.0))*sc[1]*isc[0]);
    a[2] = (T)((-0.161*beta*dt/(-beta*dt*(-0.0012942725*y[0] - 77.27*y[1] + 77.27) + 1.0))*sc[2]*isc[0]);
    a[3] = (T)((-beta*dt*(77.27 - 77.27*y[0]))*sc[0]*isc[1]);
    a[4] = (T)((0.0129416332341141*((beta)*(beta))*((dt)*(dt))*y[1]*(77.27 - 77.27*y[0])/(-beta*dt*(-0.0012942725*y[0] - 77.27*y[1] + 77.27) + 1.0) - beta*dt*(-0.0129416332341141*y[0] - 0.0129416332341141) + 1.0)*sc[1]*isc[1]);
    a[5] = (T)((-0.161*((beta)*(beta))*((dt)*(dt))*(77.27 - 77.27*y[0])/((-beta*dt*(-0.0012942725*y[0] - 77.27*y[1] + 77.27) + 1.0)*(0.0129416332341141*((beta)*(beta))*((dt)*(dt))*y[1]*(77.27 - 77.27*y[0])/(-beta*dt*(-0.0012942725*y[0] - 77.27*y[1] + 77.27) + 1.0) - beta*dt*(-0.0129416332341141*y[0] - 0.0129416332341141) + 1.0)))*sc[2]*isc[1]);
    a[6] = (T)((-0.0129416332341141*beta*dt)*sc[1]*isc[2]);
    a[7] = (T)((-0.00208360295069238*((beta)*((beta)*(beta)))*((dt)*((dt)*(dt)))*(77.27 - 77.27*y[0])/((-beta*dt*(-0.0012942725*y[0] - 77.27*y[1] + 77.27) + 1.0)*(0.0129416332341141*((beta)*(beta))*((dt)*(dt))*y[1]*(77.27 - 77.27*y[0])/(-beta*dt*(-0.0012942725*y[0] - 77.27*y[1] + 77.27) + 1.0) - beta*dt*(-0.0129416332341141*y[0] - 0.0129416332341141) + 1.0)) + 0.161*beta*dt + 1.0)*sc[2]*isc[2]);
  }
  /* in-place numeric LU of the packed dynamic block a[0..NNZ-1]; A is a
     pointer or an accessor whose operator[] yields T& */
  template <class T, class A> OV_HD static OV_INLINE void lu_factor(A a) {
    (void)a;
    a[7] = ov_pivot<T>(a[7]);
    a[4] = ov_pivot<T>(a[4]);
    a[0] = ov_pivot<T>(a[0]);
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
    d1 = d1 - a[1]*d0;
    d2 = d2 - (a[2]*d0 + a[5]*d1);
    d2 = ov_divp<T>(d2, a[7]);
    d1 = ov_divp<T>((d1 - a[6]*d2), a[4]);
    d0 = ov_divp<T>((d0 - a[3]*d1), a[0]);
    x[0] = (double)d0*OV_ISC(0);
    x[1] = (double)d1*OV_ISC(1);
    x[2] = (double)d2*OV_ISC(2);
#undef OV_SC
#undef OV_ISC
  }
};
