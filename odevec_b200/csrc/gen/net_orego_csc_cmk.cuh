/* Generated by odevec_b200.pre_odevec -- do not edit.
 * CUDA traits of network variant OREGO_CSC_CMK for the BDF kernel: straight-line
 * LU factorisation and solve over the fill pattern (left-looking Crout, CSC). */
#pragma once
#include "net_orego_csc_cmk.h"


/* warp-per-cell tables (odevec_b200/wpc.py) */
static __device__ const int ov_wpc_orego_csc_cmk_rhs_ptr[4] = {
    0, 4, 7, 9};
static __device__ const double ov_wpc_orego_csc_cmk_rhs_coef[9] = {
    -0.00064713625, -77.27, 77.27, 77.27,
    -0.0129416332341141, -0.0129416332341141, 0.0129416332341141, 0.161,
    -0.161};
static __device__ const int ov_wpc_orego_csc_cmk_rhs_fac[27] = {
    1, -1, -1, 0, 2, -1, 0, -1, -1, 2, -1, -1, 0, 2, -1, 2,
    -1, -1, 4, -1, -1, 0, -1, -1, 4, -1, -1};
static __device__ const int ov_wpc_orego_csc_cmk_jac_ptr[8] = {
    0, 7, 13, 26, 36, 42, 49, 66};
static __device__ const int ov_wpc_orego_csc_cmk_jac_code[66] = {
    0, 2, 7, 3, 7, 16, 5, 32, 4, 2, 7, 3, 7, 2, 4, 3,
    7, 48, 4, 1, 7, 64, 6, 7, 80, 5, 2, 4, 3, 7, 96, 112,
    1, 7, 6, 7, 128, 4, 2, 7, 3, 7, 144, 2, 7, 3, 7, 17,
    7, 2, 4, 3, 7, 160, 4, 1, 7, 176, 17, 7, 6, 192, 5, 7,
    208, 5};
static __device__ const double ov_wpc_orego_csc_cmk_jac_const[14] = {
    0.161, 1.0, 0.0129416332341141, 0.0129416332341141,
    0.0129416332341141, 1.0, 77.27, 77.27,
    0.161, 0.0129416332341141, 0.0012942725, 77.27,
    77.27, 1.0};
static __device__ const int ov_wpc_orego_csc_cmk_jac_rc[7] = {
    131074, 131073, 65537, 65536, 2, 1, 0};
static __device__ const long long ov_wpc_orego_csc_cmk_fac_op[128] = {
    2305840810190438408LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    2199031644171LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    2305840810194632714LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    6597080252429LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL};
static __device__ const long long ov_wpc_orego_csc_cmk_sol_op[192] = {
    2199021158400LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    2199023255555LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    6597067669506LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    6597071863813LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    15393160691716LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    8796097216513LL, 10995120472067LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL};
static __device__ const long long ov_wpc_orego_csc_cmk_fac_op16[64] = {
    2305840810190438408LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    2199031644171LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    2305840810194632714LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    6597080252429LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL};
static __device__ const long long ov_wpc_orego_csc_cmk_sol_op16[96] = {
    2199021158400LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    2199023255555LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    6597067669506LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    6597071863813LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    15393160691716LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    8796097216513LL, 10995120472067LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL};
static __device__ const long long ov_wpc_orego_csc_cmk_fac_op8[32] = {
    2305840810190438408LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    2199031644171LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    2305840810194632714LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    6597080252429LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL};
static __device__ const long long ov_wpc_orego_csc_cmk_sol_op8[48] = {
    2199021158400LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    2199023255555LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    6597067669506LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    6597071863813LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    15393160691716LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL,
    8796097216513LL, 10995120472067LL, -1LL, -1LL, -1LL, -1LL, -1LL, -1LL};
static __device__ const int ov_wpc_orego_csc_cmk_srow[3] = {
    2, 1, 0};
static __device__ const int ov_wpc_orego_csc_cmk_dyn[3] = {
    0, 1, 2};
struct ov_wpc_orego_csc_cmk {
  static constexpr int NTERM = 9, NPROG = 7, DEPTH = 4, NFL = 4, NSL = 6;
  static constexpr int NFL16 = 4, NSL16 = 6;
  static constexpr int NFL8 = 4, NSL8 = 6;
  __device__ static const int* rhs_ptr() { return ov_wpc_orego_csc_cmk_rhs_ptr; }
  __device__ static const int* rhs_fac() { return ov_wpc_orego_csc_cmk_rhs_fac; }
  __device__ static const int* jac_ptr() { return ov_wpc_orego_csc_cmk_jac_ptr; }
  __device__ static const int* jac_code() { return ov_wpc_orego_csc_cmk_jac_code; }
  __device__ static const int* jac_rc() { return ov_wpc_orego_csc_cmk_jac_rc; }
  __device__ static const int* srow() { return ov_wpc_orego_csc_cmk_srow; }
  __device__ static const int* dyn() { return ov_wpc_orego_csc_cmk_dyn; }
  __device__ static const double* rhs_coef() { return ov_wpc_orego_csc_cmk_rhs_coef; }
  __device__ static const double* jac_const() { return ov_wpc_orego_csc_cmk_jac_const; }
  __device__ static const long long* fac_op() { return ov_wpc_orego_csc_cmk_fac_op; }
  __device__ static const long long* sol_op() { return ov_wpc_orego_csc_cmk_sol_op; }
  __device__ static const long long* fac_op16() { return ov_wpc_orego_csc_cmk_fac_op16; }
  __device__ static const long long* sol_op16() { return ov_wpc_orego_csc_cmk_sol_op16; }
  __device__ static const long long* fac_op8() { return ov_wpc_orego_csc_cmk_fac_op8; }
  __device__ static const long long* sol_op8() { return ov_wpc_orego_csc_cmk_sol_op8; }
};

struct ov_net_orego_csc_cmk {
  /* warp-per-cell tables (staging 7) */
  static constexpr bool HAS_WPC = true;
  using Wpc = ov_wpc_orego_csc_cmk;
  static constexpr int NEQ = 3;   /* all species (state vector) */
  static constexpr int ND = 3;    /* species in the solver state */
  static constexpr int NNZ = 7;   /* packed LU entries of the dynamic block */
  static constexpr int NREA = 0;
  static constexpr int IDX_TGAS = -1;
  static constexpr bool DENSE = false;
  /* 1: symbolic Jacobian + numeric LU, 2: symbolic LU, 3: difference quotients */
  static constexpr int LU_METHOD = 1;
  /* the Tgas row is the heating/cooling term (--heatcool=1); HC_FD: GetJac writes
     its difference quotients and leaves some entries as the storage holds them */
  static constexpr bool HEATCOOL = false;
  static constexpr bool HC_FD = false;
  static constexpr const char* TAG = "OREGO_CSC_CMK";
  /* dynamic species (solver state index -> species) and frozen ones */
  OV_HD static constexpr int dyn(int i) { return i == 0 ? 0 : (i == 1 ? 1 : (2)); }
  static constexpr int NF = 0;
  OV_HD static constexpr int frozen(int i) { return 0; }
  OV_HD static OV_INLINE void rhs(const double* y, const double* k, double* f) { ov_orego_csc_cmk_rhs(y, k, f); }
  static OV_INLINE __device__ void rates_k(const double*, const double*, double*) {}
  static OV_INLINE __device__ void rates_T(const double*, double*) {}
  /* P = I - dt*beta*J on the dynamic block, packed CSC order */
  template <class T, class A> OV_HD static OV_INLINE void jac(const double* OV_RESTRICT y, const double* OV_RESTRICT k, double beta, double dt, A a) {
    (void)y; (void)k; (void)beta; (void)dt; (void)a;
    a[0] = (T)(0.161*beta*dt + 1.0);
    a[1] = (T)(-0.0129416332341141*beta*dt);
    a[2] = (T)(-beta*dt*(-0.0129416332341141*y[0] - 0.0129416332341141) + 1.0);
    a[3] = (T)(-beta*dt*(77.27 - 77.27*y[0]));
    a[4] = (T)(-0.161*beta*dt);
    a[5] = (T)(0.0129416332341141*beta*dt*y[1]);
    a[6] = (T)(-beta*dt*(-0.0012942725*y[0] - 77.27*y[1] + 77.27) + 1.0);
  }
  /* a = D P D^-1 rounded to T, D = diag(sc) over solver-state indices */
  template <class T, class A> OV_HD static OV_INLINE void store_scaled(const double* OV_RESTRICT P, A a, const double* OV_RESTRICT sc, const double* OV_RESTRICT isc) {
    a[0] = (T)(P[0]*sc[2]*isc[2]);
    a[1] = (T)(P[1]*sc[1]*isc[2]);
    a[2] = (T)(P[2]*sc[1]*isc[1]);
    a[3] = (T)(P[3]*sc[0]*isc[1]);
    a[4] = (T)(P[4]*sc[2]*isc[0]);
    a[5] = (T)(P[5]*sc[1]*isc[0]);
    a[6] = (T)(P[6]*sc[0]*isc[0]);
  }
  /* the same, each entry evaluated in FP64, scaled by powers of two and
     rounded to T on the fly */
  template <class T, class A> OV_HD static OV_INLINE void jac_scaled(const double* OV_RESTRICT y, const double* OV_RESTRICT k, double beta, double dt, A a, const double* OV_RESTRICT sc, const double* OV_RESTRICT isc) {
    (void)y; (void)k; (void)beta; (void)dt; (void)a; (void)sc; (void)isc;
    a[0] = (T)((0.161*beta*dt + 1.0)*sc[2]*isc[2]);
    a[1] = (T)((-0.0129416332341141*beta*dt)*sc[1]*isc[2]);
    a[2] = (T)((-beta*dt*(-0.0129416332341141*y[0] - 0.0129416332341141) + 1.0)*sc[1]*isc[1]);
    a[3] = (T)((-beta*dt*(77.27 - 77.27*y[0]))*sc[0]*isc[1]);
    a[4] = (T)((-0.161*beta*dt)*sc[2]*isc[0]);
    a[5] = (T)((0.0129416332341141*beta*dt*y[1])*sc[1]*isc[0]);
    a[6] = (T)((-beta*dt*(-0.0012942725*y[0] - 77.27*y[1] + 77.27) + 1.0)*sc[0]*isc[0]);
  }
  /* in-place numeric LU of the packed dynamic block a[0..NNZ-1]; A is a
     pointer or an accessor whose operator[] yields T& */
  template <class T, class A> OV_HD static OV_INLINE void lu_factor(A a) {
    (void)a;
    a[0] = ov_pivot<T>(a[0]);
    a[4] = ov_divp<T>(a[4], a[0]);
    a[5] = a[5] - a[4]*a[1];
    a[2] = ov_pivot<T>(a[2]);
    a[5] = ov_divp<T>(a[5], a[2]);
    a[6] = a[6] - a[5]*a[3];
    a[6] = ov_pivot<T>(a[6]);
  }
  /* x = P^-1 r on the dynamic block; r, x over solver-state indices.  sc/isc
     scale entry i by sc[i] on the way in and isc[i] on the way out (pass
     nullptr for none); T is the precision of the solve. */
  template <class T, class A> OV_HD static OV_INLINE void lu_solve(A a, const double* OV_RESTRICT r, double* OV_RESTRICT x, const double* OV_RESTRICT sc, const double* OV_RESTRICT isc) {
#define OV_SC(i) (sc ? sc[i] : 1.0)
#define OV_ISC(i) (isc ? isc[i] : 1.0)
    T d0 = (T)(r[2]*OV_SC(2));
    T d1 = (T)(r[1]*OV_SC(1));
    T d2 = (T)(r[0]*OV_SC(0));
    d0 = ov_divp<T>(d0, a[0]);
    d1 = d1 - d0*a[1];
    d1 = ov_divp<T>(d1, a[2]);
    d2 = d2 - d1*a[3];
    d2 = ov_divp<T>(d2, a[6]);
    d0 = d0 - d2*a[4];
    d1 = d1 - d2*a[5];
    x[2] = (double)d0*OV_ISC(2);
    x[1] = (double)d1*OV_ISC(1);
    x[0] = (double)d2*OV_ISC(0);
#undef OV_SC
#undef OV_ISC
  }
};
