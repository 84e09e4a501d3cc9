// harm_device.cuh -- per-zone GRMHD physics as sm_100a device functions.
//
// Every function keeps the floating-point operation order of the reference
// routine it cites, and the translation unit is compiled with -fmad=false, so
// that the FP64 path reproduces the reference CPU build bit for bit (the
// reference is built with -ffp-contract=off).  sqrt and '/' are IEEE
// correctly rounded on both sides.
//
// Build options mirrored: WHICHVEL=VELREL4, REMOVERESTMASSFROMUU=2,
// WHICHEOM=WITHGDET, EOMTYPE=EOMGRMHD, ideal-gas EOS (eos.c:58-194),
// MAXWELL=PRIMMAXWELL (phys.c:140), TRUEFAST=0 (vchar.c:33),
// UTOPRIMVERSION=UTOPRIM2DFINAL with PRECISEINVERSION=1 (u2p_defs.h).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace hg {

constexpr int NPR = 8;
constexpr int RHO = 0, UU = 1, U1 = 2, U2 = 3, U3 = 4, B1 = 5, B2 = 6, B3 = 7;
constexpr int TT = 0;

// failure codes (global.h:782-799)
constexpr int UTOPRIMFAILFIXED = -1;
constexpr int UTOPRIMNOFAIL = 0;
constexpr int UTOPRIMFAILCONVW = 2;
constexpr int UTOPRIMFAILCONVUTSQ = 3;
constexpr int UTOPRIMFAILCONVGUESSUTSQ = 4;
constexpr int UTOPRIMFAILRHONEG = 9;
constexpr int UTOPRIMFAILUNEG = 10;
constexpr int UTOPRIMFAILRHOUNEG = 11;
constexpr int UTOPRIMFAILGAMMAPERC = 12;
constexpr int UTOPRIMFAILUPERC = 13;
constexpr int UTOPRIMFAILU2AVG1 = 14;
constexpr int UTOPRIMFAILU2AVG2 = 15;

constexpr double NUMEPSILON = 2.2204460492503131e-16;
constexpr double BIGNUM = 1.e+50;

// error bits (conditions where the reference calls fail() or myexit())
constexpr int ERR_UTCALC_DISCR = 1;
constexpr int ERR_COEFF_NEG = 2;
constexpr int ERR_COEFF_SUP = 4;
constexpr int ERR_VCHAR_DISCR = 8;
constexpr int ERR_VSQ_NEG = 16;
constexpr int ERR_NONFINITE_SPEED = 32;
constexpr int ERR_PREF_NEG = 64;
constexpr int ERR_BONDI = 128;  // bondi_invert_integrals' myexit (bounds.c:1040-1066)

// Tolerances of the reference's round-off guards, per arithmetic type.  The
// FP64 values are the reference's own (NUMEPSILON = DBL_EPSILON, global.h);
// the FP32 ones scale the same guards to FP32 round-off for the mixed
// precision path (reconstruction, wave speeds and Riemann fluxes in FP32).
template <typename T> struct Tol;
template <> struct Tol<double> {
  static constexpr double numeps = NUMEPSILON;       // gamma_calc, vchar cms2 guards
  static constexpr double discr = 1E-10;             // simplefast discriminant (vchar.c:268)
  static constexpr double cs2cap = 1e-9;             // vchar cs2 cap (vchar.c:77)
};
template <> struct Tol<float> {
  static constexpr float numeps = 1.1920929e-07f;    // FLT_EPSILON
  static constexpr float discr = 1E-5f;
  static constexpr float cs2cap = 1e-6f;
};

// Metric at one grid location.  gcov is stored in full because the
// reference's gcov is not exactly symmetric (differences ~1e-13) and its
// routines read different triangles in different places.
template <typename T>
struct MetricT {
  T gcov[16];
  T gcon[16];
  T gcovpert_tt;
  T g;
};
using Metric = MetricT<double>;

template <typename T>
struct StateT {
  T ucon[4], ucov[4], bcon[4], bcov[4];
};
using State = StateT<double>;

// Per-state electromagnetic pieces reused by every T^dir_mu row
// (Mcon_calc phys.c:178, lower_A phys.ffde.c:1707, Msq and 1+u_t).
template <typename T>
struct EMT {
  T Mcon[4][4];
  T Mcov[4][4];
  T Msq;
  T plus1ud0;
};
using EM = EMT<double>;

#define GCOV(m, a, b) ((m).gcov[(a) * 4 + (b)])
#define GCON(m, a, b) ((m).gcon[(a) * 4 + (b)])

template <typename T>
__device__ __forceinline__ T dot4(const T *a, const T *b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3];
}

// lower_vec (phys.c:766-787)
template <typename T>
__device__ __forceinline__ void lower_vec(const T *ucon, const MetricT<T> &m, T *ucov) {
  ucov[0] = GCOV(m, 0, 0) * ucon[0] + GCOV(m, 0, 1) * ucon[1] + GCOV(m, 0, 2) * ucon[2] + GCOV(m, 0, 3) * ucon[3];
  ucov[1] = GCOV(m, 0, 1) * ucon[0] + GCOV(m, 1, 1) * ucon[1] + GCOV(m, 1, 2) * ucon[2] + GCOV(m, 1, 3) * ucon[3];
  ucov[2] = GCOV(m, 0, 2) * ucon[0] + GCOV(m, 1, 2) * ucon[1] + GCOV(m, 2, 2) * ucon[2] + GCOV(m, 2, 3) * ucon[3];
  ucov[3] = GCOV(m, 0, 3) * ucon[0] + GCOV(m, 1, 3) * ucon[1] + GCOV(m, 2, 3) * ucon[2] + GCOV(m, 3, 3) * ucon[3];
}

// raise_vec (phys.c:826-846)
template <typename T>
__device__ __forceinline__ void raise_vec(const T *ucov, const MetricT<T> &m, T *ucon) {
  ucon[0] = GCON(m, 0, 0) * ucov[0] + GCON(m, 0, 1) * ucov[1] + GCON(m, 0, 2) * ucov[2] + GCON(m, 0, 3) * ucov[3];
  ucon[1] = GCON(m, 0, 1) * ucov[0] + GCON(m, 1, 1) * ucov[1] + GCON(m, 1, 2) * ucov[2] + GCON(m, 1, 3) * ucov[3];
  ucon[2] = GCON(m, 0, 2) * ucov[0] + GCON(m, 1, 2) * ucov[1] + GCON(m, 2, 2) * ucov[2] + GCON(m, 2, 3) * ucov[3];
  ucon[3] = GCON(m, 0, 3) * ucov[0] + GCON(m, 1, 3) * ucov[1] + GCON(m, 2, 3) * ucov[2] + GCON(m, 3, 3) * ucov[3];
}

// qsq_calc (phys.c:1077-1090) on the relative 4-velocity u~^i
template <typename T>
__device__ __forceinline__ T qsq_calc(T u1, T u2, T u3, const MetricT<T> &m) {
  return +GCOV(m, 1, 1) * u1 * u1 + GCOV(m, 2, 2) * u2 * u2 + GCOV(m, 3, 3) * u3 * u3 +
         T(2.) * (GCOV(m, 1, 2) * u1 * u2 + GCOV(m, 1, 3) * u1 * u3 + GCOV(m, 2, 3) * u2 * u3);
}

// gamma_calc (phys.c:1022-1074); returns nonzero if qsq is negative beyond
// round-off (the reference calls fail(FAIL_UTCALC_DISCR))
template <typename T>
__device__ __forceinline__ int gamma_calc(const T *pr, const MetricT<T> &m, T *gamma) {
  T qsq = qsq_calc(pr[U1], pr[U2], pr[U3], m);
  if (qsq < T(0.0)) {
    if (qsq > -Tol<T>::numeps * T(100)) qsq = T(0.0);
    else return 1;
  }
  *gamma = sqrt(T(1.) + qsq);
  return 0;
}

// ucon_calc_rel4vel (phys.c:983-1019)
template <typename T>
__device__ __forceinline__ int ucon_calc(const T *pr, const MetricT<T> &m, T *ucon) {
  T alpha = T(1.) / sqrt(-GCON(m, 0, 0));
  T beta1 = GCON(m, 0, 1) * alpha * alpha;
  T beta2 = GCON(m, 0, 2) * alpha * alpha;
  T beta3 = GCON(m, 0, 3) * alpha * alpha;
  T gamma;
  if (gamma_calc(pr, m, &gamma)) return 1;
  ucon[0] = gamma / alpha;
  ucon[1] = pr[U1] - ucon[0] * beta1;
  ucon[2] = pr[U2] - ucon[0] * beta2;
  ucon[3] = pr[U3] - ucon[0] * beta3;
  return 0;
}

// get_state (phys.c:849-859) with bcon_calc (phys.c:309-318)
template <typename T>
__device__ __forceinline__ int get_state(const T *pr, const MetricT<T> &m, StateT<T> &q) {
  if (ucon_calc(pr, m, q.ucon)) return 1;
  lower_vec(q.ucon, m, q.ucov);
  q.bcon[0] = pr[B1] * q.ucov[1] + pr[B2] * q.ucov[2] + pr[B3] * q.ucov[3];
#pragma unroll
  for (int j = 1; j <= 3; j++) q.bcon[j] = (pr[B1 - 1 + j] + q.bcon[0] * q.ucon[j]) / q.ucon[0];
  lower_vec(q.bcon, m, q.bcov);
  return 0;
}

// compute_1plusud0 (phys.c:541-575)
template <typename T>
__device__ __forceinline__ T compute_1plusud0(const MetricT<T> &m, const StateT<T> &q) {
  T vcon[4];
#pragma unroll
  for (int j = 1; j < 4; j++) vcon[j] = q.ucon[j] / q.ucon[0];
  T plus1gv00 = m.gcovpert_tt;
  T vsq = m.gcovpert_tt;
#pragma unroll
  for (int j = 1; j < 4; j++) vsq += T(2.0) * GCOV(m, 0, j) * vcon[j];
#pragma unroll
  for (int j = 1; j < 4; j++)
#pragma unroll
    for (int k = 1; k < 4; k++) vsq += GCOV(m, j, k) * vcon[j] * vcon[k];
  T gvtt = GCOV(m, 0, 0);
  T alpha = T(0.0);
#pragma unroll
  for (int j = 1; j < 4; j++) alpha += GCOV(m, j, 0) * q.ucon[j];
  T uu0 = q.ucon[0];
  return alpha + ((T(1.0) - gvtt) * plus1gv00 - uu0 * uu0 * vsq * gvtt * gvtt) / (T(1.0) - gvtt * uu0);
}

// Mcon_calc PRIMMAXWELL (phys.c:178-210), lower_A (phys.ffde.c:1707-1735),
// Msq (phys.ffde.c:1507) and 1+u_t
template <typename T>
__device__ __forceinline__ void em_prepare(const T *pr, const MetricT<T> &m, const StateT<T> &q, EMT<T> &e) {
#pragma unroll
  for (int j = 0; j < 4; j++) e.Mcon[j][j] = T(0.0);
#pragma unroll
  for (int k = 1; k < 4; k++) {
    e.Mcon[k][0] = pr[B1 + k - 1];
    e.Mcon[0][k] = -e.Mcon[k][0];
  }
#pragma unroll
  for (int j = 1; j < 4; j++)
#pragma unroll
    for (int k = 1; k < 4; k++) e.Mcon[j][k] = (pr[B1 + j - 1] * q.ucon[k] - pr[B1 + k - 1] * q.ucon[j]) / q.ucon[0];
  T a01 = T(0.), a02 = T(0.), a03 = T(0.), a12 = T(0.), a23 = T(0.), a31 = T(0.);
#pragma unroll
  for (int j = 0; j < 4; j++)
#pragma unroll
    for (int k = 0; k < 4; k++) {
      T A = e.Mcon[j][k];
      a01 += (GCOV(m, 0, j)) * (GCOV(m, 1, k)) * A;
      a02 += (GCOV(m, 0, j)) * (GCOV(m, 2, k)) * A;
      a03 += (GCOV(m, 0, j)) * (GCOV(m, 3, k)) * A;
      a12 += (GCOV(m, 1, j)) * (GCOV(m, 2, k)) * A;
      a23 += (GCOV(m, 2, j)) * (GCOV(m, 3, k)) * A;
      a31 += (GCOV(m, 3, j)) * (GCOV(m, 1, k)) * A;
    }
  e.Mcov[0][0] = T(0.);
  e.Mcov[1][1] = T(0.);
  e.Mcov[2][2] = T(0.);
  e.Mcov[3][3] = T(0.);
  e.Mcov[0][1] = a01;
  e.Mcov[0][2] = a02;
  e.Mcov[0][3] = a03;
  e.Mcov[1][2] = a12;
  e.Mcov[2][3] = a23;
  e.Mcov[3][1] = a31;
  e.Mcov[1][0] = -a01;
  e.Mcov[2][0] = -a02;
  e.Mcov[3][0] = -a03;
  e.Mcov[2][1] = -a12;
  e.Mcov[3][2] = -a23;
  e.Mcov[1][3] = -a31;
  T Msq = T(0.);
#pragma unroll
  for (int j = 0; j < 4; j++)
#pragma unroll
    for (int k = 0; k < 4; k++) Msq += e.Mcov[j][k] * e.Mcon[j][k];
  e.Msq = Msq;
  e.plus1ud0 = compute_1plusud0(m, q);
}

// mhd_calc_norestmass (phys.c:442-506) + ffdestresstensor_dir
// (phys.ffde.c:1483-1515): one row T^dir_mu without rest mass
template <typename T>
__device__ __forceinline__ void mhd_row(const T *pr, int dir, T gam, const StateT<T> &q, const EMT<T> &e, T *mhd) {
  T rho = pr[RHO], u = pr[UU];
  T P = (gam - T(1.)) * u;
  T w = P + rho + u;
  T eta = w, ptot = P;
  mhd[0] = (P + u) * q.ucon[dir] * q.ucov[0] + rho * q.ucon[dir] * e.plus1ud0 + ptot * ((dir == 0) ? T(1.) : T(0.));
#pragma unroll
  for (int j = 1; j < 4; j++) mhd[j] = eta * q.ucon[dir] * q.ucov[j] + ptot * ((dir == j) ? T(1.) : T(0.));
  T TEM[4];
#pragma unroll
  for (int j = 0; j < 4; j++) {
    TEM[j] = T(0.);
#pragma unroll
    for (int i = 0; i < 4; i++) TEM[j] += e.Mcon[dir][i] * e.Mcov[j][i];
  }
  TEM[dir] -= T(0.25) * e.Msq;
#pragma unroll
  for (int j = 0; j < 4; j++) mhd[j] += TEM[j];
}

// primtoflux (phys.c:16-55), UEVOLVE, every EOM factor = gdet
template <typename T>
__device__ __forceinline__ void primtoflux(const T *pr, const StateT<T> &q, const EMT<T> &e, int dir,
                                           const MetricT<T> &m, T gam, T *flux) {
  T fin[NPR];
  fin[RHO] = pr[RHO] * q.ucon[dir];
  mhd_row(pr, dir, gam, q, e, &fin[UU]);
  if (dir > 0) {
    fin[B1] = (pr[B1] * q.ucon[dir] - pr[B1 + dir - 1] * q.ucon[1]) / q.ucon[0];
    fin[B2] = (pr[B2] * q.ucon[dir] - pr[B1 + dir - 1] * q.ucon[2]) / q.ucon[0];
    fin[B3] = (pr[B3] * q.ucon[dir] - pr[B1 + dir - 1] * q.ucon[3]) / q.ucon[0];
  } else {
    fin[B1] = pr[B1];
    fin[B2] = pr[B2];
    fin[B3] = pr[B3];
  }
#pragma unroll
  for (int pl = 0; pl < NPR; pl++) flux[pl] = fin[pl] * m.g;
}

// simplefast (vchar.c:213-312) with Acov = e_dir, Bcov = e_t
template <typename T>
__device__ __forceinline__ int simplefast(int dir, const MetricT<T> &m, const StateT<T> &q, T cms2, T *vmin,
                                          T *vmax) {
  T Acov[4] = {T(0.), T(0.), T(0.), T(0.)}, Bcov[4] = {T(0.), T(0.), T(0.), T(0.)}, Acon[4], Bcon[4];
  Acov[dir] = T(1.);
  raise_vec(Acov, m, Acon);
  Bcov[0] = T(1.);
  raise_vec(Bcov, m, Bcon);
  T Asq = dot4(Acon, Acov);
  T Bsq = dot4(Bcon, Bcov);
  T Au = dot4(Acov, q.ucon);
  T Bu = dot4(Bcov, q.ucon);
  T AB = dot4(Acon, Bcov);
  T Au2 = Au * Au;
  T Bu2 = Bu * Bu;
  T AuBu = Au * Bu;
  T A = Bu2 * (T(1.0) - cms2) - Bsq * cms2;
  T B = T(2.) * (AuBu * (T(1.0) - cms2) - AB * cms2);
  T discr = T(4.0) * cms2 *
            ((AB * AB - Asq * Bsq) * cms2 + (T(2.0) * AB * Au * Bu - Asq * Bu2 - Bsq * Au2) * (cms2 - T(1.0)));
  if ((discr < T(0.0)) && (discr > -Tol<T>::discr)) discr = T(0.0);
  else if (discr < T(0.0)) return ERR_VCHAR_DISCR;
  discr = sqrt(discr);
  T vm = -(-B + discr) / (T(2.) * A);
  T vp = -(-B - discr) / (T(2.) * A);
  if ((!isfinite(vm)) || (!isfinite(vp))) return ERR_NONFINITE_SPEED;
  if (vp < vm) {
    *vmax = vm;
    *vmin = vp;
  } else {
    *vmax = vp;
    *vmin = vm;
  }
  return 0;
}

// vchar (vchar.c:37-171)
template <typename T>
__device__ __forceinline__ int vchar(const T *pr, const StateT<T> &q, int dir, const MetricT<T> &m, T gam, T *vmax,
                                     T *vmin) {
  T bsq = dot4(q.bcon, q.bcov);
  T rho = pr[RHO], u = pr[UU], cs2, va2, EF, WW, P;
  if (u < T(0)) u = T(0);
  if (rho < T(0)) rho = T(0);
  P = (gam - T(1.)) * u;
  WW = rho + u + P;
  if (WW > T(0.0)) {
    T pressure = (gam - T(1.)) * u;
    T h = rho + u + pressure;
    cs2 = gam * pressure / h;
  } else WW = cs2 = T(0.0);
  if (cs2 >= T(1.0)) cs2 = T(1.0) - Tol<T>::cs2cap;
  else if (cs2 <= T(0.0)) cs2 = T(0.0);
  EF = bsq + WW;
  if (EF > T(0.0)) va2 = bsq / EF;
  else EF = va2 = T(0.0);
  T cms2 = cs2 + va2 - cs2 * va2;
  if (cms2 < T(0.0)) {
    if (cms2 / (cs2 + va2) > -Tol<T>::numeps * T(100.0)) cms2 = T(0.0);
    else return ERR_COEFF_NEG;
  }
  if (cms2 > T(1.)) {
    if (cms2 < T(1.0) + Tol<T>::numeps * T(100.0)) cms2 = T(1.0);
    else if (rho < T(0.0)) cms2 = T(1.0);
    else return ERR_COEFF_SUP;
  }
  return simplefast(dir, m, q, cms2, vmin, vmax);
}

// vchar with FP32 arithmetic on an FP64 state (the mixed-precision Riemann
// kernel of WENO5: fluxes and states stay FP64, the wave speeds, which only
// scale the HLL dissipation and the CFL limit, are formed in FP32).  Reads
// what vchar reads: rho, u, b^mu, b_mu, u^mu and g^{mu nu}.
template <typename T>
__device__ __forceinline__ int vchar_f32(const T *pr, const StateT<T> &q, int dir, const MetricT<T> &m, T gam,
                                         T *vmax, T *vmin) {
  float prf[NPR];
  prf[RHO] = (float)pr[RHO];
  prf[UU] = (float)pr[UU];
  StateT<float> qf;
  MetricT<float> mf;
#pragma unroll
  for (int a = 0; a < 4; a++) {
    qf.ucon[a] = (float)q.ucon[a];
    qf.bcon[a] = (float)q.bcon[a];
    qf.bcov[a] = (float)q.bcov[a];
  }
#pragma unroll
  for (int a = 0; a < 16; a++) mf.gcon[a] = (float)m.gcon[a];
  float vmx = 0.f, vmn = 0.f;
  const int r = vchar<float>(prf, qf, dir, mf, (float)gam, &vmx, &vmn);
  *vmax = (T)vmx;
  *vmin = (T)vmn;
  return r;
}

template <typename T>
__device__ __forceinline__ T max_ref(T a, T b) { return (a > b) ? a : b; }  // phys.c:1797
template <typename T>
__device__ __forceinline__ T min_ref(T a, T b) { return (a > b) ? b : a; }  // phys.c:1804
__device__ __forceinline__ double min_macro(double a, double b) { return ((a) < (b)) ? (a) : (b); }  // global.h:751

// limit_gamma (fixup.c:1859-1905); returns -1 if it changed pr
__device__ __forceinline__ int limit_gamma(double gammamax, double *pr, const Metric &m, int *err) {
  if (gammamax <= 1.0) return 0;
  double gamma;
  if (gamma_calc(pr, m, &gamma)) {
    *err |= ERR_UTCALC_DISCR;
    return 1;
  }
  if ((gamma > gammamax && (gamma != 1.0))) {
    double pref = (gammamax * gammamax - 1.) / (gamma * gamma - 1.);
    if (pref < 0.0) {
      *err |= ERR_PREF_NEG;
      return 1;
    }
    double f = sqrt(pref);
    pr[U1] *= f;
    pr[U2] *= f;
    pr[U3] *= f;
    return -1;
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Con-to-prim: Utoprimgen (utoprimgen.c:23) -> Utoprim_2d_final
// (utoprim_2d_final.c:34-453) with the 2D Newton on (W, v^2)
// (general_newton_raphson :736-1119, func_vsq2 :1189-1278, USE_LINE_SEARCH=-2)
// ---------------------------------------------------------------------------
struct U2P {
  double Bsq, QdotBsq, Qtsq, Qdotn, D, wglobal, gam, gammasq_too_big, vsq_too_big;
};

__device__ __forceinline__ double vsq_calc(const U2P &c, double W) {
  double Wsq = W * W;
  double Xsq = (c.Bsq + W) * (c.Bsq + W);
  return ((Wsq * c.Qtsq + c.QdotBsq * (c.Bsq + 2. * W)) / (Wsq * Xsq));
}

// func_vsq2 with the EOS pieces of utoprim_jon_eos.c (pressure_W_vsq :83,
// dpdW_calc_vsq :214, dpdvsq_calc :316) for the ideal gas
__device__ __forceinline__ void func_vsq2(const U2P &c, double W, double vsq, double *dx0, double *dx1, double *f,
                                          double *df) {
  double Wsq = W * W;
  double D = c.D;
  double gamma = 1.0 / sqrt(1.0 - vsq);
  double gammasq = gamma * gamma;
  double Wp = W - D;
  double wmrho0 = (Wp / gammasq - D * vsq / (1.0 + gamma));
  double igr = (c.gam - 1.0) / c.gam;
  double p_tmp = igr * wmrho0;
  double dPdW = 0.0 * 0.0 + (1.0 - vsq) * igr;
  double dwmrho0dvsq = (D * (gamma * 0.5 - 1.0) - Wp);
  double drho0dvsq = -D * gamma * 0.5;
  double dPdvsq = drho0dvsq * 0.0 + dwmrho0dvsq * igr;
  double Bsq = c.Bsq, QdotBsq = c.QdotBsq, Qtsq = c.Qtsq, Qdotn = c.Qdotn;
  double t2 = -0.5 * Bsq + dPdvsq;
  double t3 = Bsq + W;
  double t4 = t3 * t3;
  double t9 = 1 / Wsq;
  double t11 = Qtsq - vsq * t4 + QdotBsq * (Bsq + 2.0 * W) * t9;
  double t16 = QdotBsq * t9;
  double t18 = -Qdotn - 0.5 * Bsq * (1.0 + vsq) + 0.5 * t16 - W + p_tmp;
  double t21 = 1 / t3;
  double t23 = 1 / W;
  double t24 = t16 * t23;
  double t25 = -1.0 + dPdW - t24;
  double t35 = t25 * t3 + (Bsq - 2.0 * dPdvsq) * (QdotBsq + vsq * Wsq * W) * t9 * t23;
  double t36 = 1 / t35;
  *dx0 = -(t2 * t11 + t4 * t18) * t21 * t36;
  double t40 = (vsq + t24) * t3;
  *dx1 = -(-t25 * t11 - 2.0 * t40 * t18) * t21 * t36;
  *df = -t11 * t11 - t18 * t18;
  *f = -0.5 * (*df);
}

// Inversion of the evolved conserved vector U (includes gdet) with guess in
// prim; returns the pflag code and the Newton iteration count.
__device__ __forceinline__ int utoprimgen(const double *U, const Metric &m, double gam, double gammafail, double *prim,
                                          int *iters) {
  constexpr int MAX_NEWT_ITER = 200;
  constexpr double NEWT_TOL = 1E3 * NUMEPSILON;
  constexpr double MIN_NEWT_TOL = 1E-6;
  constexpr double MAXNEGUTSQ = 1E-10;
  const double MAXNEGVSQ = (1.0 - 1.0 / (MAXNEGUTSQ + 1.0));
  U2P c;
  c.gam = gam;
  c.gammasq_too_big = gammafail * gammafail;
  c.vsq_too_big = (c.gammasq_too_big - 1.0) / (c.gammasq_too_big);
  double Ugf[NPR], Ut[NPR];
  // UtoU(UEVOLVE->UNOTHING) and rest-mass convention (utoprimgen.c:55,76-85)
#pragma unroll
  for (int pl = 0; pl < NPR; pl++) Ugf[pl] = U[pl] / m.g;
  Ugf[UU] -= Ugf[RHO];
  // Utoprim_2d_final (utoprim_2d_final.c:34-117)
  prim[B1] = Ugf[B1];
  prim[B2] = Ugf[B2];
  prim[B3] = Ugf[B3];
  double alpha = 1.0 / sqrt(-GCON(m, 0, 0));
#pragma unroll
  for (int i = 0; i < NPR; i++) Ut[i] = alpha * Ugf[i];
  // Utoprim_new_body (:152-453)
  double Bcon[4], Bcov[4], Qcov[4], Qcon[4], ncov[4], ncon[4];
  Bcon[0] = 0.;
  Bcon[1] = Ut[B1];
  Bcon[2] = Ut[B2];
  Bcon[3] = Ut[B3];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    double s = 0.;
#pragma unroll
    for (int j = 0; j < 4; j++) s += GCOV(m, i, j) * Bcon[j];
    Bcov[i] = s;
  }
#pragma unroll
  for (int i = 0; i < 4; i++) Qcov[i] = Ut[UU + i];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    double s = 0.;
#pragma unroll
    for (int j = 0; j < 4; j++) s += GCON(m, i, j) * Qcov[j];
    Qcon[i] = s;
  }
  double Bsq = 0.;
#pragma unroll
  for (int i = 1; i < 4; i++) Bsq += Bcon[i] * Bcov[i];
  c.Bsq = Bsq;
  double QdotB = 0.;
#pragma unroll
  for (int i = 0; i < 4; i++) QdotB += Qcov[i] * Bcon[i];
  c.QdotBsq = QdotB * QdotB;
  double lapse = sqrt(-1. / GCON(m, 0, 0));
  ncov[0] = -lapse;
  ncov[1] = 0.;
  ncov[2] = 0.;
  ncov[3] = 0.;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    double s = 0.;
#pragma unroll
    for (int j = 0; j < 4; j++) s += GCON(m, i, j) * ncov[j];
    ncon[i] = s;
  }
  c.Qdotn = Qcon[0] * ncov[0];
  double Qsq = 0.;
#pragma unroll
  for (int i = 0; i < 4; i++) Qsq += Qcov[i] * Qcon[i];
  c.Qtsq = Qsq + c.Qdotn * c.Qdotn;
  c.D = Ut[RHO];
  double utsq = 0.;
#pragma unroll
  for (int i = 1; i < 4; i++)
#pragma unroll
    for (int j = 1; j < 4; j++) utsq += GCOV(m, i, j) * prim[U1 + i - 1] * prim[U1 + j - 1];
  *iters = 0;
  if ((utsq < 0.) && (fabs(utsq) < MAXNEGUTSQ)) utsq = 0.0;
  if (utsq < 0. || utsq > ((gammafail - 1.0) * (gammafail - 1.0))) return UTOPRIMFAILCONVGUESSUTSQ;
  double gammasq = 1. + utsq;
  double gamma = sqrt(gammasq);
  double rho0 = c.D / gamma;
  double u = prim[UU];
  double p = (gam - 1.) * u;
  double w = rho0 + u + p;
  double W_last = w * gammasq;
  int i_increase = 0;
  while (((W_last * W_last * W_last * (W_last + 2. * c.Bsq) - c.QdotBsq * (2. * W_last + c.Bsq)) <=
          W_last * W_last * (c.Qtsq - c.Bsq * c.Bsq)) &&
         (i_increase < 10)) {
    W_last *= 10.;
    i_increase++;
  }
  c.wglobal = w;
  // find_root_2D_gen (:573-644)
  double x0 = fabs(W_last);
  double vs0 = vsq_calc(c, W_last);
  double x1 = (vs0 > 1.) ? c.vsq_too_big : vs0;
  // general_newton_raphson (:736-1119) with plain Newton steps
  double f = 1., df = 1., errx = 1.;
  int n_iter = 0;
  bool keep = true;
  while (keep) {
    double dx0, dx1;
    func_vsq2(c, x0, x1, &dx0, &dx1, &f, &df);
    double x0old = x0;
    x0 += dx0;
    x1 += dx1;
    errx = (x0 == 0.) ? fabs(dx0) : fabs(dx0 / x0);
    // validate_x (:708-728)
    x0 = fabs(x0);
    x0 = (x0 / c.wglobal > c.gammasq_too_big) ? x0old : x0;
    x1 = (x1 > 1.) ? c.vsq_too_big : x1;
    if ((fabs(errx) <= NEWT_TOL) || (n_iter >= (MAX_NEWT_ITER - 1))) keep = false;
    n_iter++;
  }
  *iters = n_iter;
  int retval = 0;
  if ((isfinite(f) == 0) || (isfinite(df) == 0) || (isfinite(x0) == 0) || (isfinite(x1) == 0)) retval = 1;
  else if (fabs(errx) > MIN_NEWT_TOL) retval = 1;
  double W = x0;
  if ((retval != 0) || (W == 1.e30)) return retval * 100 + 1;
  double Wtest = W / c.wglobal;
  if (Wtest <= 0. || Wtest > c.gammasq_too_big) return UTOPRIMFAILCONVW;
  double vsq = vsq_calc(c, W);
  if ((vsq < 0.) && (fabs(vsq) < MAXNEGVSQ)) vsq = 0.0;
  if ((vsq > c.vsq_too_big) || (vsq < 0.0)) return UTOPRIMFAILCONVUTSQ;
  double gtmp = sqrt(1. - vsq);
  gamma = 1. / gtmp;
  rho0 = c.D * gtmp;
  w = W * (1. - vsq);
  p = ((gam - 1.0) / gam) * (w - rho0);
  u = w - (rho0 + p);
  int lpflag = UTOPRIMNOFAIL;
  if ((rho0 <= 0.) || (u < 0.)) {
    if ((rho0 <= 0.) && (u >= 0.)) lpflag = UTOPRIMFAILRHONEG;
    if ((rho0 > 0.) && (u < 0.)) lpflag = UTOPRIMFAILUNEG;
    if ((rho0 <= 0.) && (u < 0.)) lpflag = UTOPRIMFAILRHOUNEG;
  }
  prim[RHO] = rho0;
  prim[UU] = u;
#pragma unroll
  for (int i = 1; i < 4; i++) {
    double Qtcon = Qcon[i] + ncon[i] * c.Qdotn;
    prim[U1 + i - 1] = gamma / (W + c.Bsq) * (Qtcon + QdotB * Bcon[i] / W);
  }
  return lpflag;
}

// ---------------------------------------------------------------------------
// Con-to-prim: Utoprimgen -> Utoprim_jon_nonrelcompat_inputnorestmass
// (utoprim_jon.c:65-205, UTOPRIMVERSION=UTOPRIMJONNONRELCOMPAT, the FM torus
// default set in init.fishmon.c:46): a 1-D Newton solve of E'(W') = 0 in
// W' = W - D (WHICHHOTINVERTER 3, PRIMFROMVSQ 0, JONGENNEWTSTUFF 1,
// USE_LINE_SEARCH -2), u2p_defs.h with PRECISEINVERSION 1, ideal gas.
// ---------------------------------------------------------------------------
struct JonU2P {
  double Bsq, QdotB, QdotBsq, Qtsq, Qdotnp, D, wglobal, igammar, gammasq_too_big;
};

// utsq_calc (utoprim_jon.c:1294-1315)
__device__ __forceinline__ double jon_utsq(const JonU2P &c, double W) {
  double SoW = c.QdotB / W;
  double top = c.Qtsq + (c.Bsq + 2.0 * W) * SoW * SoW;
  double bottom = (c.Bsq * c.Bsq - c.Qtsq) + 2.0 * c.Bsq * W + W * W - SoW * SoW * (c.Bsq + 2.0 * W);
  return top / bottom;
}

// coldgrhd (utoprim_jon.c:1402-1425)
__device__ __forceinline__ int jon_coldgrhd(double Qtsq, double D, double *Wp) {
  double det = D * D + Qtsq;
  if (det < 0.0) return 1;
  if (D > 0.0) *Wp = Qtsq / (D + sqrt(det));
  else *Wp = Qtsq / (D - sqrt(det));
  return 0;
}

__device__ __forceinline__ double jon_max(double a, double b) { return ((a) > (b)) ? (a) : (b); }  // global.h:750
__device__ __forceinline__ double jon_sign(double a) {  // phys.c:1778
  return (a > 0.0) ? 1.0 : ((a < 0.0) ? -1.0 : 0.0);
}

// func_Eprime (utoprim_jon.c:2258-2281): the Newton step -E'/(dE'/dW') from
// Eprime_Wp (:1529-1554) and dEprimedWp (:1558-1587) with the ideal-gas EOS
// pieces of utoprim_jon_eos.c (pressure_Wp_utsq :134, dpdWp_calc_utsq :262,
// dpdvsq_calc2_Wp :391, wmrho0_compute_utsq :474) and eos.c:178-194.  Both
// evaluate utsq_calc at the same W'; it is computed once here.
__device__ __forceinline__ void jon_func(const JonU2P &c, double Wp, double *resid, double *dx) {
  const double D = c.D;
  const double W = Wp + D;
  const double X = c.Bsq + W + 1.e-50;  // SMALL (global.h:1041)
  double utsq = jon_utsq(c, W);
  if (utsq < -0.1) utsq = 0.0;
  const double gammasq = 1.0 + utsq;
  const double gamma = sqrt(gammasq);
  const double wmrho0 = (Wp - D * utsq / (1.0 + gamma)) / gammasq;
  const double p_tmp = c.igammar * wmrho0;
  const double X2 = X * X;
  const double r = c.Qdotnp + Wp - p_tmp + 0.5 * c.Bsq + 0.5 * (c.Bsq * c.Qtsq - c.QdotBsq) / X2;
  // dvsq_dW (:1378-1398)
  const double Xv = c.Bsq + W;
  const double Wsq = W * W;
  const double W3 = Wsq * W;
  const double X3v = Xv * Xv * Xv;
  const double dvsq = -2. * (c.Qtsq / X3v + c.QdotBsq * (3.0 * W * Xv + c.Bsq * c.Bsq) / (W3 * X3v));
  const double dp1 = 0.0 * 0.0 + (1.0 / gammasq) * c.igammar;
  const double dp2 = (-D * gamma * 0.5) * 0.0 + (D * (gamma * 0.5 - 1.0) - Wp) * c.igammar;
  const double dpdWp = dp1 + dp2 * dvsq;
  const double X3 = X * X * X;
  const double drdW = (1.0 - dpdWp) - (c.Bsq * c.Qtsq - c.QdotBsq) / X3;
  *resid = r;
  *dx = -r / drdW;
}

// Inversion of the evolved conserved vector U (includes gdet; U[UU] without
// rest mass, as REMOVERESTMASSFROMUU 2 evolves it) with the guess in prim;
// returns the pflag code and the Newton iteration count.  Flags follow the
// reference: the non-B primitives are replaced whenever the Newton solve
// returned 0 (UTOPRIMFAILCONVW, negative rho/u and a root equal to FAIL_VAL
// come with new primitives, NaN components keep the guess with flag 8),
// UTOPRIMFAILCONVRET keeps the guess.  A guess with u~^2 outside
// [-MAXNEGUTSQ, UTSQ_TOO_BIG] or with no 4-velocity keeps the guess with
// UTOPRIMFAILCONVGUESSUTSQ (the reference proceeds there with an unset W').
__device__ __forceinline__ int utoprimgen_jon(const double *U, const Metric &m, double gam, double gammafail,
                                              double *prim, int *iters) {
  constexpr int MAX_NEWT_ITER = 200;
  constexpr double NEWT_TOL = 1E3 * NUMEPSILON;
  constexpr double NEWT_TOL_ULTRAREL = NUMEPSILON;
  constexpr double MIN_NEWT_TOL = 1E-6;
  constexpr int EXTRA_NEWT_ITER = 0;
  constexpr int EXTRA_NEWT_ITER_ULTRAREL = 2;
  constexpr double GAMMASQCHECKRESID = 1e2;
  constexpr double MAXNEGUTSQ = 1E-10;
  JonU2P c;
  c.igammar = (gam - 1.0) / gam;
  c.gammasq_too_big = gammafail * gammafail;
  double Ut[NPR], pt[NPR];
  // UtoU(UEVOLVE->UNOTHING); U[UU] stays without rest mass (utoprimgen.c:76-85)
  double Ugf[NPR];
#pragma unroll
  for (int pl = 0; pl < NPR; pl++) Ugf[pl] = U[pl] / m.g;
  prim[B1] = Ugf[B1];
  prim[B2] = Ugf[B2];
  prim[B3] = Ugf[B3];
  const double alpha = 1.0 / sqrt(-GCON(m, 0, 0));
#pragma unroll
  for (int i = 0; i < NPR; i++) Ut[i] = alpha * Ugf[i];
#pragma unroll
  for (int i = 0; i < B1; i++) pt[i] = prim[i];
#pragma unroll
  for (int i = B1; i <= B3; i++) pt[i] = Ut[i];
  // compute_setup_quantities (:494-636)
  c.D = Ut[RHO];
  double Bcon[4], Bcov[4], ncov[4], ncon[4], Qconp[4], Qcov[4], Qtcon[4];
  Bcon[0] = 0.;
  Bcon[1] = Ut[B1];
  Bcon[2] = Ut[B2];
  Bcon[3] = Ut[B3];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    double s = 0.;
#pragma unroll
    for (int j = 0; j < 4; j++) s += GCOV(m, i, j) * Bcon[j];
    Bcov[i] = s;
  }
  double Bsq = 0.;
#pragma unroll
  for (int i = 1; i < 4; i++) Bsq += Bcon[i] * Bcov[i];
  c.Bsq = Bsq;
  const double lapse = sqrt(-1. / GCON(m, 0, 0));
  ncov[0] = -lapse;
  ncov[1] = 0.;
  ncov[2] = 0.;
  ncov[3] = 0.;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    double s = 0.;
#pragma unroll
    for (int j = 0; j < 4; j++) s += GCON(m, i, j) * ncov[j];
    ncon[i] = s;
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    double s = 0.;
#pragma unroll
    for (int j = 0; j < 4; j++) s += GCON(m, i, j) * Ut[UU + j];
    Qconp[i] = s;
  }
  Qtcon[0] = 0.0;
#pragma unroll
  for (int j = 1; j < 4; j++) {
    double s = 0.0;
#pragma unroll
    for (int i = 1; i < 4; i++) s += Ut[UU + i] * (GCON(m, i, j) + ncon[i] * ncon[j]);
    Qtcon[j] = s;
  }
  double Qtsq = 0.;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    double s = 0.;
#pragma unroll
    for (int j = 0; j < 4; j++) s += GCOV(m, i, j) * Qtcon[j];
    Qtsq += s * Qtcon[i];
  }
  c.Qtsq = Qtsq;
#pragma unroll
  for (int i = 0; i < 4; i++) Qcov[i] = (i == 0) ? Ut[UU] - c.D : Ut[UU + i];
  double QdotB = 0.;
#pragma unroll
  for (int i = 1; i < 4; i++) QdotB += Qcov[i] * Bcon[i];
  c.QdotB = QdotB;
  c.QdotBsq = QdotB * QdotB;
  c.Qdotnp = Qconp[0] * ncov[0] + c.D * (1.0 - 1.0 / fabs(ncov[TT]));
  // set_guess_Wp (:640-745)
  *iters = 0;
  double utsq = 0.;
#pragma unroll
  for (int i = 1; i < 4; i++)
#pragma unroll
    for (int j = 1; j < 4; j++) utsq += GCOV(m, i, j) * pt[U1 + i - 1] * pt[U1 + j - 1];
  if ((utsq < 0.) && (fabs(utsq) < MAXNEGUTSQ)) utsq = 0.0;
  if (utsq < 0. || utsq > ((gammafail - 1.0) * (gammafail - 1.0))) return UTOPRIMFAILCONVGUESSUTSQ;
  double gammasq = 1. + utsq;
  double gamma = sqrt(gammasq);
  double rho0 = c.D / gamma;
  double u = pt[UU];
  double p = (gam - 1.) * u;
  double w = rho0 + u + p;
  double bsq;
  {
    State q;
    if (get_state(pt, m, q)) return UTOPRIMFAILCONVGUESSUTSQ;
    bsq = dot4(q.bcon, q.bcov);
  }
  double Wp_last = c.D * utsq / (1.0 + gamma) + (u + p) * gammasq;
  double W_last = Wp_last + c.D;
  if ((w + bsq) * gammasq >= GAMMASQCHECKRESID) {
    double Wpcoldhd;
    if (jon_coldgrhd(c.Qtsq, c.D, &Wpcoldhd)) Wpcoldhd = Wp_last;
    c.wglobal = 1E-5 * jon_max(jon_max(Wpcoldhd, Wp_last), w + bsq);
    Wp_last = jon_max(jon_max(2.0 * Wpcoldhd, Wp_last), w + bsq);
  } else {
    c.wglobal = w + bsq;
  }
  // verify_Wlast (:752-812)
  if (W_last < -c.D || Wp_last < 0) {
    W_last = -c.D;
    Wp_last = 0;
  }
  for (int i_increase = 0; i_increase < 10; i_increase++) {
    if (!(W_last * W_last * W_last * (W_last + 2. * c.Bsq) - c.QdotBsq * (2. * W_last + c.Bsq) <=
          W_last * W_last * (c.Qtsq - c.Bsq * c.Bsq)))
      break;
    Wp_last *= 10.;
    W_last = Wp_last + c.D;
  }
  // general_newton_raphson (:2896-3424), n = 1, no line search
  double x = Wp_last, x_old = x, x_older = x, dx = 0., dx_old = 1E30 * x, resid = 0.;
  double errx = 1., xold0 = 0., residold = 0., damp = 1.0;
  int n_iter = 0, doing_extra = 0, i_extra = 0;
  const bool ultrarel_w = fabs(c.wglobal) > GAMMASQCHECKRESID;
  bool keep = true;
  while (keep) {
    jon_func(c, x, &resid, &dx);
    x_older = x_old;
    x_old = x;
    if (n_iter == 0) {
      xold0 = x;
      residold = resid;
    } else if (jon_sign(residold) != jon_sign(resid)) {
      if (fabs(xold0) > GAMMASQCHECKRESID || fabs(x_old) > GAMMASQCHECKRESID) {
        damp = 0.5 * damp;
        x = x_older;
        dx = dx_old;
      }
    }
    x += damp * dx;
    errx = (c.wglobal == 0.) ? fabs(dx_old) : fabs(dx_old / jon_max(fabs(c.wglobal), fabs(x)));
    // validate_Wp (:1726-1758)
    if (x < -c.D && c.D > 0.0) {
      double Wpc;
      if (!jon_coldgrhd(c.Qtsq, c.D, &Wpc)) x = Wpc * 10.0;
    }
    x = (fabs(x / c.wglobal) > c.gammasq_too_big) ? 0.5 * (x_old + x) : x;
    dx_old = dx;
    // newt_errorcheck / newt_extracheck (:3430-3458)
    const bool ur = ultrarel_w || (fabs(x) > GAMMASQCHECKRESID);
    const bool conv = ur ? (fabs(errx) <= NEWT_TOL_ULTRAREL) : (fabs(errx) <= NEWT_TOL);
    const int extra = ur ? EXTRA_NEWT_ITER_ULTRAREL : EXTRA_NEWT_ITER;
    if (conv && (doing_extra == 0) && (extra > 0)) doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if ((conv && (doing_extra == 0)) || (i_extra > extra) || (n_iter >= (MAX_NEWT_ITER - 1))) keep = false;
    n_iter++;
  }
  *iters = n_iter;
  // f = resid^2/2 and df = -2 f are finite exactly when resid^2 is
  int retval;
  const double f = 0.5 * resid * resid;
  if ((isfinite(f) == 0) || (isfinite(-2. * f) == 0) || (isfinite(x) == 0)) {
    retval = 1;
  } else {
    x = x_old;
    const bool ur = ultrarel_w || (fabs(x) > GAMMASQCHECKRESID);
    const bool conv = ur ? (fabs(errx) <= NEWT_TOL_ULTRAREL) : (fabs(errx) <= NEWT_TOL);
    retval = (conv || fabs(errx) <= MIN_NEWT_TOL) ? 0 : 1;
  }
  // check_Wp (:819-903)
  const double Wp = x;
  int lpflag = UTOPRIMNOFAIL;
  if ((retval != 0) || (Wp == 1.e30)) {
    lpflag = retval * 100 + 1;
    if (retval != 0) return lpflag;
  } else {
    const double Wtest = Wp / c.wglobal;
    if (!(Wtest <= 0.0) && (Wtest > c.gammasq_too_big)) lpflag = UTOPRIMFAILCONVW;
  }
  // Wp2prim (:949-1165), PRIMFROMVSQ 0
  double pr0[NPR];
#pragma unroll
  for (int i = 0; i < NPR; i++) pr0[i] = pt[i];
  const double W = Wp + c.D;
  utsq = jon_utsq(c, W);
  gammasq = 1.0 + utsq;
  gamma = sqrt(gammasq);
  const double wmrho0 = (Wp - c.D * utsq / (1.0 + gamma)) / gammasq;
  rho0 = c.D / gamma;
  p = c.igammar * wmrho0;
  u = wmrho0 - p;
  if ((rho0 <= 0.) || (u < 0.)) {
    if ((rho0 <= 0.) && (u >= 0.)) lpflag = UTOPRIMFAILRHONEG;
    if ((rho0 > 0.) && (u < 0.)) lpflag = UTOPRIMFAILUNEG;
    if ((rho0 <= 0.) && (u < 0.)) lpflag = UTOPRIMFAILRHOUNEG;
  }
  pt[RHO] = rho0;
  pt[UU] = u;
#pragma unroll
  for (int i = 1; i < 4; i++) pt[U1 + i - 1] = gamma / (W + c.Bsq) * (Qtcon[i] + QdotB * Bcon[i] / W);
#pragma unroll
  for (int i = 0; i < NPR; i++)
    if (!isfinite(pt[i])) {
      pt[i] = pr0[i];
      lpflag = 8;  // UTOPRIMFAILNANRESULT
    }
#pragma unroll
  for (int i = 0; i < B1; i++) prim[i] = pt[i];
  return lpflag;
}

// Utoprimgen dispatch on UTOPRIMVERSION (0/6: UTOPRIM2DFINAL, 8: Jon)
template <int UV>
__device__ __forceinline__ int utoprimgen_v(const double *U, const Metric &m, double gam, double gammafail,
                                            double *prim, int *iters) {
  if (UV == 8) return utoprimgen_jon(U, m, gam, gammafail, prim, iters);
  return utoprimgen(U, m, gam, gammafail, prim, iters);
}

}  // namespace hg
