// weno5.cuh -- device side of the reference's WENO5 centre-to-edge line
// reconstruction (lim = WENO5): slope_lim_linetype_c2e (interpline.c:517-678)
// -> compute_smonotonicity_line (smonointerp.c:15-175) -> eno_line_reconstruct
// (reconstructeno.c:261-563) for the torus build options: PRIMTOINTERP,
// COMPUTEDRHODP=1, SMONO with smooth transition, "AND" stencil reduction,
// post/pre-shock dP/P reduction, smooth adjustment of the unoptimised
// weights, no stencil shift, default (non-PPM) reduction.
//
// The reference reconstructs whole lines; every quantity of one output cell
// c depends only on the line from c-5 to c+5 (for the reference's MAXBND=11
// lines no stencil reaches a line end, so its boundary-truncation branches
// are dead).  These are the per-cell pieces; weno5_kernel (common.cuh)
// stages them over tiles of a line in shared memory:
//   per cell, per primitive: SMONO cusp test and indicator, and the
//          unoptimised order-3 weights (compute_cf_stencil_weights +
//          mono_adjust_unoptimized_weights)
//   per output cell: weight ratios of c-1..c+1 (compute_weights_ratios),
//          dP/P reduction (apply_additional_reduction_to_weights), optimised
//          weights, order-2 weights when reduced (choose_weno_order) and the
//          face values (eno_cvt + the SMONO blend).
// Every expression keeps the reference's operation order; the library is
// compiled with -fmad=false, so results are bit-identical to the reference.
#pragma once

namespace hg {
namespace w5 {

// Constants of the scheme per arithmetic type.  FP64: the reference's own.
// FP32 (mixed-precision path): the same WENO and SMONO epsilons -- the FP32
// path reconstructs on differences from the cell's own value (exact zeros
// where the line is flat, as in FP64) and forms the nonlinear weights from
// ratios to the smallest smoothness term (no 1/eps^2 overflow); BIG, SMALL
// and DBL_MIN become FP32-range values.  The FP32 path is not bit-compatible
// with the reference; its error against the FP64 path is measured and stated.
template <typename T> struct K;
template <> struct K<double> {
  static constexpr double eps = 1.e-26;       // WENO_EPSILON = REDUCEEPSILON (reconstructeno.h:195-200)
  static constexpr double smono = 1.e-13;     // SMONO_EPSILON = SQRT_WENO_EPSILON (reconstructeno.h:73,196)
  static constexpr double big = 1.e+50;       // BIG (global.h:1040)
  static constexpr double small = 1.e-50;     // SMALL (global.h:1041)
  static constexpr double tiny = 2.2250738585072014e-308;  // DBL_MIN
};
template <> struct K<float> {
  static constexpr float eps = 1.e-26f;
  static constexpr float smono = 1.e-13f;
  static constexpr float big = 1.e+30f;
  static constexpr float small = 1.e-30f;
  static constexpr float tiny = 1.17549435e-38f;  // FLT_MIN
};
constexpr double kMinRat = 1.3;      // MIN/MAX_TRANSITION_RATIO of the AND reduction (reconstructeno.h:175-176)
constexpr double kMaxRat = 1.6;
constexpr double kDpFrac = 0.5;      // REDUCE_DP_FRACTION (reconstructeno.h:96)
constexpr double kDblMin = K<double>::tiny;

template <typename T>
__device__ __forceinline__ T wmin(T a, T b) { return (a < b) ? a : b; }  // MIN global.h:751
template <typename T>
__device__ __forceinline__ T wmax(T a, T b) { return (a > b) ? a : b; }  // MAX global.h:750
template <typename T>
__device__ __forceinline__ T minmod(T a, T b) {                          // global.h:361-362
  return ((a) * (b) <= T(0)) ? T(0.0) : ((fabs(a) < fabs(b)) ? (a) : (b));
}
template <typename T>
__device__ __forceinline__ T sgn(T a) { return (a > T(0.0)) ? T(1.0) : ((a < T(0.0)) ? T(-1.0) : T(0.0)); }  // phys.c:1778

// get_sum_of_elements with SYMMETRIZE_WENO (reconstructeno.c:1920-1946)
template <typename T>
__device__ __forceinline__ T sum2(T a0, T a1) {
  T s = T(0.0);
  s += a0 + a1;
  s += a1 * T(0.0);
  return s;
}
template <typename T>
__device__ __forceinline__ T sum3(T a0, T a1, T a2) {
  T s = T(0.0);
  s += a0 + a2;
  s += a1 * T(1.0);
  return s;
}
template <typename T>
__device__ __forceinline__ T sum5(const T *a) {
  T s = T(0.0);
  s += a[0] + a[4];
  s += a[1] + a[3];
  s += a[2] * T(1.0);
  return s;
}

// x / 12 rounded to nearest without a division instruction.  q = RN(x r)
// with r = RN(1/12) is within 2 ulp of x/12, so e = x - 12 q is exact (a
// small multiple of 4 ulp(q)), and q + e r, rounded once by the FMA, differs
// from x/12 by at most 2^-52 ulp.  x/12 = (x/3)/4, and x/3 has a significand
// fraction of 0, 1/3 or 2/3 ulp, so x/12 lies at least 1/6 ulp from every
// rounding midpoint (or is a float): the result is RN(x/12), the bits of
// the IEEE division.  Magnitudes outside [2^-960, 2^1000] (where the steps
// could underflow or overflow), zeros, infinities and NaN take the division.
// The FP32 kernels of the mixed-precision path are built with approximate
// division and keep it.
template <typename T>
__device__ __forceinline__ T div12(T x) { return x / T(12.); }
template <>
__device__ __forceinline__ double div12<double>(double x) {
  const double ax = fabs(x);
  if (!(ax >= 0x1p-960 && ax <= 0x1p1000)) return x / 12.0;
  const double r = 1.0 / 12.0;
  const double q = x * r;
  const double e = fma(-q, 12.0, x);
  return fma(e, r, q);
}

// The routines below take the line at the cell twice: y (y[-2..2] valid)
// for every difference and linear combination, and yn for the magnitudes
// that scale the epsilons.  The FP64 path passes the primitives as both; the
// FP32 path passes y[k] = y_k - y_0 (formed in FP64) and the primitives as
// yn, and adds y_0 back to the face values in FP64.  The stencil formulas
// used on y are differences or rows summing to one, so both forms agree in
// exact arithmetic.

// check_for_cusp_new (smonointerp.c:439-476)
template <typename T>
__device__ __forceinline__ bool cusp(const T *y, const T *yn) {
  T df_m1 = y[-1] - y[-2], df0 = y[0] - y[-1], df1 = y[1] - y[0], df2 = y[2] - y[1];
  T ddf_m1 = df0 - df_m1, ddf0 = df1 - df0, ddf1 = df2 - df1;
  T norm = (fabs(yn[-2]) + fabs(yn[-1]) + fabs(yn[0]) + fabs(yn[1]) + fabs(yn[2]) + K<T>::small);
  norm = norm * K<T>::smono;
  T s0 = sgn(df0);
  T f1a = fabs(df0) - norm;
  T f1 = ddf_m1 * s0 - norm;
  T f2 = -ddf0 * s0 - norm;
  T f3 = -df2 * s0 - norm;
  T f3a = fabs(-df2 - df0) - T(0.25) * (fabs(df2) + fabs(df0));
  T f4 = -df1 * s0 - norm;
  T f4a = fabs(-df1 - df0) - T(0.25) * (fabs(df1) + fabs(df0));
  if (f1a > 0 && f1 > 0 && f2 > 0 && ((f3 > 0 && f3a > 0) || (f4 > 0 && f4a > 0))) return true;
  T s1 = sgn(df1);
  T f5a = fabs(df1) - norm;
  T f5 = -ddf1 * s1 - norm;
  T f6 = ddf0 * s1 - norm;
  T f7 = -df_m1 * s1 - norm;
  T f7a = fabs(-df_m1 - df1) - T(0.25) * (fabs(df_m1) + fabs(df1));
  T f8 = -df0 * s1 - norm;
  T f8a = fabs(-df0 - df1) - T(0.25) * (fabs(df0) + fabs(df1));
  if (f5a > 0 && f5 > 0 && f6 > 0 && ((f7 > 0 && f7a > 0) || (f8 > 0 && f8a > 0))) return true;
  return false;
}

// compute_mono_indicator_point_eno5 (smonointerp.c:296-425) + transition_function (:428-437)
template <typename T>
__device__ __forceinline__ T mono(const T *y, const T *yn) {
  // (division by 2 is the exact multiplication by 1/2)
  T l1 = div12((((-3 * y[-2] + y[2]) + (-10 * y[-1] - 6 * y[1])) + 18 * y[0]));
  T l2 = div12((((11 * y[-2] - y[2]) + (-20 * y[-1] + 4 * y[1])) + 6 * y[0]));
  T l3 = (((-3 * y[-2] - y[2]) + (10 * y[-1] + 6 * y[1])) - 12 * y[0]) * T(0.5);
  T r1 = div12((((-y[-2] + 3 * y[2]) + (6 * y[-1] + 10 * y[1])) - 18 * y[0]));
  T r2 = div12((((-y[-2] + 11 * y[2]) + (4 * y[-1] - 20 * y[1])) + 6 * y[0]));
  T r3 = (((y[-2] + 3 * y[2]) - (6 * y[-1] + 10 * y[1])) + 12 * y[0]) * T(0.5);
  l1 = minmod(l1, y[-1] - y[-2]);
  r1 = minmod(r1, y[2] - y[1]);
  T minabs = K<T>::big;
  minabs = wmin(minabs, fabs(minmod(l1, r1)));
  minabs = wmin(minabs, fabs(minmod(l2, r2)));
  minabs = wmin(minabs, fabs(minmod(l3, r3)));
  T norm = fabs(yn[0]) + ((fabs(yn[-1]) + fabs(yn[1])) + (fabs(yn[-2]) + fabs(yn[2])));
  T cut = norm * K<T>::smono + K<T>::tiny;
  T v = (minabs - T(0.0)) / (cut - T(0.0));
  return wmax(T(0.), wmin(T(1.), v));
}

// c2e_simple_eno(5, ...) (reconstructeno.c:826-901): central row of the
// 5-point centre-to-left (right=false) / centre-to-right matrix
template <typename T>
__device__ __forceinline__ T eno5(bool right, const T *y) {
  T d[5];
  if (!right) {
    d[0] = (-T(5.) / T(128.)) * y[-2];
    d[1] = (T(15.) / T(32.)) * y[-1];
    d[2] = (T(45.) / T(64.)) * y[0];
    d[3] = (-T(5.) / T(32.)) * y[1];
    d[4] = (T(3.) / T(128.)) * y[2];
  } else {
    d[0] = (T(3.) / T(128.)) * y[-2];
    d[1] = (-T(5.) / T(32.)) * y[-1];
    d[2] = (T(45.) / T(64.)) * y[0];
    d[3] = (T(15.) / T(32.)) * y[1];
    d[4] = (-T(5.) / T(128.)) * y[2];
  }
  return sum5(d);
}

// Unoptimised order-3 weights of compute_cf_stencil_weights
// (reconstructeno.c:1406-1614; desensitise :1687-1707, normalisation
// :1948-1960, compute_weights_from_smoothness_indicators :1878-1917) followed
// by mono_adjust_unoptimized_weights (:702-728).  m0 is monoindicator[0]
// (0 at a cusp); the cusp's lower_order_fraction=1 is kept by the caller.
template <typename T>
__device__ __forceinline__ void unopt3(T m0, const T *u, const T *un, T w[3]) {
  if (m0 == 1) {
    w[0] = w[1] = w[2] = T(1.0) / 3;
    return;
  }
  T fd0 = -(3 * u[0] + u[2]) + 4 * u[1];
  T fd1 = u[1] - u[-1];
  T fd2 = (3 * u[0] + u[-2]) - 4 * u[-1];
  T sd0 = (u[0] + u[2]) - 2 * u[1];
  T sd1 = (u[-1] + u[1]) - 2 * u[0];
  T sd2 = (u[0] + u[-2]) - 2 * u[-1];
  T si0 = T(13.) / T(12.) * sd0 * sd0 + T(1.) / T(4.) * fd0 * fd0;
  T si1 = T(13.) / T(12.) * sd1 * sd1 + T(1.) / T(4.) * fd1 * fd1;
  T si2 = T(13.) / T(12.) * sd2 * sd2 + T(1.) / T(4.) * fd2 * fd2;
  T u2[5] = {un[-2] * un[-2], un[-1] * un[-1], un[0] * un[0], un[1] * un[1], un[2] * un[2]};
  T e = sum5(u2) * K<T>::eps;
  si0 += e;
  si1 += e;
  si2 += e;
  T s = sum3(si0, si1, si2);
  si0 /= (s + K<T>::tiny);
  si1 /= (s + K<T>::tiny);
  si2 /= (s + K<T>::tiny);
  T t0 = si0 + K<T>::eps / T(1.), t1 = si1 + K<T>::eps / T(1.), t2 = si2 + K<T>::eps / T(1.);
  if constexpr (sizeof(T) == 4) {
    // 1/t^2 normalised, formed as (tmin/t)^2 (each in (0, 1])
    const T tm = wmin(t0, wmin(t1, t2));
    t0 = tm / t0;
    t1 = tm / t1;
    t2 = tm / t2;
    w[0] = t0 * t0;
    w[1] = t1 * t1;
    w[2] = t2 * t2;
  } else {
    t0 *= t0;
    t1 *= t1;
    t2 *= t2;
    w[0] = T(1.) / t0;
    w[1] = T(1.) / t1;
    w[2] = T(1.) / t2;
  }
  s = sum3(w[0], w[1], w[2]);
  w[0] /= (s + T(0.0));
  w[1] /= (s + T(0.0));
  w[2] /= (s + T(0.0));
  if (m0 > T(0.0) && m0 < T(1.0)) {
    T simple = T(1.0) / T(3.0);
    w[0] = (T(1.0) - m0) * w[0] + m0 * simple;
    w[1] = (T(1.0) - m0) * w[1] + m0 * simple;
    w[2] = (T(1.0) - m0) * w[2] + m0 * simple;
  }
}

// order-2 unoptimised weights (compute_cf_stencil_weights with order 2)
template <typename T>
__device__ __forceinline__ void unopt2(T m0, const T *u, const T *un, T w[2]) {
  if (m0 == 1) {
    w[0] = w[1] = T(1.0) / 2;
    return;
  }
  T fd0 = u[1] - u[0];
  T fd1 = u[0] - u[-1];
  T si0 = fd0 * fd0, si1 = fd1 * fd1;
  T e = sum3(un[-1] * un[-1], un[0] * un[0], un[1] * un[1]) * K<T>::eps;
  si0 += e;
  si1 += e;
  T s = sum2(si0, si1);
  si0 /= (s + K<T>::tiny);
  si1 /= (s + K<T>::tiny);
  T t0 = si0 + K<T>::eps / T(1.), t1 = si1 + K<T>::eps / T(1.);
  if constexpr (sizeof(T) == 4) {
    const T tm = wmin(t0, t1);
    t0 = tm / t0;
    t1 = tm / t1;
    w[0] = t0 * t0;
    w[1] = t1 * t1;
  } else {
    t0 *= t0;
    t1 *= t1;
    w[0] = T(1.) / t0;
    w[1] = T(1.) / t1;
  }
  s = sum2(w[0], w[1]);
  w[0] /= (s + T(0.0));
  w[1] /= (s + T(0.0));
}

// lower_order_fraction of compute_weights_ratios (reconstructeno.c:1962-2083),
// AND reduction, centre-to-edge ratios; wc = weights of the cell,
// wl0 = weights[0] of cell-2, wr2 = weights[2] of cell+2; lof0 = 1 at a cusp
template <typename T>
__device__ __forceinline__ T ratio_lof(const T wc[3], T wl0, T wr2, T lof0) {
  T minr = kMinRat, maxr = kMaxRat;
  T wrl = (wc[2] + K<T>::eps) / (wl0 + K<T>::eps);
  T wrr = (wc[0] + K<T>::eps) / (wr2 + K<T>::eps);
  T wr = wmin(wrl, wrr);
  T lof = (wr - minr) / (maxr - minr);
  lof = wmax(T(0.), wmin(lof, T(1.0)));
  return wmax(lof, lof0);
}

// eno_cvt (reconstructeno.c:730-823) with order-3 centre-to-face matrices
template <typename T>
__device__ __forceinline__ T cvt3(bool right, const T *wo, const T *u) {
  T su[3];
  // shift 0 uses u[0..2], shift 1 u[-1..1], shift 2 u[-2..0]
  if (!right) {
    su[0] = T(0.0);
    if (wo[0] != T(0.0)) su[0] = wo[0] * sum3((T(15.) / T(8.)) * u[0], (-T(5.) / T(4.)) * u[1], (T(3.) / T(8.)) * u[2]);
    su[1] = T(0.0);
    if (wo[1] != T(0.0)) su[1] = wo[1] * sum3((T(3.) / T(8.)) * u[-1], (T(3.) / T(4.)) * u[0], (-T(1.) / T(8.)) * u[1]);
    su[2] = T(0.0);
    if (wo[2] != T(0.0)) su[2] = wo[2] * sum3((-T(1.) / T(8.)) * u[-2], (T(3.) / T(4.)) * u[-1], (T(3.) / T(8.)) * u[0]);
  } else {
    su[0] = T(0.0);
    if (wo[0] != T(0.0)) su[0] = wo[0] * sum3((T(3.) / T(8.)) * u[0], (T(3.) / T(4.)) * u[1], (-T(1.) / T(8.)) * u[2]);
    su[1] = T(0.0);
    if (wo[1] != T(0.0)) su[1] = wo[1] * sum3((-T(1.) / T(8.)) * u[-1], (T(3.) / T(4.)) * u[0], (T(3.) / T(8.)) * u[1]);
    su[2] = T(0.0);
    if (wo[2] != T(0.0)) su[2] = wo[2] * sum3((T(3.) / T(8.)) * u[-2], (-T(5.) / T(4.)) * u[-1], (T(15.) / T(8.)) * u[0]);
  }
  return sum3(su[0], su[1], su[2]);
}

// eno_cvt with order-2 centre-to-face matrices
template <typename T>
__device__ __forceinline__ T cvt2(bool right, const T *wo, const T *u) {
  T s0 = T(0.0), s1 = T(0.0);
  if (!right) {
    if (wo[0] != T(0.0)) s0 = wo[0] * sum2((T(3.) / T(2.)) * u[0], (-T(1.) / T(2.)) * u[1]);
    if (wo[1] != T(0.0)) s1 = wo[1] * sum2((T(1.) / T(2.)) * u[-1], (T(1.) / T(2.)) * u[0]);
  } else {
    if (wo[0] != T(0.0)) s0 = wo[0] * sum2((T(1.) / T(2.)) * u[0], (T(1.) / T(2.)) * u[1]);
    if (wo[1] != T(0.0)) s1 = wo[1] * sum2((-T(1.) / T(2.)) * u[-1], (T(3.) / T(2.)) * u[0]);
  }
  return sum2(s0, s1);
}

// Face values of one cell (eno_line_reconstruct output loop,
// reconstructeno.c:444-545, with choose_weno_order :2087-2247 and the
// optimised weights of compute_optimized_cf_stencil_weights :1617-1683).
// u: the line at the cell (u[-2..2]); m0: SMONO indicator (0 at a cusp);
// is_cusp; w: unoptimised order-3 weights; lof: final lower-order fraction.
template <typename T>
__device__ __forceinline__ void faces(const T *u, const T *un, T m0, bool is_cusp, const T w[3], T lof,
                                      T *yl, T *yr) {
  // optimised order-3 weights, left face then right face (c2e_optimal_weights_*face[1])
  T wl[3], wr[3];
  wl[0] = w[0] * (T(1.) / T(16.));
  wl[1] = w[1] * (T(5.) / T(8.));
  wl[2] = w[2] * (T(5.) / T(16.));
  wr[0] = w[0] * (T(5.) / T(16.));
  wr[1] = w[1] * (T(5.) / T(8.));
  wr[2] = w[2] * (T(1.) / T(16.));
  T s = sum3(wl[0], wl[1], wl[2]);
  wl[0] /= (s + K<T>::tiny);
  wl[1] /= (s + K<T>::tiny);
  wl[2] /= (s + K<T>::tiny);
  s = sum3(wr[0], wr[1], wr[2]);
  wr[0] /= (s + K<T>::tiny);
  wr[1] /= (s + K<T>::tiny);
  wr[2] /= (s + K<T>::tiny);
  T ll[2], lr[2];
  bool two = (T(0.0) < lof);
  if (two) {
    T f = (T(1.) - lof);
    wl[0] *= f;
    wl[1] *= f;
    wl[2] *= f;
    wr[0] *= f;
    wr[1] *= f;
    wr[2] *= f;
    T w2[2];
    unopt2(m0, u, un, w2);
    // order-2 optimised weights (c2e_optimal_weights_*face[0]), then scaled by lof
    ll[0] = w2[0] * (T(1.) / T(4.));
    ll[1] = w2[1] * (T(3.) / 4);
    lr[0] = w2[0] * (T(3.) / T(4.));
    lr[1] = w2[1] * (T(1.) / T(4.));
    s = sum2(ll[0], ll[1]);
    ll[0] /= (s + K<T>::tiny);
    ll[1] /= (s + K<T>::tiny);
    s = sum2(lr[0], lr[1]);
    lr[0] /= (s + K<T>::tiny);
    lr[1] /= (s + K<T>::tiny);
    ll[0] *= lof;
    ll[1] *= lof;
    lr[0] *= lof;
    lr[1] *= lof;
  }
  (void)is_cusp;
  for (int side = 0; side < 2; side++) {
    bool right = side == 1;
    T prev = (m0 != T(0.0)) ? eno5(right, u) : T(0.0);
    if (m0 >= T(0.0) && m0 < T(1.0)) {
      T v = T(0.0);
      v += cvt3(right, right ? wr : wl, u);
      if (two) v += cvt2(right, right ? lr : ll, u);
      prev = (T(1.0) - m0) * v + m0 * prev;
    }
    if (right) *yr = prev;
    else *yl = prev;
  }
}

}  // namespace w5
}  // namespace hg
