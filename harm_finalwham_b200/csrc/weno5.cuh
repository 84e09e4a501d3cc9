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
// are dead).  The GPU splits the line work into two cell-parallel passes:
//   pass A (per cell, per primitive): SMONO cusp test and indicator, and the
//          unoptimised order-3 weights (compute_cf_stencil_weights +
//          mono_adjust_unoptimized_weights)
//   pass B (per output cell): weight ratios of c-1..c+1 (compute_weights_ratios),
//          dP/P reduction (apply_additional_reduction_to_weights), optimised
//          weights, order-2 weights when reduced (choose_weno_order) and the
//          face values (eno_cvt + the SMONO blend).
// Every expression keeps the reference's operation order; the library is
// compiled with -fmad=false, so results are bit-identical to the reference.
#pragma once

namespace hg {
namespace w5 {

constexpr double kEps = 1.e-26;      // WENO_EPSILON = REDUCEEPSILON (reconstructeno.h:195-200)
constexpr double kSmonoEps = 1.e-13; // SMONO_EPSILON = SQRT_WENO_EPSILON (reconstructeno.h:73,196)
constexpr double kMinRat = 1.3;      // MIN/MAX_TRANSITION_RATIO of the AND reduction (reconstructeno.h:175-176)
constexpr double kMaxRat = 1.6;
constexpr double kDpFrac = 0.5;      // REDUCE_DP_FRACTION (reconstructeno.h:96)
constexpr double kBig = 1.e+50;      // BIG (global.h:1040)
constexpr double kSmall = 1.e-50;    // SMALL (global.h:1041)
constexpr double kDblMin = 2.2250738585072014e-308;  // DBL_MIN

__device__ __forceinline__ double wmin(double a, double b) { return (a < b) ? a : b; }  // MIN global.h:751
__device__ __forceinline__ double wmax(double a, double b) { return (a > b) ? a : b; }  // MAX global.h:750
__device__ __forceinline__ double minmod(double a, double b) {                          // global.h:361-362
  return ((a) * (b) <= 0) ? 0.0 : ((fabs(a) < fabs(b)) ? (a) : (b));
}
__device__ __forceinline__ double sgn(double a) { return (a > 0.0) ? 1.0 : ((a < 0.0) ? -1.0 : 0.0); }  // phys.c:1778

// get_sum_of_elements with SYMMETRIZE_WENO (reconstructeno.c:1920-1946)
__device__ __forceinline__ double sum2(double a0, double a1) {
  double s = 0.0;
  s += a0 + a1;
  s += a1 * 0.0;
  return s;
}
__device__ __forceinline__ double sum3(double a0, double a1, double a2) {
  double s = 0.0;
  s += a0 + a2;
  s += a1 * 1.0;
  return s;
}
__device__ __forceinline__ double sum5(const double *a) {
  double s = 0.0;
  s += a[0] + a[4];
  s += a[1] + a[3];
  s += a[2] * 1.0;
  return s;
}

// check_for_cusp_new (smonointerp.c:439-476); y points at the cell (y[-2..2] valid)
__device__ __forceinline__ bool cusp(const double *y) {
  double df_m1 = y[-1] - y[-2], df0 = y[0] - y[-1], df1 = y[1] - y[0], df2 = y[2] - y[1];
  double ddf_m1 = df0 - df_m1, ddf0 = df1 - df0, ddf1 = df2 - df1;
  double norm = (fabs(y[-2]) + fabs(y[-1]) + fabs(y[0]) + fabs(y[1]) + fabs(y[2]) + kSmall);
  norm = norm * kSmonoEps;
  double s0 = sgn(df0);
  double f1a = fabs(df0) - norm;
  double f1 = ddf_m1 * s0 - norm;
  double f2 = -ddf0 * s0 - norm;
  double f3 = -df2 * s0 - norm;
  double f3a = fabs(-df2 - df0) - 0.25 * (fabs(df2) + fabs(df0));
  double f4 = -df1 * s0 - norm;
  double f4a = fabs(-df1 - df0) - 0.25 * (fabs(df1) + fabs(df0));
  if (f1a > 0 && f1 > 0 && f2 > 0 && ((f3 > 0 && f3a > 0) || (f4 > 0 && f4a > 0))) return true;
  double s1 = sgn(df1);
  double f5a = fabs(df1) - norm;
  double f5 = -ddf1 * s1 - norm;
  double f6 = ddf0 * s1 - norm;
  double f7 = -df_m1 * s1 - norm;
  double f7a = fabs(-df_m1 - df1) - 0.25 * (fabs(df_m1) + fabs(df1));
  double f8 = -df0 * s1 - norm;
  double f8a = fabs(-df0 - df1) - 0.25 * (fabs(df0) + fabs(df1));
  if (f5a > 0 && f5 > 0 && f6 > 0 && ((f7 > 0 && f7a > 0) || (f8 > 0 && f8a > 0))) return true;
  return false;
}

// compute_mono_indicator_point_eno5 (smonointerp.c:296-425) + transition_function (:428-437)
__device__ __forceinline__ double mono(const double *y) {
  double l1 = (((-3 * y[-2] + y[2]) + (-10 * y[-1] - 6 * y[1])) + 18 * y[0]) / 12.;
  double l2 = (((11 * y[-2] - y[2]) + (-20 * y[-1] + 4 * y[1])) + 6 * y[0]) / 12.;
  double l3 = (((-3 * y[-2] - y[2]) + (10 * y[-1] + 6 * y[1])) - 12 * y[0]) / 2.;
  double r1 = (((-y[-2] + 3 * y[2]) + (6 * y[-1] + 10 * y[1])) - 18 * y[0]) / 12.;
  double r2 = (((-y[-2] + 11 * y[2]) + (4 * y[-1] - 20 * y[1])) + 6 * y[0]) / 12.;
  double r3 = (((y[-2] + 3 * y[2]) - (6 * y[-1] + 10 * y[1])) + 12 * y[0]) / 2.;
  l1 = minmod(l1, y[-1] - y[-2]);
  r1 = minmod(r1, y[2] - y[1]);
  double minabs = kBig;
  minabs = wmin(minabs, fabs(minmod(l1, r1)));
  minabs = wmin(minabs, fabs(minmod(l2, r2)));
  minabs = wmin(minabs, fabs(minmod(l3, r3)));
  double norm = fabs(y[0]) + ((fabs(y[-1]) + fabs(y[1])) + (fabs(y[-2]) + fabs(y[2])));
  double cut = norm * kSmonoEps + kDblMin;
  double v = (minabs - 0.0) / (cut - 0.0);
  return wmax(0., wmin(1., v));
}

// c2e_simple_eno(5, ...) (reconstructeno.c:826-901): central row of the
// 5-point centre-to-left (right=false) / centre-to-right matrix
__device__ __forceinline__ double eno5(bool right, const double *y) {
  double d[5];
  if (!right) {
    d[0] = (-5. / 128.) * y[-2];
    d[1] = (15. / 32.) * y[-1];
    d[2] = (45. / 64.) * y[0];
    d[3] = (-5. / 32.) * y[1];
    d[4] = (3. / 128.) * y[2];
  } else {
    d[0] = (3. / 128.) * y[-2];
    d[1] = (-5. / 32.) * y[-1];
    d[2] = (45. / 64.) * y[0];
    d[3] = (15. / 32.) * y[1];
    d[4] = (-5. / 128.) * y[2];
  }
  return sum5(d);
}

// Unoptimised order-3 weights of compute_cf_stencil_weights
// (reconstructeno.c:1406-1614; desensitise :1687-1707, normalisation
// :1948-1960, compute_weights_from_smoothness_indicators :1878-1917) followed
// by mono_adjust_unoptimized_weights (:702-728).  m0 is monoindicator[0]
// (0 at a cusp); the cusp's lower_order_fraction=1 is kept by the caller.
__device__ __forceinline__ void unopt3(double m0, const double *u, double w[3]) {
  if (m0 == 1) {
    w[0] = w[1] = w[2] = 1.0 / 3;
    return;
  }
  double fd0 = -(3 * u[0] + u[2]) + 4 * u[1];
  double fd1 = u[1] - u[-1];
  double fd2 = (3 * u[0] + u[-2]) - 4 * u[-1];
  double sd0 = (u[0] + u[2]) - 2 * u[1];
  double sd1 = (u[-1] + u[1]) - 2 * u[0];
  double sd2 = (u[0] + u[-2]) - 2 * u[-1];
  double si0 = 13. / 12. * sd0 * sd0 + 1. / 4. * fd0 * fd0;
  double si1 = 13. / 12. * sd1 * sd1 + 1. / 4. * fd1 * fd1;
  double si2 = 13. / 12. * sd2 * sd2 + 1. / 4. * fd2 * fd2;
  double u2[5] = {u[-2] * u[-2], u[-1] * u[-1], u[0] * u[0], u[1] * u[1], u[2] * u[2]};
  double e = sum5(u2) * kEps;
  si0 += e;
  si1 += e;
  si2 += e;
  double s = sum3(si0, si1, si2);
  si0 /= (s + kDblMin);
  si1 /= (s + kDblMin);
  si2 /= (s + kDblMin);
  double t0 = si0 + kEps / 1., t1 = si1 + kEps / 1., t2 = si2 + kEps / 1.;
  t0 *= t0;
  t1 *= t1;
  t2 *= t2;
  w[0] = 1. / t0;
  w[1] = 1. / t1;
  w[2] = 1. / t2;
  s = sum3(w[0], w[1], w[2]);
  w[0] /= (s + 0.0);
  w[1] /= (s + 0.0);
  w[2] /= (s + 0.0);
  if (m0 > 0.0 && m0 < 1.0) {
    double simple = 1.0 / 3.0;
    w[0] = (1.0 - m0) * w[0] + m0 * simple;
    w[1] = (1.0 - m0) * w[1] + m0 * simple;
    w[2] = (1.0 - m0) * w[2] + m0 * simple;
  }
}

// order-2 unoptimised weights (compute_cf_stencil_weights with order 2)
__device__ __forceinline__ void unopt2(double m0, const double *u, double w[2]) {
  if (m0 == 1) {
    w[0] = w[1] = 1.0 / 2;
    return;
  }
  double fd0 = u[1] - u[0];
  double fd1 = u[0] - u[-1];
  double si0 = fd0 * fd0, si1 = fd1 * fd1;
  double e = sum3(u[-1] * u[-1], u[0] * u[0], u[1] * u[1]) * kEps;
  si0 += e;
  si1 += e;
  double s = sum2(si0, si1);
  si0 /= (s + kDblMin);
  si1 /= (s + kDblMin);
  double t0 = si0 + kEps / 1., t1 = si1 + kEps / 1.;
  t0 *= t0;
  t1 *= t1;
  w[0] = 1. / t0;
  w[1] = 1. / t1;
  s = sum2(w[0], w[1]);
  w[0] /= (s + 0.0);
  w[1] /= (s + 0.0);
}

// lower_order_fraction of compute_weights_ratios (reconstructeno.c:1962-2083),
// AND reduction, centre-to-edge ratios; wc = weights of the cell,
// wl0 = weights[0] of cell-2, wr2 = weights[2] of cell+2; lof0 = 1 at a cusp
__device__ __forceinline__ double ratio_lof(const double wc[3], double wl0, double wr2, double lof0) {
  double minr = kMinRat, maxr = kMaxRat;
  double wrl = (wc[2] + kEps) / (wl0 + kEps);
  double wrr = (wc[0] + kEps) / (wr2 + kEps);
  double wr = wmin(wrl, wrr);
  double lof = (wr - minr) / (maxr - minr);
  lof = wmax(0., wmin(lof, 1.0));
  return wmax(lof, lof0);
}

// eno_cvt (reconstructeno.c:730-823) with order-3 centre-to-face matrices
__device__ __forceinline__ double cvt3(bool right, const double *wo, const double *u) {
  double su[3];
  // shift 0 uses u[0..2], shift 1 u[-1..1], shift 2 u[-2..0]
  if (!right) {
    su[0] = 0.0;
    if (wo[0] != 0.0) su[0] = wo[0] * sum3((15. / 8.) * u[0], (-5. / 4.) * u[1], (3. / 8.) * u[2]);
    su[1] = 0.0;
    if (wo[1] != 0.0) su[1] = wo[1] * sum3((3. / 8.) * u[-1], (3. / 4.) * u[0], (-1. / 8.) * u[1]);
    su[2] = 0.0;
    if (wo[2] != 0.0) su[2] = wo[2] * sum3((-1. / 8.) * u[-2], (3. / 4.) * u[-1], (3. / 8.) * u[0]);
  } else {
    su[0] = 0.0;
    if (wo[0] != 0.0) su[0] = wo[0] * sum3((3. / 8.) * u[0], (3. / 4.) * u[1], (-1. / 8.) * u[2]);
    su[1] = 0.0;
    if (wo[1] != 0.0) su[1] = wo[1] * sum3((-1. / 8.) * u[-1], (3. / 4.) * u[0], (3. / 8.) * u[1]);
    su[2] = 0.0;
    if (wo[2] != 0.0) su[2] = wo[2] * sum3((3. / 8.) * u[-2], (-5. / 4.) * u[-1], (15. / 8.) * u[0]);
  }
  return sum3(su[0], su[1], su[2]);
}

// eno_cvt with order-2 centre-to-face matrices
__device__ __forceinline__ double cvt2(bool right, const double *wo, const double *u) {
  double s0 = 0.0, s1 = 0.0;
  if (!right) {
    if (wo[0] != 0.0) s0 = wo[0] * sum2((3. / 2.) * u[0], (-1. / 2.) * u[1]);
    if (wo[1] != 0.0) s1 = wo[1] * sum2((1. / 2.) * u[-1], (1. / 2.) * u[0]);
  } else {
    if (wo[0] != 0.0) s0 = wo[0] * sum2((1. / 2.) * u[0], (1. / 2.) * u[1]);
    if (wo[1] != 0.0) s1 = wo[1] * sum2((-1. / 2.) * u[-1], (3. / 2.) * u[0]);
  }
  return sum2(s0, s1);
}

// Face values of one cell (eno_line_reconstruct output loop,
// reconstructeno.c:444-545, with choose_weno_order :2087-2247 and the
// optimised weights of compute_optimized_cf_stencil_weights :1617-1683).
// u: the line at the cell (u[-2..2]); m0: SMONO indicator (0 at a cusp);
// is_cusp; w: unoptimised order-3 weights; lof: final lower-order fraction.
__device__ __forceinline__ void faces(const double *u, double m0, bool is_cusp, const double w[3], double lof,
                                      double *yl, double *yr) {
  // optimised order-3 weights, left face then right face (c2e_optimal_weights_*face[1])
  double wl[3], wr[3];
  wl[0] = w[0] * (1. / 16.);
  wl[1] = w[1] * (5. / 8.);
  wl[2] = w[2] * (5. / 16.);
  wr[0] = w[0] * (5. / 16.);
  wr[1] = w[1] * (5. / 8.);
  wr[2] = w[2] * (1. / 16.);
  double s = sum3(wl[0], wl[1], wl[2]);
  wl[0] /= (s + kDblMin);
  wl[1] /= (s + kDblMin);
  wl[2] /= (s + kDblMin);
  s = sum3(wr[0], wr[1], wr[2]);
  wr[0] /= (s + kDblMin);
  wr[1] /= (s + kDblMin);
  wr[2] /= (s + kDblMin);
  double ll[2], lr[2];
  bool two = (0.0 < lof);
  if (two) {
    double f = (1. - lof);
    wl[0] *= f;
    wl[1] *= f;
    wl[2] *= f;
    wr[0] *= f;
    wr[1] *= f;
    wr[2] *= f;
    double w2[2];
    unopt2(m0, u, w2);
    // order-2 optimised weights (c2e_optimal_weights_*face[0]), then scaled by lof
    ll[0] = w2[0] * (1. / 4.);
    ll[1] = w2[1] * (3. / 4);
    lr[0] = w2[0] * (3. / 4.);
    lr[1] = w2[1] * (1. / 4.);
    s = sum2(ll[0], ll[1]);
    ll[0] /= (s + kDblMin);
    ll[1] /= (s + kDblMin);
    s = sum2(lr[0], lr[1]);
    lr[0] /= (s + kDblMin);
    lr[1] /= (s + kDblMin);
    ll[0] *= lof;
    ll[1] *= lof;
    lr[0] *= lof;
    lr[1] *= lof;
  }
  (void)is_cusp;
  for (int side = 0; side < 2; side++) {
    bool right = side == 1;
    double prev = (m0 != 0.0) ? eno5(right, u) : 0.0;
    if (m0 >= 0.0 && m0 < 1.0) {
      double v = 0.0;
      v += cvt3(right, right ? wr : wl, u);
      if (two) v += cvt2(right, right ? lr : ll, u);
      prev = (1.0 - m0) * v + m0 * prev;
    }
    if (right) *yr = prev;
    else *yl = prev;
  }
}

}  // namespace w5
}  // namespace hg
