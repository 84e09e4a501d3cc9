// harm_gpu.cu -- sm_100a kernels of HARM's per-zone conservative update and
// the C ABI declared in include/harmgpu.h.
//
// Device data layout (resident in HBM for the whole run):
//   primitives, conserved accumulators, fluxes: SoA planes [8][nt1][nt2][nt3]
//     with x3 fastest, so that the 32 threads of a warp walk x3 at one (i,j)
//     and read one metric row (broadcast) -- the metric depends on (i,j) only.
//   geometry: SoA [component][gt1*gt2], 205 doubles per (i,j):
//     4 locations (FACE1, FACE2, FACE3, CENT) x {gcov 16, gcon 16, gcovpert_tt, gdet},
//     CORN1..3 gdet, conn[64] at CENT, floors[2].
//
// Work per RK substep (the reference's advance(), step_ch.c:94-186):
//   weno5_kernel<dir> WENO5 line reconstruction (interpline.c:517-678), one
//                     kernel per direction over tiles staged in shared
//                     memory (lim = WENO5 only; weno5.cuh, common.cuh)
//   flux_kernel<dir>  fluxcalc_standard (flux.c:469-680) fused with the
//                     MC/PARA reconstruction (or reading the WENO5 face
//                     values), both Riemann states, vchar, HLL/LaxF, the gdet
//                     strip of flux_ct and the dt-min (common.cuh; the FP32
//                     instances of the mixed path are built in flux_f32.cu)
//   emf_kernel        corner EMFs of flux_ct (fluxct.c:148-218)
//   conserve_kernel   advance_standard zone loop (advance.c:143-213): U(pi),
//                     source_conn, flux divergence (B fluxes rebuilt from the
//                     EMFs, fluxct.c:724-781), dUtoU
//   invert_kernel     Utoprimgen and, on the final substep, fixup1zone
//   bound kernels     bound_prim (bounds.fishmon.c:29-345)
//   fixup kernels     post_fixup (fixup.c:37-96) in an order-independent
//                     formulation that reproduces the reference's sequential
//                     sweep exactly (see checksol_resolve / fixup_compute)
//   finalize_kernel   ndt combine (advance.c:231) and dt update (step_ch.c:236-247)
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <mutex>
#include <new>
#include <utility>
#include <vector>

#include "common.cuh"
#include "harm_device.cuh"
#include "harmgpu.h"
#include "weno5.cuh"

using namespace hg;

// FP32 instantiations of the reconstruction and flux kernels are compiled in
// flux_f32.cu (FMA and fast FP32 division there; this unit keeps -fmad=false)
namespace hg {
#define HG_F32_EXTERN(DIR)                                                                                         \
  extern template __global__ void weno5_kernel<DIR, true, float>(Dims, Params, W5Tile, const double *,            \
                                                                 const float *, double *, double *);              \
  extern template __global__ void weno5_kernel<DIR, false, float>(Dims, Params, W5Tile, const double *,           \
                                                                  const float *, double *, double *);             \
  extern template __global__ void flux_kernel<DIR, 0, float>(Dims, Params, Box, const double *, const float *,    \
                                                             const float *, const double *, double *, Scalars *);   \
  extern template __global__ void flux_kernel<DIR, 2, float>(Dims, Params, Box, const double *, const float *,    \
                                                             const float *, const double *, double *, Scalars *);   \
  extern template __global__ void flux_kernel<DIR, 1, double, kFluxMB[0], double, 1>(                             \
      Dims, Params, Box, const double *, const double *, const double *, const double *, double *, Scalars *);      \
  extern template __global__ void flux_kernel<DIR, 1, double, kFluxMB[1], double, 1>(                             \
      Dims, Params, Box, const double *, const double *, const double *, const double *, double *, Scalars *);
HG_F32_EXTERN(1)
HG_F32_EXTERN(2)
HG_F32_EXTERN(3)
extern template __global__ void w5_state_kernel<float>(Dims, Params, Box, const double *, const double *, float *);
}  // namespace hg

namespace {

thread_local char g_errbuf[512] = "";

void set_err(const char *fmt, const char *a = "", int b = 0) {
  snprintf(g_errbuf, sizeof(g_errbuf), fmt, a, b);
}

#define CUDA_TRY(call)                                                         \
  do {                                                                         \
    cudaError_t e__ = (call);                                                  \
    if (e__ != cudaSuccess) {                                                  \
      set_err("CUDA error: %s (line %d)", cudaGetErrorString(e__), __LINE__);  \
      return HGPU_E_CUDA;                                                      \
    }                                                                          \
  } while (0)

// ---------------------------------------------------------------------------
// corner EMFs (fluxct.c:104-218) on the corners the updated faces read
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) emf_kernel(Dims d, Box box, const double *__restrict__ F1,
                                                  const double *__restrict__ F2, const double *__restrict__ F3,
                                                  const double *__restrict__ G, double *__restrict__ E) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= box.size()) return;
  int i, j, k;
  box_ijk(box, t, i, j, k);
  long long z = zix(d, i, j, k);
  const long long o1 = (long long)d.nt2 * d.nt3, o2 = d.nt3, o3 = 1;
  const long long ij = gix(d, i, j);
  const int n1 = d.n1, n2 = d.n2, n3 = d.n3;
  double coef1 = ((n2 > 1) && (n3 > 1)) ? 0.25 : 0.5;
  double coef2 = ((n1 > 1) && (n3 > 1)) ? 0.25 : 0.5;
  double coef3 = ((n1 > 1) && (n2 > 1)) ? 0.25 : 0.5;
  const long long nz = d.nz;
  if (i <= n1 - 1) {
    double v;
    if (n2 > 1 && n3 > 1)
      v = coef1 * (+F2[B3 * nz + z] + F2[B3 * nz + z - d.s3 * o3] - F3[B2 * nz + z] - F3[B2 * nz + z - d.s2 * o2]);
    else if (n2 > 1)
      v = coef1 * (+F2[B3 * nz + z] + F2[B3 * nz + z - d.s3 * o3]);
    else if (n3 > 1)
      v = coef1 * (-F3[B2 * nz + z] - F3[B2 * nz + z - d.s2 * o2]);
    else
      v = 0.0;
    E[0 * nz + z] = v * __ldg(G + (long long)(G_CORN + 0) * d.nij + ij);
  }
  if (j <= n2 - 1) {
    double v;
    if (n1 > 1 && n3 > 1)
      v = coef2 * (+F3[B1 * nz + z] + F3[B1 * nz + z - d.s1 * o1] - F1[B3 * nz + z] - F1[B3 * nz + z - d.s3 * o3]);
    else if (n3 > 1)
      v = coef2 * (+F3[B1 * nz + z] + F3[B1 * nz + z - d.s1 * o1]);
    else if (n1 > 1)
      v = coef2 * (-F1[B3 * nz + z] - F1[B3 * nz + z - d.s3 * o3]);
    else
      v = 0.0;
    E[1 * nz + z] = v * __ldg(G + (long long)(G_CORN + 1) * d.nij + ij);
  }
  if (k <= n3 - 1) {
    double v;
    if (n1 > 1 && n2 > 1)
      v = coef3 * (+F1[B2 * nz + z] + F1[B2 * nz + z - d.s2 * o2] - F2[B1 * nz + z] - F2[B1 * nz + z - d.s1 * o1]);
    else if (n1 > 1)
      v = coef3 * (+F1[B2 * nz + z] + F1[B2 * nz + z - d.s2 * o2]);
    else if (n2 > 1)
      v = coef3 * (-F2[B1 * nz + z] - F2[B1 * nz + z - d.s1 * o1]);
    else
      v = 0.0;
    E[2 * nz + z] = v * __ldg(G + (long long)(G_CORN + 2) * d.nij + ij);
  }
}

// ---------------------------------------------------------------------------
// zone update: advance_standard's CZLOOP body (advance.c:143-213), split in
// two kernels with the same arithmetic: the conserved update (U(pi), the
// geometric source, the flux divergence, dUtoU) and the inversion with the
// final-substep fixup1zone.  Each holds half the live state of the fused
// loop body, so more warps fit per SM.
// ---------------------------------------------------------------------------
// per-zone step parameters: dt, gamma, dx1 of the domain or of the zone's
// batch instance; false if the zone does not advance
__device__ __forceinline__ bool zone_step(const Params &P, const Scalars *sc, long long z, int i, double &dt,
                                          double &gam, double &dx1) {
  dt = sc->dt;
  gam = P.gam;
  dx1 = P.dx1;
  if (P.cell_inst) {
    const Inst &I = P.inst[P.cell_inst[z]];
    int loc = i - I.i0;
    dt = I.dt;
    gam = I.gam;
    dx1 = I.dx;
    return loc >= 0 && loc < I.n && !I.done;
  }
  return !sc->done;
}

// diag_fixup's correction of the evolved conserved state under
// ENOFINITEVOLUME with DOENOFLUXMEMORY (fixup.c:196-252), final substep only:
// unew += UtoU(UDIAG->UEVOLVE, U(pr)) - UtoU(UDIAG->UEVOLVE, U(pr0)) where
// U = primtoU(UDIAG) and UtoU divides by gdet and multiplies by e = gdet
// (phys.c:243-285).  It runs once per energy region (NUMENERREGIONS = 3
// with DOJETDIAG, global.h:435-439, every active zone being in the
// correctable region), so the difference is added three times.
__device__ __forceinline__ void fv_diag_fixup(const double *pr0, const double *pr, const Metric &m, double gam,
                                              double *__restrict__ ucum, long long z, long long nz, int *err) {
  double Ui[NPR], Uf[NPR];
  {
    State q;
    EM e;
    if (get_state(pr0, m, q)) {
      *err |= ERR_UTCALC_DISCR;
      return;
    }
    em_prepare(pr0, m, q, e);
    primtoflux(pr0, q, e, 0, m, gam, Ui);
  }
  {
    State q;
    EM e;
    if (get_state(pr, m, q)) {
      *err |= ERR_UTCALC_DISCR;
      return;
    }
    em_prepare(pr, m, q, e);
    primtoflux(pr, q, e, 0, m, gam, Uf);
  }
#pragma unroll
  for (int pl = 0; pl < NPR; pl++) {
    const double upre = (Ui[pl] / m.g) * m.g;
    const double upost = (Uf[pl] / m.g) * m.g;
    double u = ucum[pl * nz + z];
    u += upost - upre;
    u += upost - upre;
    u += upost - upre;
    ucum[pl * nz + z] = u;
  }
}

// pi2Uavg (initbase.c:1833-1880) with avgscheme=DONOR: the conserved state
// U(p) in every zone, ghosts included
__global__ void pi2u_kernel(Dims d, Params P, const double *__restrict__ p, const double *__restrict__ G,
                            double *__restrict__ u, Scalars *sc) {
  long long z = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= d.nz) return;
  int k = (int)(z % d.nt3) - d.g3;
  long long r = z / d.nt3;
  int j = (int)(r % d.nt2) - d.g2;
  int i = (int)(r / d.nt2) - d.g1;
  Metric m;
  load_metric(G, d, gix(d, i, j), G_CENT, m);
  double pr[NPR], U[NPR];
  load_prim(p, d, z, pr);
  State q;
  EM e;
  if (get_state(pr, m, q)) {
    atomicOr(&sc->err, ERR_UTCALC_DISCR);
    return;
  }
  em_prepare(pr, m, q, e);
  primtoflux(pr, q, e, 0, m, P.gam, U);
#pragma unroll
  for (int pl = 0; pl < NPR; pl++) u[pl * d.nz + z] = U[pl];
}

// source() -> source_conn() (phys.c:578-752): the connection contraction of
// T^mu_nu for the state pbz (q, e formed from it), times gdet
__device__ __forceinline__ void source_conn(const Dims &d, const double *__restrict__ G, long long ij,
                                            const double *pbz, const State &q, const EM &e, const Metric &m,
                                            double gam, double *dUg) {
  double dUconn[4] = {0., 0., 0., 0.};
  const double *conn = G + (long long)G_CONN * d.nij + ij;
  // each T^jj_kk row is contracted as soon as it is formed; every
  // dUconn[l] still adds its terms in the order jj, then kk
#pragma unroll
  for (int jj = 0; jj < 4; jj++) {
    double row[4];
    mhd_row(pbz, jj, gam, q, e, row);
#pragma unroll
    for (int l = 0; l < 4; l++) {
      double s = dUconn[l];
#pragma unroll
      for (int kk = 0; kk < 4; kk++) s += row[kk] * __ldg(conn + (long long)((kk * 4 + l) * 4 + jj) * d.nij);
      dUconn[l] = s;
    }
  }
#pragma unroll
  for (int l = 0; l < 4; l++) {
    double s = dUconn[l];
#pragma unroll
    for (int jj = 0; jj < 4; jj++) s += -pbz[RHO] * q.ucon[jj] * __ldg(conn + (long long)((0 * 4 + l) * 4 + jj) * d.nij);
    dUconn[l] = s;
  }
  // dU = sum of the NUMSOURCES components; only GEOMSOURCE is nonzero
  double full[NPR] = {0., dUconn[0], dUconn[1], dUconn[2], dUconn[3], 0., 0., 0.};
#pragma unroll
  for (int pl = 0; pl < NPR; pl++) {
    double comp0 = 0. + m.g * full[pl];
    double acc = 0.;
    acc += comp0;
#pragma unroll
    for (int l = 1; l < 7; l++) acc += 0.0;
    dUg[pl] = acc;
  }
}

template <int MB>
__global__ void __launch_bounds__(128, MB) conserve_kernel(
    Dims d, Params P, Box box, const double *pi, const double *pb, double *__restrict__ uf,
    double *__restrict__ ucum, const double *__restrict__ F1, const double *__restrict__ F2,
    const double *__restrict__ F3, const double *__restrict__ E, const double *__restrict__ G, Scalars *sc,
    double CUf0, double CUf1, double CUf2, double Cunew0, double Cunew1, double Cunew2, int timeorder,
    double *__restrict__ ui, int fv) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= box.size()) return;
  int i, j, k;
  box_ijk(box, t, i, j, k);
  const long long z = zix(d, i, j, k);
  const long long nz = d.nz;
  const long long o1 = (long long)d.nt2 * d.nt3, o2 = d.nt3, o3 = 1;
  const long long ij = gix(d, i, j);
  double dt, gam, dx1;
  if (!zone_step(P, sc, z, i, dt, gam, dx1)) return;
    double Ui[NPR], dUg[NPR], dUr[NPR];
    // the flux differences first: their ~50 independent loads are in flight
    // together before the arithmetic of U(pi) and the source term
    // flux2dUavg (advance.c:741-914) with the B fluxes of flux_ct (fluxct.c:724-781)
    {
      const double idx1 = 1.0 / dx1, idx2 = 1.0 / P.dx2, idx3 = 1.0 / P.dx3;
      const double *e1 = E, *e2 = E + nz, *e3 = E + 2 * nz;
#pragma unroll
      for (int pl = 0; pl < NPR; pl++) {
        double a1 = 0, a2 = 0, a3 = 0;
        if (d.n1 > 1) {
          double fa, fb;
          if (pl == B1) { fa = 0.; fb = 0.; }
          else if (pl == B2) { fa = 0.5 * (e3[z] + e3[z + d.s2 * o2]); fb = 0.5 * (e3[z + o1] + e3[z + o1 + d.s2 * o2]); }
          else if (pl == B3) { fa = -0.5 * (e2[z] + e2[z + d.s3 * o3]); fb = -0.5 * (e2[z + o1] + e2[z + o1 + d.s3 * o3]); }
          else { fa = F1[pl * nz + z]; fb = F1[pl * nz + z + o1]; }
          a1 = (-(fb - fa) * idx1);
        }
        if (d.n2 > 1) {
          double fa, fb;
          if (pl == B1) { fa = -0.5 * (e3[z] + e3[z + d.s1 * o1]); fb = -0.5 * (e3[z + o2] + e3[z + o2 + d.s1 * o1]); }
          else if (pl == B2) { fa = 0.; fb = 0.; }
          else if (pl == B3) { fa = 0.5 * (e1[z] + e1[z + d.s3 * o3]); fb = 0.5 * (e1[z + o2] + e1[z + o2 + d.s3 * o3]); }
          else { fa = F2[pl * nz + z]; fb = F2[pl * nz + z + o2]; }
          a2 = (-(fb - fa) * idx2);
        }
        if (d.n3 > 1) {
          double fa, fb;
          if (pl == B1) { fa = 0.5 * (e2[z] + e2[z + d.s1 * o1]); fb = 0.5 * (e2[z + o3] + e2[z + o3 + d.s1 * o1]); }
          else if (pl == B2) { fa = -0.5 * (e1[z] + e1[z + d.s2 * o2]); fb = -0.5 * (e1[z + o3] + e1[z + o3 + d.s2 * o2]); }
          else if (pl == B3) { fa = 0.; fb = 0.; }
          else { fa = F3[pl * nz + z]; fb = F3[pl * nz + z + o3]; }
          a3 = (-(fb - fa) * idx3);
        }
        dUr[pl] = a1 + a2 + a3;
      }
    }
    Metric m;
    load_metric(G, d, ij, G_CENT, m);
    int err = 0;
    if (fv) {
      // advance_finitevolume (advance.c:245-501): Ui is the stored conserved
      // state; the first substep takes the last step's ucum as ui
      // (advance.c:330-343)
      if (timeorder == 0) {
#pragma unroll
        for (int pl = 0; pl < NPR; pl++) {
          Ui[pl] = ucum[pl * nz + z];
          ui[pl * nz + z] = Ui[pl];
        }
      } else {
#pragma unroll
        for (int pl = 0; pl < NPR; pl++) Ui[pl] = ui[pl * nz + z];
      }
      double pbz[NPR];
      load_prim(pb, d, z, pbz);
      State q;
      EM e;
      if (get_state(pbz, m, q)) err |= ERR_UTCALC_DISCR;
      em_prepare(pbz, m, q, e);
      source_conn(d, G, ij, pbz, q, e, m, gam, dUg);
    } else if (pi == pb) {
      // a first substep: U(pi) and the source read the same state, whose
      // get_state and field terms are formed once
      double pbz[NPR];
      load_prim(pb, d, z, pbz);
      State q;
      EM e;
      if (get_state(pbz, m, q)) err |= ERR_UTCALC_DISCR;
      em_prepare(pbz, m, q, e);
      primtoflux(pbz, q, e, 0, m, gam, Ui);
      source_conn(d, G, ij, pbz, q, e, m, gam, dUg);
    } else {
      {
        double pr[NPR];
        load_prim(pi, d, z, pr);
        State qi;
        EM ei;
        if (get_state(pr, m, qi)) err |= ERR_UTCALC_DISCR;
        em_prepare(pr, m, qi, ei);
        primtoflux(pr, qi, ei, 0, m, gam, Ui);
      }
      double pbz[NPR];
      load_prim(pb, d, z, pbz);
      State q;
      EM e;
      if (get_state(pbz, m, q)) err |= ERR_UTCALC_DISCR;
      em_prepare(pbz, m, q, e);
      source_conn(d, G, ij, pbz, q, e, m, gam, dUg);
    }
    // dUtoU (advance.c:922-949)
    double Uf[NPR], Ucum[NPR];
#pragma unroll
    for (int pl = 0; pl < NPR; pl++) {
      double ufo = (timeorder == 0) ? 0.0 : uf[pl * nz + z];
      double uco = (timeorder == 0) ? 0.0 : ucum[pl * nz + z];
      Uf[pl] = CUf0 * Ui[pl] + CUf1 * ufo + CUf2 * dt * (dUr[pl] + dUg[pl]);
      Ucum[pl] = uco + (Cunew0 * Ui[pl] + Cunew1 * dt * (dUr[pl] + dUg[pl]) + Cunew2 * Uf[pl]);
      uf[pl * nz + z] = Uf[pl];
      ucum[pl * nz + z] = Ucum[pl];
    }
    if (err) atomicOr(&sc->err, err);
}

template <int UV, int MB>
__global__ void __launch_bounds__(128, MB) invert_kernel(Dims d, Params P, Box box, const double *pb,
                                                                     double *pf, const double *__restrict__ uf,
                                                                     const double *__restrict__ ucum,
                                                                     const double *__restrict__ G,
                                                                     int *__restrict__ pflag, Scalars *sc,
                                                                     int finalstep, double *__restrict__ ufv) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long my_iters = 0;
  int my_fail = 0;
  if (t < box.size()) {
    int i, j, k;
    box_ijk(box, t, i, j, k);
    const long long z = zix(d, i, j, k);
    const long long nz = d.nz;
    const long long ij = gix(d, i, j);
    double dt, gam, dx1;
    if (zone_step(P, sc, z, i, dt, gam, dx1)) {
    Metric m;
    load_metric(G, d, ij, G_CENT, m);
    int err = 0;
    double pbz[NPR], Uin[NPR];
    load_prim(pb, d, z, pbz);
    const double *src = finalstep ? ucum : uf;
#pragma unroll
    for (int pl = 0; pl < NPR; pl++) Uin[pl] = src[pl * nz + z];
    // guess = pb, invert (advance.c:188-205)
    double pr[NPR];
#pragma unroll
    for (int v = 0; v < NPR; v++) pr[v] = pbz[v];
    int it = 0;
    int flag = utoprimgen_v<UV>(Uin, m, gam, P.gammafail, pr, &it);
    my_iters = (unsigned long long)it;
    my_fail = (flag != 0);
    if (finalstep) {
      // fixup1zone (fixup.c:341-447)
      const double *fl = G + (long long)G_FLOOR * d.nij + ij;
      double fr = __ldg(fl), fu = __ldg(fl + d.nij);
      if (fr < P.rhominlimit) fr = P.rhominlimit;
      if (fu < P.uuminlimit) fu = P.uuminlimit;
      bool floored = (fr > pr[RHO]) || (fu > pr[UU]);
      double pr0[NPR];
#pragma unroll
      for (int v = 0; v < NPR; v++) pr0[v] = pr[v];
      if (fr > pr[RHO]) pr[RHO] = fr;
      if (fu > pr[UU]) pr[UU] = fu;
      const int lg = limit_gamma(P.gammamax, pr, m, &err);
      if (floored) atomicAdd(&sc->nfloor, 1ULL);
      // diag_fixup's counts: limit_gamma's own when it rescaled
      // (fixup.c:1913), fixup1zone's when floors or the gamma limit changed
      // the zone (fixup.c:443; a failed limit_gamma returns before either)
      if (lg == -1) ffc_count(P, nz, z, CNT_LIMITGAMMAACT);
      if (lg < 1 && (floored || lg == -1)) ffc_count(P, nz, z, CNT_FLOORACT);
      // diag_fixup (fixup.c:443) when fixup1zone changed the primitives
      if (ufv && lg < 1 && (floored || lg == -1)) fv_diag_fixup(pr0, pr, m, gam, ufv, z, nz, &err);
    }
    store_prim(pf, d, z, pr);
    pflag[z] = flag;
    if (err) atomicOr(&sc->err, err);
    }
  }
  // block-level aggregation of counters
  unsigned long long s_it = my_iters;
  int s_f = my_fail;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s_it += __shfl_xor_sync(0xffffffffu, s_it, o);
    s_f += __shfl_xor_sync(0xffffffffu, s_f, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (s_it) atomicAdd(&sc->iters, s_it);
    if (s_f) atomicAdd(&sc->nfail, s_f);
  }
}

// ---------------------------------------------------------------------------
// boundaries: bound_prim_user (bounds.fishmon.c:29-345)
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool is_polar(int bc) { return bc == HGPU_BC_POLARAXIS || bc == HGPU_BC_POLARAXIS_FLIP; }
__device__ __forceinline__ bool is_bondi(int bc) {
  return bc == HGPU_BC_BONDIINTOUTFLOW || bc == HGPU_BC_BONDIMDOTOUTFLOW;
}

// Source index of a ghost zone along one direction.  The Bondi-integral
// ghosts are computed (bondi_bc_kernel), so they are their own source.
__device__ __forceinline__ int map_idx(int i, int n, int bcdn, int bcup) {
  if (i < 0) {
    if (bcdn == HGPU_BC_PERIODIC) return i + n;
    if (is_polar(bcdn)) return -i - 1;
    if (is_bondi(bcdn)) return i;
    return 0;  // OUTFLOW
  }
  if (i >= n) {
    if (bcup == HGPU_BC_PERIODIC) return i - n;
    if (is_polar(bcup)) return (n - 1) + ((n - 1) - i + 1);
    if (is_bondi(bcup)) return i;
    return n - 1;
  }
  return i;
}

// inflow_check_rel4vel for dir 1 at CENT (fixup.c:2271-2407)
__device__ __forceinline__ void inflow_check_x1(const Dims &d, const Params &P, int i, double *pr, const Metric &m,
                                                int *err) {
  double ucon[4];
  if (ucon_calc(pr, m, ucon)) {
    *err |= ERR_UTCALC_DISCR;
    return;
  }
  bool dofix = ((i <= -1) && (P.bc[1] == HGPU_BC_OUTFLOW) && (ucon[1] > 0.)) ||
               ((i >= d.n1) && (P.bc[0] == HGPU_BC_OUTFLOW) && (ucon[1] < 0.));
  if (!dofix) return;
  double gamma;
  if (gamma_calc(pr, m, &gamma)) {
    *err |= ERR_UTCALC_DISCR;
    return;
  }
  pr[U1] /= gamma;
  pr[U2] /= gamma;
  pr[U3] /= gamma;
  double alpha = 1. / sqrt(-GCON(m, 0, 0));
  double betacon = GCON(m, 0, 1) * alpha * alpha;
  pr[U1] = betacon / alpha;
  double vsq = 0.;
#pragma unroll
  for (int j = 1; j < 4; j++)
#pragma unroll
    for (int k = 1; k < 4; k++) vsq += GCOV(m, j, k) * pr[U1 + j - 1] * pr[U1 + k - 1];
  if (vsq < 0.0) {
    if (vsq > -NUMEPSILON * 100.0) vsq = 0.0;
    else {
      *err |= ERR_VSQ_NEG;
      return;
    }
  }
  if (vsq >= 1.0) vsq = 1.0 - 1.0 / (P.gammamax * P.gammamax);
  gamma = 1. / sqrt(1. - vsq);
  pr[U1] *= gamma;
  pr[U2] *= gamma;
  pr[U3] *= gamma;
}

// Bondi-integral x1 boundaries (bounds.c:140-156, 295-308): one thread per
// ghost zone (i, j, k) of active j, k.  The edge zone's integrals
// (bondi_compute_integrals, bounds.c:788-836: its relative 4-velocity to
// u^mu, metptomet to Kerr-Schild u^r, transforms.c:51-84, 310-328), carried
// unchanged to the ghost (interpn of order 1), then the ghost's primitives
// (bondi_generate_solution, bounds.c:839-888).  Runs before
// bound_ghost_kernel, which takes these zones as the sources of the x2/x3
// ghost corners.
__device__ __forceinline__ void mat4_vec(const double *M, const double *u, double *out) {
#pragma unroll
  for (int j = 0; j < 4; j++) {
    double t = 0.;
#pragma unroll
    for (int k = 0; k < 4; k++) t += M[4 * j + k] * u[k];
    out[j] = t;
  }
}

__global__ void bondi_bc_kernel(Dims d, Params P, double *p, const double *__restrict__ G, Scalars *sc) {
  const long long per_side = (long long)d.g1 * d.n2 * d.n3;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * per_side || sc->done) return;
  const int side = (int)(t / per_side);
  long long r = t % per_side;
  const int k = (int)(r % d.n3);
  r /= d.n3;
  const int j = (int)(r % d.n2);
  const int q = 1 + (int)(r / d.n2);
  if (side == 0 && P.bc[1] != HGPU_BC_BONDIINTOUTFLOW) return;
  if (side == 1 && P.bc[0] != HGPU_BC_BONDIMDOTOUTFLOW) return;
  const int i0 = side == 0 ? 0 : d.n1 - 1;
  const int i = side == 0 ? -q : d.n1 - 1 + q;
  const double *e = P.bondi + ((long long)(side * (d.g1 + 1)) * d.n2 + j) * 49;
  const double *g = P.bondi + ((long long)(side * (d.g1 + 1) + q) * d.n2 + j) * 49;
  const double gam = P.gam;
  const double n = 1 / (gam - 1);
  int err = 0;
  // the edge zone's integrals
  double pr0[NPR];
  load_prim(p, d, zix(d, i0, j, k), pr0);
  Metric m0;
  load_metric(G, d, gix(d, i0, j), G_CENT, m0);
  double ucp[4], uks[4];
  if (ucon_calc(pr0, m0, ucp)) err |= ERR_UTCALC_DISCR;
  mat4_vec(e + 1, ucp, uks);
  const double pres = (gam - 1) * pr0[UU];
  const double T = pres / pr0[RHO];
  const double re = e[0];
  double C1 = pow(T, n) * uks[1] * re * re;
  double C2 = pow(1 + (1 + n) * T, 2.) * (1 - 2. / re + uks[1] * uks[1]);
  double K = pres / pow(pr0[RHO], gam);
  if (side == 1) {
    C2 = 1.373125;  // bounds.c:48-49 (bondigrid4acc.nb)
    K = 1.;
  }
  // bondi_invert_integrals at the ghost's radius
  const double rg = g[0];
  double T0 = 0.2, T1 = 0.1;
  int it = 0;
  if (rg > 0.35 && rg < 2.5) {
    for (; it < 250 && fabs((T0 - T1) / T1) > 1.0e-15; it++) {
      T0 = T1;
      const double u1 = C1 / (rg * rg * pow(T0, n));
      T1 = T0 + 0.02 * (T0 - (sqrt(C2 / (1 - 2 / rg + u1 * u1)) - 1) / (1 + n));
    }
  } else if (rg > 9) {
    for (; it < 250 && (T0 - T1) / T1 > 1.0e-15; it++) {
      T0 = T1;
      const double u1 = C1 / (rg * rg * pow(T0, n));
      T1 = (sqrt(C2 / (1 - 2 / rg + u1 * u1)) - 1) / (1 + n);
    }
    if (T1 > T0) err |= ERR_BONDI;
  } else {
    err |= ERR_BONDI;
  }
  if (err & ERR_BONDI) {
    atomicOr(&sc->err, err);
    return;
  }
  double pr[NPR];
#pragma unroll
  for (int v = 0; v < NPR; v++) pr[v] = 0.0;
  pr[RHO] = pow(T1 / K, n);
  pr[UU] = pr[RHO] * T1 * n;
  // u^t from the Kerr-Schild metric (pr2ucon VEL4: get_4velterms, phys.c:1192-1262)
  const double *gk = g + 33;
  double uc[4] = {0., C1 / (pow(T1, n) * rg * rg), 0., 0.};
  const double AA = gk[0];
  const double BB = 2. * (gk[1] * uc[1] + gk[2] * uc[2] + gk[3] * uc[3]);
  const double CCM1 = gk[5] * uc[1] * uc[1] + gk[10] * uc[2] * uc[2] + gk[15] * uc[3] * uc[3] +
                      2. * (gk[6] * uc[1] * uc[2] + gk[7] * uc[1] * uc[3] + gk[11] * uc[2] * uc[3]);
  const double discr = BB * BB - 4. * AA * (CCM1 + 1.0);
  if (discr < 0.) err |= ERR_UTCALC_DISCR;
  uc[0] = (-BB - sqrt(discr)) / (2. * AA);
  // to the internal coordinates (mettometpface) and the relative 4-velocity (ucon2pr VELREL4)
  double ucp2[4];
  mat4_vec(g + 17, uc, ucp2);
  Metric mg;
  load_metric(G, d, gix(d, i, j), G_CENT, mg);
  const double alphasq = 1. / (-GCON(mg, 0, 0));
  pr[U1] = ucp2[1] + (alphasq * GCON(mg, 0, 1)) * ucp2[0];
  pr[U2] = ucp2[2] + (alphasq * GCON(mg, 0, 2)) * ucp2[0];
  pr[U3] = ucp2[3] + (alphasq * GCON(mg, 0, 3)) * ucp2[0];
  store_prim(p, d, zix(d, i, j, k), pr);
  if (err) atomicOr(&sc->err, err);
}

// Every ghost zone of the full box as the composition of the reference's
// sequential fills: x1 (active j,k: copy + inflow check + gamma limit with the
// ghost's own metric; the Bondi-integral ghosts come from bondi_bc_kernel),
// then x2 (full i, active k: reflection, and either POLEDEATH zeroing of u~2
// and B2 (bounds.fishmon.c) or their negation (the generic bounds.c,
// HGPU_BC_POLARAXIS_FLIP)), then x3 (full i, full j: periodic copy).  Reads
// only zones this kernel does not write.
__global__ void __launch_bounds__(128) bound_ghost_kernel(Dims d, Params P, double *p, const double *__restrict__ G,
                                                          Scalars *sc) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= d.nz) return;
  int k = (int)(t % d.nt3) - d.g3;
  long long r = t / d.nt3;
  int j = (int)(r % d.nt2) - d.g2;
  int i = (int)(r / d.nt2) - d.g1;
  bool gi = (i < 0 || i >= d.n1), gj = (j < 0 || j >= d.n2), gk = (k < 0 || k >= d.n3);
  if (!(gi || gj || gk)) return;
  // x1 ghosts of active j, k on a Bondi-integral side: bondi_bc_kernel's
  if (gi && !gj && !gk && is_bondi(i < 0 ? P.bc[1] : P.bc[0])) return;
  int si = map_idx(i, d.n1, P.bc[1], P.bc[0]);
  int sj = map_idx(j, d.n2, P.bc[3], P.bc[2]);
  int sk = map_idx(k, d.n3, P.bc[5], P.bc[4]);
  double pr[NPR];
  load_prim(p, d, zix(d, si, sj, sk), pr);
  int err = 0;
  // the generic bounds.c's polar reflection (bounds.c:477-489)
  if (gj && ((j < 0 && P.bc[3] == HGPU_BC_POLARAXIS_FLIP) || (j >= d.n2 && P.bc[2] == HGPU_BC_POLARAXIS_FLIP))) {
    pr[U2] *= -1.;
    pr[B2] *= -1.;
  }
  if (gi && (P.bc[1] == HGPU_BC_OUTFLOW || P.bc[0] == HGPU_BC_OUTFLOW) &&
      ((i < 0 && P.bc[1] == HGPU_BC_OUTFLOW) || (i >= d.n1 && P.bc[0] == HGPU_BC_OUTFLOW))) {
    Metric m;
    load_metric(G, d, gix(d, i, sj), G_CENT, m);
    inflow_check_x1(d, P, i, pr, m, &err);
    limit_gamma(P.gammamax, pr, m, &err);
  }
  // POLEDEATH rows: x2 ghosts and the first/last active row (bounds.fishmon.c:238-250, 300-312)
  bool pole_dn = (P.bc[3] == HGPU_BC_POLARAXIS) && (j <= 0) && d.n2 > 1;
  bool pole_up = (P.bc[2] == HGPU_BC_POLARAXIS) && (j >= d.n2 - 1) && d.n2 > 1;
  if (pole_dn || pole_up) {
    pr[U2] *= 0;
    pr[B2] *= 0.;
  }
  store_prim(p, d, t, pr);
  if (err) atomicOr(&sc->err, err);
}

// POLEDEATH on the active first/last x2 rows (after the ghosts have read them)
__global__ void bound_pole_kernel(Dims d, Params P, double *p) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long rows = (long long)d.n1 * d.n3;
  if (t >= 2 * rows) return;
  int side = (int)(t / rows);
  long long r = t % rows;
  int i = (int)(r / d.n3), k = (int)(r % d.n3);
  int j;
  if (side == 0) {
    if (!(P.bc[3] == HGPU_BC_POLARAXIS)) return;
    j = 0;
  } else {
    if (!(P.bc[2] == HGPU_BC_POLARAXIS)) return;
    j = d.n2 - 1;
  }
  long long z = zix(d, i, j, k);
  p[(long long)U2 * d.nz + z] *= 0;
  p[(long long)B2 * d.nz + z] *= 0.;
}

// bound_pflag_user (boundsint.c:6-266) as the same composition
// get_bsqflags (fixup.c:1751-1849), which pre_fixup runs on the stage's
// input state at the start of every RK stage (step_ch.c:117-120): per zone,
// with the CENT metric, b^2/rho against BSQORHOLIMIT and b^2/u against
// BSQOULIMIT (initbase.c:465-466), 2 above the limit, 1 above 0.9 of it,
// else 0: the FLAGBSQORHO and FLAGBSQOU slots of pflag, packed as
// FLAGBSQORHO | FLAGBSQOU << 2.  With LIMADJUST = FLUXADJUST = 0 they change
// no state; the last stage's values are what the reference leaves in pflag.
// A state whose u^t has no real solution sets ERR_UTCALC_DISCR, as the
// reference's FAILSTATEMENT ends the step.
constexpr double BSQORHOLIMIT = 20.0, BSQOULIMIT = 100.0;
__global__ void bsqflags_kernel(Dims d, const double *__restrict__ pv, const double *__restrict__ G,
                                unsigned char *__restrict__ bf, Scalars *sc) {
  const long long z = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= d.nz) return;
  const int k = (int)(z % d.nt3) - d.g3;
  const long long r = z / d.nt3;
  const int j = (int)(r % d.nt2) - d.g2;
  const int i = (int)(r / d.nt2) - d.g1;
  double pr[NPR];
  load_prim(pv, d, z, pr);
  Metric m;
  load_metric(G, d, gix(d, i, j), G_CENT, m);
  State q;
  if (get_state(pr, m, q)) {
    atomicOr(&sc->err, ERR_UTCALC_DISCR);
    bf[z] = 0;
    return;
  }
  const double bsq = dot4(q.bcon, q.bcov);
  int f0, f3;
  if (bsq / pr[RHO] > BSQORHOLIMIT) f0 = 2;
  else if (bsq / pr[RHO] > 0.9 * BSQORHOLIMIT) f0 = 1;
  else f0 = 0;
  if (bsq / pr[UU] > BSQOULIMIT) f3 = 2;
  else if (bsq / pr[UU] > 0.9 * BSQOULIMIT) f3 = 1;
  else f3 = 0;
  bf[z] = (unsigned char)(f0 | (f3 << 2));
}

__global__ void bound_pflag_kernel(Dims d, Params P, int *pflag, const Scalars *sc) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  // a finished domain is frozen: its ghost flags keep the values of its last step
  if (t >= d.nz || sc->done) return;
  int k = (int)(t % d.nt3) - d.g3;
  long long r = t / d.nt3;
  int j = (int)(r % d.nt2) - d.g2;
  int i = (int)(r / d.nt2) - d.g1;
  bool gi = (i < 0 || i >= d.n1), gj = (j < 0 || j >= d.n2), gk = (k < 0 || k >= d.n3);
  if (!(gi || gj || gk)) return;
  int si = map_idx(i, d.n1, P.bc[1], P.bc[0]);
  int sj = map_idx(j, d.n2, P.bc[3], P.bc[2]);
  int sk = map_idx(k, d.n3, P.bc[5], P.bc[4]);
  pflag[t] = pflag[zix(d, si, sj, sk)];
}

// Batch of 1D instances: every instance's ghost cells are a plain copy of its
// first / last active cell (bounds.c OUTFLOW, bounds.c:84-135, 218-292), for
// the primitives (pv != nullptr) or the failure flags (pflag != nullptr).
__global__ void bound_batch_kernel(Dims d, Params P, double *pv, int *pflag) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= d.nz) return;
  int i = (int)t - d.g1;  // the batch line is 1D
  const Inst &I = P.inst[P.cell_inst[t]];
  // a finished instance is frozen: its ghosts keep the values of its last step
  if (I.done) return;
  int loc = i - I.i0;
  int src;
  if (loc < 0) src = I.i0;
  else if (loc >= I.n) src = I.i0 + I.n - 1;
  else return;
  long long zs = zix(d, src, 0, 0);
  if (pv) {
#pragma unroll
    for (int v = 0; v < NPR; v++) pv[(long long)v * d.nz + t] = pv[(long long)v * d.nz + zs];
  }
  if (pflag) pflag[t] = pflag[zs];
}

// ---------------------------------------------------------------------------
// post_fixup (fixup.c:37-96)
// ---------------------------------------------------------------------------
// fixup_checksolution (fixup.c:460-560), part 1: gamma on i,j,k = -1..N and
// the list of active candidate zones (gamma >= 2)
__global__ void checksol_gamma_kernel(Dims d, Params P, Box box, const double *__restrict__ pv,
                                      const double *__restrict__ G,
                                      double *__restrict__ gammacheck, long long *__restrict__ cand, int cap,
                                      Scalars *sc) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= box.size()) return;
  int i, j, k;
  box_ijk(box, t, i, j, k);
  long long z = zix(d, i, j, k);
  Metric m;
  load_metric(G, d, gix(d, i, j), G_CENT, m);
  double pr[NPR];
  load_prim(pv, d, z, pr);
  double gamma = 0.0;
  if (gamma_calc(pr, m, &gamma)) atomicOr(&sc->err, ERR_UTCALC_DISCR);
  gammacheck[z] = gamma;
  bool activez = (i >= 0 && i < d.n1 && j >= 0 && j < d.n2 && k >= 0 && k < d.n3);
  if (P.cell_inst) {
    const Inst &I = P.inst[P.cell_inst[z]];
    int loc = i - I.i0;
    activez = (loc >= 0 && loc < I.n && !I.done);
  }
  if (activez && gamma >= 2.0 && !sc->done) {
    int slot = atomicAdd(&sc->ncand, 1);
    if (slot < cap) cand[slot] = z;
    else atomicOr(&sc->overflow, 1);
  }
}

// In the reference the candidates are visited in loop order (i, then j, then
// k) and each visit may overwrite the zone's pflag with 12/13, which later
// visits of its neighbours read.  The zone index z is lexicographic in
// (i,j,k), so "visited earlier" is "smaller z".  Four kernels resolve it:
//   checksol_map_kernel     candidate slots in candmap, the original flags;
//   checksol_prep_kernel    per candidate, what does not change while the
//                           decisions settle: for each of its 8 neighbours
//                           (fixup.c:508-526) the vote bits of the gamma and
//                           u ratios (the divisions), whether a neighbour's
//                           flag is fixed and not failed (a non-candidate or
//                           a later candidate: its original flag) and whether
//                           it is an earlier candidate (its decision counts);
//                           the decision of every candidate that earlier
//                           ones cannot change, the list of the others;
//   checksol_resolve_kernel one block iterating a fixpoint over that list in
//                           which every candidate sees the current decision
//                           of its earlier candidate neighbours and the fixed
//                           flags of everything else; the dependencies point
//                           to strictly earlier zones, so the fixpoint is
//                           unique and a chain of length L settles after L
//                           sweeps: exactly the reference's sequential result;
//   checksol_apply_kernel   the decisions into pflag, candmap back to -1.
// A failed neighbour's ratio is -1 in the reference, whose |.| = 1 votes for
// nothing, so a neighbour's vote is its precomputed bit while it is not
// failed; the votes count only while neighbour 0's ratio is >= 0, i.e. while
// neighbour 0 is not failed and its gamma ratio is not negative or NaN
// (pd[0] >= 0 gates every vote in fixup.c:530-540).
__device__ __forceinline__ void checksol_neighbours(const Dims &d, long long z, long long nb[8]) {
  const long long o1 = (long long)d.nt2 * d.nt3, o2 = d.nt3;
  // neighbour order of fixup.c:508-526
  nb[0] = z + d.s2 * o2;
  nb[1] = z - d.s2 * o2;
  nb[2] = z + d.s1 * o1;
  nb[3] = z - d.s1 * o1;
  nb[4] = z + d.s1 * o1 + d.s2 * o2;
  nb[5] = z + d.s1 * o1 - d.s2 * o2;
  nb[6] = z + d.s1 * o1 + d.s2 * o2;
  nb[7] = z - d.s1 * o1 - d.s2 * o2;
}

__constant__ int kChecksolCodes[3] = {0, UTOPRIMFAILGAMMAPERC, UTOPRIMFAILUPERC};

// The vote of fixup_checksolution for one candidate (fixup.c:530-556) from
// its packed bits and the "not failed" mask of its neighbours: 0 = keep the
// flag, 1 = UTOPRIMFAILGAMMAPERC, 2 = UTOPRIMFAILUPERC.
__device__ __forceinline__ int checksol_vote(unsigned int b, unsigned int ok) {
  int vote0 = 0, vote1 = 0, numvotes = 0;
  if (ok & 1u) {
    vote0 = __popc(ok & b & 0xffu);
    vote1 = __popc(ok & (b >> 8) & 0xffu);
    numvotes = 8;
  }
  int v = 0;
  if (vote0 > numvotes * 0.5) v = 1;
  if (vote1 > numvotes * 0.5) v = 2;
  return v;
}

__global__ void checksol_map_kernel(const long long *__restrict__ cand, const int *__restrict__ pflag, int *candmap,
                                    int *orig, int cap, const Scalars *sc) {
  int n = sc->ncand;
  if (n > cap) n = cap;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    const long long z = cand[a];
    candmap[z] = a;
    orig[a] = pflag[z];
  }
}

// packed per candidate: bits 0-7 gamma vote, 8-15 u vote, 16-23 fixed
// neighbour not failed, 24-31 neighbour is an earlier candidate.  The
// earlier candidates' decisions can change this one's when neighbour 0 is
// such a candidate or when the vote differs between all of them failed and
// all of them not (the votes only grow with more neighbours not failed):
// those candidates go to deplist with their original flag as the first
// guess; every other candidate's decision is final here.
__global__ void checksol_prep_kernel(Dims d, const double *__restrict__ pv, const double *__restrict__ gammacheck,
                                     const int *__restrict__ pflag, const long long *__restrict__ cand,
                                     const int *__restrict__ candmap, const int *__restrict__ orig,
                                     int *__restrict__ dec, unsigned int *__restrict__ bits,
                                     int *__restrict__ deplist, int cap, Scalars *sc) {
  int n = sc->ncand;
  if (n > cap) n = cap;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    const long long z = cand[a];
    const double gc = gammacheck[z], uc = pv[(long long)UU * d.nz + z];
    long long nb[8];
    checksol_neighbours(d, z, nb);
    unsigned int v0 = 0, v1 = 0, okfix = 0, earlier = 0;
    bool gate = true;
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const double pd = gammacheck[nb[q]] / gc;
      const double pd2 = pv[(long long)UU * d.nz + nb[q]] / uc;
      if (q == 0) gate = pd >= 0.0;
      if ((fabs(pd) > 2.0) || (fabs(pd) < 1.0 / 2.0)) v0 |= 1u << q;
      if ((fabs(pd2) > 10.0) || (fabs(pd2) < 1.0 / 10.0)) v1 |= 1u << q;
      if (nb[q] < z && candmap[nb[q]] >= 0) earlier |= 1u << q;
      else if (pflag[nb[q]] <= UTOPRIMNOFAIL) okfix |= 1u << q;
    }
    // a not-failed neighbour 0 with a negative (or NaN) ratio gates all votes
    if (!gate) v0 = v1 = 0;
    const unsigned int bw = v0 | (v1 << 8) | (okfix << 16) | (earlier << 24);
    bits[a] = bw;
    const int vlo = checksol_vote(bw, okfix);
    if (earlier != 0 && ((earlier & 1u) || vlo != checksol_vote(bw, okfix | earlier))) {
      dec[a] = orig[a];
      deplist[atomicAdd(&sc->ndep, 1)] = a;
    } else {
      dec[a] = vlo ? kChecksolCodes[vlo] : orig[a];
    }
  }
}

// one block: sweeps over the dependent candidates until no decision changes
__global__ void __launch_bounds__(1024) checksol_resolve_kernel(Dims d, const long long *__restrict__ cand,
                                                                const int *__restrict__ candmap,
                                                                const int *__restrict__ orig, int *dec,
                                                                const unsigned int *__restrict__ bits,
                                                                const int *__restrict__ deplist, int cap, Scalars *sc) {
  int m = sc->ndep;
  if (m > cap) m = cap;
  if (m == 0) return;
  __shared__ int changed;
  // a chain can be at most m long; the sweep count is also capped so that a
  // pathological input ends with an error bit instead of a long kernel
  const int max_sweeps = m + 1 < 4096 ? m + 1 : 4096;
  for (int sweep = 0; sweep < max_sweeps; sweep++) {
    if (sweep == max_sweeps - 1 && threadIdx.x == 0 && max_sweeps < m + 1) atomicOr(&sc->overflow, 4);
    if (threadIdx.x == 0) changed = 0;
    __syncthreads();
    for (int e = threadIdx.x; e < m; e += blockDim.x) {
      const int a = deplist[e];
      const unsigned int b = bits[a];
      unsigned int ok = (b >> 16) & 0xffu;
      const unsigned int earlier = b >> 24;
      long long nb[8];
      checksol_neighbours(d, cand[a], nb);
#pragma unroll
      for (int q = 0; q < 8; q++)
        if ((earlier >> q) & 1u)
          if (dec[candmap[nb[q]]] <= UTOPRIMNOFAIL) ok |= 1u << q;
      const int v = checksol_vote(b, ok);
      const int nd = v ? kChecksolCodes[v] : orig[a];
      if (nd != dec[a]) {
        dec[a] = nd;
        changed = 1;
      }
    }
    __syncthreads();
    if (!changed) break;
    __syncthreads();
  }
}

// the decisions into pflag; candmap back to -1
__global__ void checksol_apply_kernel(const long long *__restrict__ cand, const int *__restrict__ dec, int *pflag,
                                      int *candmap, int cap, const Scalars *sc) {
  int n = sc->ncand;
  if (n > cap) n = cap;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    const long long z = cand[a];
    pflag[z] = dec[a];
    candmap[z] = -1;
  }
}

// fixup_utoprim (fixup.c:669-1470), part 1: list the active failed zones
__global__ void fixup_collect_kernel(Dims d, Params P, Box box, const int *__restrict__ pflag,
                                     long long *__restrict__ list, int cap, Scalars *sc) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= box.size()) return;
  int i, j, k;
  box_ijk(box, t, i, j, k);
  long long z = zix(d, i, j, k);
  if (P.cell_inst) {
    const Inst &I = P.inst[P.cell_inst[z]];
    int loc = i - I.i0;
    if (!(loc >= 0 && loc < I.n && !I.done)) return;
  }
  if (pflag[z] != 0 && !sc->done) {
    int slot = atomicAdd(&sc->nfixlist, 1);
    if (slot < cap) list[slot] = z;
    else atomicOr(&sc->overflow, 2);
  }
}

// counter of a failure code that becomes fixed (fixup.c:1340-1425, with the
// reference's settings STEPOVERNEG*=-1 and DOCOUNTNEG*=1)
__device__ __forceinline__ int failure_counter(int f) {
  if (f == UTOPRIMFAILRHONEG) return CNT_UTOPRIMFAILRHONEG;
  if (f == UTOPRIMFAILUNEG || f == UTOPRIMFAILU2AVG1 || f == UTOPRIMFAILU2AVG2) return CNT_UTOPRIMFAILUNEG;
  if (f == UTOPRIMFAILRHOUNEG) return CNT_UTOPRIMFAILRHOUNEG;
  if (f == UTOPRIMFAILGAMMAPERC) return CNT_GAMMAPERC;
  if (f == UTOPRIMFAILUPERC) return CNT_UPERC;
  return CNT_UTOPRIMFAILCONV;  // the non-convergence and NaN codes
}

__device__ __forceinline__ bool becomes_fixed(int f, int finalstep) {
  // accounting branch of fixup.c:1399-1470: which codes are reset to
  // UTOPRIMFAILFIXED (STEPOVERNEG*=-1, DOCOUNTNEG*=1)
  if (f == 0) return false;
  if (f == UTOPRIMFAILRHONEG || f == UTOPRIMFAILUNEG || f == UTOPRIMFAILU2AVG1 || f == UTOPRIMFAILU2AVG2 ||
      f == UTOPRIMFAILRHOUNEG)
    return finalstep != 0;
  return true;
}

// part 2: new primitives of each listed zone.  The reference averages
// neighbour values from a snapshot of pv taken before the sweep (ptoavg) and
// tests neighbour pflags that earlier visits may already have reset to -1; a
// neighbour's reset depends only on its own code, so "earlier active failed
// neighbour that becomes fixed" counts as good here.
__global__ void fixup_compute_kernel(Dims d, Params P, const double *__restrict__ pv, const int *__restrict__ pflag,
                                     const double *__restrict__ G, const long long *__restrict__ list,
                                     double *__restrict__ outv, int cap, int finalstep, Scalars *sc) {
  int n = sc->nfixlist;
  if (n > cap) n = cap;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
  long long z = list[a];
  int k = (int)(z % d.nt3) - d.g3;
  long long r = z / d.nt3;
  int j = (int)(r % d.nt2) - d.g2;
  int i = (int)(r / d.nt2) - d.g1;
  int mypflag = pflag[z];
  double pr[NPR];
  load_prim(pv, d, z, pr);
  int err = 0;
  bool fixed = (mypflag == UTOPRIMFAILUNEG || mypflag == UTOPRIMFAILRHONEG || mypflag == UTOPRIMFAILRHOUNEG);
  if (!fixed) {
    Metric m;
    load_metric(G, d, gix(d, i, j), G_CENT, m);
    double gamma = 1.0;
    if (gamma_calc(pr, m, &gamma)) err |= ERR_UTCALC_DISCR;
    if (gamma > P.gammamax) gamma = P.gammamax;
    int startpl, endpl, looptype;
    if (mypflag == UTOPRIMFAILU2AVG1 || mypflag == UTOPRIMFAILU2AVG2) {
      startpl = UU;
      endpl = UU;
      looptype = 1;
    } else {
      startpl = RHO;
      endpl = U3;
      looptype = 0;
    }
    double mysum0[5] = {0, 0, 0, 0, 0}, mysum1[5] = {0, 0, 0, 0, 0}, lastmin[5] = {1E50, 1E50, 1E50, 1E50, 1E50};
    const int s1 = d.s1, s2 = d.s2, s3 = d.s3;
    const int rnx = (s1 == 1) ? 3 : 1, rny = (s2 == 1) ? 3 : 1;
    const int npow = s1 + s2 + s3;
    int p3 = 1;
    for (int q = 0; q < npow; q++) p3 *= 3;
    const int numupairs = (p3 - 1) / 2;
    int numavg0 = 0, numavg1 = 0;
    for (int qq = 0; qq < numupairs; qq++) {
      int ii = (qq % rnx) - s1;
      int jj = ((qq % (rnx * rny)) / rnx) - s2;
      int kk = (qq / (rnx * rny)) - s3;
      long long za = zix(d, i + ii, j + jj, k + kk), zb = zix(d, i - ii, j - jj, k - kk);
      int ia = i + ii, ja = j + jj, ka = k + kk, ib = i - ii, jb = j - jj, kb = k - kk;
      bool act_a = ia >= 0 && ia < d.n1 && ja >= 0 && ja < d.n2 && ka >= 0 && ka < d.n3;
      bool act_b = ib >= 0 && ib < d.n1 && jb >= 0 && jb < d.n2 && kb >= 0 && kb < d.n3;
      int fa = pflag[za], fb = pflag[zb];
      int thisnotfail = (fa <= UTOPRIMNOFAIL) || (act_a && za < z && becomes_fixed(fa, finalstep));
      int thatnotfail = (fb <= UTOPRIMNOFAIL) || (act_b && zb < z && becomes_fixed(fb, finalstep));
      numavg1 += (pv[(long long)UU * d.nz + za] > 0.0);
      numavg1 += (pv[(long long)UU * d.nz + zb] > 0.0);
      numavg0 += thisnotfail + thatnotfail;
      for (int pl = startpl; pl <= endpl; pl++) {
        double va = pv[(long long)pl * d.nz + za], vb = pv[(long long)pl * d.nz + zb];
        if (looptype == 0) {
          double add = va * thisnotfail + vb * thatnotfail;
          if (qq % 2) mysum1[pl] += add;
          else mysum0[pl] += add;
        } else {
          if (va >= 0.0) lastmin[pl] = min_macro(lastmin[pl], va);
          if (vb >= 0.0) lastmin[pl] = min_macro(lastmin[pl], vb);
        }
      }
    }
    int numavg;
    if (looptype == 0) {
      if (numavg0 != 0)
        for (int pl = startpl; pl <= endpl; pl++) pr[pl] = (mysum0[pl] + mysum1[pl]) / ((double)(numavg0));
      numavg = numavg0;
    } else {
      if (numavg1 != 0)
        for (int pl = startpl; pl <= endpl; pl++) pr[pl] = lastmin[pl];
      numavg = numavg1;
    }
    if (mypflag == UTOPRIMFAILU2AVG2) numavg++;
    if (numavg == 0) {
      for (int pl = startpl; pl <= endpl; pl++) {
        const double *pp = pv + (long long)pl * d.nz;
        double a41 = (0.25 * ((pp[zix(d, i, j + s2, k)] + pp[zix(d, i, j - s2, k)]) +
                              (pp[zix(d, i - s1, j, k)] + pp[zix(d, i + s1, j, k)])));
        double a42 = (0.25 * ((pp[zix(d, i + s1, j + s2, k)] + pp[zix(d, i + s1, j - s2, k)]) +
                              (pp[zix(d, i - s1, j + s2, k)] + pp[zix(d, i - s1, j - s2, k)])));
        pr[pl] = 0.5 * (a41 + a42);
      }
    }
    // the averaged state's gamma limited to the zone's own (fixup.c:1326),
    // counted by limit_gamma when it rescaled (fixup.c:1913)
    if (limit_gamma(gamma, pr, m, &err) == -1) ffc_count(P, d.nz, z, CNT_LIMITGAMMAACT);
  }
#pragma unroll
  for (int v = 0; v < 5; v++) outv[(long long)a * 5 + v] = pr[v];
  if (err) atomicOr(&sc->err, err);
  }
}

__global__ void fixup_scatter_kernel(Dims d, Params P, double *pv, int *pflag, const long long *__restrict__ list,
                                     const double *__restrict__ outv, int cap, int finalstep, Scalars *sc,
                                     const double *__restrict__ G, double *__restrict__ ufv) {
  int n = sc->nfixlist;
  if (n > cap) n = cap;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    long long z = list[a];
    double pr0[NPR], pr[NPR];
    if (ufv && finalstep) load_prim(pv, d, z, pr0);
#pragma unroll
    for (int v = 0; v < 5; v++) pv[(long long)v * d.nz + z] = outv[(long long)a * 5 + v];
    int f = pflag[z];
    if (becomes_fixed(f, finalstep)) {
      if (ufv && finalstep) {
        // diag_fixup(pr0 = ptoavg, pv) (fixup.c:1428), pr0 = the zone before the fixup
        int k = (int)(z % d.nt3) - d.g3;
        long long r = z / d.nt3;
        int j = (int)(r % d.nt2) - d.g2;
        int i = (int)(r / d.nt2) - d.g1;
        (void)k;
        Metric m;
        load_metric(G, d, gix(d, i, j), G_CENT, m);
#pragma unroll
        for (int v = 0; v < 5; v++) pr[v] = outv[(long long)a * 5 + v];
#pragma unroll
        for (int v = 5; v < NPR; v++) pr[v] = pr0[v];
        int err = 0;
        fv_diag_fixup(pr0, pr, m, P.gam, ufv, z, d.nz, &err);
        if (err) atomicOr(&sc->err, err);
      }
      // diag_fixup's count of the failure type (fixup.c:1428)
      if (f > 0) ffc_count(P, d.nz, z, failure_counter(f));
      pflag[z] = UTOPRIMFAILFIXED;
      atomicAdd(&sc->nfixed, 1);
    }
  }
}

// B components of the fluxes after flux_ct (fluxct.c:724-781) on the faces
// the update reads; used only to hand fluxes back through hgpu_fluxcalc (the
// update kernel rebuilds them from the EMFs on the fly)
__global__ void bflux_kernel(Dims d, int dir, Box box, const double *__restrict__ E, double *__restrict__ F) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= box.size()) return;
  int i, j, k;
  box_ijk(box, t, i, j, k);
  long long z = zix(d, i, j, k), nz = d.nz;
  const long long o1 = (long long)d.nt2 * d.nt3, o2 = d.nt3, o3 = 1;
  const double *e1 = E, *e2 = E + nz, *e3 = E + 2 * nz;
  if (dir == 1) {
    F[B1 * nz + z] = 0.;
    F[B2 * nz + z] = 0.5 * (e3[z] + e3[z + d.s2 * o2]);
    F[B3 * nz + z] = -0.5 * (e2[z] + e2[z + d.s3 * o3]);
  } else if (dir == 2) {
    F[B1 * nz + z] = -0.5 * (e3[z] + e3[z + d.s1 * o1]);
    F[B2 * nz + z] = 0.;
    F[B3 * nz + z] = 0.5 * (e1[z] + e1[z + d.s3 * o3]);
  } else {
    F[B1 * nz + z] = 0.5 * (e2[z] + e2[z + d.s1 * o1]);
    F[B2 * nz + z] = -0.5 * (e1[z] + e1[z + d.s2 * o2]);
    F[B3 * nz + z] = 0.;
  }
}

// ndt (advance.c:231) and the dt update of step_ch (step_ch.c:236-247)
__global__ void finalize_kernel(Params P, Scalars *sc, int advance_time) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double n1 = __longlong_as_double((long long)sc->ndtbits[1]);
  double n2 = __longlong_as_double((long long)sc->ndtbits[2]);
  double n3 = __longlong_as_double((long long)sc->ndtbits[3]);
  double ndt = P.defcon * 1. / (1. / n1 + 1. / n2 + 1. / n3);
  if (advance_time && !sc->done) {
    double dt = sc->dt;
    sc->t += dt;
    if (ndt > P.safe * dt) ndt = P.safe * dt;
    dt = ndt;
    if (sc->t + dt > P.tf) dt = P.tf - sc->t;
    sc->dt = dt;
    // the reference's main loop runs while t < tf (main.c:33)
    sc->nsteps++;
    if (!(sc->t < P.tf)) sc->done = 1;
  }
  // keep the last ndt where the host can read it
  sc->ndtbits[0] = (unsigned long long)__double_as_longlong(ndt);
}

// batch: per-instance ndt combine and dt update (the same formulas per
// instance; dims of size 1 contribute BIG as in the one-domain case)
__global__ void finalize_batch_kernel(Params P, int advance_time) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= P.ninst) return;
  Inst &I = P.inst[b];
  double n1 = __longlong_as_double((long long)I.ndtbits);
  double ndt = P.defcon * 1. / (1. / n1 + 1. / BIGNUM + 1. / BIGNUM);
  if (advance_time) {
    if (I.done) return;
    double dt = I.dt;
    I.t += dt;
    I.nsteps++;
    if (ndt > P.safe * dt) ndt = P.safe * dt;
    dt = ndt;
    if (I.t + dt > I.tf) dt = I.tf - I.t;
    I.dt = dt;
    if (!(I.t < I.tf)) I.done = 1;
  } else {
    I.dt = ndt;
  }
}

__global__ void reset_batch_kernel(Params P) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= P.ninst) return;
  P.inst[b].ndtbits = (unsigned long long)__double_as_longlong(BIGNUM);
}

__global__ void reset_stage_kernel(Scalars *sc) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  unsigned long long big = (unsigned long long)__double_as_longlong(BIGNUM);
  sc->ndtbits[1] = big;
  sc->ndtbits[2] = big;
  sc->ndtbits[3] = big;
  sc->nfail = 0;
  sc->ncand = 0;
  sc->ndep = 0;
  sc->nfixlist = 0;
}

// reference AoS [zone][8] <-> device SoA [8][zone]
// Active zones only, host layout [n1][n2][n3][8] (and [n1][n2][n3] for the
// flags) <-> the device's planes with ghosts: thread per (zone, primitive),
// so the host-layout side is read/written contiguously.
__global__ void active_scatter_kernel(Dims d, const double *__restrict__ a, double *__restrict__ s) {
  const long long na = (long long)d.n1 * d.n2 * d.n3;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= na * NPR) return;
  const long long z = t / NPR;
  const int pl = (int)(t % NPR);
  const int k = (int)(z % d.n3), j = (int)((z / d.n3) % d.n2), i = (int)(z / ((long long)d.n2 * d.n3));
  s[(long long)pl * d.nz + zix(d, i, j, k)] = a[t];
}

__global__ void active_gather_kernel(Dims d, const double *__restrict__ s, double *__restrict__ a) {
  const long long na = (long long)d.n1 * d.n2 * d.n3;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= na * NPR) return;
  const long long z = t / NPR;
  const int pl = (int)(t % NPR);
  const int k = (int)(z % d.n3), j = (int)((z / d.n3) % d.n2), i = (int)(z / ((long long)d.n2 * d.n3));
  a[t] = s[(long long)pl * d.nz + zix(d, i, j, k)];
}

__global__ void active_gather_flags_kernel(Dims d, const int *__restrict__ f, int *__restrict__ a) {
  const long long na = (long long)d.n1 * d.n2 * d.n3;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= na) return;
  const int k = (int)(t % d.n3), j = (int)((t / d.n3) % d.n2), i = (int)(t / ((long long)d.n2 * d.n3));
  a[t] = f[zix(d, i, j, k)];
}

__global__ void aos_to_soa_kernel(const double *__restrict__ a, double *__restrict__ s, long long nz) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nz * NPR) return;
  long long z = t / NPR;
  int v = (int)(t % NPR);
  s[(long long)v * nz + z] = a[t];
}
__global__ void soa_to_aos_kernel(const double *__restrict__ s, double *__restrict__ a, long long nz) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nz * NPR) return;
  long long z = t / NPR;
  int v = (int)(t % NPR);
  a[t] = s[(long long)v * nz + z];
}

// geometry packing: the reference-layout arrays (per (i,j): gcov and gcon
// [8 locations][16], gcovpert [8][4], gdet [8], conn [64], floors [2]) into
// the SoA planes: FACE1/FACE2/FACE3/CENT x {gcov 16, gcon 16, 1+g_tt, gdet},
// the three corner gdets, conn, floors
constexpr int GRAW_WORDS = 128 + 128 + 32 + 8 + 64 + 2;
__global__ void pack_geometry_kernel(const double *__restrict__ raw, long long nij, double *__restrict__ G) {
  long long ij = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (ij >= nij) return;
  const double *rcov = raw, *rcon = raw + 128 * nij, *rpert = raw + 256 * nij, *rgdet = raw + 288 * nij,
               *rconn = raw + 296 * nij, *rfl = raw + 360 * nij;
  const int locs[4] = {R_FACE1, R_FACE2, R_FACE3, R_CENT};
#pragma unroll
  for (int s = 0; s < 4; s++) {
    const int L = locs[s];
#pragma unroll
    for (int q = 0; q < 16; q++) {
      G[(long long)(s * GLOC + q) * nij + ij] = rcov[(ij * 8 + L) * 16 + q];
      G[(long long)(s * GLOC + 16 + q) * nij + ij] = rcon[(ij * 8 + L) * 16 + q];
    }
    G[(long long)(s * GLOC + 32) * nij + ij] = rpert[(ij * 8 + L) * 4 + 0];
    G[(long long)(s * GLOC + 33) * nij + ij] = rgdet[ij * 8 + L];
  }
  G[(long long)(G_CORN + 0) * nij + ij] = rgdet[ij * 8 + R_CORN1];
  G[(long long)(G_CORN + 1) * nij + ij] = rgdet[ij * 8 + R_CORN2];
  G[(long long)(G_CORN + 2) * nij + ij] = rgdet[ij * 8 + R_CORN3];
#pragma unroll 8
  for (int q = 0; q < 64; q++) G[(long long)(G_CONN + q) * nij + ij] = rconn[ij * 64 + q];
  G[(long long)(G_FLOOR + 0) * nij + ij] = rfl[ij * 2 + 0];
  G[(long long)(G_FLOOR + 1) * nij + ij] = rfl[ij * 2 + 1];
}

// batched inversion on arbitrary per-zone metrics (hgpu_utoprim_batch,
// hgpu_utoprimgen_batch)
template <int UV>
__global__ void utoprim_batch_kernel(const double *__restrict__ U, const double *__restrict__ gcov,
                                     const double *__restrict__ gcon, const double *__restrict__ gdet, double *pr,
                                     int *pflag, long long n, double gam, double gammafail,
                                     unsigned long long *iters) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long it_total = 0;
  if (t < n) {
    Metric m;
#pragma unroll
    for (int q = 0; q < 16; q++) {
      m.gcov[q] = gcov[t * 16 + q];
      m.gcon[q] = gcon[t * 16 + q];
    }
    m.gcovpert_tt = 0.0;
    m.g = gdet[t];
    double u[NPR], p[NPR];
#pragma unroll
    for (int v = 0; v < NPR; v++) {
      u[v] = U[t * NPR + v];
      p[v] = pr[t * NPR + v];
    }
    int it = 0;
    pflag[t] = utoprimgen_v<UV>(u, m, gam, gammafail, p, &it);
#pragma unroll
    for (int v = 0; v < NPR; v++) pr[t * NPR + v] = p[v];
    it_total = (unsigned long long)it;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) it_total += __shfl_xor_sync(0xffffffffu, it_total, o);
  if ((threadIdx.x & 31) == 0 && it_total) atomicAdd(iters, it_total);
}

inline unsigned grid_for(long long n, int block) { return (unsigned)((n + block - 1) / block); }

// Dynamic shared memory the WENO5 kernel may use per block (its tilings are
// sized to fit, for FP64 elements)
constexpr size_t W5_SMEM_MAX = 72 * 1024;

// Cost of a WENO5 tiling in block rounds (a stage's items over the 256
// threads, whole rounds), weighted by each stage's work per item, plus the
// barriers: S (shock factor) once, then per primitive Y (line loads), A
// (SMONO + weights), R (ratios), F (face values) and four barriers.
double w5_cost(int nout, long long nlines, int lb, int w, bool fs) {
  const int nseg = (nout + lb - 1) / lb;
  const long long ntile = (nlines + w - 1) / w;
  const int tl = W5_THREADS / w;
  auto rounds = [&](int n) {
    return fs ? (double)((n + tl - 1) / tl) : (double)(((long long)n * w + W5_THREADS - 1) / W5_THREADS);
  };
  double per = 0.0;
  for (int sgi = 0; sgi < 2; sgi++) {
    const int nv = sgi == 0 ? lb : nout - (nseg - 1) * lb;  // full tiles, then the last one
    const double count = sgi == 0 ? (double)(nseg - 1) : 1.0;
    per += count * (rounds(nv) +
                    8.0 * (0.3 * rounds(nv + 10) + 2.0 * rounds(nv + 6) + 0.3 * rounds(nv + 2) + 1.5 * rounds(nv) + 2.0));
  }
  return per * (double)ntile;
}

// WENO5 tilings of the output box b along direction dir, best first (at
// most `max` of them, one per line count).  Lines whose cells are contiguous
// in memory (x3, or any direction of a domain flat across it) are walked
// along by consecutive threads, a warp or more per line; the others across,
// consecutive threads on neighbouring lines (x3 fastest), at least 8 of them
// for 64-byte rows.  Every tiling fits the shared-memory budget.
int w5_candidates(const Dims &d, const Box &b, int dir, W5Tile *out, int max) {
  const int nout = dir == 1 ? b.ni : (dir == 2 ? b.nj : b.nk);
  const long long nlines = dir == 1 ? (long long)b.nj * b.nk : (dir == 2 ? (long long)b.ni * b.nk : (long long)b.ni * b.nj);
  const long long stride = dir == 1 ? (long long)d.nt2 * d.nt3 : (dir == 2 ? (long long)d.nt3 : 1LL);
  const bool fs = stride == 1;
  double cost[6];
  W5Tile cand[6];
  int n = 0;
  const int ws[] = {1, 2, 4, 8, 16, 32};
  for (int w : ws) {
    if (w > nlines && w > 1) break;
    if (!fs && w < 8 && nlines >= 8) continue;
    if (fs && w > 8 && nout >= 32) continue;
    double best = -1.0;
    int blb = 0;
    for (int nseg = 1; nseg <= nout; nseg++) {
      const int lb = (nout + nseg - 1) / nseg;
      if (w5_smem_bytes(lb, w, 8) > (long long)W5_SMEM_MAX) continue;
      if (lb < 8 && nseg > 1) break;
      const double c = w5_cost(nout, nlines, lb, w, fs);
      if (best < 0.0 || c < best) {
        best = c;
        blb = lb;
      }
      if (nseg > 64 && lb < 256) break;
    }
    if (blb == 0) continue;
    W5Tile t;
    t.box = b;
    t.nlines = (int)nlines;
    t.fast_s = fs;
    t.lb = blb;
    t.w = w;
    t.nseg = (nout + blb - 1) / blb;
    t.ntile = (int)((nlines + w - 1) / w);
    t.wshift = 0;
    while ((1 << t.wshift) < w) t.wshift++;
    cost[n] = best;
    cand[n++] = t;
  }
  // best first
  for (int i = 1; i < n; i++)
    for (int j = i; j > 0 && cost[j] < cost[j - 1]; j--) {
      std::swap(cost[j], cost[j - 1]);
      std::swap(cand[j], cand[j - 1]);
    }
  if (n > max) n = max;
  for (int i = 0; i < n; i++) out[i] = cand[i];
  return n;
}

W5Tile w5_tiling(const Dims &d, const Box &b, int dir) {
  W5Tile t[1];
  w5_candidates(d, b, dir, t, 1);
  return t[0];
}

// the WENO5 kernels may use up to W5_SMEM_MAX of dynamic shared memory
void w5_allow_smem_all() {
  static std::once_flag once;
  std::call_once(once, [] {
    const int m = (int)W5_SMEM_MAX;
    const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    cudaFuncSetAttribute(weno5_kernel<1, false, double, kWenoMB[0]>, a, m);
    cudaFuncSetAttribute(weno5_kernel<1, true, double, kWenoMB[0]>, a, m);
    cudaFuncSetAttribute(weno5_kernel<2, false, double, kWenoMB[0]>, a, m);
    cudaFuncSetAttribute(weno5_kernel<2, true, double, kWenoMB[0]>, a, m);
    cudaFuncSetAttribute(weno5_kernel<3, true, double, kWenoMB[0]>, a, m);
    cudaFuncSetAttribute(weno5_kernel<1, false, double, kWenoMB[1]>, a, m);
    cudaFuncSetAttribute(weno5_kernel<1, true, double, kWenoMB[1]>, a, m);
    cudaFuncSetAttribute(weno5_kernel<2, false, double, kWenoMB[1]>, a, m);
    cudaFuncSetAttribute(weno5_kernel<2, true, double, kWenoMB[1]>, a, m);
    cudaFuncSetAttribute(weno5_kernel<3, true, double, kWenoMB[1]>, a, m);
    cudaFuncSetAttribute(weno5_kernel<1, false, float>, a, m);
    cudaFuncSetAttribute(weno5_kernel<1, true, float>, a, m);
    cudaFuncSetAttribute(weno5_kernel<2, false, float>, a, m);
    cudaFuncSetAttribute(weno5_kernel<2, true, float>, a, m);
    cudaFuncSetAttribute(weno5_kernel<3, true, float>, a, m);
    cudaGetLastError();
  });
}

}  // namespace

// ---------------------------------------------------------------------------
// host context
// ---------------------------------------------------------------------------
enum KernelId {
  K_RESET, K_FLUX1, K_FLUX2, K_FLUX3, K_EMF, K_UPDATE, K_BOUND_GHOST, K_BOUND_POLE, K_BOUND_PFLAG, K_CHECK_GAMMA,
  K_CHECK_RESOLVE, K_FIX_COLLECT, K_FIX_COMPUTE, K_FIX_SCATTER, K_FINALIZE, K_WENO5, K_W5STATE, K_INVERT, K_OTHER, K_NKERNELS
};
static const char *kKernelNames[K_NKERNELS] = {
    "reset_stage",  "flux_x1",         "flux_x2",       "flux_x3",       "emf",           "update",
    "bound_ghost",  "bound_pole",      "bound_pflag",   "checksol_gamma", "checksol_resolve", "fixup_collect",
    "fixup_compute", "fixup_scatter",  "finalize",      "weno5",         "w5_state",      "invert",        "other"};

struct ProfEvent {
  int kid;
  cudaEvent_t a, b;
};

struct hgpu_ctx {
  long long launches = 0;
  bool profiling = false;
  std::vector<ProfEvent> pending;
  std::vector<cudaEvent_t> freelist;
  double kms[K_NKERNELS] = {0};
  long long kcount[K_NKERNELS] = {0};
  hgpu_config cfg;
  Dims d;
  Params P;
  cudaStream_t stream;
  double *p = nullptr, *pk = nullptr, *uf = nullptr, *ucum = nullptr;
  double *pk1 = nullptr;  // second intermediate state of TIMEORDER 3 and 4
  double *ui = nullptr;   // ENOFINITEVOLUME: the conserved state at the start of the step (uinitial)
  struct {
    int flux = 0, weno = 0, conserve = 0, invert = 0;  // variant index per kernel family (hgpu_autotune)
  } tune;
  double *F[4] = {nullptr, nullptr, nullptr, nullptr};
  double *E = nullptr;
  double *G = nullptr;
  int *pflag = nullptr;
  double *gammacheck = nullptr;
  long long *cand = nullptr, *fixlist = nullptr;
  int *cand_orig = nullptr, *cand_dec = nullptr, *candmap = nullptr;
  unsigned int *cand_bits = nullptr;  // checksolution: per-candidate vote and neighbour bits
  int *cand_deplist = nullptr;        // checksolution: candidates whose vote earlier ones can change
  double *fixvals = nullptr;
  int cap = 0;
  Scalars *sc = nullptr;
  double *staging = nullptr;  // AoS staging for uploads/downloads
  double *pL = nullptr, *pR = nullptr;  // WENO5 face values
  double *w5pu = nullptr;               // WENO5: per-zone dP/P state pieces (2 planes)
  unsigned char *bsqf = nullptr;        // FLAGBSQORHO | FLAGBSQOU << 2 per zone
  unsigned int *ffc = nullptr;          // failure/floor counters, NFFC planes
  double *bondi_tab = nullptr;          // Bondi-integral boundaries' coordinate data
  double *progress = nullptr;                          // 4 doubles for hg_progress_async
  W5Tile w5[4];  // WENO5 tiling per direction
  Box w5_state_box;  // zones whose dP/P state pieces some direction reads
  int *istaging = nullptr;
  // batch of 1D instances (hgpu_create_batch)
  int *cell_inst = nullptr;
  Inst *inst = nullptr;
  int ninst = 0;
  // one captured time step (hgpu_step_graph)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  long long launches_per_step = 0;
  Box face_box[4], emf_box, active_box, dq_box;
};

static cudaEvent_t take_event(hgpu_ctx *x) {
  if (!x->freelist.empty()) {
    cudaEvent_t e = x->freelist.back();
    x->freelist.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

struct ProfScope {
  hgpu_ctx *x;
  int kid;
  cudaEvent_t a = nullptr;
  ProfScope(hgpu_ctx *x_, int kid_) : x(x_), kid(kid_) {
    if (x->profiling) {
      a = take_event(x);
      cudaEventRecord(a, x->stream);
    }
  }
  ~ProfScope() {
    x->launches++;
    if (x->profiling) {
      cudaEvent_t b = take_event(x);
      cudaEventRecord(b, x->stream);
      x->pending.push_back(ProfEvent{kid, a, b});
    }
  }
};

// every launch of the library goes through this macro: it counts the launch
// and, when profiling is on, brackets it with events on the context's stream
#define LAUNCH(x, kid, kernel, grid, block, ...)                 \
  do {                                                          \
    ProfScope ps__(x, kid);                                     \
    kernel<<<(grid), (block), 0, (x)->stream>>>(__VA_ARGS__);   \
  } while (0)

static void collect_profile(hgpu_ctx *x) {
  for (auto &pe : x->pending) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, pe.a, pe.b) == cudaSuccess) {
      x->kms[pe.kid] += ms;
      x->kcount[pe.kid] += 1;
    }
    x->freelist.push_back(pe.a);
    x->freelist.push_back(pe.b);
  }
  x->pending.clear();
}

static int validate(const hgpu_config *c) {
  if (!c) return HGPU_E_INVALID;
  if (c->n1 < 1 || c->n2 < 1 || c->n3 < 1 || c->ng < 2) return HGPU_E_INVALID;
  if (c->lim != HGPU_LIM_MC && c->lim != HGPU_LIM_VANL && c->lim != HGPU_LIM_MINM && c->lim != HGPU_LIM_DONOR &&
      c->lim != HGPU_LIM_PARA && c->lim != HGPU_LIM_WENO5)
    return HGPU_E_INVALID;
  // PARA reads 3 zones beyond the faces' cells
  if (c->lim == HGPU_LIM_PARA && c->ng < 3) return HGPU_E_INVALID;
  // WENO5 reads the line up to 5 cells beyond the faces' cells -1..n
  if (c->lim == HGPU_LIM_WENO5 && c->ng < 6) return HGPU_E_INVALID;
  if (c->fluxmethod != HGPU_FLUX_HLL && c->fluxmethod != HGPU_FLUX_LAXF) return HGPU_E_INVALID;
  for (int f = 0; f < 6; f++)
    if (c->bc[f] != HGPU_BC_OUTFLOW && c->bc[f] != HGPU_BC_POLARAXIS && c->bc[f] != HGPU_BC_PERIODIC &&
        c->bc[f] != HGPU_BC_OUTFLOW_COPY && c->bc[f] != HGPU_BC_POLARAXIS_FLIP &&
        !(f == 0 && c->bc[f] == HGPU_BC_BONDIMDOTOUTFLOW) && !(f == 1 && c->bc[f] == HGPU_BC_BONDIINTOUTFLOW))
      return HGPU_E_INVALID;
  // the Bondi-integral boundaries: x1 ghosts exist, and the edge zone's
  // integrals come from the zone itself
  if ((c->bc[0] == HGPU_BC_BONDIMDOTOUTFLOW || c->bc[1] == HGPU_BC_BONDIINTOUTFLOW) && c->n1 < 2) return HGPU_E_INVALID;
  // reflections and periodic wraps read inside the active range
  if (c->n2 > 1 && c->n2 < c->ng) return HGPU_E_INVALID;
  if (c->n3 > 1 && c->n3 < c->ng) return HGPU_E_INVALID;
  if (c->n1 > 1 && c->n1 < c->ng) return HGPU_E_INVALID;
  if (c->precision != HGPU_PREC_FP64 && c->precision != HGPU_PREC_MIXED) return HGPU_E_INVALID;
  if (c->timeorder < 0 || c->timeorder > 4) return HGPU_E_INVALID;
  if (c->utoprimversion != 0 && c->utoprimversion != HGPU_UTOPRIM2DFINAL &&
      c->utoprimversion != HGPU_UTOPRIMJONNONRELCOMPAT)
    return HGPU_E_INVALID;
  if (c->doenoflux != HGPU_NOENOFLUX && c->doenoflux != HGPU_ENOFINITEVOLUME) return HGPU_E_INVALID;
  return HGPU_OK;
}

extern "C" {

int hgpu_abi_version(void) { return HGPU_ABI_VERSION; }

int hgpu_set_device(int device) {
  CUDA_TRY(cudaSetDevice(device));
  return HGPU_OK;
}

const char *hgpu_last_error(void) { return g_errbuf; }

// error text of a failing call made elsewhere in the library (host code)
void hg_set_error(const char *msg) { snprintf(g_errbuf, sizeof(g_errbuf), "%s", msg); }

void hgpu_destroy(hgpu_ctx *x) {
  if (!x) return;
  cudaStreamSynchronize(x->stream);
  if (x->graph_exec) cudaGraphExecDestroy(x->graph_exec);
  if (x->graph) cudaGraphDestroy(x->graph);
  collect_profile(x);
  for (cudaEvent_t e : x->freelist) cudaEventDestroy(e);
  void *ptrs[] = {x->p, x->pk, x->uf, x->ucum, x->F[1], x->F[2], x->F[3], x->E, x->G, x->pflag, x->gammacheck,
                  x->cand, x->fixlist, x->cand_orig, x->cand_dec, x->cand_bits, x->cand_deplist, x->candmap, x->fixvals, x->sc, x->staging, x->istaging,
                  x->pL, x->pR, x->w5pu, x->bsqf, x->ffc, x->bondi_tab, x->cell_inst, x->inst, x->progress, x->pk1, x->ui};
  for (void *q : ptrs)
    if (q) cudaFree(q);
  cudaStreamDestroy(x->stream);
  delete x;
}

// the scalar parameters every kernel takes by value
static void fill_params(Params &P, const hgpu_config *cfg) {
  P.gam = cfg->gam;
  P.cour = cfg->cour;
  P.gammamax = cfg->gammamax;
  P.gammafail = cfg->gammafail;
  P.rhominlimit = cfg->rhominlimit;
  P.uuminlimit = cfg->uuminlimit;
  P.defcon = cfg->defcon;
  P.safe = cfg->safe;
  P.tf = cfg->tf;
  P.dx1 = cfg->dx[1];
  P.dx2 = cfg->dx[2];
  P.dx3 = cfg->dx[3];
  P.lim = cfg->lim;
  P.flux = cfg->fluxmethod;
  for (int f = 0; f < 6; f++) P.bc[f] = cfg->bc[f];
  P.fvring = (cfg->doenoflux == HGPU_ENOFINITEVOLUME);
}

// Two configurations with the same allocation shape: the same device
// buffers serve both (only the by-value parameters differ).
bool hg_same_shape(const hgpu_config *a, const hgpu_config *b) {
  return a->n1 == b->n1 && a->n2 == b->n2 && a->n3 == b->n3 && a->ng == b->ng && a->lim == b->lim &&
         a->fluxmethod == b->fluxmethod && a->precision == b->precision &&
         (a->timeorder >= 3) == (b->timeorder >= 3) && a->utoprimversion == b->utoprimversion &&
         a->doenoflux == b->doenoflux;
}

// Give an idle context a new configuration of the same shape (a pool of
// contexts reuses device memory across solves): new by-value parameters,
// and the captured step graph, which holds the old ones, is dropped.
int hg_reconfigure(hgpu_ctx *x, const hgpu_config *cfg) {
  if (!x || validate(cfg) || !hg_same_shape(&x->cfg, cfg)) return HGPU_E_INVALID;
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  if (x->graph_exec) cudaGraphExecDestroy(x->graph_exec);
  if (x->graph) cudaGraphDestroy(x->graph);
  x->graph_exec = nullptr;
  x->graph = nullptr;
  x->cfg = *cfg;
  fill_params(x->P, cfg);
  CUDA_TRY(cudaMemsetAsync(x->ffc, 0, sizeof(unsigned int) * NFFC * x->d.nz, x->stream));
  return HGPU_OK;
}

int hgpu_reconfigure(hgpu_ctx *x, const hgpu_config *cfg) {
  const int rc = hg_reconfigure(x, cfg);
  if (rc == HGPU_E_INVALID) set_err("hgpu_reconfigure: configuration invalid or of another allocation shape");
  return rc;
}

int hgpu_create(const hgpu_config *cfg, hgpu_ctx **out) {
  if (!out) return HGPU_E_INVALID;
  *out = nullptr;
  int rc = validate(cfg);
  if (rc) {
    set_err("invalid configuration");
    return rc;
  }
  hgpu_ctx *x = new (std::nothrow) hgpu_ctx();
  if (!x) return HGPU_E_NOMEM;
  x->cfg = *cfg;
  Dims &d = x->d;
  d.n1 = cfg->n1;
  d.n2 = cfg->n2;
  d.n3 = cfg->n3;
  d.s1 = d.n1 > 1;
  d.s2 = d.n2 > 1;
  d.s3 = d.n3 > 1;
  d.g1 = d.s1 ? cfg->ng : 0;
  d.g2 = d.s2 ? cfg->ng : 0;
  d.g3 = d.s3 ? cfg->ng : 0;
  d.nt1 = d.n1 + 2 * d.g1;
  d.nt2 = d.n2 + 2 * d.g2;
  d.nt3 = d.n3 + 2 * d.g3;
  d.gt1 = d.nt1 + d.s1;
  d.gt2 = d.nt2 + d.s2;
  d.nz = (long long)d.nt1 * d.nt2 * d.nt3;
  d.nij = (long long)d.gt1 * d.gt2;
  fill_params(x->P, cfg);
  // loop ranges (initbase.c:1010-1058 and fixup.c:477 DQZLOOP)
  if (cfg->doenoflux == HGPU_ENOFINITEVOLUME) {
    // ENOFINITEVOLUME with avgo = 0 (initbase.c:952-994): faces along the
    // direction, every transverse zone including all ghosts; the dt minimum
    // runs over all of them
    x->face_box[1] = Box{0, -d.g2, -d.g3, d.n1 + 1, d.n2 + 2 * d.g2, d.n3 + 2 * d.g3};
    x->face_box[2] = Box{-d.g1, 0, -d.g3, d.n1 + 2 * d.g1, d.n2 + 1, d.n3 + 2 * d.g3};
    x->face_box[3] = Box{-d.g1, -d.g2, 0, d.n1 + 2 * d.g1, d.n2 + 2 * d.g2, d.n3 + 1};
  } else {
    x->face_box[1] = Box{0, -d.s2, -d.s3, d.n1 + 1, d.n2 + 2 * d.s2, d.n3 + 2 * d.s3};
    x->face_box[2] = Box{-d.s1, 0, -d.s3, d.n1 + 2 * d.s1, d.n2 + 1, d.n3 + 2 * d.s3};
    x->face_box[3] = Box{-d.s1, -d.s2, 0, d.n1 + 2 * d.s1, d.n2 + 2 * d.s2, d.n3 + 1};
  }
  x->emf_box = Box{0, 0, 0, d.n1 + d.s1, d.n2 + d.s2, d.n3 + d.s3};
  x->active_box = Box{0, 0, 0, d.n1, d.n2, d.n3};
  x->dq_box = Box{-d.s1, -d.s2, -d.s3, d.n1 + 2 * d.s1, d.n2 + 2 * d.s2, d.n3 + 2 * d.s3};
  // WENO5: output cells -1..n along the direction, the flux loop's
  // transverse ranges across it
  for (int q = 1; q <= 3; q++) {
    Box b = x->face_box[q];
    int n = (q == 1) ? d.n1 : ((q == 2) ? d.n2 : d.n3);
    if (q == 1) { b.i0 = -1; b.ni = n + 2; }
    if (q == 2) { b.j0 = -1; b.nj = n + 2; }
    if (q == 3) { b.k0 = -1; b.nk = n + 2; }
    x->w5[q] = w5_tiling(d, b, q);
  }
  // the state pieces are read at cells -2..n+1 along each direction, across
  // it over the flux loop's transverse range (every ghost for the
  // finite-volume scheme)
  {
    const int fvg = cfg->doenoflux == HGPU_ENOFINITEVOLUME;
    const int e1 = fvg ? d.g1 : 2 * d.s1, e2 = fvg ? d.g2 : 2 * d.s2, e3 = fvg ? d.g3 : 2 * d.s3;
    x->w5_state_box = Box{-e1, -e2, -e3, d.n1 + 2 * e1, d.n2 + 2 * e2, d.n3 + 2 * e3};
  }
  if (cfg->lim == HGPU_LIM_WENO5) w5_allow_smem_all();
  long long nz = d.nz;
  x->cap = (int)((long long)d.n1 * d.n2 * d.n3 < (1LL << 22) ? (long long)d.n1 * d.n2 * d.n3 : (1LL << 22));
  if (cudaStreamCreateWithFlags(&x->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete x;
    set_err("cudaStreamCreate failed");
    return HGPU_E_CUDA;
  }
  size_t pb = sizeof(double) * NPR * nz;
  bool ok = cudaMalloc(&x->p, pb) == cudaSuccess && cudaMalloc(&x->pk, pb) == cudaSuccess &&
            cudaMalloc(&x->uf, pb) == cudaSuccess && cudaMalloc(&x->ucum, pb) == cudaSuccess &&
            cudaMalloc(&x->E, sizeof(double) * 3 * nz) == cudaSuccess &&
            cudaMalloc(&x->G, sizeof(double) * G_NCOMP * d.nij) == cudaSuccess &&
            cudaMalloc(&x->pflag, sizeof(int) * nz) == cudaSuccess &&
            cudaMalloc(&x->gammacheck, sizeof(double) * nz) == cudaSuccess &&
            cudaMalloc(&x->cand, sizeof(long long) * x->cap) == cudaSuccess &&
            cudaMalloc(&x->fixlist, sizeof(long long) * x->cap) == cudaSuccess &&
            cudaMalloc(&x->cand_orig, sizeof(int) * x->cap) == cudaSuccess &&
            cudaMalloc(&x->cand_dec, sizeof(int) * x->cap) == cudaSuccess &&
            cudaMalloc(&x->cand_bits, sizeof(unsigned int) * x->cap) == cudaSuccess &&
            cudaMalloc(&x->cand_deplist, sizeof(int) * x->cap) == cudaSuccess &&
            cudaMalloc(&x->candmap, sizeof(int) * nz) == cudaSuccess &&
            cudaMalloc(&x->fixvals, sizeof(double) * 5 * x->cap) == cudaSuccess &&
            cudaMalloc(&x->sc, sizeof(Scalars)) == cudaSuccess &&
            cudaMalloc(&x->bsqf, nz) == cudaSuccess && cudaMemset(x->bsqf, 0, nz) == cudaSuccess &&
            cudaMalloc(&x->ffc, sizeof(unsigned int) * NFFC * nz) == cudaSuccess &&
            cudaMemset(x->ffc, 0, sizeof(unsigned int) * NFFC * nz) == cudaSuccess;
  for (int dd = 1; dd <= 3 && ok; dd++) ok = cudaMalloc(&x->F[dd], pb) == cudaSuccess;
  if (ok && cfg->timeorder >= 3) ok = cudaMalloc(&x->pk1, pb) == cudaSuccess && cudaMemset(x->pk1, 0, pb) == cudaSuccess;
  if (ok && cfg->doenoflux == HGPU_ENOFINITEVOLUME)
    ok = cudaMalloc(&x->ui, pb) == cudaSuccess && cudaMemset(x->ui, 0, pb) == cudaSuccess &&
         cudaMemset(x->ucum, 0, pb) == cudaSuccess;
  if (ok && cfg->lim == HGPU_LIM_WENO5)
    ok = cudaMalloc(&x->pL, pb) == cudaSuccess && cudaMalloc(&x->pR, pb) == cudaSuccess &&
         cudaMalloc(&x->w5pu, sizeof(double) * 2 * nz) == cudaSuccess;
  if (!ok) {
    hgpu_destroy(x);
    set_err("device allocation failed");
    return HGPU_E_NOMEM;
  }
  x->P.ffc = x->ffc;
  cudaMemsetAsync(x->p, 0, pb, x->stream);
  cudaMemsetAsync(x->pk, 0, pb, x->stream);
  cudaMemsetAsync(x->uf, 0, pb, x->stream);
  cudaMemsetAsync(x->ucum, 0, pb, x->stream);
  cudaMemsetAsync(x->E, 0, sizeof(double) * 3 * nz, x->stream);
  for (int dd = 1; dd <= 3; dd++) cudaMemsetAsync(x->F[dd], 0, pb, x->stream);
  cudaMemsetAsync(x->pflag, 0, sizeof(int) * nz, x->stream);
  cudaMemsetAsync(x->candmap, 0xFF, sizeof(int) * nz, x->stream);
  cudaMemsetAsync(x->sc, 0, sizeof(Scalars), x->stream);
  if (cudaStreamSynchronize(x->stream) != cudaSuccess) {
    hgpu_destroy(x);
    set_err("initialisation failed");
    return HGPU_E_CUDA;
  }
  *out = x;
  return HGPU_OK;
}

int hgpu_create_batch(const hgpu_config *cfg, int ninst, const int *n1, const double *dx1, const double *gam,
                      const double *tf, hgpu_ctx **out) {
  if (!cfg || !out || ninst < 1 || !n1 || !dx1 || !gam || !tf) return HGPU_E_INVALID;
  *out = nullptr;
  if (cfg->n2 != 1 || cfg->n3 != 1) {
    set_err("a batch holds 1D instances: n2 = n3 = 1");
    return HGPU_E_INVALID;
  }
  if (cfg->bc[0] != HGPU_BC_OUTFLOW_COPY || cfg->bc[1] != HGPU_BC_OUTFLOW_COPY) {
    set_err("a batch needs HGPU_BC_OUTFLOW_COPY at both x1 ends");
    return HGPU_E_INVALID;
  }
  if (cfg->doenoflux != HGPU_NOENOFLUX) {
    set_err("a batch runs the standard (NOENOFLUX) scheme");
    return HGPU_E_INVALID;
  }
  long long total = 0;
  for (int b = 0; b < ninst; b++) {
    if (n1[b] < cfg->ng || !(dx1[b] > 0.0) || !(gam[b] > 1.0)) {
      set_err("instance %s%d: n1 < ng, dx1 <= 0 or gam <= 1", "", b);
      return HGPU_E_INVALID;
    }
    total += n1[b] + 2LL * cfg->ng;
  }
  if (total - 2LL * cfg->ng > (1LL << 30)) return HGPU_E_INVALID;
  hgpu_config c = *cfg;
  c.n1 = (int)(total - 2LL * cfg->ng);
  int rc = hgpu_create(&c, out);
  if (rc) return rc;
  hgpu_ctx *x = *out;
  const Dims &d = x->d;
  std::vector<Inst> hi(ninst);
  std::vector<int> hc(d.nz);
  long long start = 0;  // global x1 index of the instance's first ghost is start - ng
  for (int b = 0; b < ninst; b++) {
    Inst I;
    memset(&I, 0, sizeof(I));
    I.i0 = (int)start;
    I.n = n1[b];
    I.dx = dx1[b];
    I.gam = gam[b];
    I.tf = tf[b];
    hi[b] = I;
    for (long long q = start - cfg->ng; q < start + n1[b] + cfg->ng; q++) hc[q + d.g1] = b;
    start += n1[b] + 2LL * cfg->ng;
  }
  if (cudaMalloc(&x->inst, sizeof(Inst) * ninst) != cudaSuccess ||
      cudaMalloc(&x->cell_inst, sizeof(int) * d.nz) != cudaSuccess) {
    hgpu_destroy(x);
    *out = nullptr;
    set_err("device allocation failed");
    return HGPU_E_NOMEM;
  }
  if (cudaMemcpy(x->inst, hi.data(), sizeof(Inst) * ninst, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(x->cell_inst, hc.data(), sizeof(int) * d.nz, cudaMemcpyHostToDevice) != cudaSuccess) {
    hgpu_destroy(x);
    *out = nullptr;
    set_err("batch table upload failed");
    return HGPU_E_CUDA;
  }
  x->ninst = ninst;
  x->P.cell_inst = x->cell_inst;
  x->P.inst = x->inst;
  x->P.ninst = ninst;
  return HGPU_OK;
}

int hgpu_batch_layout(hgpu_ctx *x, int *i0) {
  if (!x || !x->inst || !i0) return HGPU_E_INVALID;
  std::vector<Inst> hi(x->ninst);
  CUDA_TRY(cudaMemcpy(hi.data(), x->inst, sizeof(Inst) * x->ninst, cudaMemcpyDeviceToHost));
  for (int b = 0; b < x->ninst; b++) i0[b] = hi[b].i0;
  return HGPU_OK;
}

int hgpu_batch_status(hgpu_ctx *x, double *t, double *dt, int *done, int *ndone) {
  if (!x || !x->inst) return HGPU_E_INVALID;
  std::vector<Inst> hi(x->ninst);
  CUDA_TRY(cudaMemcpyAsync(hi.data(), x->inst, sizeof(Inst) * x->ninst, cudaMemcpyDeviceToHost, x->stream));
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  int nd = 0;
  for (int b = 0; b < x->ninst; b++) {
    if (t) t[b] = hi[b].t;
    if (dt) dt[b] = hi[b].dt;
    if (done) done[b] = hi[b].done;
    nd += hi[b].done != 0;
  }
  if (ndone) *ndone = nd;
  return HGPU_OK;
}

int hgpu_batch_set_time(hgpu_ctx *x, const double *t, const double *dt) {
  if (!x || !x->inst || !t || !dt) return HGPU_E_INVALID;
  std::vector<Inst> hi(x->ninst);
  CUDA_TRY(cudaMemcpyAsync(hi.data(), x->inst, sizeof(Inst) * x->ninst, cudaMemcpyDeviceToHost, x->stream));
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  for (int b = 0; b < x->ninst; b++) {
    hi[b].t = t[b];
    hi[b].dt = dt[b];
    hi[b].done = !(t[b] < hi[b].tf);
    hi[b].nsteps = 0;
  }
  CUDA_TRY(cudaMemcpyAsync(x->inst, hi.data(), sizeof(Inst) * x->ninst, cudaMemcpyHostToDevice, x->stream));
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  return HGPU_OK;
}

int hgpu_upload_geometry(hgpu_ctx *x, const double *gcov, const double *gcon, const double *gcovpert,
                         const double *gdet, const double *conn, const double *floors) {
  if (!x || !gcov || !gcon || !gcovpert || !gdet || !conn || !floors) return HGPU_E_INVALID;
  const long long nij = x->d.nij;
  // the host arrays go up as they are (six large copies); the device packs
  // them into the SoA planes of the library's layout
  const long long words = nij * GRAW_WORDS;
  double *raw = nullptr;
  CUDA_TRY(cudaMallocAsync(&raw, sizeof(double) * words, x->stream));
  double *rcov = raw, *rcon = raw + 128 * nij, *rpert = raw + 256 * nij, *rgdet = raw + 288 * nij,
         *rconn = raw + 296 * nij, *rfl = raw + 360 * nij;
  cudaError_t e = cudaMemcpyAsync(rcov, gcov, sizeof(double) * 128 * nij, cudaMemcpyHostToDevice, x->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(rcon, gcon, sizeof(double) * 128 * nij, cudaMemcpyHostToDevice, x->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(rpert, gcovpert, sizeof(double) * 32 * nij, cudaMemcpyHostToDevice, x->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(rgdet, gdet, sizeof(double) * 8 * nij, cudaMemcpyHostToDevice, x->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(rconn, conn, sizeof(double) * 64 * nij, cudaMemcpyHostToDevice, x->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(rfl, floors, sizeof(double) * 2 * nij, cudaMemcpyHostToDevice, x->stream);
  if (e == cudaSuccess) {
    LAUNCH(x, K_OTHER, pack_geometry_kernel, grid_for(nij, 128), 128, raw, nij, x->G);
    e = cudaGetLastError();
  }
  cudaFreeAsync(raw, x->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(x->stream);
  if (e != cudaSuccess) {
    set_err("geometry upload: %s", cudaGetErrorString(e));
    return HGPU_E_CUDA;
  }
  return HGPU_OK;
}

static int ensure_staging(hgpu_ctx *x) {
  if (!x->staging) CUDA_TRY(cudaMalloc(&x->staging, sizeof(double) * NPR * x->d.nz));
  return HGPU_OK;
}

int hgpu_upload_state(hgpu_ctx *x, const double *p, const int *pflag, double t, double dt) {
  if (!x || !p) return HGPU_E_INVALID;
  int rc = ensure_staging(x);
  if (rc) return rc;
  long long nz = x->d.nz;
  CUDA_TRY(cudaMemcpyAsync(x->staging, p, sizeof(double) * NPR * nz, cudaMemcpyHostToDevice, x->stream));
  LAUNCH(x, K_OTHER, aos_to_soa_kernel, grid_for(nz * NPR, 256), 256, x->staging, x->p, nz);
  if (pflag) CUDA_TRY(cudaMemcpyAsync(x->pflag, pflag, sizeof(int) * nz, cudaMemcpyHostToDevice, x->stream));
  Scalars s;
  memset(&s, 0, sizeof(s));
  s.t = t;
  s.dt = dt;
  CUDA_TRY(cudaMemcpyAsync(x->sc, &s, sizeof(Scalars), cudaMemcpyHostToDevice, x->stream));
  // the finite-volume scheme's conserved state: init_conservatives (pi2Uavg)
  if (x->cfg.doenoflux == HGPU_ENOFINITEVOLUME)
    LAUNCH(x, K_OTHER, pi2u_kernel, grid_for(nz, 128), 128, x->d, x->P, x->p, x->G, x->ucum, x->sc);
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  CUDA_TRY(cudaGetLastError());
  return HGPU_OK;
}

int hgpu_download_state(hgpu_ctx *x, double *p, int *pflag, double *t, double *dt) {
  if (!x) return HGPU_E_INVALID;
  long long nz = x->d.nz;
  if (p) {
    int rc = ensure_staging(x);
    if (rc) return rc;
    LAUNCH(x, K_OTHER, soa_to_aos_kernel, grid_for(nz * NPR, 256), 256, x->p, x->staging, nz);
    CUDA_TRY(cudaMemcpyAsync(p, x->staging, sizeof(double) * NPR * nz, cudaMemcpyDeviceToHost, x->stream));
  }
  if (pflag) CUDA_TRY(cudaMemcpyAsync(pflag, x->pflag, sizeof(int) * nz, cudaMemcpyDeviceToHost, x->stream));
  Scalars s;
  CUDA_TRY(cudaMemcpyAsync(&s, x->sc, sizeof(Scalars), cudaMemcpyDeviceToHost, x->stream));
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  CUDA_TRY(cudaGetLastError());
  if (t) *t = s.t;
  if (dt) *dt = s.dt;
  return HGPU_OK;
}

// one stage: fluxes, EMFs, update, bound, post_fixup, bound
extern "C++" {
// one direction's reconstruction + flux launches.  TW: arithmetic of the
// WENO5 reconstruction, TF: of the Riemann kernel (the MC/PARA
// reconstruction happens inside it); FMB / BMB: resident blocks per SM asked
// of the flux and WENO5 kernels (autotuned variants)
// the WENO5 reconstruction of one direction with the context's tiling
template <int DIR, typename TW, int BMB>
static void launch_w5(hgpu_ctx *x, const double *pb) {
  const Dims &d = x->d;
  const Params &P = x->P;
  const W5Tile &tl = x->w5[DIR];
  const size_t smem = (size_t)w5_smem_bytes(tl.lb, tl.w, (int)sizeof(TW));
  const TW *PU = (const TW *)x->w5pu;
  double *pL = x->pL, *pR = x->pR;
  ProfScope ps__(x, K_WENO5);
  const unsigned grid = (unsigned)tl.nseg * tl.ntile;
  if constexpr (DIR == 3) {
    weno5_kernel<3, true, TW, BMB><<<grid, W5_THREADS, smem, x->stream>>>(d, P, tl, pb, PU, pL, pR);
  } else {
    if (tl.fast_s)
      weno5_kernel<DIR, true, TW, BMB><<<grid, W5_THREADS, smem, x->stream>>>(d, P, tl, pb, PU, pL, pR);
    else
      weno5_kernel<DIR, false, TW, BMB><<<grid, W5_THREADS, smem, x->stream>>>(d, P, tl, pb, PU, pL, pR);
  }
}

template <int DIR, typename TW, typename TF, int FMB, int BMB, int MIX = 0>
static void launch_dir(hgpu_ctx *x, const double *pb) {
  const Dims &d = x->d;
  const Params &P = x->P;
  const int kid = (DIR == 1) ? K_FLUX1 : ((DIR == 2) ? K_FLUX2 : K_FLUX3);
  unsigned gf = grid_for(x->face_box[DIR].size(), 128);
  if (P.lim == HGPU_LIM_WENO5) {
    launch_w5<DIR, TW, BMB>(x, pb);
    LAUNCH(x, kid, (flux_kernel<DIR, 1, TF, FMB, double, MIX>), gf, 128, d, P, x->face_box[DIR], pb, x->pL, x->pR, x->G,
           x->F[DIR], x->sc);
  } else if (P.lim == HGPU_LIM_PARA) {
    LAUNCH(x, kid, (flux_kernel<DIR, 2, TF, FMB, TF>), gf, 128, d, P, x->face_box[DIR], pb, nullptr, nullptr, x->G,
           x->F[DIR], x->sc);
  } else {
    LAUNCH(x, kid, (flux_kernel<DIR, 0, TF, FMB, TF>), gf, 128, d, P, x->face_box[DIR], pb, nullptr, nullptr, x->G,
           x->F[DIR], x->sc);
  }
}

template <typename TW, typename TF, int FMB, int BMB, int MIX = 0>
static void launch_fluxes_t(hgpu_ctx *x, const double *pb) {
  const Dims &d = x->d;
  if (x->P.lim == HGPU_LIM_WENO5)
    LAUNCH(x, K_W5STATE, w5_state_kernel<TW>, grid_for(x->w5_state_box.size(), 128), 128, d, x->P, x->w5_state_box,
           pb, x->G, (TW *)x->w5pu);
  if (d.n1 > 1) launch_dir<1, TW, TF, FMB, BMB, MIX>(x, pb);
  if (d.n2 > 1) launch_dir<2, TW, TF, FMB, BMB, MIX>(x, pb);
  if (d.n3 > 1) launch_dir<3, TW, TF, FMB, BMB, MIX>(x, pb);
}
// the WENO5 state pieces and one direction's reconstruction with the
// context's precision and WENO5 variant (for timing tilings)
template <int DIR>
static void launch_w5_any(hgpu_ctx *x, const double *pb, bool state) {
  const Dims &d = x->d;
  if (x->cfg.precision == HGPU_PREC_MIXED) {
    if (state)
      w5_state_kernel<float><<<grid_for(x->w5_state_box.size(), 128), 128, 0, x->stream>>>(d, x->P, x->w5_state_box,
                                                                                          pb, x->G, (float *)x->w5pu);
    launch_w5<DIR, float, MinBlocks<float>::weno>(x, pb);
  } else {
    if (state)
      w5_state_kernel<double><<<grid_for(x->w5_state_box.size(), 128), 128, 0, x->stream>>>(d, x->P, x->w5_state_box,
                                                                                           pb, x->G, x->w5pu);
    if (x->tune.weno == 0) launch_w5<DIR, double, kWenoMB[0]>(x, pb);
    else launch_w5<DIR, double, kWenoMB[1]>(x, pb);
  }
}
}  // extern "C++"

// fluxcalc + the EMFs of flux_ct.  HGPU_PREC_MIXED runs the WENO5
// reconstruction in FP32 (on differences from each cell's value, face values
// returned in FP64) and the Riemann kernel in FP64: in a torus near
// equilibrium the flux divergence cancels most of each face flux, so FP32
// rounding of the fluxes themselves would dominate the error.  With MC/PARA,
// whose reconstruction runs inside the Riemann kernel, that kernel runs in
// FP32.  The fluxes are stored in FP64 and everything after them (flux-CT,
// update, inversion) stays FP64.
static void launch_fluxes(hgpu_ctx *x, const double *pb) {
  const Dims &d = x->d;
  const int fv = x->tune.flux, bv = x->tune.weno;
  if (x->cfg.precision == HGPU_PREC_MIXED) {
    constexpr int WMB = MinBlocks<float>::weno;
    if (x->P.lim != HGPU_LIM_WENO5) launch_fluxes_t<float, float, MinBlocks<float>::flux, WMB>(x, pb);
    else if (fv == 0) launch_fluxes_t<float, double, kFluxMB[0], WMB, 1>(x, pb);
    else launch_fluxes_t<float, double, kFluxMB[1], WMB, 1>(x, pb);
  } else {
    if (fv == 0 && bv == 0) launch_fluxes_t<double, double, kFluxMB[0], kWenoMB[0]>(x, pb);
    else if (fv == 0) launch_fluxes_t<double, double, kFluxMB[0], kWenoMB[1]>(x, pb);
    else if (bv == 0) launch_fluxes_t<double, double, kFluxMB[1], kWenoMB[0]>(x, pb);
    else launch_fluxes_t<double, double, kFluxMB[1], kWenoMB[1]>(x, pb);
  }
  LAUNCH(x, K_EMF, emf_kernel, grid_for(x->emf_box.size(), 256), 256, d, x->emf_box, x->F[1], x->F[2], x->F[3], x->G,
         x->E);
}

static void launch_bound(hgpu_ctx *x, double *pv) {
  const Dims &d = x->d;
  if (x->P.cell_inst) {
    LAUNCH(x, K_BOUND_GHOST, bound_batch_kernel, grid_for(d.nz, 128), 128, d, x->P, pv, (int *)nullptr);
    return;
  }
  if (x->P.bondi) {
    const long long nb = 2LL * d.g1 * d.n2 * d.n3;
    LAUNCH(x, K_BOUND_GHOST, bondi_bc_kernel, grid_for(nb, 128), 128, d, x->P, pv, x->G, x->sc);
  }
  LAUNCH(x, K_BOUND_GHOST, bound_ghost_kernel, grid_for(d.nz, 128), 128, d, x->P, pv, x->G, x->sc);
  if (d.n2 > 1) LAUNCH(x, K_BOUND_POLE, bound_pole_kernel, grid_for(2LL * d.n1 * d.n3, 128), 128, d, x->P, pv);
}

static void launch_reset(hgpu_ctx *x) {
  LAUNCH(x, K_RESET, reset_stage_kernel, 1, 32, x->sc);
  if (x->P.cell_inst) LAUNCH(x, K_RESET, reset_batch_kernel, grid_for(x->P.ninst, 128), 128, x->P);
}

static void launch_finalize(hgpu_ctx *x, int advance_time) {
  if (x->P.cell_inst)
    LAUNCH(x, K_FINALIZE, finalize_batch_kernel, grid_for(x->P.ninst, 128), 128, x->P, advance_time);
  else
    LAUNCH(x, K_FINALIZE, finalize_kernel, 1, 32, x->P, x->sc, advance_time);
}

// setup_rktimestep (step_ch.c:442-562): per stage of the TIMEORDER-stage
// method, CUf (Ui, ulast, dU) and Cunew (Ui, dU, Uf), and the arrays read as
// pb and written as pf (pi is always p): 0 = p, 1 = pk0, 2 = pk1
struct RKStage {
  double cuf[3], cun[3];
  int pb, pf;
};
static const RKStage kRK1[1] = {{{1.0, 0.0, 1.0}, {0.0, 0.0, 1.0}, 0, 0}};
static const RKStage kRK2[2] = {{{1.0, 0.0, 0.5}, {0.0, 0.0, 0.0}, 0, 1}, {{1.0, 0.0, 1.0}, {0.0, 0.0, 1.0}, 1, 0}};
static const RKStage kRK3[3] = {{{1.0, 0.0, 1.0}, {0.0, 0.0, 0.0}, 0, 1},
                                {{3.0 / 4.0, 1.0 / 4.0, 1.0 / 4.0}, {0.0, 0.0, 0.0}, 1, 2},
                                {{1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0}, {0.0, 0.0, 1.0}, 2, 0}};
static const RKStage kRK4[4] = {{{1.0, 0.0, 0.5}, {1.0, 1.0 / 6.0, 0.0}, 0, 1},
                                {{1.0, 0.0, 0.5}, {0.0, 1.0 / 3.0, 0.0}, 1, 2},
                                {{1.0, 0.0, 1.0}, {0.0, 1.0 / 3.0, 0.0}, 2, 1},
                                {{1.0, 0.0, 1.0}, {0.0, 1.0 / 6.0, 0.0}, 1, 0}};

static int num_orders(const hgpu_ctx *x) { return x->cfg.timeorder ? x->cfg.timeorder : 2; }

static const RKStage &rk_stage(const hgpu_ctx *x, int timeorder) {
  const int norders = num_orders(x);
  return (norders == 4 ? kRK4 : norders == 3 ? kRK3 : norders == 2 ? kRK2 : kRK1)[timeorder];
}

// the array stage `timeorder` writes (pf); -1 names p itself
static double *stage_output(hgpu_ctx *x, int timeorder) {
  if (timeorder < 0) return x->p;
  double *arr[3] = {x->p, x->pk, x->pk1};
  return arr[rk_stage(x, timeorder).pf];
}

// One RK stage in two halves.  The first runs advance (fluxes, conserved
// update, inversion, fixup1zone) and the bound_prim/bound_pflag that open
// post_fixup; the second runs fixup_checksolution, fixup_utoprim and the
// closing bound_prim.  A domain split along x3 exchanges the x3 ghost planes
// of pf and pflag after the first half and of pf after the second, where the
// reference's bound_prim and bound_pflag call bound_mpi / bound_mpi_int.
static void launch_stage_advance(hgpu_ctx *x, int timeorder) {
  const Dims &d = x->d;
  const int norders = num_orders(x);
  const RKStage &S = rk_stage(x, timeorder);
  double *arr[3] = {x->p, x->pk, x->pk1};
  const double *pi = x->p;
  const double *pb = arr[S.pb];
  double *pf = arr[S.pf];
  int finalstep = (timeorder == norders - 1);
  double CUf0 = S.cuf[0], CUf1 = S.cuf[1], CUf2 = S.cuf[2];
  double Cn0 = S.cun[0], Cn1 = S.cun[1], Cn2 = S.cun[2];
  launch_reset(x);
  // pre_fixup: only the last stage's flags survive the step
  if (finalstep && !x->P.cell_inst)
    LAUNCH(x, K_OTHER, bsqflags_kernel, grid_for(d.nz, 256), 256, d, pi, x->G, x->bsqf, x->sc);
  launch_fluxes(x, pb);
  const int fv = (x->cfg.doenoflux == HGPU_ENOFINITEVOLUME);
  double *ufv = (fv && finalstep) ? x->ucum : nullptr;
  if (x->tune.conserve)
    LAUNCH(x, K_UPDATE, conserve_kernel<kConserveMB[1]>, grid_for(x->active_box.size(), 128), 128, d, x->P,
           x->active_box, pi, pb, x->uf, x->ucum, x->F[1], x->F[2], x->F[3], x->E, x->G, x->sc, CUf0, CUf1, CUf2, Cn0,
           Cn1, Cn2, timeorder, x->ui, fv);
  else
    LAUNCH(x, K_UPDATE, conserve_kernel<kConserveMB[0]>, grid_for(x->active_box.size(), 128), 128, d, x->P,
           x->active_box, pi, pb, x->uf, x->ucum, x->F[1], x->F[2], x->F[3], x->E, x->G, x->sc, CUf0, CUf1, CUf2, Cn0,
           Cn1, Cn2, timeorder, x->ui, fv);
  {
    const unsigned gi = grid_for(x->active_box.size(), 128);
    const bool jon = x->cfg.utoprimversion == HGPU_UTOPRIMJONNONRELCOMPAT;
    if (jon && x->tune.invert)
      LAUNCH(x, K_INVERT, (invert_kernel<8, kInvertMB[1]>), gi, 128, d, x->P, x->active_box, pb, pf, x->uf, x->ucum,
             x->G, x->pflag, x->sc, finalstep, ufv);
    else if (jon)
      LAUNCH(x, K_INVERT, (invert_kernel<8, kInvertMB[0]>), gi, 128, d, x->P, x->active_box, pb, pf, x->uf, x->ucum,
             x->G, x->pflag, x->sc, finalstep, ufv);
    else if (x->tune.invert)
      LAUNCH(x, K_INVERT, (invert_kernel<6, kInvertMB[1]>), gi, 128, d, x->P, x->active_box, pb, pf, x->uf, x->ucum,
             x->G, x->pflag, x->sc, finalstep, ufv);
    else
      LAUNCH(x, K_INVERT, (invert_kernel<6, kInvertMB[0]>), gi, 128, d, x->P, x->active_box, pb, pf, x->uf, x->ucum,
             x->G, x->pflag, x->sc, finalstep, ufv);
  }
  launch_bound(x, pf);
  // post_fixup (fixup.c:37-96)
  if (x->P.cell_inst)
    LAUNCH(x, K_BOUND_PFLAG, bound_batch_kernel, grid_for(d.nz, 256), 256, d, x->P, (double *)nullptr, x->pflag);
  else
    LAUNCH(x, K_BOUND_PFLAG, bound_pflag_kernel, grid_for(d.nz, 256), 256, d, x->P, x->pflag, x->sc);
}

// fixup_checksolution and fixup_utoprim on pf with the context's flags
static void launch_checksol_fixup(hgpu_ctx *x, double *pf, int finalstep) {
  const Dims &d = x->d;
  double *ufv = (x->cfg.doenoflux == HGPU_ENOFINITEVOLUME && finalstep) ? x->ucum : nullptr;
  LAUNCH(x, K_CHECK_GAMMA, checksol_gamma_kernel, grid_for(x->dq_box.size(), 128), 128, d, x->P, x->dq_box, pf, x->G,
         x->gammacheck, x->cand, x->cap, x->sc);
  // grid-stride over the device-side candidate count; idle blocks exit at once
  int cgrid = (int)grid_for(x->cap, 256);
  if (cgrid > 592) cgrid = 592;
  LAUNCH(x, K_CHECK_RESOLVE, checksol_map_kernel, cgrid, 256, x->cand, x->pflag, x->candmap, x->cand_orig, x->cap,
         x->sc);
  LAUNCH(x, K_CHECK_RESOLVE, checksol_prep_kernel, cgrid, 256, d, pf, x->gammacheck, x->pflag, x->cand, x->candmap,
         x->cand_orig, x->cand_dec, x->cand_bits, x->cand_deplist, x->cap, x->sc);
  LAUNCH(x, K_CHECK_RESOLVE, checksol_resolve_kernel, 1, 1024, d, x->cand, x->candmap, x->cand_orig, x->cand_dec,
         x->cand_bits, x->cand_deplist, x->cap, x->sc);
  LAUNCH(x, K_CHECK_RESOLVE, checksol_apply_kernel, cgrid, 256, x->cand, x->cand_dec, x->pflag, x->candmap, x->cap,
         x->sc);
  LAUNCH(x, K_FIX_COLLECT, fixup_collect_kernel, grid_for(x->active_box.size(), 256), 256, d, x->P, x->active_box, x->pflag,
         x->fixlist, x->cap, x->sc);
  // grid-stride over the device-side list length; idle blocks exit at once
  int fixgrid = (int)grid_for(x->cap, 128);
  if (fixgrid > 296) fixgrid = 296;
  LAUNCH(x, K_FIX_COMPUTE, fixup_compute_kernel, fixgrid, 128, d, x->P, pf, x->pflag, x->G, x->fixlist, x->fixvals,
         x->cap, finalstep, x->sc);
  LAUNCH(x, K_FIX_SCATTER, fixup_scatter_kernel, fixgrid, 128, d, x->P, pf, x->pflag, x->fixlist, x->fixvals, x->cap,
         finalstep, x->sc, x->G, ufv);
}

static void launch_stage_fixup(hgpu_ctx *x, int timeorder) {
  double *pf = stage_output(x, timeorder);
  launch_checksol_fixup(x, pf, timeorder == num_orders(x) - 1);
  launch_bound(x, pf);
}

static void launch_stage(hgpu_ctx *x, int timeorder) {
  launch_stage_advance(x, timeorder);
  launch_stage_fixup(x, timeorder);
}

static int read_stats(hgpu_ctx *x, hgpu_stats *st) {
  Scalars s;
  CUDA_TRY(cudaMemcpyAsync(&s, x->sc, sizeof(Scalars), cudaMemcpyDeviceToHost, x->stream));
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  CUDA_TRY(cudaGetLastError());
  if (st) {
    st->newton_iters = (long long)s.iters;
    st->err = s.err;
    st->nfail = s.nfail;
    st->nfixed = s.nfixed;
  }
  if (s.overflow) {
    // bit 0: checksolution candidate list full; bit 1: fixup list full;
    // bit 2: a checksolution dependency chain longer than the sweep cap
    set_err("%s (overflow bits %d)",
            (s.overflow & 3) ? "fixup list capacity exceeded" : "checksolution dependency chain over 4096 zones",
            s.overflow);
    return HGPU_E_PHYSICS;
  }
  if (s.err) {
    set_err("physics failure bits %s%d", "", s.err);
    return HGPU_E_PHYSICS;
  }
  return HGPU_OK;
}

static void clear_counters(hgpu_ctx *x) {
  // iters, err, nfixed, overflow accumulate over a call
  cudaMemsetAsync(&x->sc->iters, 0, sizeof(unsigned long long), x->stream);
  cudaMemsetAsync(&x->sc->err, 0, sizeof(int), x->stream);
  cudaMemsetAsync(&x->sc->nfixed, 0, sizeof(int), x->stream);
  cudaMemsetAsync(&x->sc->overflow, 0, sizeof(int), x->stream);
  cudaMemsetAsync(&x->sc->nfloor, 0, sizeof(unsigned long long), x->stream);
}

// the Bondi-integral boundaries need their coordinate data before any bound
static int boundaries_ready(const hgpu_ctx *x) {
  const bool bondi = x->cfg.bc[0] == HGPU_BC_BONDIMDOTOUTFLOW || x->cfg.bc[1] == HGPU_BC_BONDIINTOUTFLOW;
  if (bondi && !x->P.bondi) {
    set_err("Bondi-integral boundaries: call hgpu_set_bondi_boundaries first");
    return HGPU_E_INVALID;
  }
  return HGPU_OK;
}

int hgpu_step_ch(hgpu_ctx *x, int nsteps, hgpu_stats *stats) {
  if (!x || nsteps < 0) return HGPU_E_INVALID;
  if (boundaries_ready(x)) return HGPU_E_INVALID;
  clear_counters(x);
  for (int n = 0; n < nsteps; n++) {
    for (int o = 0; o < num_orders(x); o++) launch_stage(x, o);
    launch_finalize(x, 1);
  }
  CUDA_TRY(cudaGetLastError());
  if (stats) return read_stats(x, stats);
  return HGPU_OK;
}

// The active zones from / to host arrays; the ghost zones are the device's
// bound_prim of them (what the end of every step leaves there).
int hgpu_upload_active(hgpu_ctx *x, const double *p, double t, double dt) {
  if (!x || !p || x->ninst > 0) return HGPU_E_INVALID;
  if (boundaries_ready(x)) return HGPU_E_INVALID;
  int rc = ensure_staging(x);
  if (rc) return rc;
  const Dims &d = x->d;
  const long long na = (long long)d.n1 * d.n2 * d.n3;
  CUDA_TRY(cudaMemcpyAsync(x->staging, p, sizeof(double) * NPR * na, cudaMemcpyHostToDevice, x->stream));
  LAUNCH(x, K_OTHER, active_scatter_kernel, grid_for(na * NPR, 256), 256, d, x->staging, x->p);
  Scalars s;
  memset(&s, 0, sizeof(s));
  s.t = t;
  s.dt = dt;
  CUDA_TRY(cudaMemcpyAsync(x->sc, &s, sizeof(Scalars), cudaMemcpyHostToDevice, x->stream));
  launch_bound(x, x->p);
  if (x->cfg.doenoflux == HGPU_ENOFINITEVOLUME)
    LAUNCH(x, K_OTHER, pi2u_kernel, grid_for(d.nz, 128), 128, d, x->P, x->p, x->G, x->ucum, x->sc);
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  CUDA_TRY(cudaGetLastError());
  return HGPU_OK;
}

int hgpu_download_active(hgpu_ctx *x, double *p, int *pflag, double *t, double *dt) {
  if (!x || x->ninst > 0) return HGPU_E_INVALID;
  int rc = ensure_staging(x);
  if (rc) return rc;
  const Dims &d = x->d;
  const long long na = (long long)d.n1 * d.n2 * d.n3;
  if (p) {
    LAUNCH(x, K_OTHER, active_gather_kernel, grid_for(na * NPR, 256), 256, d, x->p, x->staging);
    CUDA_TRY(cudaMemcpyAsync(p, x->staging, sizeof(double) * NPR * na, cudaMemcpyDeviceToHost, x->stream));
  }
  if (pflag) {
    // the flags follow the primitives in the staging buffer (it holds 8 nz doubles)
    int *fs = (int *)(x->staging + NPR * na);
    LAUNCH(x, K_OTHER, active_gather_flags_kernel, grid_for(na, 256), 256, d, x->pflag, fs);
    CUDA_TRY(cudaMemcpyAsync(pflag, fs, sizeof(int) * na, cudaMemcpyDeviceToHost, x->stream));
  }
  Scalars s;
  CUDA_TRY(cudaMemcpyAsync(&s, x->sc, sizeof(Scalars), cudaMemcpyDeviceToHost, x->stream));
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  CUDA_TRY(cudaGetLastError());
  if (t) *t = s.t;
  if (dt) *dt = s.dt;
  return HGPU_OK;
}

// nsteps replays of one captured time step.  The capture is made on the
// first call (profiling must be off) and reused; the step's launches read t,
// dt and every bound from device memory, so the same graph advances any state.
int hgpu_step_graph(hgpu_ctx *x, int nsteps, hgpu_stats *stats) {
  if (!x || nsteps < 0) return HGPU_E_INVALID;
  if (boundaries_ready(x)) return HGPU_E_INVALID;
  if (x->profiling) {
    set_err("hgpu_step_graph: turn profiling off first");
    return HGPU_E_INVALID;
  }
  if (!x->graph_exec) {
    CUDA_TRY(cudaStreamSynchronize(x->stream));
    CUDA_TRY(cudaStreamBeginCapture(x->stream, cudaStreamCaptureModeThreadLocal));
    long long l0 = x->launches;
    for (int o = 0; o < num_orders(x); o++) launch_stage(x, o);
    launch_finalize(x, 1);
    x->launches_per_step = x->launches - l0;
    x->launches = l0;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(x->stream, &g);
    if (e != cudaSuccess) {
      set_err("step capture failed: %s", cudaGetErrorString(e));
      return HGPU_E_CUDA;
    }
    e = cudaGraphInstantiate(&x->graph_exec, g, 0);
    if (e != cudaSuccess) {
      cudaGraphDestroy(g);
      set_err("graph instantiation failed: %s", cudaGetErrorString(e));
      return HGPU_E_CUDA;
    }
    x->graph = g;
  }
  clear_counters(x);
  for (int n = 0; n < nsteps; n++) {
    CUDA_TRY(cudaGraphLaunch(x->graph_exec, x->stream));
    x->launches += x->launches_per_step;
  }
  if (stats) return read_stats(x, stats);
  return HGPU_OK;
}

int hgpu_advance_stage(hgpu_ctx *x, int timeorder, double *ndt, hgpu_stats *stats) {
  if (!x || timeorder < 0 || timeorder >= num_orders(x)) return HGPU_E_INVALID;
  if (boundaries_ready(x)) return HGPU_E_INVALID;
  clear_counters(x);
  launch_stage(x, timeorder);
  launch_finalize(x, 0);
  CUDA_TRY(cudaGetLastError());
  int rc = read_stats(x, stats);
  if (ndt) {
    unsigned long long b;
    CUDA_TRY(cudaMemcpy(&b, &x->sc->ndtbits[0], sizeof(b), cudaMemcpyDeviceToHost));
    double v;
    memcpy(&v, &b, sizeof(v));
    *ndt = v;
  }
  return rc;
}

int hgpu_fluxcalc(hgpu_ctx *x, int which, double *F1, double *F2, double *F3, double *ndt1, double *ndt2,
                  double *ndt3) {
  if (!x || (which != 0 && which != 1)) return HGPU_E_INVALID;
  launch_reset(x);
  launch_fluxes(x, which ? x->pk : x->p);
  CUDA_TRY(cudaGetLastError());
  Scalars s;
  CUDA_TRY(cudaMemcpyAsync(&s, x->sc, sizeof(Scalars), cudaMemcpyDeviceToHost, x->stream));
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  double v[4];
  for (int q = 1; q <= 3; q++) memcpy(&v[q], &s.ndtbits[q], sizeof(double));
  if (ndt1) *ndt1 = v[1];
  if (ndt2) *ndt2 = v[2];
  if (ndt3) *ndt3 = v[3];
  {
    // faces read by the update (advance.c:777-790)
    const Dims &d = x->d;
    Box fb[4] = {Box{0, 0, 0, 0, 0, 0}, Box{0, 0, 0, d.n1 + 1, d.n2, d.n3}, Box{0, 0, 0, d.n1, d.n2 + 1, d.n3},
                 Box{0, 0, 0, d.n1, d.n2, d.n3 + 1}};
    int nd[4] = {0, d.n1, d.n2, d.n3};
    for (int q = 1; q <= 3; q++)
      if (nd[q] > 1) bflux_kernel<<<grid_for(fb[q].size(), 256), 256, 0, x->stream>>>(d, q, fb[q], x->E, x->F[q]);
  }
  double *outs[4] = {nullptr, F1, F2, F3};
  int rc = ensure_staging(x);
  if (rc) return rc;
  long long nz = x->d.nz;
  for (int q = 1; q <= 3; q++) {
    if (!outs[q]) continue;
    soa_to_aos_kernel<<<grid_for(nz * NPR, 256), 256, 0, x->stream>>>(x->F[q], x->staging, nz);
    CUDA_TRY(cudaMemcpyAsync(outs[q], x->staging, sizeof(double) * NPR * nz, cudaMemcpyDeviceToHost, x->stream));
    CUDA_TRY(cudaStreamSynchronize(x->stream));
  }
  return HGPU_OK;
}

int hgpu_bound_prim(hgpu_ctx *x, int which) {
  if (!x || (which != 0 && which != 1)) return HGPU_E_INVALID;
  if (boundaries_ready(x)) return HGPU_E_INVALID;
  launch_bound(x, which ? x->pk : x->p);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  return HGPU_OK;
}

int hgpu_device_prims(hgpu_ctx *x, int which, double **dptr) {
  if (!x || !dptr) return HGPU_E_INVALID;
  *dptr = which ? x->pk : x->p;
  return HGPU_OK;
}

int hgpu_sync(hgpu_ctx *x) {
  if (!x) return HGPU_E_INVALID;
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  CUDA_TRY(cudaGetLastError());
  return HGPU_OK;
}

static int utoprim_batch_impl(const double *U, const double *gcov, const double *gcon, const double *gdet, double *pr,
                              int *pflag, long long n, double gam, double gammafail, int uv, long long *iters) {
  if (n < 0 || (n > 0 && (!U || !gcov || !gcon || !gdet || !pr || !pflag))) return HGPU_E_INVALID;
  if (uv != 0 && uv != HGPU_UTOPRIM2DFINAL && uv != HGPU_UTOPRIMJONNONRELCOMPAT) return HGPU_E_INVALID;
  if (n == 0) {
    if (iters) *iters = 0;
    return HGPU_OK;
  }
  double *dU = nullptr, *dgcov = nullptr, *dgcon = nullptr, *dg = nullptr, *dpr = nullptr;
  int *dpf = nullptr;
  unsigned long long *dit = nullptr;
  int rc = HGPU_OK;
  cudaError_t e = cudaSuccess;
  if ((e = cudaMalloc(&dU, sizeof(double) * 8 * n)) != cudaSuccess ||
      (e = cudaMalloc(&dgcov, sizeof(double) * 16 * n)) != cudaSuccess ||
      (e = cudaMalloc(&dgcon, sizeof(double) * 16 * n)) != cudaSuccess ||
      (e = cudaMalloc(&dg, sizeof(double) * n)) != cudaSuccess ||
      (e = cudaMalloc(&dpr, sizeof(double) * 8 * n)) != cudaSuccess ||
      (e = cudaMalloc(&dpf, sizeof(int) * n)) != cudaSuccess ||
      (e = cudaMalloc(&dit, sizeof(unsigned long long))) != cudaSuccess) {
    rc = HGPU_E_NOMEM;
  } else {
    cudaMemcpy(dU, U, sizeof(double) * 8 * n, cudaMemcpyHostToDevice);
    cudaMemcpy(dgcov, gcov, sizeof(double) * 16 * n, cudaMemcpyHostToDevice);
    cudaMemcpy(dgcon, gcon, sizeof(double) * 16 * n, cudaMemcpyHostToDevice);
    cudaMemcpy(dg, gdet, sizeof(double) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(dpr, pr, sizeof(double) * 8 * n, cudaMemcpyHostToDevice);
    cudaMemset(dit, 0, sizeof(unsigned long long));
    if (uv == HGPU_UTOPRIMJONNONRELCOMPAT)
      utoprim_batch_kernel<8><<<grid_for(n, 128), 128>>>(dU, dgcov, dgcon, dg, dpr, dpf, n, gam, gammafail, dit);
    else
      utoprim_batch_kernel<6><<<grid_for(n, 128), 128>>>(dU, dgcov, dgcon, dg, dpr, dpf, n, gam, gammafail, dit);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) {
      unsigned long long it = 0;
      cudaMemcpy(pr, dpr, sizeof(double) * 8 * n, cudaMemcpyDeviceToHost);
      cudaMemcpy(pflag, dpf, sizeof(int) * n, cudaMemcpyDeviceToHost);
      cudaMemcpy(&it, dit, sizeof(it), cudaMemcpyDeviceToHost);
      if (iters) *iters = (long long)it;
    } else {
      set_err("utoprim batch: %s", cudaGetErrorString(e));
      rc = HGPU_E_CUDA;
    }
  }
  cudaFree(dU);
  cudaFree(dgcov);
  cudaFree(dgcon);
  cudaFree(dg);
  cudaFree(dpr);
  cudaFree(dpf);
  cudaFree(dit);
  return rc;
}

int hgpu_utoprim_batch(const double *U, const double *gcov, const double *gcon, const double *gdet, double *pr,
                       int *pflag, long long n, double gam, double gammafail, long long *iters) {
  return utoprim_batch_impl(U, gcov, gcon, gdet, pr, pflag, n, gam, gammafail, HGPU_UTOPRIM2DFINAL, iters);
}

int hgpu_utoprimgen_batch(const double *U, const double *gcov, const double *gcon, const double *gdet, double *pr,
                          int *pflag, long long n, double gam, double gammafail, int utoprimversion,
                          long long *iters) {
  return utoprim_batch_impl(U, gcov, gcon, gdet, pr, pflag, n, gam, gammafail, utoprimversion, iters);
}

// ---------------------------------------------------------------------------
// Diagnostics (dump_ener.c): integrals of the conserved quantities and the
// flux-CT div B of the reference's divbmaxavg (dump_ener.c:482-520), over
// the active zones, with a deterministic two-pass reduction.
// ---------------------------------------------------------------------------
constexpr int DIAG_VALS = 12;  // 8 integrals, divb sum, divb max, failed zones, interior divb max
__device__ __forceinline__ bool diag_is_max(int q) { return q == 9 || q == 11; }
constexpr int DIAG_BLOCK = 256;

// DIVBFLUXCT (global.h:1586-1645) at the corner (i,j,k): B*gdet(CENT)
// averaged onto the corner and differenced, normalised; dims of size 1 use
// the same zone on both sides (im1mac(i) = i)
__device__ double divb_fluxct(const Dims &d, const Params &P, const double *__restrict__ p,
                              const double *__restrict__ G, int i, int j, int k) {
  const int s1 = d.s1, s2 = d.s2, s3 = d.s3;
  auto Fg = [&](int ii, int jj, int kk, int pl) {
    return p[(long long)pl * d.nz + zix(d, ii, jj, kk)] * __ldg(G + (long long)(G_CENT * GLOC + 33) * d.nij + gix(d, ii, jj));
  };
  auto avg1 = [&](int ii, int jj, int kk, int pl) { return 0.5 * (Fg(ii, jj, kk, pl) + Fg(ii - s1, jj, kk, pl)); };
  auto avg2 = [&](int ii, int jj, int kk, int pl) { return 0.5 * (Fg(ii, jj, kk, pl) + Fg(ii, jj - s2, kk, pl)); };
  auto for1 = [&](int ii, int jj, int kk) { return 0.5 * (avg2(ii, jj, kk, B1) + avg2(ii, jj, kk - s3, B1)); };
  auto for2 = [&](int ii, int jj, int kk) { return 0.5 * (avg1(ii, jj, kk, B2) + avg1(ii, jj, kk - s3, B2)); };
  auto for3 = [&](int ii, int jj, int kk) { return 0.5 * (avg2(ii, jj, kk, B3) + avg2(ii - s1, jj, kk, B3)); };
  double dfx = for1(i, j, k) - for1(i - s1, j, k);
  double dfy = for2(i, j, k) - for2(i, j - s2, k);
  double dfz = for3(i, j, k) - for3(i, j, k - s3);
  double nx = for1(i, j, k) + for1(i - s1, j, k);
  double ny = for2(i, j, k) + for2(i, j - s2, k);
  double nz = for3(i, j, k) + for3(i, j, k - s3);
  // corner gdet: CORNT is not kept on the device; the metric does not depend
  // on x3, so gdet at the true corner equals CORN3's
  double gc = __ldg(G + (long long)(G_CORN + 2) * d.nij + gix(d, i, j));
  double mx = max_ref(max_ref(P.dx1, P.dx2), P.dx3);
  double norm = mx / ((1.0 / 3.0) * gc * fabs(nx + ny + nz) + 1.e-50);
  return fabs((dfx / P.dx1 + dfy / P.dx2 + dfz / P.dx3) * norm);
}

// ufv: the evolved conserved state of the finite-volume scheme, which the
// reference's constotal integrates directly (dump_ener.c:611-619); nullptr:
// U(p) (dump_ener.c:622-630)
__global__ void __launch_bounds__(DIAG_BLOCK) diag_kernel(Dims d, Params P, Box box, const double *__restrict__ p,
                                                          const int *__restrict__ pflag, const double *__restrict__ G,
                                                          const double *__restrict__ ufv, double *__restrict__ part) {
  __shared__ double sh[DIAG_VALS][DIAG_BLOCK];
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double v[DIAG_VALS];
#pragma unroll
  for (int q = 0; q < DIAG_VALS; q++) v[q] = 0.0;
  if (t < box.size()) {
    int i, j, k;
    box_ijk(box, t, i, j, k);
    long long z = zix(d, i, j, k);
    Metric m;
    load_metric(G, d, gix(d, i, j), G_CENT, m);
    double pr[NPR], U[NPR];
    if (ufv) {
      load_prim(ufv, d, z, U);
    } else {
      load_prim(p, d, z, pr);
      State q;
      EM e;
      get_state(pr, m, q);
      em_prepare(pr, m, q, e);
      primtoflux(pr, q, e, 0, m, P.gam, U);
    }
    double dV = P.dx1 * P.dx2 * P.dx3;
#pragma unroll
    for (int pl = 0; pl < NPR; pl++) v[pl] = U[pl] * dV;
    double db = divb_fluxct(d, P, p, G, i, j, k);
    v[8] = db;
    v[9] = db;
    v[10] = (pflag[z] > 0) ? 1.0 : 0.0;
    // corners constrained by flux-CT: x1 corners 1..n1-1, x2 corners
    // 2..n2-2 (POLEDEATH resets B2 in the first and last rows, and gdet
    // vanishes at the axis corners), all x3 corners
    bool in1 = !d.s1 || (i >= 1 && i <= d.n1 - 1);
    bool in2 = !d.s2 || (j >= 2 && j <= d.n2 - 2);
    v[11] = (in1 && in2) ? db : 0.0;
  }
#pragma unroll
  for (int q = 0; q < DIAG_VALS; q++) sh[q][threadIdx.x] = v[q];
  __syncthreads();
  for (int w = DIAG_BLOCK / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
#pragma unroll
      for (int q = 0; q < DIAG_VALS; q++) {
        double a = sh[q][threadIdx.x], b = sh[q][threadIdx.x + w];
        sh[q][threadIdx.x] = diag_is_max(q) ? max_ref(a, b) : a + b;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x < DIAG_VALS) part[(long long)blockIdx.x * DIAG_VALS + threadIdx.x] = sh[threadIdx.x][0];
}

__global__ void __launch_bounds__(DIAG_BLOCK) diag_final_kernel(const double *__restrict__ part, int nblocks,
                                                                double *__restrict__ out) {
  __shared__ double sh[DIAG_BLOCK];
  for (int q = 0; q < DIAG_VALS; q++) {
    double a = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += DIAG_BLOCK) {
      double x = part[(long long)b * DIAG_VALS + q];
      a = diag_is_max(q) ? max_ref(a, x) : a + x;
    }
    sh[threadIdx.x] = a;
    __syncthreads();
    for (int w = DIAG_BLOCK / 2; w > 0; w >>= 1) {
      if (threadIdx.x < w) sh[threadIdx.x] = diag_is_max(q) ? max_ref(sh[threadIdx.x], sh[threadIdx.x + w])
                                                        : sh[threadIdx.x] + sh[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[q] = sh[0];
    __syncthreads();
  }
}

// progress of a context for a host that polls without blocking: t, dt,
// done, steps
__global__ void progress_kernel(const Scalars *sc, double *q) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    q[0] = sc->t;
    q[1] = sc->dt;
    q[2] = sc->done;
    q[3] = sc->nsteps;
  }
}

__global__ void set_dt_kernel(Scalars *sc) {
  if (threadIdx.x == 0 && blockIdx.x == 0) sc->dt = __longlong_as_double((long long)sc->ndtbits[0]);
}

int hgpu_init_dt(hgpu_ctx *x, double *dt) {
  if (!x) return HGPU_E_INVALID;
  launch_reset(x);
  launch_fluxes(x, x->p);
  launch_finalize(x, 0);
  if (!x->P.cell_inst) LAUNCH(x, K_OTHER, set_dt_kernel, 1, 32, x->sc);
  CUDA_TRY(cudaGetLastError());
  Scalars s;
  CUDA_TRY(cudaMemcpyAsync(&s, x->sc, sizeof(Scalars), cudaMemcpyDeviceToHost, x->stream));
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  if (dt) *dt = s.dt;
  return HGPU_OK;
}

int hgpu_step_ch_timed(hgpu_ctx *x, int nsteps, float *ms, hgpu_stats *stats) {
  if (!x || nsteps < 0) return HGPU_E_INVALID;
  if (boundaries_ready(x)) return HGPU_E_INVALID;
  cudaEvent_t a, b;
  CUDA_TRY(cudaEventCreate(&a));
  CUDA_TRY(cudaEventCreate(&b));
  clear_counters(x);
  CUDA_TRY(cudaEventRecord(a, x->stream));
  for (int n = 0; n < nsteps; n++) {
    for (int o = 0; o < num_orders(x); o++) launch_stage(x, o);
    launch_finalize(x, 1);
  }
  CUDA_TRY(cudaEventRecord(b, x->stream));
  CUDA_TRY(cudaEventSynchronize(b));
  float t = 0.f;
  cudaEventElapsedTime(&t, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (ms) *ms = t;
  return read_stats(x, stats);
}

// Autotuner: for each FP64 kernel family (flux, WENO5, conserve, invert)
// time both resident-block variants on the context's own state (one warm-up
// step and one timed step each, kernel times from the profiling events, the
// state restored before every trial) and keep the faster.  The variants
// differ only in register allocation, so results are identical whichever
// is chosen; the state is restored at the end.
int hgpu_autotune(hgpu_ctx *x, hgpu_tuning *out) {
  if (!x) return HGPU_E_INVALID;
  if (x->profiling) {
    set_err("hgpu_autotune: turn profiling off first");
    return HGPU_E_INVALID;
  }
  const long long nz = x->d.nz;
  const size_t pb = sizeof(double) * NPR * nz;
  const bool fv = x->cfg.doenoflux == HGPU_ENOFINITEVOLUME;
  double *sp = nullptr, *su = nullptr;
  int *sf = nullptr;
  Scalars *ss = nullptr;
  Inst *si = nullptr;  // a batch's per-instance t, dt, done, step count
  const size_t ib = sizeof(Inst) * (size_t)x->ninst;
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  CUDA_TRY(cudaMallocAsync(&sp, pb, x->stream));
  if (ib) {
    CUDA_TRY(cudaMallocAsync(&si, ib, x->stream));
    CUDA_TRY(cudaMemcpyAsync(si, x->inst, ib, cudaMemcpyDeviceToDevice, x->stream));
  }
  CUDA_TRY(cudaMallocAsync(&sf, sizeof(int) * nz, x->stream));
  CUDA_TRY(cudaMallocAsync(&ss, sizeof(Scalars), x->stream));
  if (fv) CUDA_TRY(cudaMallocAsync(&su, pb, x->stream));
  CUDA_TRY(cudaMemcpyAsync(sp, x->p, pb, cudaMemcpyDeviceToDevice, x->stream));
  CUDA_TRY(cudaMemcpyAsync(sf, x->pflag, sizeof(int) * nz, cudaMemcpyDeviceToDevice, x->stream));
  CUDA_TRY(cudaMemcpyAsync(ss, x->sc, sizeof(Scalars), cudaMemcpyDeviceToDevice, x->stream));
  if (fv) CUDA_TRY(cudaMemcpyAsync(su, x->ucum, pb, cudaMemcpyDeviceToDevice, x->stream));
  auto restore = [&]() {
    cudaMemcpyAsync(x->p, sp, pb, cudaMemcpyDeviceToDevice, x->stream);
    cudaMemcpyAsync(x->pflag, sf, sizeof(int) * nz, cudaMemcpyDeviceToDevice, x->stream);
    cudaMemcpyAsync(x->sc, ss, sizeof(Scalars), cudaMemcpyDeviceToDevice, x->stream);
    if (fv) cudaMemcpyAsync(x->ucum, su, pb, cudaMemcpyDeviceToDevice, x->stream);
    if (ib) cudaMemcpyAsync(x->inst, si, ib, cudaMemcpyDeviceToDevice, x->stream);
  };
  auto one_step = [&]() {
    clear_counters(x);
    for (int o = 0; o < num_orders(x); o++) launch_stage(x, o);
    launch_finalize(x, 1);
  };
  const bool fp64 = x->cfg.precision == HGPU_PREC_FP64;
  int *knob[4] = {&x->tune.flux, &x->tune.weno, &x->tune.conserve, &x->tune.invert};
  // the mixed-precision path runs the FP64 Riemann kernel after a WENO5
  // reconstruction (its FP32 kernels have fixed variants)
  const bool applies[4] = {fp64 || x->P.lim == HGPU_LIM_WENO5, fp64 && x->P.lim == HGPU_LIM_WENO5, true, true};
  const int kids[4][3] = {{K_FLUX1, K_FLUX2, K_FLUX3}, {K_WENO5, -1, -1}, {K_UPDATE, -1, -1}, {K_INVERT, -1, -1}};
  float ms[4][2] = {{0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}};
  int rc = HGPU_OK;
  x->profiling = true;
  for (int f = 0; f < 4 && !rc; f++) {
    if (!applies[f]) continue;
    for (int v = 0; v < 2 && !rc; v++) {
      *knob[f] = v;
      for (int rep = 0; rep < 2; rep++) {
        restore();
        one_step();
        if (cudaStreamSynchronize(x->stream) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
          rc = HGPU_E_CUDA;
          break;
        }
        collect_profile(x);
        double t = 0.0;
        for (int q = 0; q < 3; q++)
          if (kids[f][q] >= 0) t += x->kms[kids[f][q]];
        if (rep == 1) ms[f][v] = (float)t;
        for (int k = 0; k < K_NKERNELS; k++) {
          x->kms[k] = 0.0;
          x->kcount[k] = 0;
        }
      }
    }
    *knob[f] = (ms[f][1] < ms[f][0]) ? 1 : 0;
  }
  x->profiling = false;
  restore();
  // WENO5 tile shapes: per direction, the candidates of the cost model timed
  // on the current state (the face values are scratch: nothing else changes)
  float tile_ms[4] = {0.f, 0.f, 0.f, 0.f};
  if (!rc && x->P.lim == HGPU_LIM_WENO5) {
    const Dims &d = x->d;
    const int nd[4] = {0, d.n1, d.n2, d.n3};
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int dir = 1; dir <= 3 && !rc; dir++) {
      if (nd[dir] <= 1) continue;
      W5Tile cand[4];
      const int nc = w5_candidates(d, x->w5[dir].box, dir, cand, 4);
      float best = -1.f;
      W5Tile bt = x->w5[dir];
      for (int c = 0; c < nc; c++) {
        x->w5[dir] = cand[c];
        auto go = [&](bool state) {
          if (dir == 1) launch_w5_any<1>(x, x->p, state);
          else if (dir == 2) launch_w5_any<2>(x, x->p, state);
          else launch_w5_any<3>(x, x->p, state);
        };
        go(true);  // warm-up, with the state pieces
        cudaEventRecord(e0, x->stream);
        go(false);
        go(false);
        cudaEventRecord(e1, x->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
          rc = HGPU_E_CUDA;
          break;
        }
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        t *= 0.5f;
        if (best < 0.f || t < best) {
          best = t;
          bt = cand[c];
        }
      }
      x->w5[dir] = bt;
      tile_ms[dir] = best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (int k = 0; k < K_NKERNELS; k++) {
      x->kms[k] = 0.0;
      x->kcount[k] = 0;
    }
  }
  cudaFreeAsync(sp, x->stream);
  cudaFreeAsync(sf, x->stream);
  cudaFreeAsync(ss, x->stream);
  if (su) cudaFreeAsync(su, x->stream);
  if (si) cudaFreeAsync(si, x->stream);
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  // the captured step holds the old variants
  if (x->graph_exec) cudaGraphExecDestroy(x->graph_exec);
  if (x->graph) cudaGraphDestroy(x->graph);
  x->graph_exec = nullptr;
  x->graph = nullptr;
  if (out) {
    out->flux_minb = kFluxMB[x->tune.flux];
    out->weno_minb = kWenoMB[x->tune.weno];
    out->update_minb = kConserveMB[x->tune.conserve];
    out->invert_minb = kInvertMB[x->tune.invert];
    for (int q = 0; q < 4; q++) {
      const bool on = q >= 1 && x->P.lim == HGPU_LIM_WENO5;
      out->weno_lb[q] = on ? x->w5[q].lb : 0;
      out->weno_lines[q] = on ? x->w5[q].w : 0;
      out->weno_tile_ms[q] = tile_ms[q];
    }
    for (int v = 0; v < 2; v++) {
      out->flux_ms[v] = ms[0][v];
      out->weno_ms[v] = ms[1][v];
      out->update_ms[v] = ms[2][v];
      out->invert_ms[v] = ms[3][v];
      out->flux_cand[v] = kFluxMB[v];
      out->weno_cand[v] = kWenoMB[v];
      out->update_cand[v] = kConserveMB[v];
      out->invert_cand[v] = kInvertMB[v];
    }
  }
  return rc;
}

// apply a known choice (e.g. from an earlier hgpu_autotune of the same shape)
int hgpu_set_tuning(hgpu_ctx *x, const hgpu_tuning *t) {
  if (!x || !t) return HGPU_E_INVALID;
  auto pick = [](const int *cand, int minb) { return cand[1] == minb ? 1 : (cand[0] == minb ? 0 : -1); };
  const int f = pick(kFluxMB, t->flux_minb), b = pick(kWenoMB, t->weno_minb);
  const int u = pick(kConserveMB, t->update_minb), v = pick(kInvertMB, t->invert_minb);
  if (f < 0 || b < 0 || u < 0 || v < 0) return HGPU_E_INVALID;
  // WENO5 tilings (0: keep the current one)
  W5Tile w5[4];
  for (int q = 1; q <= 3; q++) {
    w5[q] = x->w5[q];
    const int lb = t->weno_lb[q], w = t->weno_lines[q];
    if (lb <= 0 || x->P.lim != HGPU_LIM_WENO5) continue;
    const Box &bx = x->w5[q].box;
    const int nout = q == 1 ? bx.ni : (q == 2 ? bx.nj : bx.nk);
    if (w < 1 || w > 32 || (w & (w - 1)) || lb > nout || w5_smem_bytes(lb, w, 8) > (long long)W5_SMEM_MAX) {
      set_err("hgpu_set_tuning: invalid WENO5 tiling");
      return HGPU_E_INVALID;
    }
    w5[q].lb = lb;
    w5[q].w = w;
    w5[q].nseg = (nout + lb - 1) / lb;
    w5[q].ntile = (w5[q].nlines + w - 1) / w;
    w5[q].wshift = 0;
    while ((1 << w5[q].wshift) < w) w5[q].wshift++;
  }
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  for (int q = 1; q <= 3; q++) x->w5[q] = w5[q];
  x->tune.flux = f;
  x->tune.weno = b;
  x->tune.conserve = u;
  x->tune.invert = v;
  if (x->graph_exec) cudaGraphExecDestroy(x->graph_exec);
  if (x->graph) cudaGraphDestroy(x->graph);
  x->graph_exec = nullptr;
  x->graph = nullptr;
  return HGPU_OK;
}

int hgpu_set_profiling(hgpu_ctx *x, int on) {
  if (!x) return HGPU_E_INVALID;
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  collect_profile(x);
  x->profiling = (on != 0);
  for (int k = 0; k < K_NKERNELS; k++) {
    x->kms[k] = 0.0;
    x->kcount[k] = 0;
  }
  return HGPU_OK;
}

int hgpu_kernel_times(hgpu_ctx *x, const char **names, double *ms, long long *launches, int n) {
  if (!x) return -HGPU_E_INVALID;
  if (cudaStreamSynchronize(x->stream) != cudaSuccess) return -HGPU_E_CUDA;
  collect_profile(x);
  for (int k = 0; k < K_NKERNELS && k < n; k++) {
    if (names) names[k] = kKernelNames[k];
    if (ms) ms[k] = x->kms[k];
    if (launches) launches[k] = x->kcount[k];
  }
  return K_NKERNELS;
}

long long hgpu_launch_count(hgpu_ctx *x) { return x ? x->launches : -1; }

// 8 independent multiply/add chains per thread; -fmad=false keeps DMUL and
// DADD separate (the instruction mix of the FP64 path)
__global__ void fp64_probe_kernel(double *out, int iters, double b, double c) {
  double a0 = threadIdx.x * 1e-9, a1 = a0 + 1e-3, a2 = a0 + 2e-3, a3 = a0 + 3e-3;
  double a4 = a0 + 4e-3, a5 = a0 + 5e-3, a6 = a0 + 6e-3, a7 = a0 + 7e-3;
  for (int it = 0; it < iters; it++) {
    a0 = a0 * b + c; a1 = a1 * b + c; a2 = a2 * b + c; a3 = a3 * b + c;
    a4 = a4 * b + c; a5 = a5 * b + c; a6 = a6 * b + c; a7 = a7 * b + c;
  }
  double s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (s == 12345.678) out[blockIdx.x] = s;  // keeps the chains alive
}

int hgpu_fp64_peak(double *tflops) {
  if (!tflops) return HGPU_E_INVALID;
  int dev = 0, sms = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  double *out = nullptr;
  CUDA_TRY(cudaMalloc(&out, sizeof(double) * sms * 8));
  const int iters = 4096, blocks = sms * 8, threads = 256;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  fp64_probe_kernel<<<blocks, threads>>>(out, 64, 0.999999, 1e-7);  // warm-up
  cudaEventRecord(a);
  fp64_probe_kernel<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
  cudaEventRecord(b);
  cudaError_t e = cudaEventSynchronize(b);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  if (e != cudaSuccess) {
    set_err("fp64 probe: %s", cudaGetErrorString(e));
    return HGPU_E_CUDA;
  }
  double ops = 2.0 * 8.0 * (double)iters * (double)blocks * (double)threads;
  *tflops = ops / (ms * 1e-3) / 1e12;
  return HGPU_OK;
}

int hgpu_alloc_pinned(size_t bytes, void **ptr) {
  if (!ptr) return HGPU_E_INVALID;
  CUDA_TRY(cudaHostAlloc(ptr, bytes, cudaHostAllocDefault));
  return HGPU_OK;
}

int hgpu_free_pinned(void *ptr) {
  if (ptr) CUDA_TRY(cudaFreeHost(ptr));
  return HGPU_OK;
}

int hgpu_batch_run(hgpu_ctx *x, int check_every, int max_steps, int *steps, float *ms, int *steps_per_instance,
                   float *done_ms) {
  if (!x || !x->inst || check_every < 1 || max_steps < 0) return HGPU_E_INVALID;
  cudaEvent_t a, b;
  CUDA_TRY(cudaEventCreate(&a));
  CUDA_TRY(cudaEventCreate(&b));
  std::vector<Inst> hi(x->ninst);
  std::vector<float> fin(x->ninst, -1.f);
  int taken = 0, rc = HGPU_OK;
  CUDA_TRY(cudaEventRecord(a, x->stream));
  while (taken < max_steps) {
    int k = check_every < max_steps - taken ? check_every : max_steps - taken;
    rc = hgpu_step_graph(x, k, nullptr);
    if (rc) break;
    taken += k;
    CUDA_TRY(cudaMemcpyAsync(hi.data(), x->inst, sizeof(Inst) * x->ninst, cudaMemcpyDeviceToHost, x->stream));
    CUDA_TRY(cudaEventRecord(b, x->stream));
    CUDA_TRY(cudaEventSynchronize(b));
    float now = 0.f;
    cudaEventElapsedTime(&now, a, b);
    int nd = 0;
    for (int q = 0; q < x->ninst; q++) {
      if (hi[q].done && fin[q] < 0.f) fin[q] = now;
      nd += hi[q].done != 0;
    }
    if (nd == x->ninst) break;
  }
  float total = 0.f;
  cudaEventElapsedTime(&total, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (rc) return rc;
  if (steps) *steps = taken;
  if (ms) *ms = total;
  for (int q = 0; q < x->ninst; q++) {
    if (steps_per_instance) steps_per_instance[q] = hi[q].nsteps;
    if (done_ms) done_ms[q] = fin[q];
  }
  return read_stats(x, nullptr);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// hgpu_utoprim_batch_noalloc: the batched inversion with its device scratch in
// a fixed file-scope array instead of cudaMalloc'd buffers.
// ---------------------------------------------------------------------------
namespace {

// per zone: U 8, gcov 16, gcon 16, gdet 1, pr 8 doubles; then pflag ints and
// the iteration counter
constexpr long long NA_DOUBLES_PER_ZONE = 8 + 16 + 16 + 1 + 8;
constexpr long long NA_MAX = HGPU_NOALLOC_MAX_ZONES;
constexpr size_t NA_BYTES = sizeof(double) * NA_DOUBLES_PER_ZONE * NA_MAX + sizeof(int) * NA_MAX + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

constexpr int NA_MAX_DEVICES = 64;
std::mutex g_na_mutex;
unsigned char *g_na_addr[NA_MAX_DEVICES] = {nullptr};

// device address of the scratch array on the current device (looked up once
// per device; the host-side symbol is only a handle, never a device pointer)
int noalloc_scratch_address(unsigned char **out) {
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NA_MAX_DEVICES) {
    set_err("device index %s%d out of range", "", dev);
    return HGPU_E_INVALID;
  }
  std::lock_guard<std::mutex> lock(g_na_mutex);
  if (!g_na_addr[dev]) {
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) {
      set_err("cudaGetSymbolAddress: %s", cudaGetErrorString(e));
      return HGPU_E_CUDA;
    }
    g_na_addr[dev] = (unsigned char *)ptr;
  }
  *out = g_na_addr[dev];
  return HGPU_OK;
}

}  // namespace

extern "C" int hgpu_utoprim_batch_noalloc(const double *U, const double *gcov, const double *gcon, const double *gdet,
                                          double *pr, int *pflag, long long n, double gam, double gammafail,
                                          long long *iters) {
  if (n < 0 || (n > 0 && (!U || !gcov || !gcon || !gdet || !pr || !pflag))) {
    set_err("invalid arguments");
    return HGPU_E_INVALID;
  }
  if (n > NA_MAX) {
    snprintf(g_errbuf, sizeof(g_errbuf), "batch of %lld zones exceeds HGPU_NOALLOC_MAX_ZONES=%lld; split the batch",
             n, (long long)NA_MAX);
    return HGPU_E_INVALID;
  }
  if (n == 0) {
    if (iters) *iters = 0;
    return HGPU_OK;
  }
  unsigned char *base = nullptr;
  int rc = noalloc_scratch_address(&base);
  if (rc) return rc;
  double *dU = (double *)base;
  double *dgcov = dU + 8 * NA_MAX;
  double *dgcon = dgcov + 16 * NA_MAX;
  double *dg = dgcon + 16 * NA_MAX;
  double *dpr = dg + NA_MAX;
  int *dpf = (int *)(dpr + 8 * NA_MAX);
  unsigned long long *dit = (unsigned long long *)(((uintptr_t)(dpf + NA_MAX) + 255) & ~(uintptr_t)255);
  CUDA_TRY(cudaMemcpy(dU, U, sizeof(double) * 8 * n, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(dgcov, gcov, sizeof(double) * 16 * n, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(dgcon, gcon, sizeof(double) * 16 * n, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(dg, gdet, sizeof(double) * n, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(dpr, pr, sizeof(double) * 8 * n, cudaMemcpyHostToDevice));
  // the counter keeps the previous call's value: clear it
  CUDA_TRY(cudaMemset(dit, 0, sizeof(unsigned long long)));
  utoprim_batch_kernel<6><<<grid_for(n, 128), 128>>>(dU, dgcov, dgcon, dg, dpr, dpf, n, gam, gammafail, dit);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaDeviceSynchronize());
  unsigned long long it = 0;
  CUDA_TRY(cudaMemcpy(pr, dpr, sizeof(double) * 8 * n, cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpy(pflag, dpf, sizeof(int) * n, cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpy(&it, dit, sizeof(it), cudaMemcpyDeviceToHost));
  if (iters) *iters = (long long)it;
  return HGPU_OK;

}

// ---------------------------------------------------------------------------
// Interfaces used by the serving loop (serve.cu)
// ---------------------------------------------------------------------------
cudaStream_t hg_stream(hgpu_ctx *x) { return x->stream; }

// Configuration of a context and whether it is a batch of 1D instances
// (host code elsewhere in the library: the restart dump writer).
const hgpu_config *hg_config(const hgpu_ctx *x, int *is_batch) {
  if (is_batch) *is_batch = x->ninst > 0;
  return &x->cfg;
}

// Enqueue on the context's stream a copy of (t, dt, done, steps) into host
// memory dst[4] (pinned) and record ev after it; the host tests ev with
// cudaEventQuery and reads dst once it has completed.
int hg_progress_async(hgpu_ctx *x, double *dst, cudaEvent_t ev) {
  if (!x->progress) CUDA_TRY(cudaMalloc(&x->progress, 4 * sizeof(double)));
  progress_kernel<<<1, 32, 0, x->stream>>>(x->sc, x->progress);
  CUDA_TRY(cudaMemcpyAsync(dst, x->progress, 4 * sizeof(double), cudaMemcpyDeviceToHost, x->stream));
  CUDA_TRY(cudaEventRecord(ev, x->stream));
  return HGPU_OK;
}

extern "C" size_t hgpu_context_bytes(const hgpu_config *c) {
  if (!c || validate(c)) return 0;
  auto tot = [&](int n) { return (size_t)(n > 1 ? n + 2 * c->ng : 1); };
  size_t nt1 = tot(c->n1), nt2 = tot(c->n2), nt3 = tot(c->n3);
  size_t nz = nt1 * nt2 * nt3;
  size_t nij = (nt1 + (c->n1 > 1)) * (nt2 + (c->n2 > 1));
  size_t zones = (size_t)c->n1 * c->n2 * c->n3;
  size_t cap = zones < (1u << 22) ? zones : (1u << 22);
  size_t plane = sizeof(double) * NPR * nz;
  size_t b = 7 * plane                       // p, pk, uf, ucum, F1..F3
             + sizeof(double) * 3 * nz        // corner EMFs
             + sizeof(double) * G_NCOMP * nij // geometry
             + sizeof(int) * 2 * nz           // pflag, candidate map
             + (size_t)nz                     // b^2 flags
             + sizeof(unsigned int) * NFFC * nz  // failure/floor counters
             + sizeof(double) * nz            // gamma check
             + cap * (2 * sizeof(long long) + 4 * sizeof(int) + 5 * sizeof(double))
             + plane;                         // staging for uploads and downloads
  if (c->lim == HGPU_LIM_WENO5) b += 2 * plane + sizeof(double) * 2 * nz;  // pL, pR, dP/P state pieces
  if (c->timeorder >= 3) b += plane;                     // pk1
  if (c->doenoflux == HGPU_ENOFINITEVOLUME) b += plane;  // ui
  if (c->bc[0] == HGPU_BC_BONDIMDOTOUTFLOW || c->bc[1] == HGPU_BC_BONDIINTOUTFLOW)
    b += sizeof(double) * 2 * (size_t)((c->n1 > 1 ? c->ng : 0) + 1) * c->n2 * 49;  // Bondi boundary table
  return b;
}

extern "C" int hgpu_diagnostics(hgpu_ctx *x, hgpu_diag *out) {
  if (!x || !out) return HGPU_E_INVALID;
  const Box &box = x->active_box;
  int nb = (int)grid_for(box.size(), DIAG_BLOCK);
  double *part = nullptr;
  CUDA_TRY(cudaMallocAsync(&part, sizeof(double) * ((size_t)nb * DIAG_VALS + DIAG_VALS), x->stream));
  const double *ufv = x->cfg.doenoflux == HGPU_ENOFINITEVOLUME ? x->ucum : nullptr;
  diag_kernel<<<nb, DIAG_BLOCK, 0, x->stream>>>(x->d, x->P, box, x->p, x->pflag, x->G, ufv, part);
  diag_final_kernel<<<1, DIAG_BLOCK, 0, x->stream>>>(part, nb, part + (size_t)nb * DIAG_VALS);
  double h[DIAG_VALS];
  Scalars s;
  cudaError_t e1 = cudaMemcpyAsync(h, part + (size_t)nb * DIAG_VALS, sizeof(h), cudaMemcpyDeviceToHost, x->stream);
  cudaError_t e2 = cudaMemcpyAsync(&s, x->sc, sizeof(Scalars), cudaMemcpyDeviceToHost, x->stream);
  cudaFreeAsync(part, x->stream);
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  if (e1 != cudaSuccess || e2 != cudaSuccess) return HGPU_E_CUDA;
  for (int q = 0; q < NPR; q++) out->integral[q] = h[q];
  long long zones = (long long)x->d.n1 * x->d.n2 * x->d.n3;
  out->divb_avg = h[8] / (double)zones;
  out->divb_max = h[9];
  out->divb_max_interior = h[11];
  out->nfail = (int)h[10];
  out->t = s.t;
  out->dt = s.dt;
  out->nsteps = s.nsteps;
  out->nfloor = (long long)s.nfloor;
  return HGPU_OK;
}

// unew of the reference (the conserved state U^{n+1} = the last stage's ucum,
// with gdet) in the reference's AoS layout, for restart dumps
// (rdump_content, restart.c:244-250, writes p and unew per zone)
extern "C" int hgpu_upload_conserved(hgpu_ctx *x, const double *unew) {
  if (!x || !unew || x->ninst > 0) return HGPU_E_INVALID;
  long long nz = x->d.nz;
  int rc = ensure_staging(x);
  if (rc) return rc;
  CUDA_TRY(cudaMemcpyAsync(x->staging, unew, sizeof(double) * NPR * nz, cudaMemcpyHostToDevice, x->stream));
  LAUNCH(x, K_OTHER, aos_to_soa_kernel, grid_for(nz * NPR, 256), 256, x->staging, x->ucum, nz);
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  CUDA_TRY(cudaGetLastError());
  return HGPU_OK;
}

extern "C" int hgpu_download_bsqflags(hgpu_ctx *x, int *flags) {
  if (!x || !flags) return HGPU_E_INVALID;
  const long long nz = x->d.nz;
  std::vector<unsigned char> h((size_t)nz);
  CUDA_TRY(cudaMemcpyAsync(h.data(), x->bsqf, (size_t)nz, cudaMemcpyDeviceToHost, x->stream));
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  for (long long z = 0; z < nz; z++) {
    flags[2 * z] = h[z] & 3;
    flags[2 * z + 1] = (h[z] >> 2) & 3;
  }
  return HGPU_OK;
}

extern "C" int hgpu_set_bondi_boundaries(hgpu_ctx *x, const double *table) {
  if (!x || !table || x->ninst > 0) return HGPU_E_INVALID;
  const size_t n = (size_t)2 * (x->d.g1 + 1) * x->d.n2 * 49;
  if (!x->bondi_tab) CUDA_TRY(cudaMalloc(&x->bondi_tab, sizeof(double) * n));
  CUDA_TRY(cudaMemcpyAsync(x->bondi_tab, table, sizeof(double) * n, cudaMemcpyHostToDevice, x->stream));
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  x->P.bondi = x->bondi_tab;
  // a captured step holds the parameters by value
  if (x->graph_exec) cudaGraphExecDestroy(x->graph_exec);
  if (x->graph) cudaGraphDestroy(x->graph);
  x->graph_exec = nullptr;
  x->graph = nullptr;
  return HGPU_OK;
}

extern "C" int hgpu_download_failfloorcount(hgpu_ctx *x, long long *counts, int clear) {
  if (!x || !counts) return HGPU_E_INVALID;
  const long long nz = x->d.nz;
  std::vector<unsigned int> h((size_t)(NFFC * nz));
  CUDA_TRY(cudaMemcpyAsync(h.data(), x->ffc, sizeof(unsigned int) * NFFC * nz, cudaMemcpyDeviceToHost, x->stream));
  if (clear) CUDA_TRY(cudaMemsetAsync(x->ffc, 0, sizeof(unsigned int) * NFFC * nz, x->stream));
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  for (long long z = 0; z < nz; z++)
    for (int c = 0; c < NFFC; c++) counts[z * NFFC + c] = (long long)h[(size_t)(c * nz + z)];
  return HGPU_OK;
}

extern "C" int hgpu_download_conserved(hgpu_ctx *x, double *unew) {
  if (!x || !unew) return HGPU_E_INVALID;
  long long nz = x->d.nz;
  int rc = ensure_staging(x);
  if (rc) return rc;
  LAUNCH(x, K_OTHER, soa_to_aos_kernel, grid_for(nz * NPR, 256), 256, x->ucum, x->staging, nz);
  CUDA_TRY(cudaMemcpyAsync(unew, x->staging, sizeof(double) * NPR * nz, cudaMemcpyDeviceToHost, x->stream));
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  return HGPU_OK;
}

// ---------------------------------------------------------------------------
// Domain split along x3 (the reference's MPI decomposition with ncpux3 ranks,
// boundmpi.c:6-180; pack / send-receive / unpack boundmpi.c:185-290).  A rank
// owns n3 planes of the global domain; its x3 ghost planes are the
// neighbours' edge planes.  The step runs as phases so that the caller can
// move the planes between phases (NCCL between GPUs, or device copies
// between domains on one GPU):
//   hgpu_stats_clear
//   per stage s: hgpu_stage_advance(s); exchange pf and pflag planes;
//                hgpu_stage_fixup(s);   exchange pf planes
//   exchange the per-direction ndt minima (minimum over ranks); hgpu_step_end(1)
// Every kernel reads the x3 ghosts only after the exchange that fills them,
// so the phases reproduce a whole-domain step bit for bit wherever the
// per-rank loops of fixup_utoprim see the same "already visited" neighbours
// (fixup.c:669-1470 counts an earlier failed neighbour that becomes fixed as
// good; across a rank boundary that neighbour is a ghost zone).
// Halo buffer of one face: [8 primitives][i][j][plane] doubles, then, with
// pflag, [i][j][plane] ints; i and j run over the ghosts too, so the x1/x2
// ghost corners travel with the planes.
// ---------------------------------------------------------------------------
__global__ void halo_x3_kernel(Dims d, double *p, int *pflag, unsigned char *buf, int side, int unpack,
                               int with_pflag) {
  const long long per_var = (long long)d.nt1 * d.nt2 * d.g3;
  const long long nvals = per_var * (NPR + (with_pflag ? 1 : 0));
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nvals) return;
  const int v = (int)(t / per_var);
  const long long r = t % per_var;
  // consecutive threads walk the planes of one (i,j) column, contiguous in k
  const long long ij = r / d.g3;
  const int layer = (int)(r % d.g3);
  int k;
  if (unpack) k = side == 0 ? layer - d.g3 : d.n3 + layer;
  else k = side == 0 ? layer : d.n3 - d.g3 + layer;
  const long long z = ij * d.nt3 + (k + d.g3);
  double *vb = (double *)buf;
  if (v < NPR) {
    const long long b = (long long)v * per_var + r;
    if (unpack) p[(long long)v * d.nz + z] = vb[b];
    else vb[b] = p[(long long)v * d.nz + z];
  } else {
    int *fb = (int *)(vb + (long long)NPR * per_var);
    if (unpack) pflag[z] = fb[r];
    else fb[r] = pflag[z];
  }
}

static int decomposable(const hgpu_ctx *x) { return x && !x->P.cell_inst && x->d.n3 > 1; }

extern "C" int hgpu_halo_bytes(hgpu_ctx *x, size_t *bytes) {
  if (!decomposable(x) || !bytes) return HGPU_E_INVALID;
  *bytes = (size_t)x->d.nt1 * x->d.nt2 * x->d.g3 * (NPR * sizeof(double) + sizeof(int));
  return HGPU_OK;
}

static int halo_io(hgpu_ctx *x, int stage, int side, int with_pflag, void *buf, int unpack) {
  if (!decomposable(x) || !buf || (side != 0 && side != 1) || stage < -1 || stage >= num_orders(x))
    return HGPU_E_INVALID;
  const long long n = (long long)x->d.nt1 * x->d.nt2 * x->d.g3 * (NPR + (with_pflag ? 1 : 0));
  LAUNCH(x, K_OTHER, halo_x3_kernel, grid_for(n, 256), 256, x->d, stage_output(x, stage), x->pflag,
         (unsigned char *)buf, side, unpack, with_pflag ? 1 : 0);
  CUDA_TRY(cudaGetLastError());
  return HGPU_OK;
}

extern "C" int hgpu_halo_pack(hgpu_ctx *x, int stage, int side, int with_pflag, void *dev_buf) {
  return halo_io(x, stage, side, with_pflag, dev_buf, 0);
}

extern "C" int hgpu_halo_unpack(hgpu_ctx *x, int stage, int side, int with_pflag, const void *dev_buf) {
  return halo_io(x, stage, side, with_pflag, const_cast<void *>(dev_buf), 1);
}

extern "C" int hgpu_stats_clear(hgpu_ctx *x) {
  if (!x) return HGPU_E_INVALID;
  clear_counters(x);
  CUDA_TRY(cudaGetLastError());
  return HGPU_OK;
}

extern "C" int hgpu_stats_read(hgpu_ctx *x, hgpu_stats *stats) {
  if (!x) return HGPU_E_INVALID;
  return read_stats(x, stats);
}

extern "C" int hgpu_stage_advance(hgpu_ctx *x, int stage) {
  if (!decomposable(x) || stage < 0 || stage >= num_orders(x)) return HGPU_E_INVALID;
  if (boundaries_ready(x)) return HGPU_E_INVALID;
  launch_stage_advance(x, stage);
  CUDA_TRY(cudaGetLastError());
  return HGPU_OK;
}

extern "C" int hgpu_stage_fixup(hgpu_ctx *x, int stage) {
  if (!decomposable(x) || stage < 0 || stage >= num_orders(x)) return HGPU_E_INVALID;
  if (boundaries_ready(x)) return HGPU_E_INVALID;
  launch_stage_fixup(x, stage);
  CUDA_TRY(cudaGetLastError());
  return HGPU_OK;
}

// post_fixup (fixup.c:37-96) on the context's state and flags, between
// steps: bound_pflag, fixup_checksolution, fixup_utoprim.  The candidate and
// fixup lists start empty; the stage's dt accumulators are left alone.
extern "C" int hgpu_post_fixup(hgpu_ctx *x, int finalstep, hgpu_stats *stats) {
  if (!x || x->P.cell_inst) return HGPU_E_INVALID;
  if (boundaries_ready(x)) return HGPU_E_INVALID;
  const Dims &d = x->d;
  clear_counters(x);
  CUDA_TRY(cudaMemsetAsync(&x->sc->ncand, 0, sizeof(int), x->stream));
  CUDA_TRY(cudaMemsetAsync(&x->sc->ndep, 0, sizeof(int), x->stream));
  CUDA_TRY(cudaMemsetAsync(&x->sc->nfixlist, 0, sizeof(int), x->stream));
  LAUNCH(x, K_BOUND_PFLAG, bound_pflag_kernel, grid_for(d.nz, 256), 256, d, x->P, x->pflag, x->sc);
  launch_checksol_fixup(x, x->p, finalstep ? 1 : 0);
  CUDA_TRY(cudaGetLastError());
  return read_stats(x, stats);
}

// start-up ndt (set_dt, advance.c:957) of a split domain: the fluxes of p,
// then the ndt exchange, then hgpu_step_end(x, 0)
extern "C" int hgpu_dt_probe(hgpu_ctx *x) {
  if (!decomposable(x)) return HGPU_E_INVALID;
  launch_reset(x);
  launch_fluxes(x, x->p);
  CUDA_TRY(cudaGetLastError());
  return HGPU_OK;
}

// advance_time 1: the dt update closing a step (step_ch.c:236-247);
// 0: dt = ndt, the start-up value
extern "C" int hgpu_step_end(hgpu_ctx *x, int advance_time) {
  if (!decomposable(x)) return HGPU_E_INVALID;
  launch_finalize(x, advance_time ? 1 : 0);
  if (!advance_time) LAUNCH(x, K_OTHER, set_dt_kernel, 1, 32, x->sc);
  CUDA_TRY(cudaGetLastError());
  return HGPU_OK;
}

// the three per-direction minima of cour*dx/ctop as order-preserving 64-bit
// patterns (positive doubles compare as integers), for a minimum over ranks
extern "C" int hgpu_ndt_pack(hgpu_ctx *x, unsigned long long *dev3) {
  if (!decomposable(x) || !dev3) return HGPU_E_INVALID;
  CUDA_TRY(cudaMemcpyAsync(dev3, &x->sc->ndtbits[1], 3 * sizeof(unsigned long long), cudaMemcpyDeviceToDevice,
                           x->stream));
  return HGPU_OK;
}

extern "C" int hgpu_ndt_unpack(hgpu_ctx *x, const unsigned long long *dev3) {
  if (!decomposable(x) || !dev3) return HGPU_E_INVALID;
  CUDA_TRY(cudaMemcpyAsync(&x->sc->ndtbits[1], dev3, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToDevice,
                           x->stream));
  return HGPU_OK;
}

extern "C" int hgpu_stream(hgpu_ctx *x, void **stream) {
  if (!x || !stream) return HGPU_E_INVALID;
  *stream = (void *)x->stream;
  return HGPU_OK;
}
