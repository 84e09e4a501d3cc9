// common.cuh -- device data layout and the reconstruction + Riemann-flux
// kernels shared by the FP64 translation unit (harm_gpu.cu, built with
// -fmad=false for bit-identity with the reference) and the FP32 one of the
// mixed-precision path (flux_f32.cu, built with FMA contraction and fast
// FP32 division/square root, which leave FP64 arithmetic untouched).
#pragma once
#include <cuda_runtime.h>

#include "harm_device.cuh"
#include "harmgpu.h"
#include "weno5.cuh"

namespace hg {

// geometry component offsets
constexpr int GLOC = 34;                  // per location: gcov 16, gcon 16, gcovpert_tt, gdet
constexpr int G_FACE1 = 0, G_FACE2 = 1, G_FACE3 = 2, G_CENT = 3;
constexpr int G_CORN = 4 * GLOC;          // CORN1, CORN2, CORN3 gdet
constexpr int G_CONN = G_CORN + 3;        // 64
constexpr int G_FLOOR = G_CONN + 64;      // 2
constexpr int G_NCOMP = G_FLOOR + 2;      // 205

// reference location ids (global.h:948-955)
constexpr int R_FACE1 = 0, R_FACE2 = 1, R_FACE3 = 2, R_CORN1 = 3, R_CORN2 = 4, R_CORN3 = 5, R_CENT = 7;

struct Dims {
  int n1, n2, n3;
  int g1, g2, g3;
  int nt1, nt2, nt3;
  int s1, s2, s3;
  int gt1, gt2;
  long long nz, nij;
};

// One instance of a batch: a 1D problem occupying the x1 cells
// i0-ng .. i0+n+ng-1 of the concatenated line (its own ghosts included),
// with its own gamma, dx, time and dt (step_ch's t, dt, tf per problem).
struct Inst {
  int i0, n;
  double dx, gam, tf;
  double t, dt;
  unsigned long long ndtbits;  // x1 min of cour*dx/ctop as ordered bits
  int done;                    // t reached tf: the instance no longer advances
  int nsteps;                  // time steps this instance has taken
};

struct Params {
  double gam, cour, gammamax, gammafail, rhominlimit, uuminlimit, defcon, safe, tf;
  double dx1, dx2, dx3;
  int lim, flux;
  int bc[6];
  // finite-volume scheme: faces beyond one zone across the grid (its flux
  // loops run over all transverse ghosts) feed only the dt minimum
  int fvring;
  // batch of independent 1D instances (nullptr: one domain)
  const int *cell_inst;  // instance of every cell of the line
  Inst *inst;
  int ninst;
  // failure and floor counters per zone, NFFC planes of nz (failfloorcount,
  // fixup.c:206): incremented where the reference's diag_fixup counts
  unsigned int *ffc;
  // Bondi-integral x1 boundaries: [2][g1+1][n2][49] coordinate data (nullptr: none)
  const double *bondi;
};

// counter categories (global.h:769-779)
enum {
  CNT_UTOPRIMFAILCONV = 0,
  CNT_FLOORACT = 1,
  CNT_LIMITGAMMAACT = 2,
  CNT_INFLOWACT = 3,
  CNT_UTOPRIMFAILRHONEG = 4,
  CNT_UTOPRIMFAILUNEG = 5,
  CNT_UTOPRIMFAILRHOUNEG = 6,
  CNT_GAMMAPERC = 7,
  CNT_UPERC = 8,
  NFFC = 9
};

__device__ __forceinline__ void ffc_count(const Params &P, long long nz, long long z, int what) {
  if (P.ffc) P.ffc[(long long)what * nz + z] += 1u;
}

// device scalars
struct Scalars {
  double t, dt;
  unsigned long long ndtbits[4];   // per-direction min of cour*dx/ctop as ordered bits
  unsigned long long iters;        // Newton iterations
  int err;
  int nfail;                       // failures after Utoprimgen in the last stage
  int ncand;                       // checksolution candidates
  int ndep;                        // checksolution candidates that depend on earlier ones
  int nfixlist;                    // fixup_utoprim list length
  int nfixed;
  int overflow;
  int done;                        // t reached tf: later steps leave the state unchanged
  int nsteps;                      // time steps taken since the last upload
  unsigned long long nfloor;       // zone floorings by fixup1zone (summed over a call's final substeps)
};

__device__ __forceinline__ long long zix(const Dims &d, int i, int j, int k) {
  return ((long long)(i + d.g1) * d.nt2 + (j + d.g2)) * d.nt3 + (k + d.g3);
}
__device__ __forceinline__ long long gix(const Dims &d, int i, int j) {
  return (long long)(i + d.g1) * d.gt2 + (j + d.g2);
}

__device__ __forceinline__ void load_metric(const double *__restrict__ G, const Dims &d, long long ij, int slot,
                                            Metric &m) {
  const double *b = G + (long long)slot * GLOC * d.nij + ij;
#pragma unroll
  for (int q = 0; q < 16; q++) m.gcov[q] = __ldg(b + (long long)q * d.nij);
#pragma unroll
  for (int q = 0; q < 16; q++) m.gcon[q] = __ldg(b + (long long)(16 + q) * d.nij);
  m.gcovpert_tt = __ldg(b + (long long)32 * d.nij);
  m.g = __ldg(b + (long long)33 * d.nij);
}

__device__ __forceinline__ void load_prim(const double *__restrict__ P, const Dims &d, long long z, double *pr) {
#pragma unroll
  for (int v = 0; v < NPR; v++) pr[v] = P[(long long)v * d.nz + z];
}
__device__ __forceinline__ void store_prim(double *__restrict__ P, const Dims &d, long long z, const double *pr) {
#pragma unroll
  for (int v = 0; v < NPR; v++) P[(long long)v * d.nz + z] = pr[v];
}

// box iteration helper: flat index -> (i,j,k) with k fastest
struct Box {
  int i0, j0, k0, ni, nj, nk;
  __host__ __device__ long long size() const { return (long long)ni * nj * nk; }
};
__device__ __forceinline__ void box_ijk(const Box &b, long long t, int &i, int &j, int &k) {
  k = (int)(t % b.nk);
  long long r = t / b.nk;
  j = (int)(r % b.nj);
  i = (int)(r / b.nj);
  i += b.i0;
  j += b.j0;
  k += b.k0;
}

__device__ __forceinline__ void warp_min_atomic(unsigned long long *dst, double v, bool active) {
  unsigned long long bits = active ? (unsigned long long)__double_as_longlong(v) : 0xFFFFFFFFFFFFFFFFull;
  // NaN is never selected by the reference's `if (dtij < ndt)`: map it out
  if (active && !(v == v)) bits = 0xFFFFFFFFFFFFFFFFull;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long ob = __shfl_xor_sync(0xffffffffu, bits, o);
    bits = ob < bits ? ob : bits;
  }
  if ((threadIdx.x & 31) == 0 && bits != 0xFFFFFFFFFFFFFFFFull) atomicMin(dst, bits);
}

// MC / VANL / MINM / DONOR slopes (interppoint.c:387-443)
template <typename T>
__device__ __forceinline__ T slope3(int lim, T yl, T yc, T yr) {
  if (lim == HGPU_LIM_MC) {
    T Dqm = T(2.0) * (yc - yl);
    T Dqp = T(2.0) * (yr - yc);
    T Dqc = T(0.5) * (yr - yl);
    T mm = ((Dqm) * (Dqp) <= T(0)) ? T(0.0) : ((fabs(Dqm) < fabs(Dqp)) ? (Dqm) : (Dqp));
    return ((Dqc) * (mm) <= T(0)) ? T(0.0) : ((fabs(Dqc) < fabs(mm)) ? (Dqc) : (mm));
  } else if (lim == HGPU_LIM_VANL) {
    T Dqm = (yc - yl);
    T Dqp = (yr - yc);
    T s = Dqm * Dqp;
    if (s <= T(0.)) return T(0.);
    return (T(2.0) * s / (Dqm + Dqp));
  } else if (lim == HGPU_LIM_MINM) {
    T Dqm = T(1.0) * (yc - yl);
    T Dqp = T(1.0) * (yr - yc);
    T Dqc = T(0.5) * (yr - yl);
    T mm = ((Dqm) * (Dqc) <= T(0)) ? T(0.0) : ((fabs(Dqm) < fabs(Dqc)) ? (Dqm) : (Dqc));
    return ((mm) * (Dqp) <= T(0)) ? T(0.0) : ((fabs(mm) < fabs(Dqp)) ? (mm) : (Dqp));
  }
  return T(0.0);
}

// para4 (interppoint.c:736-869) with PARA2LIM=MC and JONPARAREDUCE=0: face
// values of the cell at y[0] from y[-2..2]
template <typename T>
__device__ __forceinline__ void para4(const T *y, T *lout, T *rout) {
  T dq[3];
#pragma unroll
  for (int mm = -1; mm <= 1; mm++) {
    T Dqm = T(2.0) * (y[mm] - y[mm - 1]);
    T Dqp = T(2.0) * (y[mm + 1] - y[mm]);
    T Dqc = T(0.5) * (y[mm + 1] - y[mm - 1]);
    T aDqm = fabs(Dqm), aDqp = fabs(Dqp), aDqc = fabs(Dqc);
    T s = Dqm * Dqp;
    T sg = (Dqc > T(0.0)) ? T(1.0) : ((Dqc < T(0.0)) ? T(-1.0) : T(0.0));
    dq[mm + 1] = (s <= T(0.)) ? T(0.) : min_ref(aDqc, min_ref(aDqm, aDqp)) * sg;
  }
  T l = T(0.5) * (y[0] + y[-1]) - (dq[1] - dq[0]) / T(8.0);
  T r = T(0.5) * (y[1] + y[0]) - (dq[2] - dq[1]) / T(8.0);
  l = max_ref(min_ref(y[0], y[-1]), l);
  l = min_ref(max_ref(y[0], y[-1]), l);
  r = max_ref(min_ref(y[0], y[1]), r);
  r = min_ref(max_ref(y[0], y[1]), r);
  T qa = (r - y[0]) * (y[0] - l);
  T qd = (r - l);
  T qe = T(6.0) * (y[0] - T(0.5) * (l + r));
  if (qa <= T(0.)) {
    l = y[0];
    r = y[0];
  } else {
    if (qd * (qd - qe) < T(0.0)) l = T(3.0) * y[0] - T(2.0) * r;
    if (qd * (qd + qe) < T(0.0)) r = T(3.0) * y[0] - T(2.0) * l;
  }
  *lout = l;
  *rout = r;
}

// Minimum resident blocks per SM asked of the register allocator for the
// FP64-heavy kernels (launch_bounds' second argument).  With 64K registers
// per SM, B blocks of 128 threads cap a thread at 65536 / (128 B) registers:
// 1-2 -> 255 (8 warps/SM), 3 -> 170 (12 warps), 4 -> 128 (16 warps), more
// warps to hide FP64 latency at the price of spills to local memory.
// Defaults from a B200 sweep (256x128x128 torus, 1/3/4/5 blocks for flux and
// update): flux 4 (-11% WENO5, -21% MC); update is fastest unconstrained.
// The WENO5 kernel runs blocks of 256 threads (W5_THREADS).
#ifndef HG_MINB_FLUX
#define HG_MINB_FLUX 4
#endif
#ifndef HG_MINB_UPDATE
#define HG_MINB_UPDATE 4
#endif
#ifndef HG_MINB_INVERT
#define HG_MINB_INVERT 1
#endif
#ifndef HG_MINB_WENO
#define HG_MINB_WENO 3
#endif
// the same for the FP32 kernels of the mixed-precision path (B200 sweep of
// 4/6/8 for flux: 8 -4%)
#ifndef HG_MINB_FLUX_F32
#define HG_MINB_FLUX_F32 8
#endif
#ifndef HG_MINB_WENO_F32
#define HG_MINB_WENO_F32 4
#endif
template <typename T> struct MinBlocks;
template <> struct MinBlocks<double> {
  static constexpr int flux = HG_MINB_FLUX, weno = HG_MINB_WENO;
};
template <> struct MinBlocks<float> {
  static constexpr int flux = HG_MINB_FLUX_F32, weno = HG_MINB_WENO_F32;
};

// the FP64 variants the autotuner chooses between (resident blocks per SM
// for each heavy kernel; variant 0 is the default above)
constexpr int kFluxMB[2] = {HG_MINB_FLUX, HG_MINB_FLUX - 1};
constexpr int kWenoMB[2] = {HG_MINB_WENO, HG_MINB_WENO + 1};
constexpr int kConserveMB[2] = {HG_MINB_UPDATE, 3};
constexpr int kInvertMB[2] = {HG_MINB_INVERT, 2};

template <int DIR>
__device__ __forceinline__ long long dir_stride(const Dims &d) {
  return (DIR == 1) ? (long long)d.nt2 * d.nt3 : ((DIR == 2) ? (long long)d.nt3 : 1);
}

// metric of one location converted to the arithmetic type of a kernel
template <typename T>
__device__ __forceinline__ void load_metric_t(const double *__restrict__ G, const Dims &d, long long ij, int slot,
                                              MetricT<T> &m) {
  const double *b = G + (long long)slot * GLOC * d.nij + ij;
#pragma unroll
  for (int q = 0; q < 16; q++) m.gcov[q] = (T)__ldg(b + (long long)q * d.nij);
#pragma unroll
  for (int q = 0; q < 16; q++) m.gcon[q] = (T)__ldg(b + (long long)(16 + q) * d.nij);
  m.gcovpert_tt = (T)__ldg(b + (long long)32 * d.nij);
  m.g = (T)__ldg(b + (long long)33 * d.nij);
}

// ---------------------------------------------------------------------------
// WENO5 line reconstruction (slope_lim_linetype_c2e, interpline.c:517-678),
// one kernel per direction.  The reference sweeps whole lines serially; here
// a block owns a tile: `lb` consecutive output cells along the direction on
// `w` lines, and stages what the cells of the tile share in shared memory so
// that every per-cell quantity is computed once:
//   S  per output cell: the post/pre-shock reduction factor of
//      apply_additional_reduction_to_weights (reconstructeno.c:650-700) from
//      the dP/P jump of compute_df_line_new (interpline.c:2148-2222) over
//      cells -1, 0, +1, whose state pieces w5_state_kernel formed once per
//      zone for all three directions
//   for each primitive v:
//   Y  the line of v, cells -5..lb+4
//   A  per cell -3..lb+2: SMONO cusp test and indicator, unoptimised order-3
//      weights (compute_cf_stencil_weights + mono_adjust_unoptimized_weights)
//   R  per cell -1..lb: lower-order fraction of compute_weights_ratios
//   F  per output cell: the final fraction (the cell's own, and the shock
//      factor times its neighbours'), optimised and order-2 weights and the
//      two face values -> pL, pR
// The output cells of a direction are the line cells -1..n (the box), every
// line across it that the flux loop covers.  Every quantity is formed by the
// same device functions, in the same operation order, as before tiling, so
// the FP64 results stay bit-identical to the reference.  T = float is the
// reconstruction of the mixed-precision path: its line is kept in FP64, it
// works on differences from each cell's own value and writes FP64 face
// values (the cell's value plus the FP32 offset), which the FP64 Riemann
// kernel reads.
// ---------------------------------------------------------------------------
constexpr int W5_THREADS = 256;

struct W5Tile {
  Box box;      // output cells
  int lb;       // output cells per tile along the direction
  int w;        // lines per tile (a power of two, at most 32)
  int wshift;   // log2(w)
  int nseg;     // tiles along the direction
  int ntile;    // tiles across (ceil(nlines / w))
  int nlines;   // lines of the box
  int fast_s;   // 1: threads walk along the line (its cells are contiguous in memory), 0: across lines
};

// The dP/P pieces of compute_df_line_new (interpline.c:2148-2222) of one
// zone, (1 + u_t) u^t and gam u (u^t u_t) + (gam - 1) u, into PU[0][z] and
// PU[1][z]: they depend on the zone's state only, so one pass serves the
// WENO5 reconstruction of every direction.
template <typename T>
__global__ void __launch_bounds__(128) w5_state_kernel(Dims d, Params P, Box box, const double *__restrict__ pb,
                                                       const double *__restrict__ G, T *__restrict__ PU) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= box.size()) return;
  int i, j, k;
  box_ijk(box, t, i, j, k);
  const long long z = zix(d, i, j, k);
  const T gam = (T)(P.cell_inst ? P.inst[P.cell_inst[z]].gam : P.gam);
  T pc[NPR];
#pragma unroll
  for (int v = 0; v < NPR; v++) pc[v] = (T)pb[(long long)v * d.nz + z];
  MetricT<T> m;
  load_metric_t(G, d, gix(d, i, j), G_CENT, m);
  StateT<T> q;
  get_state(pc, m, q);
  const T a = compute_1plusud0(m, q);
  PU[z] = a * (q.ucon[0]);
  PU[d.nz + z] = gam * pc[UU] * (q.ucon[0] * q.ucov[0]) + (gam - T(1.0)) * pc[UU];
}

// shared-memory bytes of a tile with lb output cells on w lines: per line
// Y (lb+10) in FP64, and in the arithmetic type (tsize bytes) A 4 (lb+6),
// R (lb+2) and the shock factor lb
__host__ __device__ inline long long w5_smem_bytes(int lb, int w, int tsize) {
  return (long long)w * (8LL * (lb + 10) + (long long)tsize * (6LL * lb + 26));
}

// zone index of cell 0 of line `line` of box b (along the line the index
// steps by dir_stride)
template <int DIR>
__device__ __forceinline__ long long w5_line(const Dims &d, const Box &b, int line) {
  int i = 0, j = 0, k = 0;
  if (DIR == 1) {
    j = b.j0 + line / b.nk;
    k = b.k0 + line % b.nk;
  } else if (DIR == 2) {
    i = b.i0 + line / b.nk;
    k = b.k0 + line % b.nk;
  } else {
    i = b.i0 + line / b.nj;
    j = b.j0 + line % b.nj;
  }
  return zix(d, i, j, k);
}

template <int DIR, bool FS, typename T, int MB = MinBlocks<T>::weno>
__global__ void __launch_bounds__(W5_THREADS, MB) weno5_kernel(Dims d, Params P, W5Tile tl,
                                                               const double *__restrict__ pb,
                                                               const T *__restrict__ PU, double *__restrict__ pL,
                                                               double *__restrict__ pR) {
  extern __shared__ __align__(16) unsigned char w5_smem[];
  __shared__ long long zb[32];
  const int W = tl.w;
  const int seg = blockIdx.x % tl.nseg;
  const int line0 = (blockIdx.x / tl.nseg) * W;
  const int nl = min(W, tl.nlines - line0);
  const int nout = (DIR == 1) ? tl.box.ni : ((DIR == 2) ? tl.box.nj : tl.box.nk);
  const int c0 = ((DIR == 1) ? tl.box.i0 : ((DIR == 2) ? tl.box.j0 : tl.box.k0)) + seg * tl.lb;
  const int nv = min(tl.lb, nout - seg * tl.lb);  // output cells of this tile
  const int NS = nv + 10, NA = nv + 6, NL = nv + 2;
  const long long o = dir_stride<DIR>(d);
  // this thread's line w and first cell r; it steps along the line by TL
  const int TL = W5_THREADS >> tl.wshift;
  const int w = FS ? (int)(threadIdx.x / TL) : (int)(threadIdx.x & (W - 1));
  const int r = FS ? (int)(threadIdx.x & (TL - 1)) : (int)(threadIdx.x >> tl.wshift);
  const bool on = w < nl;
  if (threadIdx.x < nl) zb[threadIdx.x] = w5_line<DIR>(d, tl.box, line0 + threadIdx.x);
  double *Y = reinterpret_cast<double *>(w5_smem);                  // cells -5 .. nv+4
  T *A = reinterpret_cast<T *>(Y + (long long)NS * W);  // 4 planes, cells -3 .. nv+2: code (indicator, -1 at a cusp), w0, w1, w2
  T *R = A + 4LL * NA * W;          // cells -1 .. nv: lower-order fraction
  T *SS = R + (long long)NL * W;    // output cells: shock reduction factor
  // element s of this thread's line in a plane with n cells per line
  auto at = [&](T *plane, int n, int s) -> T & { return FS ? plane[w * n + s] : plane[s * W + w]; };
  auto aty = [&](int s) -> double & { return FS ? Y[w * NS + s] : Y[s * W + w]; };
  // the stencil of the cell at Y index sc: yd[] for differences and linear
  // combinations, yn[] for magnitudes (the same values in FP64; in FP32 the
  // offsets from the cell's own value and the values)
  auto stencil = [&](int sc, T *yd, T *yn, double &yc) {
    yc = aty(sc);
#pragma unroll
    for (int q = 0; q < 5; q++) {
      const double yq = aty(sc - 2 + q);
      if constexpr (sizeof(T) == 4) {
        yd[q] = (T)(yq - yc);
        yn[q] = (T)yq;
      } else {
        yd[q] = yq;
        yn[q] = yq;
      }
    }
  };
  __syncthreads();
  const long long zl = on ? zb[w] : 0;

  // S: the reduction factor of each output cell from the state pieces of
  // cells -1, 0, +1 (no barrier needed before stage Y: different planes)
  if (on)
    for (int s = r; s < nv; s += TL) {
      const long long z = zl + (long long)(c0 + s) * o;
      const T parl = __ldg(PU + z - o), par = __ldg(PU + z), parr = __ldg(PU + z + o);
      const T uparl = __ldg(PU + d.nz + z - o), upar = __ldg(PU + d.nz + z), uparr = __ldg(PU + d.nz + z + o);
      const T r0 = (T)__ldg(pb + z);
      const T dP =
          (fabs(r0 * (parr - parl)) + fabs(uparr - uparl)) / (fabs(r0 * par) + fabs(upar) + w5::K<T>::tiny);
      // (x / 0.25 is the exact multiplication by 4)
      at(SS, nv, s) = w5::wmin((fabs(dP) - T(0.5 * w5::kDpFrac)) * T(1.0 / (0.5 * w5::kDpFrac)), T(1.));
    }

  T *CODE = A, *W0 = A + (long long)NA * W, *W1 = A + 2LL * NA * W, *W2 = A + 3LL * NA * W;
  for (int v = 0; v < NPR; v++) {
    const double *pv = pb + (long long)v * d.nz + zl;
    // Y: the line of primitive v
    if (on)
      for (int s = r; s < NS; s += TL) aty(s) = __ldg(pv + (long long)(c0 - 5 + s) * o);
    __syncthreads();
    // A: cusp test, SMONO indicator, unoptimised weights of cells -3..nv+2
    if (on)
      for (int s = r; s < NA; s += TL) {
        T ya[5], yb[5];
        double yc;
        stencil(s + 2, ya, yb, yc);
        const T *y = ya + 2, *yn = yb + 2;
        const bool c = w5::cusp(y, yn);
        const T m0 = c ? T(0.0) : w5::mono(y, yn);
        T wt[3];
        w5::unopt3(m0, y, yn, wt);
        at(CODE, NA, s) = c ? T(-1.0) : m0;
        at(W0, NA, s) = wt[0];
        at(W1, NA, s) = wt[1];
        at(W2, NA, s) = wt[2];
      }
    __syncthreads();
    // R: lower-order fraction of cells -1..nv from the weights of cells -3..nv+2
    if (on)
      for (int s = r; s < NL; s += TL) {
        const int a = s + 2;  // cell s-1 in the A planes
        const T wc[3] = {at(W0, NA, a), T(0.0), at(W2, NA, a)};
        at(R, NL, s) =
            w5::ratio_lof(wc, at(W0, NA, a - 2), at(W2, NA, a + 2), at(CODE, NA, a) == T(-1.0) ? T(1.0) : T(0.0));
      }
    __syncthreads();
    // F: face values of the output cells
    if (on)
      for (int s = r; s < nv; s += TL) {
        const T ss = at(SS, nv, s);
        T lof = at(R, NL, s + 1);
        lof = w5::wmax(lof, ss * at(R, NL, s + 2));
        lof = w5::wmax(lof, ss * at(R, NL, s));
        const int a = s + 3;
        const T c0v = at(CODE, NA, a);
        const T wc[3] = {at(W0, NA, a), at(W1, NA, a), at(W2, NA, a)};
        T ya[5], yb[5];
        double yc;
        stencil(s + 5, ya, yb, yc);
        const bool cu = (c0v == T(-1.0));
        T yl, yr;
        w5::faces(ya + 2, yb + 2, cu ? T(0.0) : c0v, cu, wc, lof, &yl, &yr);
        const long long z = zl + (long long)(c0 + s) * o + (long long)v * d.nz;
        if constexpr (sizeof(T) == 4) {
          pL[z] = yc + (double)yl;
          pR[z] = yc + (double)yr;
        } else {
          pL[z] = yl;
          pR[z] = yr;
        }
      }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// face flux kernel (one per direction); RECON 0: MC-type slopes in the
// kernel, RECON 1: Riemann states from the WENO5 face values pL/pR (stored
// as TR), RECON 2: PARA
// ---------------------------------------------------------------------------
// MIX = 1: the mixed-precision variant of the FP64 kernel (wave speeds in
// FP32, vchar_f32; instantiated only in flux_f32.cu, whose FP64 arithmetic
// may contract a*b+c into FMA)
template <int DIR, int RECON, typename T, int MB = MinBlocks<T>::flux, typename TR = T, int MIX = 0>
__global__ void __launch_bounds__(128, MB) flux_kernel(Dims d, Params P, Box box,
                                                                 const double *__restrict__ pb,
                                                                 const TR *__restrict__ pL, const TR *__restrict__ pR,
                                                                 const double *__restrict__ G, double *__restrict__ F,
                                                                 Scalars *sc) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  bool active = t < box.size();
  double dtij = 0.0;
  if (active) {
    int i, j, k;
    box_ijk(box, t, i, j, k);
    long long z = zix(d, i, j, k);
    const long long o = dir_stride<DIR>(d);
    T p_l[NPR], p_r[NPR];
    if (RECON == 1) {
      // getp2interplr (flux.c:788-808), line-type branch
#pragma unroll
      for (int v = 0; v < NPR; v++) {
        p_l[v] = (T)__ldg(pR + (long long)v * d.nz + z - o);
        p_r[v] = (T)__ldg(pL + (long long)v * d.nz + z);
      }
    } else if (RECON == 2) {
      // PARA: pright of the cell on the left, pleft of the cell on the right
#pragma unroll
      for (int v = 0; v < NPR; v++) {
        const double *q = pb + (long long)v * d.nz + z;
        T y[6];
#pragma unroll
        for (int l = 0; l < 6; l++) y[l] = (T)__ldg(q + (l - 3) * o);
        T dummy;
        para4(y + 2, &dummy, &p_l[v]);
        para4(y + 3, &p_r[v], &dummy);
      }
    } else {
#pragma unroll
      for (int v = 0; v < NPR; v++) {
        const double *q = pb + (long long)v * d.nz + z;
        T ym2 = (T)__ldg(q - 2 * o), ym1 = (T)__ldg(q - o), y0 = (T)__ldg(q), yp1 = (T)__ldg(q + o);
        T dqm = slope3(P.lim, ym2, ym1, y0);
        T dq0 = slope3(P.lim, ym1, y0, yp1);
        // getp2interplr (flux.c:788-808)
        p_l[v] = ym1 + T(0.5) * dqm;
        p_r[v] = y0 - T(0.5) * dq0;
      }
    }
    // BDIRCONT (flux.c:629-633)
    p_l[B1 + DIR - 1] = p_r[B1 + DIR - 1] = T(0.5) * (p_l[B1 + DIR - 1] + p_r[B1 + DIR - 1]);
    MetricT<T> m;
    load_metric_t(G, d, gix(d, i, j), DIR - 1, m);
    int b = P.cell_inst ? P.cell_inst[z] : -1;
    const T gam = (T)(b >= 0 ? P.inst[b].gam : P.gam);
    int err = 0;
    // a face that only feeds the dt minimum needs the wave speeds alone
    bool ring = false;
    if (P.fvring) {
      if (DIR != 1 && (i < -d.s1 || i > d.n1 - 1 + d.s1)) ring = true;
      if (DIR != 2 && (j < -d.s2 || j > d.n2 - 1 + d.s2)) ring = true;
      if (DIR != 3 && (k < -d.s3 || k > d.n3 - 1 + d.s3)) ring = true;
    }
    T cmaxl = T(0.), cminl = T(0.), cmaxr = T(0.), cminr = T(0.);
    T Fl[NPR], Fr[NPR], Ul[NPR], Ur[NPR];
    {
      StateT<T> q;
      if (get_state(p_l, m, q)) err |= ERR_UTCALC_DISCR;
      if constexpr (MIX != 0) err |= vchar_f32(p_l, q, DIR, m, gam, &cmaxl, &cminl);
      else err |= vchar(p_l, q, DIR, m, gam, &cmaxl, &cminl);
      if (!ring) {
        EMT<T> e;
        em_prepare(p_l, m, q, e);
        primtoflux(p_l, q, e, DIR, m, gam, Fl);
        primtoflux(p_l, q, e, 0, m, gam, Ul);
      }
    }
    {
      StateT<T> q;
      if (get_state(p_r, m, q)) err |= ERR_UTCALC_DISCR;
      if constexpr (MIX != 0) err |= vchar_f32(p_r, q, DIR, m, gam, &cmaxr, &cminr);
      else err |= vchar(p_r, q, DIR, m, gam, &cmaxr, &cminr);
      if (!ring) {
        EMT<T> e;
        em_prepare(p_r, m, q, e);
        primtoflux(p_r, q, e, DIR, m, gam, Fr);
        primtoflux(p_r, q, e, 0, m, gam, Ur);
      }
    }
    // cminmax_calc (wavespeeds.c:325-385)
    T lmin = min_ref(cminl, cminr);
    T lmax = max_ref(cmaxl, cmaxr);
    lmin = fabs(max_ref(T(0.), -lmin));
    lmax = fabs(max_ref(T(0.), lmax));
    T cmin = lmin, cmax = lmax, ctop = max_ref(lmax, lmin);
    if (!ring) {
      double Fo[NPR];
      if (P.flux == HGPU_FLUX_HLL && (cmax + cmin != T(0.0))) {
#pragma unroll
        for (int v = 0; v < NPR; v++)
          Fo[v] = (double)(((cmax * Fl[v] + cmin * Fr[v]) - (cmax * cmin) * (Ur[v] - Ul[v])) / (cmax + cmin));
      } else {
#pragma unroll
        for (int v = 0; v < NPR; v++) Fo[v] = (double)(T(0.5) * ((Fl[v] + Fr[v]) - ctop * (Ur[v] - Ul[v])));
      }
      // flux_ct gdet strip (fluxct.c:74-96), in FP64 in both precision modes
      const double gface = __ldg(G + (long long)((DIR - 1) * GLOC + 33) * d.nij + gix(d, i, j));
      Fo[B1] /= gface;
      Fo[B2] /= gface;
      Fo[B3] /= gface;
      store_prim(F, d, z, Fo);
    }
    double dxd = (DIR == 1) ? P.dx1 : ((DIR == 2) ? P.dx2 : P.dx3);
    if (b >= 0) {
      // batch: faces 0..n of a running instance feed its own dt
      const Inst &I = P.inst[b];
      int loc = i - I.i0;
      active = false;
      if (loc >= 0 && loc <= I.n && !I.done) {
        dtij = P.cour * I.dx / (double)ctop;
        if (dtij == dtij) atomicMin(&P.inst[b].ndtbits, (unsigned long long)__double_as_longlong(dtij));
        if (err) atomicOr(&sc->err, err);
      }
    } else {
      dtij = P.cour * dxd / (double)ctop;
      if (err) atomicOr(&sc->err, err);
    }
  }
  warp_min_atomic(&sc->ndtbits[DIR], dtij, active);
}


}  // namespace hg
