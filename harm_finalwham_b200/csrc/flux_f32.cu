// flux_f32.cu -- the kernels of the mixed-precision path (HGPU_PREC_MIXED):
// the FP32 reconstruction and Riemann kernels, and the WENO5 Riemann kernel
// with FP64 states and fluxes and FP32 wave speeds (flux_kernel<.., MIX = 1>).
// This translation unit is compiled with FMA contraction and fast FP32
// division and square root (-fmad=true -prec-div=false -prec-sqrt=false
// -ftz=true).  -fmad=true also lets the FP64 arithmetic of the MIX = 1
// kernels contract a*b+c into FMA, which the mixed path allows; the
// bit-identical FP64 kernels live in harm_gpu.cu, compiled with -fmad=false.
// harm_gpu.cu launches these instantiations (declared there as extern
// templates).
#include "common.cuh"

namespace hg {

#define HG_F32_INSTANCES(DIR)                                                                                      \
  template __global__ void weno5_kernel<DIR, true, float>(Dims, Params, W5Tile, const double *, const float *,    \
                                                          double *, double *);                                      \
  template __global__ void weno5_kernel<DIR, false, float>(Dims, Params, W5Tile, const double *, const float *,   \
                                                           double *, double *);                                     \
  template __global__ void flux_kernel<DIR, 0, float>(Dims, Params, Box, const double *, const float *,           \
                                                      const float *, const double *, double *, Scalars *);          \
  template __global__ void flux_kernel<DIR, 2, float>(Dims, Params, Box, const double *, const float *,           \
                                                      const float *, const double *, double *, Scalars *);          \
  template __global__ void flux_kernel<DIR, 1, double, kFluxMB[0], double, 1>(                                    \
      Dims, Params, Box, const double *, const double *, const double *, const double *, double *, Scalars *);      \
  template __global__ void flux_kernel<DIR, 1, double, kFluxMB[1], double, 1>(                                    \
      Dims, Params, Box, const double *, const double *, const double *, const double *, double *, Scalars *);

HG_F32_INSTANCES(1)
HG_F32_INSTANCES(2)
HG_F32_INSTANCES(3)
template __global__ void w5_state_kernel<float>(Dims, Params, Box, const double *, const double *, float *);

}  // namespace hg
