// Point formulas shared by the split-precision phi-stage kernels.
#pragma once

#include <cuda_runtime.h>

namespace mt {

// magic_torch/courant.py:25-77 in FP32 arithmetic (grid values are FP32; the
// maxima keep ~1e-7 relative accuracy)
__device__ __forceinline__ void courant_point_s(int mode, float vr, float vt, float vp, float br,
                                                float bt, float bp, float or2, float or4,
                                                float orho1, float orho2, float ost2, float LFfac,
                                                float cf2, float af2, float valri2, float valhi2,
                                                float& vr2, float& vh2) {
  const float vflr2 = orho2 * vr * vr;
  const float vflh2 = (vt * vt + vp * vp) * ost2 * orho2;
  if (mode == 0) {
    vr2 = cf2 * or4 * vflr2;
    vh2 = cf2 * or2 * vflh2;
    return;
  }
  const float valr = br * br * LFfac * orho1;
  const float valh2 = (bt * bt + bp * bp) * LFfac * ost2 * orho1;
  float valr2 = valr, valh2m = valh2;
  if (mode == 1) {
    valr2 = valr * valr / (valr + valri2);
    valh2m = valh2 * valh2 / (valh2 + valhi2);
  }
  vr2 = or4 * (cf2 * vflr2 + af2 * valr2);
  vh2 = or2 * (cf2 * vflh2 + af2 * valh2m);
}

__device__ __forceinline__ double block_max_d(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[w] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < nw ? red[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  }
  return v;
}

}  // namespace mt
