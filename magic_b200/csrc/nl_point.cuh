// Point formulas shared by the phi-stage kernels.
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

// Anelastic phi stage (k_nl_anel_split in FP32, k_nl_anel_f64 in FP64).  Grid
// fields (rows 2 f, 2 f + 1 of the synthesis): 0 vr, 1 vt, 2 vp, 3 dvrdr,
// 4 dvtdr, 5 dvpdr, 6 dvrdt, 7 dvrdp, 8 dvtdp, 9 dvpdp, 10 cvr, 11 s, [12 xi],
// then br bt bp cbr cbt cbp.  Products: 0 Advr, 1 Advt, 2 Advp, 3 VSr, 4 VSt,
// 5 VSp, [VxBr VxBt VxBp], [VXir VXit VXip], heat.
template <bool MAG, bool CHEM>
struct AnelFields {
  static constexpr int NFI = 12 + (CHEM ? 1 : 0) + (MAG ? 6 : 0);
  static constexpr int NFO = 7 + (MAG ? 3 : 0) + (CHEM ? 3 : 0);
  static constexpr int NB = NFI > NFO ? NFI : NFO;
  static constexpr int IB = 12 + (CHEM ? 1 : 0);  // first magnetic grid field
  static constexpr int IX = 6 + (MAG ? 3 : 0);    // first composition product
  static constexpr int THW = 32 * ((NB + 1) / 2);  // threads of the half-warp variant
  __host__ __device__ static constexpr bool radial(int o) {
    return o == 0 || o == 3 || (MAG && o == 6) || (CHEM && o == IX) || o == NFO - 1;
  }
};

// Per-level constants of the products in the phi stage's arithmetic type.
template <typename Real>
struct AnelLevel {
  Real R, or1, or2, or4, beta, orho1, otemp1, visc, lam, LF, vhf, ohm;
};

// get_nl_anel at one grid point (magic_torch/get_nl_anel.py:63-136).
template <typename Real, bool MAG, bool CHEM>
__device__ __forceinline__ void anel_point(const Real* v, const AnelLevel<Real>& L, Real ost2,
                                           Real cosn, Real* o) {
  using F = AnelFields<MAG, CHEM>;
  const Real vr = v[0], vt = v[1], vp = v[2], dvrdr = v[3], dvtdr = v[4], dvpdr = v[5];
  const Real dvrdt = v[6], dvrdp = v[7], dvtdp = v[8], dvpdp = v[9], cvr = v[10], s = v[11];
  Real LFr = 0, LFt = 0, LFp = 0;
  Real br = 0, bt = 0, bp = 0, cbr = 0, cbt = 0, cbp = 0;
  if constexpr (MAG) {
    br = v[F::IB]; bt = v[F::IB + 1]; bp = v[F::IB + 2];
    cbr = v[F::IB + 3]; cbt = v[F::IB + 4]; cbp = v[F::IB + 5];
    LFr = L.LF * ost2 * (cbt * bp - cbp * bt);
    LFt = L.LF * L.or4 * (cbp * br - cbr * bp);
    LFp = L.LF * L.or4 * (cbr * bt - cbt * br);
  }
  o[0] = -L.or2 * L.orho1 * (vr * (dvrdr - (Real(2) * L.or1 + L.beta) * vr) +
                             ost2 * (vt * (dvrdt - L.R * vt) + vp * (dvrdp - L.R * vp))) + LFr;
  o[1] = L.or4 * L.orho1 * (-vr * (dvtdr - L.beta * vt) + vt * (cosn * vt + dvpdp + dvrdr) +
                            vp * (cosn * vp - dvtdp)) + LFt;
  o[2] = L.or4 * L.orho1 * (-vr * (dvpdr - L.beta * vp) - vt * (dvtdp + cvr) - vp * dvpdp) + LFp;
  o[3] = vr * s;
  o[4] = L.or2 * vt * s;
  o[5] = L.or2 * vp * s;
  if constexpr (MAG) {
    o[6] = L.orho1 * ost2 * (vt * bp - vp * bt);
    o[7] = L.orho1 * L.or4 * (vp * br - vr * bp);
    o[8] = L.orho1 * L.or4 * (vr * bt - vt * br);
  }
  if constexpr (CHEM) {
    const Real xi = v[12];
    o[F::IX] = vr * xi;
    o[F::IX + 1] = L.or2 * vt * xi;
    o[F::IX + 2] = L.or2 * vp * xi;
  }
  const Real prefac = L.vhf * L.or4 * L.orho1 * L.otemp1 * L.visc;
  const Real beta_r = L.beta * L.R;
  const Real e_rr = dvrdr - (Real(2) * L.or1 + L.beta) * vr;
  const Real e_tt = cosn * vt + dvpdp + dvrdr - L.or1 * vr;
  const Real e_pp = dvpdp + cosn * vt + L.or1 * vr;
  const Real e_tp = Real(2) * dvtdp + cvr - Real(2) * cosn * vp;
  const Real e_rt = L.R * dvtdr - (Real(2) + beta_r) * vt + L.or1 * dvrdt;
  const Real e_rp = L.R * dvpdr - (Real(2) + beta_r) * vp + L.or1 * dvrdp;
  const Real bv = L.beta * vr;
  Real heat = prefac * (Real(2) * e_rr * e_rr + Real(2) * e_tt * e_tt + Real(2) * e_pp * e_pp +
                        e_tp * e_tp + ost2 * (e_rt * e_rt + e_rp * e_rp) -
                        (Real(2) / Real(3)) * bv * bv);
  if constexpr (MAG)
    heat += L.ohm * L.lam * L.or2 * L.otemp1 * (L.or2 * cbr * cbr + ost2 * (cbt * cbt + cbp * cbp));
  o[F::NFO - 1] = heat;
}


}  // namespace mt
