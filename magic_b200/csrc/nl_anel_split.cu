// Fused phi stage of the split-precision anelastic radial loop (FP32).
//
// One CTA per (theta row, level), as k_nl_bouss_split_hw: the synthesis
// delivers equatorially symmetric/antisymmetric Fourier rows of the 18 (19
// with composition) grid fields, this kernel forms the hemisphere's rows,
// transforms them (half-warp FFT for n_phi = 256, 384, 512, 768, block FFT
// otherwise), evaluates get_nl_anel (magic_torch/get_nl_anel.py:41-136,
// viscous and Ohmic heating included) and the Courant maxima at every grid
// point, and writes the weighted Fourier rows of the 10-13 products for the
// analysis.  Velocity, its derivatives and cvr are zero on the two boundary
// levels (radial_loop_anel synthesises them on the bulk levels only); the
// phi-derivative fields get their 1/sin^2(theta) factor here
// (torpol_to_dphspat, magic_torch/sht.py:725-743).
//
// Grid fields (rows 2 f, 2 f + 1 of the synthesis): 0 vr, 1 vt, 2 vp,
// 3 dvrdr, 4 dvtdr, 5 dvpdr, 6 dvrdt, 7 dvrdp, 8 dvtdp, 9 dvpdp, 10 cvr,
// 11 s, [12 xi], then br bt bp cbr cbt cbp.  Products: 0 Advr, 1 Advt,
// 2 Advp, 3 VSr, 4 VSt, 5 VSp, [VxBr VxBt VxBp], [VXir VXit VXip], heat.
#include "fft.cuh"
#include "fft_hw.cuh"
#include "nl_point.cuh"
#include "split_kernels.cuh"

namespace mt {

template <bool MAG, bool CHEM, int Q>
__global__ void __launch_bounds__(Q > 0 ? AnelFields<MAG, CHEM>::THW : 256)
    k_nl_anel_split(NlAnelArgs a) {
  using F = AnelFields<MAG, CHEM>;
  constexpr int NFI = F::NFI, NFO = F::NFO, NB = F::NB;
  constexpr int T = Q > 0 ? F::THW : 256;
  extern __shared__ __align__(16) float smemf[];
  __shared__ double red[32];
  cplx<float>* buf = reinterpret_cast<cplx<float>*>(smemf);
  const Tables& t = a.t;
  const int N = t.n_phi, H = N / 2, M = t.n_m;
  const int S = Q > 0 ? H + 1 : padded_len(H);
  auto idx = [](int i) {
    if constexpr (Q > 0) return hw_swz<Q>(i);
    else return pad16(i);
  };
  const int row = blockIdx.x, r = blockIdx.y, j = row >> 1;
  const float hs = (row & 1) ? -1.f : 1.f;  // north = sym + asym, south = sym - asym
  const int tid = threadIdx.x;
  cplx<float>* tw2 = buf + NB * S;  // half-warp FFT tables (Q > 0)
  cplx<float>* tw3 = tw2 + 3 * Q;
  cplx<float>* twN = tw3 + 12 * Q;
  cplx<float>* tws = buf + (NB + kFftRowBatch) * S;  // block FFT table (Q = 0)
  if constexpr (Q > 0) hw_twiddles_to_smem<Q>(tw2, tw3, twN, t.twiddle, tid, T);
  else fft_twiddles_to_smem(tws, H, t.twiddle, t.fft_radix, t.fft_nstages);
  const float* fsym = a.Fs + (int64_t)j * a.fs_j + (int64_t)r * 2 * NFI;
#pragma unroll 4
  for (int e = tid; e < NFI * M; e += T) {
    const int k = e / NFI, f = e - k * NFI;
    const float2 sy = __ldg(reinterpret_cast<const float2*>(fsym + k * a.fs_m) + f);
    const float2 as = __ldg(reinterpret_cast<const float2*>(fsym + k * a.fs_m + a.fs_c) + f);
    buf[f * S + idx(k)] = {sy.x + hs * as.x, sy.y + hs * as.y};
  }
  for (int e = tid; e < NFI * (H - M); e += T) {
    const int k = M + e / NFI, f = e % NFI;
    buf[f * S + idx(k)] = {0.f, 0.f};
  }
  __syncthreads();
  if constexpr (Q > 0) {
    const int hw = tid >> 4, lane = tid & 15;
    if (hw < NFI)
      hw_row_fft<Q, true, true>(buf + hw * S, lane, 0xFFFFu << (16 * (hw & 1)), tw2, tw3, twN);
  } else {
    for (int e = tid; e < NFI * (H / 2 + 1); e += T) {
      const int q = e / (H / 2 + 1), k = e % (H / 2 + 1);
      cplx<float>* rw = buf + q * S;
      const int kc = H - k;
      cplx<float> Xk = rw[pad16(k)];
      if (k == 0) {
        Xk.y = 0.f;
        rw[pad16(0)] = c2r_pre(Xk, cplx<float>{0.f, 0.f}, 0, t.twiddle);
      } else {
        const cplx<float> Xc = rw[pad16(kc)];
        const cplx<float> Zk = c2r_pre(Xk, Xc, k, t.twiddle);
        const cplx<float> Zc = c2r_pre(Xc, Xk, kc, t.twiddle);
        rw[pad16(k)] = Zk;
        if (kc != k) rw[pad16(kc)] = Zc;
      }
    }
    __syncthreads();
    fft_rows<true>(buf, buf + NB * S, NFI, H, S, t.fft_radix, t.fft_nstages, tws);
  }
  __syncthreads();

  const bool bnd = r == 0 || r == a.n_r - 1;
  AnelLevel<float> L;
  L.R = (float)a.r[r];
  L.or1 = (float)a.or1[r];
  L.or2 = (float)a.or2[r];
  L.or4 = (float)a.or4[r];
  L.beta = (float)a.beta[r];
  L.orho1 = (float)a.orho1[r];
  L.otemp1 = (float)a.otemp1[r];
  L.visc = (float)a.visc[r];
  L.lam = (float)a.lambda_[r];
  L.LF = (float)a.LFfac;
  L.vhf = (float)a.ViscHeatFac;
  L.ohm = (float)a.OhmLossFac;
  const float ost2 = (float)t.ost2[row], cosn = (float)t.cosn[row];
  const float orho2 = (float)a.orho2[r];
  const float valri2 = (float)(a.valfac / a.delxr2[r]), valhi2 = (float)(a.valfac / a.delxh2[r]);
  const float cf2 = (float)a.cf2, af2 = (float)a.af2;
  float mr = 0.f, mh = 0.f;
  for (int i = tid; i < H; i += T) {
    const int si = idx(i);
    cplx<float> zin[NFI];
#pragma unroll
    for (int f = 0; f < NFI; ++f) zin[f] = buf[f * S + si];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float v[NFI];
#pragma unroll
      for (int f = 0; f < NFI; ++f) v[f] = h ? zin[f].y : zin[f].x;
      if (bnd) {
#pragma unroll
        for (int f = 0; f <= 10; ++f) v[f] = 0.f;  // velocity, derivatives, cvr
      }
      v[8] *= ost2;  // dvtdp, dvpdp: torpol_to_dphspat's 1/sin^2
      v[9] *= ost2;
      float vr2, vh2;
      if constexpr (MAG)
        courant_point_s(a.cour_mode, v[0], v[1], v[2], v[F::IB], v[F::IB + 1], v[F::IB + 2], L.or2,
                        L.or4, L.orho1, orho2, ost2, L.LF, cf2, af2, valri2, valhi2, vr2, vh2);
      else
        courant_point_s(0, v[0], v[1], v[2], 0.f, 0.f, 0.f, L.or2, L.or4, L.orho1, orho2, ost2,
                        L.LF, cf2, af2, valri2, valhi2, vr2, vh2);
      mr = fmaxf(mr, vr2);
      mh = fmaxf(mh, vh2);
      if (!bnd) {
        float o[NFO];
        anel_point<float, MAG, CHEM>(v, L, ost2, cosn, o);
#pragma unroll
        for (int q = 0; q < NFO; ++q) {
          if (h) buf[q * S + si].y = o[q];
          else buf[q * S + si].x = o[q];
        }
      }
    }
  }
  double vmr = block_max_d((double)mr, red);
  if (tid == 0) atomicMax(&a.vr2max[r], (unsigned long long)__double_as_longlong(vmr + 0.0));
  double vmh = block_max_d((double)mh, red);
  if (tid == 0) atomicMax(&a.vh2max[r], (unsigned long long)__double_as_longlong(vmh + 0.0));
  if (bnd) return;
  __syncthreads();
  if constexpr (Q > 0) {
    const int hw = tid >> 4, lane = tid & 15;
    if (hw < NFO)
      hw_row_fft<Q, false, false>(buf + hw * S, lane, 0xFFFFu << (16 * (hw & 1)), tw2, tw3, twN);
  } else {
    fft_rows<false>(buf, buf + NB * S, NFO, H, S, t.fft_radix, t.fft_nstages, tws);
  }
  __syncthreads();
  const float ws = (float)(t.wq[row] / N), wv = (float)(t.wq_v[row] / N);
  float* Gr = a.G + (int64_t)(row & 1) * a.g_h + (int64_t)j * a.g_j + (int64_t)(r - 1) * a.g_level;
  for (int e = tid; e < M * NFO; e += T) {
    const int k = e / NFO, o = e - k * NFO;
    const cplx<float>* z = buf + o * S;
    cplx<float> X;
    if constexpr (Q > 0) X = r2c_post_w(z[idx(k)], z[idx((H - k) % H)], twN[k]);
    else X = r2c_post(z[pad16(k)], z[pad16((H - k) % H)], k, t.twiddle);
    const float w = F::radial(o) ? ws : wv;
    reinterpret_cast<float2*>(Gr + k * a.g_m)[o] = make_float2(w * X.x, w * X.y);
  }
}

template <bool MAG, bool CHEM, int Q>
static int launch_anel(const NlAnelArgs& a, cudaStream_t st) {
  using F = AnelFields<MAG, CHEM>;
  const int H = a.t.n_phi / 2;
  size_t ncplx;
  if constexpr (Q > 0) ncplx = (size_t)F::NB * (H + 1) + 15 * Q + H;
  else ncplx = (size_t)(F::NB + kFftRowBatch) * padded_len(H) + H;
  const size_t sm = ncplx * sizeof(cplx<float>);
  MT_REQUIRE(sm <= 227 * 1024, MT_ERR_UNSUPPORTED, "n_phi too large for the anelastic phi stage");
  auto kern = k_nl_anel_split<MAG, CHEM, Q>;
  MT_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  MT_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     cudaSharedmemCarveoutMaxShared));
  dim3 grid(a.t.n_theta, a.n_r);
  kern<<<grid, Q > 0 ? F::THW : 256, sm, st>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

template <bool MAG, bool CHEM>
static int launch_anel_t(const NlAnelArgs& a, cudaStream_t st) {
  switch (a.t.n_phi) {
    case 256: return launch_anel<MAG, CHEM, 8>(a, st);
    case 384: return launch_anel<MAG, CHEM, 12>(a, st);
    case 512: return launch_anel<MAG, CHEM, 16>(a, st);
    case 768: return launch_anel<MAG, CHEM, 24>(a, st);
    default: return launch_anel<MAG, CHEM, 0>(a, st);
  }
}

int launch_nl_anel_split(bool mag, bool chem, const NlAnelArgs& a, cudaStream_t st) {
  if (mag) return chem ? launch_anel_t<true, true>(a, st) : launch_anel_t<true, false>(a, st);
  return chem ? launch_anel_t<false, true>(a, st) : launch_anel_t<false, false>(a, st);
}

}  // namespace mt
