// Fused phi stage of the split-precision Boussinesq radial loop (FP32).
//
// Same structure as k_nl_bouss (one CTA per (theta row, level): per-field
// half-length FFTs in shared memory, get_nl products and Courant maxima at
// every grid point, forward FFTs truncated to n_m modes), with FP32 data:
// the synthesis delivers equatorially symmetric/antisymmetric parts
// (north = sym + asym, south = sym - asym) and the analysis folds north and
// south itself, so this kernel reads and writes plain north/south rows.
#include <algorithm>

#include "fft.cuh"
#include "fft_hw.cuh"
#include "fourier.cuh"
#include "nl_point.cuh"
#include "split_kernels.cuh"

namespace mt {

struct BoussInF {
  float vr, vt, vp, cvr, cvt, cvp, s, br, bt, bp, cbr, cbt, cbp, xi;
};

// magic_torch/get_nl.py:57-85 in FP32
__device__ __forceinline__ void bouss_point_f(const BoussInF& f, float or2, float or4, float ost2,
                                              float LF, bool mag, float (&o)[12]) {
  float LFr = 0.f, LFt = 0.f, LFp = 0.f;
  if (mag) {
    LFr = LF * ost2 * (f.cbt * f.bp - f.cbp * f.bt);
    LFt = LF * or4 * (f.cbp * f.br - f.cbr * f.bp);
    LFp = LF * or4 * (f.cbr * f.bt - f.cbt * f.br);
  }
  o[0] = -ost2 * (f.cvt * f.vp - f.cvp * f.vt) + LFr;
  o[1] = -or4 * (f.cvp * f.vr - f.cvr * f.vp) + LFt;
  o[2] = -or4 * (f.cvr * f.vt - f.cvt * f.vr) + LFp;
  o[3] = f.vr * f.s;
  o[4] = or2 * f.vt * f.s;
  o[5] = or2 * f.vp * f.s;
  o[6] = ost2 * (f.vt * f.bp - f.vp * f.bt);
  o[7] = or4 * (f.vp * f.br - f.vr * f.bp);
  o[8] = or4 * (f.vr * f.bt - f.vt * f.br);
  o[9] = f.vr * f.xi;
  o[10] = or2 * f.vt * f.xi;
  o[11] = or2 * f.vp * f.xi;
}

// magic_torch/courant.py:25-77 (FP32 grid values, FP64 maxima)
__device__ __forceinline__ void courant_point_f(int mode, float vr, float vt, float vp, float br,
                                                float bt, float bp, double or2, double or4,
                                                double orho1, double orho2, double ost2,
                                                double LFfac, double cf2, double af2,
                                                double valri2, double valhi2, double& vr2,
                                                double& vh2) {
  double vflr2 = orho2 * (double)vr * vr;
  double vflh2 = ((double)vt * vt + (double)vp * vp) * ost2 * orho2;
  if (mode == 0) {
    vr2 = cf2 * or4 * vflr2;
    vh2 = cf2 * or2 * vflh2;
    return;
  }
  double valr = (double)br * br * LFfac * orho1;
  double valh2 = ((double)bt * bt + (double)bp * bp) * LFfac * ost2 * orho1;
  double valr2 = valr, valh2m = valh2;
  if (mode == 1) {
    valr2 = valr * valr / (valr + valri2);
    valh2m = valh2 * valh2 / (valh2 + valhi2);
  }
  vr2 = or4 * (cf2 * vflr2 + af2 * valr2);
  vh2 = or2 * (cf2 * vflh2 + af2 * valh2m);
}

template <bool MAG, bool CHEM>
struct SplitFields {
  static constexpr int NFI = (MAG ? 6 : 0) + 7 + (CHEM ? 1 : 0);
  static constexpr int NFO = 6 + (MAG ? 3 : 0) + (CHEM ? 3 : 0);
  static constexpr int NB = NFI > NFO ? NFI : NFO;
  static constexpr int IV = MAG ? 6 : 0;
};

constexpr int kNlSplitThreads = 256;

template <bool MAG, bool CHEM>
__global__ void __launch_bounds__(kNlSplitThreads) k_nl_bouss_split(NlSplitArgs a) {
  using BF = SplitFields<MAG, CHEM>;
  constexpr int NFI = BF::NFI, NFO = BF::NFO;
  extern __shared__ __align__(16) float smemf[];
  __shared__ double red[32];
  cplx<float>* buf = reinterpret_cast<cplx<float>*>(smemf);
  const Tables& t = a.t;
  const int N = t.n_phi, H = N / 2, M = t.n_m;
  const int stride = padded_len(H);
  const int row = blockIdx.x, r = blockIdx.y;
  const int j = row >> 1;
  const float hs = (row & 1) ? -1.f : 1.f;  // north = sym + asym, south = sym - asym
  cplx<float>* tws = buf + (BF::NB + kFftRowBatch) * stride;
  fft_twiddles_to_smem(tws, H, t.twiddle, t.fft_radix, t.fft_nstages);
  for (int i = threadIdx.x; i < NFI * stride; i += blockDim.x) buf[i] = {0.f, 0.f};
  __syncthreads();
  const float* fsym = a.Fs + (int64_t)j * a.fs_j + (int64_t)r * 2 * NFI;
  for (int e = threadIdx.x; e < M * NFI; e += blockDim.x) {
    int k = e / NFI, f = e - k * NFI;
    const float2 sy = __ldg(reinterpret_cast<const float2*>(fsym + k * a.fs_m) + f);
    const float2 as = __ldg(reinterpret_cast<const float2*>(fsym + k * a.fs_m + a.fs_c) + f);
    buf[f * stride + pad16(k)] = {sy.x + hs * as.x, sy.y + hs * as.y};
  }
  __syncthreads();
  for (int f = threadIdx.x / 32; f < NFI; f += kNlSplitThreads / 32)
    for (int k = threadIdx.x % 32; k <= H / 2; k += 32) {
      cplx<float>* rw = buf + f * stride;
      int kc = H - k;
      cplx<float> Xk = rw[pad16(k)];
      if (k == 0) {
        Xk.y = 0.f;
        rw[pad16(0)] = c2r_pre(Xk, cplx<float>{0.f, 0.f}, 0, t.twiddle);
      } else {
        cplx<float> Xc = rw[pad16(kc)];
        cplx<float> Zk = c2r_pre(Xk, Xc, k, t.twiddle);
        cplx<float> Zc = c2r_pre(Xc, Xk, kc, t.twiddle);
        rw[pad16(k)] = Zk;
        if (kc != k) rw[pad16(kc)] = Zc;
      }
    }
  __syncthreads();
  fft_rows<true>(buf, buf + BF::NB * stride, NFI, H, stride, t.fft_radix, t.fft_nstages, tws);

  const float or2 = (float)a.or2[r], or4 = (float)a.or4[r], ost2 = (float)t.ost2[row];
  const double orho1 = a.orho1[r], orho2 = a.orho2[r];
  const double valri2 = a.valfac / a.delxr2[r], valhi2 = a.valfac / a.delxh2[r];
  const double LFd = a.LFfac_r ? a.LFfac_r[r] : a.LFfac;
  double mr = 0.0, mh = 0.0;
  for (int i = threadIdx.x; i < H; i += blockDim.x) {
    cplx<float> zin[NFI];
#pragma unroll
    for (int f = 0; f < NFI; ++f) zin[f] = buf[f * stride + pad16(i)];
    float out[2][NFO];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      auto v = [&](int f) { return h ? zin[f].y : zin[f].x; };
      BoussInF fi;
      constexpr int iv = BF::IV;
      if constexpr (MAG) {
        fi.br = v(0); fi.bt = v(1); fi.bp = v(2); fi.cbr = v(3); fi.cbt = v(4); fi.cbp = v(5);
      } else {
        fi.br = fi.bt = fi.bp = fi.cbr = fi.cbt = fi.cbp = 0.f;
      }
      fi.vr = v(iv); fi.vt = v(iv + 1); fi.vp = v(iv + 2);
      fi.cvr = v(iv + 3); fi.cvt = v(iv + 4); fi.cvp = v(iv + 5);
      fi.s = v(iv + 6);
      fi.xi = 0.f;
      if constexpr (CHEM) fi.xi = v(iv + 7);
      double vr2, vh2;
      courant_point_f(a.cour_mode, fi.vr, fi.vt, fi.vp, fi.br, fi.bt, fi.bp, a.or2[r], a.or4[r],
                      orho1, orho2, t.ost2[row], LFd, a.cf2, a.af2, valri2, valhi2, vr2, vh2);
      mr = fmax(mr, vr2);
      mh = fmax(mh, vh2);
      float o[12];
      bouss_point_f(fi, or2, or4, ost2, (float)LFd, MAG, o);
#pragma unroll
      for (int q = 0; q < 6; ++q) out[h][q] = o[q];
      if constexpr (MAG) { out[h][6] = o[6]; out[h][7] = o[7]; out[h][8] = o[8]; }
      if constexpr (CHEM) {
        constexpr int c = MAG ? 9 : 6;
        out[h][c] = o[9]; out[h][c + 1] = o[10]; out[h][c + 2] = o[11];
      }
    }
#pragma unroll
    for (int q = 0; q < NFO; ++q) buf[q * stride + pad16(i)] = {out[0][q], out[1][q]};
  }
  double vmr = block_max_d(mr, red);
  if (threadIdx.x == 0) atomicMax(&a.vr2max[r], (unsigned long long)__double_as_longlong(vmr + 0.0));
  double vmh = block_max_d(mh, red);
  if (threadIdx.x == 0) atomicMax(&a.vh2max[r], (unsigned long long)__double_as_longlong(vmh + 0.0));
  if (r == 0 || r == a.n_r - 1) return;
  __syncthreads();
  fft_rows<false>(buf, buf + BF::NB * stride, NFO, H, stride, t.fft_radix, t.fft_nstages, tws);
  const float ws = (float)(t.wq[row] / N), wv = (float)(t.wq_v[row] / N);
  float* Gr = a.G + (int64_t)(row & 1) * a.g_h + (int64_t)j * a.g_j + (int64_t)(r - 1) * a.g_level;
  for (int e = threadIdx.x; e < M * NFO; e += blockDim.x) {
    int k = e / NFO, o = e - k * NFO;
    const cplx<float>* z = buf + o * stride;
    cplx<float> X = r2c_post(z[pad16(k)], z[pad16((H - k) % H)], k, t.twiddle);
    bool radial = (o == 0 || o == 3 || (MAG && o == 6) || (CHEM && o == (MAG ? 9 : 6)));
    float w = radial ? ws : wv;
    reinterpret_cast<float2*>(Gr + k * a.g_m)[o] = make_float2(w * X.x, w * X.y);
  }
}

// The same stage for n_phi = 32 Q (Q in 8, 12, 16, 24): every field row is
// transformed by one half-warp (fft_hw.cuh), so between the block-wide
// phases (load, inverse FFTs, products, forward FFTs, store) the rows
// proceed independently.  Threads: one half-warp per row of the larger of the
// input and output field sets.
template <bool MAG, bool CHEM>
__host__ __device__ constexpr int hw_threads() {
  return 32 * ((SplitFields<MAG, CHEM>::NB + 1) / 2);
}

// 72 registers (a few bytes of spill at Q = 24) let four 224-thread CTAs share
// an SM; at 96 registers only three fit and the kernel ran 35% longer.
template <bool MAG, bool CHEM, int Q>
__global__ void __maxnreg__(72)
    k_nl_bouss_split_hw(NlSplitArgs a) {
  using BF = SplitFields<MAG, CHEM>;
  constexpr int NFI = BF::NFI, NFO = BF::NFO, H = 16 * Q, S = H + 1;
  constexpr int T = hw_threads<MAG, CHEM>();
  extern __shared__ __align__(16) float smemf[];
  __shared__ double red[32];
  cplx<float>* buf = reinterpret_cast<cplx<float>*>(smemf);  // NB rows, S apart
  cplx<float>* tw2 = buf + BF::NB * S;
  cplx<float>* tw3 = tw2 + 3 * Q;
  cplx<float>* twN = tw3 + 12 * Q;
  const Tables& t = a.t;
  const int M = t.n_m;
  const int row = blockIdx.x, r = blockIdx.y;
  const int j = row >> 1;
  const float hs = (row & 1) ? -1.f : 1.f;  // north = sym + asym, south = sym - asym
  const int tid = threadIdx.x, hw = tid >> 4, lane = tid & 15;
  const unsigned mask = 0xFFFFu << (16 * (hw & 1));
  hw_twiddles_to_smem<Q>(tw2, tw3, twN, t.twiddle, tid, T);
  // Fourier rows: element e = (k, f) of the NFI (sym, asym) pairs of
  // wavenumber k (consecutive threads read consecutive fields of one k);
  // wavenumbers k >= n_m are zero.
  const float* fsym = a.Fs + (int64_t)j * a.fs_j + (int64_t)r * 2 * NFI;
#pragma unroll 4
  for (int e = tid; e < NFI * M; e += T) {
    const int k = e / NFI, f = e - k * NFI;
    const float2 sy = __ldg(reinterpret_cast<const float2*>(fsym + k * a.fs_m) + f);
    const float2 as = __ldg(reinterpret_cast<const float2*>(fsym + k * a.fs_m + a.fs_c) + f);
    buf[f * S + hw_swz<Q>(k)] = {sy.x + hs * as.x, sy.y + hs * as.y};
  }
  for (int e = tid; e < NFI * (H - M); e += T) {
    const int k = M + e / NFI, f = e % NFI;
    buf[f * S + hw_swz<Q>(k)] = {0.f, 0.f};
  }
  __syncthreads();
  if (hw < NFI) hw_row_fft<Q, true, true>(buf + hw * S, lane, mask, tw2, tw3, twN);
  __syncthreads();

  const float or2 = (float)a.or2[r], or4 = (float)a.or4[r], ost2 = (float)t.ost2[row];
  const float orho1 = (float)a.orho1[r], orho2 = (float)a.orho2[r];
  const float valri2 = (float)(a.valfac / a.delxr2[r]), valhi2 = (float)(a.valfac / a.delxh2[r]);
  const float LF = (float)(a.LFfac_r ? a.LFfac_r[r] : a.LFfac), cf2 = (float)a.cf2,
              af2 = (float)a.af2;
  float mr = 0.f, mh = 0.f;
  for (int i = tid; i < H; i += T) {
    const int si = hw_swz<Q>(i);
    cplx<float> zin[NFI];
#pragma unroll
    for (int f = 0; f < NFI; ++f) zin[f] = buf[f * S + si];
    float out[2][NFO];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      auto v = [&](int f) { return h ? zin[f].y : zin[f].x; };
      BoussInF fi;
      constexpr int iv = BF::IV;
      if constexpr (MAG) {
        fi.br = v(0); fi.bt = v(1); fi.bp = v(2); fi.cbr = v(3); fi.cbt = v(4); fi.cbp = v(5);
      } else {
        fi.br = fi.bt = fi.bp = fi.cbr = fi.cbt = fi.cbp = 0.f;
      }
      fi.vr = v(iv); fi.vt = v(iv + 1); fi.vp = v(iv + 2);
      fi.cvr = v(iv + 3); fi.cvt = v(iv + 4); fi.cvp = v(iv + 5);
      fi.s = v(iv + 6);
      fi.xi = 0.f;
      if constexpr (CHEM) fi.xi = v(iv + 7);
      float vr2, vh2;
      courant_point_s(a.cour_mode, fi.vr, fi.vt, fi.vp, fi.br, fi.bt, fi.bp, or2, or4, orho1,
                      orho2, ost2, LF, cf2, af2, valri2, valhi2, vr2, vh2);
      mr = fmaxf(mr, vr2);
      mh = fmaxf(mh, vh2);
      float o[12];
      bouss_point_f(fi, or2, or4, ost2, LF, MAG, o);
#pragma unroll
      for (int q = 0; q < 6; ++q) out[h][q] = o[q];
      if constexpr (MAG) { out[h][6] = o[6]; out[h][7] = o[7]; out[h][8] = o[8]; }
      if constexpr (CHEM) {
        constexpr int c = MAG ? 9 : 6;
        out[h][c] = o[9]; out[h][c + 1] = o[10]; out[h][c + 2] = o[11];
      }
    }
#pragma unroll
    for (int q = 0; q < NFO; ++q) buf[q * S + si] = {out[0][q], out[1][q]};
  }
  double vmr = block_max_d((double)mr, red);
  if (tid == 0) atomicMax(&a.vr2max[r], (unsigned long long)__double_as_longlong(vmr + 0.0));
  double vmh = block_max_d((double)mh, red);
  if (tid == 0) atomicMax(&a.vh2max[r], (unsigned long long)__double_as_longlong(vmh + 0.0));
  if (r == 0 || r == a.n_r - 1) return;
  __syncthreads();
  if (hw < NFO) hw_row_fft<Q, false, false>(buf + hw * S, lane, mask, tw2, tw3, twN);
  __syncthreads();
  const float ws = (float)(t.wq[row] / (2 * H)), wv = (float)(t.wq_v[row] / (2 * H));
  float* Gr = a.G + (int64_t)(row & 1) * a.g_h + (int64_t)j * a.g_j + (int64_t)(r - 1) * a.g_level;
  for (int e = tid; e < M * NFO; e += T) {
    const int k = e / NFO, o = e - k * NFO;
    const cplx<float>* z = buf + o * S;
    const cplx<float> X = r2c_post_w(z[hw_swz<Q>(k)], z[hw_swz<Q>((H - k) % H)], twN[k]);
    const bool radial = (o == 0 || o == 3 || (MAG && o == 6) || (CHEM && o == (MAG ? 9 : 6)));
    const float w = radial ? ws : wv;
    reinterpret_cast<float2*>(Gr + k * a.g_m)[o] = make_float2(w * X.x, w * X.y);
  }
}

template <bool MAG, bool CHEM, int Q>
static int launch_hw(const NlSplitArgs& a, cudaStream_t st) {
  using BF = SplitFields<MAG, CHEM>;
  constexpr int H = 16 * Q;
  const size_t sm = ((size_t)BF::NB * (H + 1) + 15 * Q + H) * sizeof(cplx<float>);
  auto kern = k_nl_bouss_split_hw<MAG, CHEM, Q>;
  MT_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  MT_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     cudaSharedmemCarveoutMaxShared));
  dim3 grid(a.t.n_theta, a.n_r);
  kern<<<grid, hw_threads<MAG, CHEM>(), sm, st>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

template <bool MAG, bool CHEM>
static int launch_t(const NlSplitArgs& a, cudaStream_t st) {
  switch (a.t.n_phi) {
    case 256: return launch_hw<MAG, CHEM, 8>(a, st);
    case 384: return launch_hw<MAG, CHEM, 12>(a, st);
    case 512: return launch_hw<MAG, CHEM, 16>(a, st);
    case 768: return launch_hw<MAG, CHEM, 24>(a, st);
    default: break;
  }
  using BF = SplitFields<MAG, CHEM>;
  size_t sm = ((size_t)(BF::NB + kFftRowBatch) * padded_len(a.t.n_phi / 2) + a.t.n_phi / 2) *
              sizeof(cplx<float>);
  auto kern = k_nl_bouss_split<MAG, CHEM>;
  MT_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  dim3 grid(a.t.n_theta, a.n_r);
  kern<<<grid, kNlSplitThreads, sm, st>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

int launch_nl_bouss_split(bool mag, bool chem, const NlSplitArgs& a, cudaStream_t st) {
  if (mag) return chem ? launch_t<true, true>(a, st) : launch_t<true, false>(a, st);
  return chem ? launch_t<false, true>(a, st) : launch_t<false, false>(a, st);
}

}  // namespace mt
