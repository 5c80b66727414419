// Grid-space nonlinear terms.
//
// * k_nl_bouss: the fused phi stage of the Boussinesq radial loop.  One CTA
//   per (interleaved theta row, radial level): the 14 Fourier rows written by
//   the Legendre synthesis are expanded and inverse-FFT'd in shared memory
//   (two real fields per complex FFT), the get_nl products
//   (magic_torch/get_nl.py:57-87) and the Courant maxima
//   (magic_torch/courant.py:25-77) are formed point by point, and the 12
//   products are forward-FFT'd and truncated to n_m modes for the Legendre
//   analysis.  Grids never reach HBM.
// * k_get_nl / k_get_nl_anel / k_courant_grid: the same formulas on grids
//   held in HBM, for the drop-in get_nl / get_nl_anel / courant_check.
#include <algorithm>

#include "fft.cuh"
#include "fft_w64.cuh"
#include "fourier.cuh"
#include "nl_point.cuh"
#include "split_kernels.cuh"

namespace mt {

// ------------------------------------------------------------ point formulas

struct BoussIn {
  double vr, vt, vp, cvr, cvt, cvp, s, br, bt, bp, cbr, cbt, cbp, xi;
};
struct BoussOut {
  double o[12];  // Advr Advt Advp VSr VSt VSp VxBr VxBt VxBp VXir VXit VXip
};

// magic_torch/get_nl.py:57-85
__device__ __forceinline__ void bouss_point(const BoussIn& f, double or2, double or4, double ost2,
                                            double LFfac, bool mag, BoussOut& r) {
  double LFr = 0.0, LFt = 0.0, LFp = 0.0;
  if (mag) {
    LFr = LFfac * ost2 * (f.cbt * f.bp - f.cbp * f.bt);
    LFt = LFfac * or4 * (f.cbp * f.br - f.cbr * f.bp);
    LFp = LFfac * or4 * (f.cbr * f.bt - f.cbt * f.br);
  }
  r.o[0] = -ost2 * (f.cvt * f.vp - f.cvp * f.vt) + LFr;
  r.o[1] = -or4 * (f.cvp * f.vr - f.cvr * f.vp) + LFt;
  r.o[2] = -or4 * (f.cvr * f.vt - f.cvt * f.vr) + LFp;
  r.o[3] = f.vr * f.s;
  r.o[4] = or2 * f.vt * f.s;
  r.o[5] = or2 * f.vp * f.s;
  r.o[6] = ost2 * (f.vt * f.bp - f.vp * f.bt);
  r.o[7] = or4 * (f.vp * f.br - f.vr * f.bp);
  r.o[8] = or4 * (f.vr * f.bt - f.vt * f.br);
  r.o[9] = f.vr * f.xi;
  r.o[10] = or2 * f.vt * f.xi;
  r.o[11] = or2 * f.vp * f.xi;
}

// magic_torch/courant.py:25-77; mode 0 non-magnetic, 1 damped, 2 undamped.
__device__ __forceinline__ void courant_point(int mode, double vr, double vt, double vp, double br,
                                              double bt, double bp, double or2, double or4,
                                              double orho1, double orho2, double ost2,
                                              double LFfac, double cf2, double af2, double valri2,
                                              double valhi2, double& vr2, double& vh2) {
  double vflr2 = orho2 * vr * vr;
  double vflh2 = (vt * vt + vp * vp) * ost2 * orho2;
  if (mode == 0) {
    vr2 = cf2 * or4 * vflr2;
    vh2 = cf2 * or2 * vflh2;
    return;
  }
  double valr = br * br * LFfac * orho1;
  double valh2 = (bt * bt + bp * bp) * LFfac * ost2 * orho1;
  double valr2 = valr, valh2m = valh2;
  if (mode == 1) {
    valr2 = valr * valr / (valr + valri2);
    valh2m = valh2 * valh2 / (valh2 + valhi2);
  }
  vr2 = or4 * (cf2 * vflr2 + af2 * valr2);
  vh2 = or2 * (cf2 * vflh2 + af2 * valh2m);
}

__device__ __forceinline__ double block_max(double v, double* red) {
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
  return v;  // valid in thread 0
}

// Block-wide maxima of two values at once (one pass through `red`, >= 2 x 16
// doubles); the results are valid in thread 0.
__device__ __forceinline__ void block_max2(double& a, double& b, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a = fmax(a, __shfl_xor_sync(0xffffffffu, a, o));
    b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
  }
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
    red[w] = a;
    red[16 + w] = b;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    a = threadIdx.x < nw ? red[threadIdx.x] : 0.0;
    b = threadIdx.x < nw ? red[16 + threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a = fmax(a, __shfl_xor_sync(0xffffffffu, a, o));
      b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
    }
  }
}

__device__ __forceinline__ void atomic_max_pos(unsigned long long* a, double v) {
  v = v + 0.0;  // -0 -> +0: bit patterns of non-negative doubles order like integers
  atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

// ------------------------------------------------------- fused Boussinesq

template <bool MAG, bool CHEM>
struct BoussFields {
  static constexpr int NFI = (MAG ? 6 : 0) + 7 + (CHEM ? 1 : 0);
  static constexpr int NFO = 6 + (MAG ? 3 : 0) + (CHEM ? 3 : 0);
  static constexpr int NB = NFI > NFO ? NFI : NFO;  // rows of the shared buffer
  static constexpr int IV = MAG ? 6 : 0;            // row of vr
};

constexpr int kNlThreads = 512;

template <typename R>
__device__ __forceinline__ void c2r_prepare_nl(cplx<R>* row, int H, const double2* __restrict__ tw,
                                               int tid, int nthr) {
  for (int k = tid; k <= H / 2; k += nthr) {
    int kc = H - k;
    cplx<R> Xk = row[pad16(k)];
    if (k == 0) {
      Xk.y = 0;
      row[pad16(0)] = c2r_pre(Xk, cplx<R>{0, 0}, 0, tw);
    } else {
      cplx<R> Xc = row[pad16(kc)];
      cplx<R> Zk = c2r_pre(Xk, Xc, k, tw);
      cplx<R> Zc = c2r_pre(Xc, Xk, kc, tw);
      row[pad16(k)] = Zk;
      if (kc != k) row[pad16(kc)] = Zc;
    }
  }
}

template <bool MAG, bool CHEM, bool SPLIT_IO>
__global__ void __launch_bounds__(kNlThreads) k_nl_bouss(NlBoussArgs a) {
  using BF = BoussFields<MAG, CHEM>;
  constexpr int NFI = BF::NFI, NFO = BF::NFO;
  extern __shared__ double smem[];
  __shared__ double red[32];
  cplx<double>* buf = reinterpret_cast<cplx<double>*>(smem);
  const Tables& t = a.t;
  const int N = t.n_phi, H = N / 2, M = t.n_m;
  const int stride = padded_len(H);
  const int row = blockIdx.x, r = blockIdx.y;
  cplx<double>* tws = buf + (BF::NB + kFftRowBatch) * stride;
  fft_twiddles_to_smem(tws, H, t.twiddle, t.fft_radix, t.fft_nstages);
  for (int i = threadIdx.x; i < NFI * stride; i += blockDim.x) buf[i] = {0.0, 0.0};
  __syncthreads();
  // half spectra of the NFI fields (one real field per buffer row)
  if constexpr (SPLIT_IO) {
    // the synthesis wrote this hemisphere's row: [m][north|south][theta pair][row]
    const double* frow = a.Fs + (int64_t)(row & 1) * a.fs_c + (int64_t)(row >> 1) * a.fs_j +
                         (int64_t)r * 2 * NFI;
    for (int e = threadIdx.x; e < M * NFI; e += blockDim.x) {
      int k = e / NFI, f = e - k * NFI;
      const double2 x = __ldg(reinterpret_cast<const double2*>(frow + k * a.fs_m) + f);
      buf[f * stride + pad16(k)] = {x.x, x.y};
    }
  } else {
    const double2* Fr = a.F + (int64_t)row * a.f_row + (int64_t)r * NFI;
    for (int e = threadIdx.x; e < M * NFI; e += blockDim.x) {
      int k = e / NFI, f = e - k * NFI;
      cp_async16(&buf[f * stride + pad16(k)], &Fr[k * a.f_m + f]);
    }
    cp_async_wait_all();
  }
  __syncthreads();
  for (int f = threadIdx.x / 32; f < NFI; f += kNlThreads / 32)
    c2r_prepare_nl(buf + f * stride, H, t.twiddle, threadIdx.x % 32, 32);
  __syncthreads();
  fft_rows<true>(buf, buf + BF::NB * stride, NFI, H, stride, t.fft_radix, t.fft_nstages, tws);

  const double or2 = a.or2[r], or4 = a.or4[r], ost2 = t.ost2[row];
  const double orho1 = a.orho1[r], orho2 = a.orho2[r];
  const double valri2 = a.valfac / a.delxr2[r], valhi2 = a.valfac / a.delxh2[r];
  const double LF = a.LFfac_r ? a.LFfac_r[r] : a.LFfac;
  double mr = 0.0, mh = 0.0;
  for (int i = threadIdx.x; i < H; i += blockDim.x) {
    cplx<double> zin[NFI];
#pragma unroll
    for (int f = 0; f < NFI; ++f) zin[f] = buf[f * stride + pad16(i)];
    double out[2][NFO];
#pragma unroll
    for (int h = 0; h < 2; ++h) {  // grid points 2i and 2i+1
      auto v = [&](int f) { return h ? zin[f].y : zin[f].x; };
      BoussIn fi;
      constexpr int iv = BF::IV;
      if constexpr (MAG) {
        fi.br = v(0); fi.bt = v(1); fi.bp = v(2); fi.cbr = v(3); fi.cbt = v(4); fi.cbp = v(5);
      } else {
        fi.br = fi.bt = fi.bp = fi.cbr = fi.cbt = fi.cbp = 0.0;
      }
      fi.vr = v(iv); fi.vt = v(iv + 1); fi.vp = v(iv + 2);
      fi.cvr = v(iv + 3); fi.cvt = v(iv + 4); fi.cvp = v(iv + 5);
      fi.s = v(iv + 6);
      fi.xi = 0.0;
      if constexpr (CHEM) fi.xi = v(iv + 7);
      double vr2, vh2;
      courant_point(a.cour_mode, fi.vr, fi.vt, fi.vp, fi.br, fi.bt, fi.bp, or2, or4, orho1, orho2,
                    ost2, LF, a.cf2, a.af2, valri2, valhi2, vr2, vh2);
      mr = fmax(mr, vr2);
      mh = fmax(mh, vh2);
      BoussOut o;
      bouss_point(fi, or2, or4, ost2, LF, MAG, o);
#pragma unroll
      for (int q = 0; q < 6; ++q) out[h][q] = o.o[q];
      if constexpr (MAG) { out[h][6] = o.o[6]; out[h][7] = o.o[7]; out[h][8] = o.o[8]; }
      if constexpr (CHEM) {
        constexpr int c = MAG ? 9 : 6;
        out[h][c] = o.o[9]; out[h][c + 1] = o.o[10]; out[h][c + 2] = o.o[11];
      }
    }
    // complex element i (points 2i, 2i+1) belongs to this thread alone
#pragma unroll
    for (int q = 0; q < NFO; ++q) buf[q * stride + pad16(i)] = {out[0][q], out[1][q]};
  }
  double vmr = block_max(mr, red);
  if (threadIdx.x == 0) atomic_max_pos(&a.vr2max[r], vmr);
  double vmh = block_max(mh, red);
  if (threadIdx.x == 0) atomic_max_pos(&a.vh2max[r], vmh);
  if (r == 0 || r == a.n_r - 1) return;  // boundary levels: Courant only
  __syncthreads();
  fft_rows<false>(buf, buf + BF::NB * stride, NFO, H, stride, t.fft_radix, t.fft_nstages, tws);
  const double ws = t.wq[row] / N, wv = t.wq_v[row] / N;
  double2* Gr = SPLIT_IO
                    ? reinterpret_cast<double2*>(a.Gs + (int64_t)(row & 1) * a.g_h +
                                                 (int64_t)(row >> 1) * a.g_j +
                                                 (int64_t)(r - 1) * a.g_level)
                    : a.G + (int64_t)row * a.g_row + (int64_t)(r - 1) * NFO;
  const int64_t gm = SPLIT_IO ? a.g_m2 / 2 : a.g_m;  // double2 stride between orders
  for (int e = threadIdx.x; e < M * NFO; e += blockDim.x) {
    int k = e / NFO, o = e - k * NFO;
    const cplx<double>* z = buf + o * stride;
    cplx<double> X = r2c_post(z[pad16(k)], z[pad16((H - k) % H)], k, t.twiddle);
    // radial components (Advr, VSr, VxBr, VXir) are scalar analyses
    bool radial = (o == 0 || o == 3 || (MAG && o == 6) || (CHEM && o == (MAG ? 9 : 6)));
    double w = radial ? ws : wv;
    Gr[k * gm + o] = make_double2(w * X.x, w * X.y);
  }
}

// The same stage for n_phi = 64 Q (Q in 4, 8, 12, 16) with warp FFTs
// (fft_w64.cuh): every field row is transformed by one warp, so between the
// block-wide phases (load, inverse FFTs, products, forward FFTs, store) rows
// proceed independently, and two CTAs of 8 warps (128 registers a thread)
// share an SM.  The load phase applies the real-row pre-processing: the
// thread of wavenumber pair (k, H - k) reads both coefficients and writes
// Z[k] and Z[H - k], so the inverse transforms read their rows once.
constexpr int kNlW64Threads = 256;

template <bool MAG, bool CHEM, bool SPLIT_IO, int Q>
__global__ void __launch_bounds__(kNlW64Threads, 2) k_nl_bouss_w64(NlBoussArgs a) {
  using BF = BoussFields<MAG, CHEM>;
  constexpr int NFI = BF::NFI, NFO = BF::NFO, H = 32 * Q, S = w64_row_stride<Q>();
  constexpr int NW = kNlW64Threads / 32;
  extern __shared__ double smem[];
  __shared__ double red[32];
  cplx<double>* buf = reinterpret_cast<cplx<double>*>(smem);  // NB rows, S apart
  cplx<double>* twsm = buf + BF::NB * S;                      // W64Tw<Q> tables
  const Tables& t = a.t;
  const int M = t.n_m;
  // levels run fastest through the grid: the CTAs resident at one time read
  // (and write) whole runs of levels of a few theta rows, contiguous in HBM
  const int row = blockIdx.y, r = blockIdx.x;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // twiddle tables: asynchronous copies, waited for before the first use
  const W64Tw<Q> tw = w64_twiddles<Q>(twsm, t.twiddle, tid, kNlW64Threads);
  const cplx<double>* twN = tw.twN;
  // coefficient X[k] of field f (k < M) of this Fourier row
  auto ldF = [&](int k, int f) -> double2 {
    if constexpr (SPLIT_IO) {
      // the synthesis wrote this hemisphere's row: [m][north|south][theta pair][row]
      const double* frow = a.Fs + (int64_t)(row & 1) * a.fs_c + (int64_t)(row >> 1) * a.fs_j +
                           (int64_t)r * 2 * NFI;
      return __ldg(reinterpret_cast<const double2*>(frow + (int64_t)k * a.fs_m) + f);
    } else {
      return __ldg(&a.F[(int64_t)row * a.f_row + (int64_t)r * NFI + (int64_t)k * a.f_m + f]);
    }
  };
  // pairs (k, H - k), k <= H / 2, of every input field: Z[k] = c2r_pre(X[k], X[H - k])
  // and Z[H - k] = c2r_pre(X[H - k], X[k]) with X[k] = 0 for k >= M (and X[H] = 0);
  // kLd pairs per thread are loaded before any is stored, so their HBM
  // latencies overlap (two rounds at n_phi = 768, the first also covering
  // the twiddle copies)
  constexpr int NP = H / 2 + 1, kLd = 6;
  for (int e0 = 0; e0 < NP * NFI; e0 += kLd * kNlW64Threads) {
    double2 xa[kLd], xb[kLd];
#pragma unroll
    for (int u = 0; u < kLd; ++u) {
      const int e = e0 + u * kNlW64Threads + tid, k = e / NFI, f = e - k * NFI;
      xa[u] = make_double2(0.0, 0.0);
      xb[u] = make_double2(0.0, 0.0);
      if (e < NP * NFI) {
        if (k < M) xa[u] = ldF(k, f);
        if (k > 0 && H - k < M) xb[u] = ldF(H - k, f);
      }
    }
    if (e0 == 0) {  // (uniform) the tables are complete once every thread's copies are
      cp_async_wait_all();
      __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < kLd; ++u) {
      const int e = e0 + u * kNlW64Threads + tid, k = e / NFI, f = e - k * NFI;
      if (e < NP * NFI) {
        cplx<double>* rowf = buf + f * S;
        const cplx<double> w = twN[k];
        const cplx<double> Xk = {xa[u].x, k ? xa[u].y : 0.0}, Xc = {xb[u].x, xb[u].y};
        rowf[w64_pos<Q>(k)] = c2r_pre_d(Xk, Xc, w);
        if (k > 0 && k < H / 2)  // exp(-2 pi i (H - k) / (2 H)) = -conj(w)
          rowf[w64_pos<Q>(H - k)] = c2r_pre_d(Xc, Xk, cplx<double>{-w.x, w.y});
      }
    }
  }
  __syncthreads();
  for (int f = warp; f < NFI; f += NW) w64_row_fft<Q, true>(buf + f * S, lane, tw);
  __syncthreads();

  const double or2 = a.or2[r], or4 = a.or4[r], ost2 = t.ost2[row];
  const double orho1 = a.orho1[r], orho2 = a.orho2[r];
  const double valri2 = a.valfac / a.delxr2[r], valhi2 = a.valfac / a.delxh2[r];
  const double LF = a.LFfac_r ? a.LFfac_r[r] : a.LFfac;
  double mr = 0.0, mh = 0.0;
  // grid points p = tid + T u, u < kPts (three at n_phi = 768): point p is
  // component p & 1 of complex element p >> 1, so every thread has the same
  // number of points; a point's outputs overwrite its own inputs.  All the
  // thread's inputs are loaded before any point is formed (so their latencies
  // overlap and the points' arithmetic can interleave).
  constexpr int NPT = 2 * H, kPts = (NPT + kNlW64Threads - 1) / kNlW64Threads;
  const double* bd = reinterpret_cast<const double*>(buf);
  double* bw = reinterpret_cast<double*>(buf);
  double in[kPts][NFI];
  int sp[kPts];
#pragma unroll
  for (int u = 0; u < kPts; ++u) {
    const int p = tid + u * kNlW64Threads;
    sp[u] = 2 * w64_pos<Q>((p < NPT ? p : 0) >> 1) + (p & 1);  // double index in a row
#pragma unroll
    for (int f = 0; f < NFI; ++f) in[u][f] = p < NPT ? bd[f * 2 * S + sp[u]] : 0.0;
  }
#pragma unroll
  for (int u = 0; u < kPts; ++u) {
    if (tid + u * kNlW64Threads >= NPT) break;
    auto v = [&](int f) { return in[u][f]; };
    BoussIn fi;
    constexpr int iv = BF::IV;
    if constexpr (MAG) {
      fi.br = v(0); fi.bt = v(1); fi.bp = v(2); fi.cbr = v(3); fi.cbt = v(4); fi.cbp = v(5);
    } else {
      fi.br = fi.bt = fi.bp = fi.cbr = fi.cbt = fi.cbp = 0.0;
    }
    fi.vr = v(iv); fi.vt = v(iv + 1); fi.vp = v(iv + 2);
    fi.cvr = v(iv + 3); fi.cvt = v(iv + 4); fi.cvp = v(iv + 5);
    fi.s = v(iv + 6);
    fi.xi = 0.0;
    if constexpr (CHEM) fi.xi = v(iv + 7);
    double vr2, vh2;
    courant_point(a.cour_mode, fi.vr, fi.vt, fi.vp, fi.br, fi.bt, fi.bp, or2, or4, orho1, orho2,
                  ost2, LF, a.cf2, a.af2, valri2, valhi2, vr2, vh2);
    mr = fmax(mr, vr2);
    mh = fmax(mh, vh2);
    BoussOut o;
    bouss_point(fi, or2, or4, ost2, LF, MAG, o);
    double out[NFO];
#pragma unroll
    for (int q = 0; q < 6; ++q) out[q] = o.o[q];
    if constexpr (MAG) { out[6] = o.o[6]; out[7] = o.o[7]; out[8] = o.o[8]; }
    if constexpr (CHEM) {
      constexpr int c = MAG ? 9 : 6;
      out[c] = o.o[9]; out[c + 1] = o.o[10]; out[c + 2] = o.o[11];
    }
#pragma unroll
    for (int q = 0; q < NFO; ++q) bw[q * 2 * S + sp[u]] = out[q];
  }
  block_max2(mr, mh, red);
  if (tid == 0) {
    atomic_max_pos(&a.vr2max[r], mr);
    atomic_max_pos(&a.vh2max[r], mh);
  }
  if (r == 0 || r == a.n_r - 1) return;  // boundary levels: Courant only
  __syncthreads();
  for (int f = warp; f < NFO; f += NW) w64_row_fft<Q, false>(buf + f * S, lane, tw);
  __syncthreads();
  const double ws = t.wq[row] / (2 * H), wv = t.wq_v[row] / (2 * H);
  double2* Gr = SPLIT_IO
                    ? reinterpret_cast<double2*>(a.Gs + (int64_t)(row & 1) * a.g_h +
                                                 (int64_t)(row >> 1) * a.g_j +
                                                 (int64_t)(r - 1) * a.g_level)
                    : a.G + (int64_t)row * a.g_row + (int64_t)(r - 1) * NFO;
  const int64_t gm = SPLIT_IO ? a.g_m2 / 2 : a.g_m;  // double2 stride between orders
  // kSt outputs per thread: their shared-memory reads are issued together
  constexpr int kSt = 4;
  for (int e0 = tid; e0 < M * NFO; e0 += kSt * kNlW64Threads) {
    cplx<double> zk[kSt], zc[kSt], wn[kSt];
#pragma unroll
    for (int u = 0; u < kSt; ++u) {
      const int e = e0 + u * kNlW64Threads, k = e / NFO, o = e - k * NFO;
      if (e < M * NFO) {
        const cplx<double>* z = buf + o * S;
        zk[u] = z[w64_pos<Q>(k)];
        zc[u] = z[w64_pos<Q>((H - k) % H)];
        wn[u] = twN[k];
      }
    }
#pragma unroll
    for (int u = 0; u < kSt; ++u) {
      const int e = e0 + u * kNlW64Threads, k = e / NFO, o = e - k * NFO;
      if (e < M * NFO) {
        const cplx<double> X = r2c_post_d(zk[u], zc[u], wn[u]);
        const bool radial =
            (o == 0 || o == 3 || (MAG && o == 6) || (CHEM && o == (MAG ? 9 : 6)));
        const double w = radial ? ws : wv;
        Gr[k * gm + o] = make_double2(w * X.x, w * X.y);
      }
    }
  }
}

template <bool MAG, bool CHEM, bool SPLIT_IO, int Q>
static int launch_nl_bouss_w64(const NlBoussArgs& a, cudaStream_t st) {
  using BF = BoussFields<MAG, CHEM>;
  constexpr int H = 32 * Q;
  const size_t sm = ((size_t)BF::NB * w64_row_stride<Q>() + W64Tw<Q>::kEntries) * sizeof(double2);
  auto kern = k_nl_bouss_w64<MAG, CHEM, SPLIT_IO, Q>;
  MT_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  MT_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     cudaSharedmemCarveoutMaxShared));
  dim3 grid(a.n_r, a.t.n_theta);
  kern<<<grid, kNlW64Threads, sm, st>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

template <bool MAG, bool CHEM, bool SPLIT_IO>
static int launch_nl_bouss_t(const NlBoussArgs& a, cudaStream_t st) {
  switch (a.t.n_phi) {
    case 256: return launch_nl_bouss_w64<MAG, CHEM, SPLIT_IO, 4>(a, st);
    case 512: return launch_nl_bouss_w64<MAG, CHEM, SPLIT_IO, 8>(a, st);
    case 768: return launch_nl_bouss_w64<MAG, CHEM, SPLIT_IO, 12>(a, st);
    case 1024: return launch_nl_bouss_w64<MAG, CHEM, SPLIT_IO, 16>(a, st);
    default: break;
  }
  using BF = BoussFields<MAG, CHEM>;
  size_t sm = ((size_t)(BF::NB + kFftRowBatch) * padded_len(a.t.n_phi / 2) + a.t.n_phi / 2) *
              sizeof(double2);
  auto kern = k_nl_bouss<MAG, CHEM, SPLIT_IO>;
  MT_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  dim3 grid(a.t.n_theta, a.n_r);
  kern<<<grid, kNlThreads, sm, st>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

template <bool SPLIT_IO>
static int launch_nl_bouss_io(bool mag, bool chem, const NlBoussArgs& a, cudaStream_t st) {
  if (mag)
    return chem ? launch_nl_bouss_t<true, true, SPLIT_IO>(a, st)
                : launch_nl_bouss_t<true, false, SPLIT_IO>(a, st);
  return chem ? launch_nl_bouss_t<false, true, SPLIT_IO>(a, st)
              : launch_nl_bouss_t<false, false, SPLIT_IO>(a, st);
}

// ------------------------------------------------------- fused anelastic (FP64)

// In-place mixed-radix FFT stages of the FP64 anelastic phi stage.  Stage
// (radix R, span Ns) has the butterflies (row, blk, j), j < Ns, over the
// elements blk R Ns + j + q Ns, q < R, of a row (row stride S; element i at
// slot anel_slot(i, sw)).  Decimation in frequency (DIF): DFT over q, then
// element q times w^(q j), w = exp(-2 pi i / (R Ns)) (conjugate for INV);
// decimation in time (DIT): the twiddle first, then the DFT.  DIF stages from
// the largest span down take a row in natural order to its transform in
// mixed-radix digit-reversed order; DIT stages from span 1 up are the
// transpose of that chain, so they take digit-reversed input to a
// natural-order transform.  The synthesis runs DIF (inverse), the analysis DIT
// (forward): the grid points in between are permuted along phi, which the
// point products and Courant maxima do not see.  A thread takes one butterfly
// position in the rows of a row group, so that its R - 1 twiddles (read from
// the plan's table tw[n] = exp(-2 pi i n / (2 H)) through L1) serve several
// rows.

// Slot of element i in a row: the low three bits XORed with the next three
// (sw = 7 when H is a multiple of 8, else 0), so that the stride-8 accesses of
// a span-1 radix-8 stage fall on distinct bank quads while aligned runs of
// eight stay conflict-free.
__device__ __forceinline__ int anel_slot(int i, int sw) { return i ^ ((i >> 3) & sw); }

template <int R, bool INV, bool DIF>
__device__ __forceinline__ void fft_stage_ip(cplx<double>* buf, int nrows, int H, int S, int sw,
                                             int Ns, const double2* __restrict__ tw) {
  const int nbr = H / R, step = 2 * H / (R * Ns);
  const int G = max(1, min(nrows, (int)blockDim.x / nbr));  // row groups
  const float rcp_nbr = 1.0f / (float)nbr, rcp_ns = 1.0f / (float)Ns;
  for (int it = threadIdx.x; it < nbr * G; it += blockDim.x) {
    const int g = fdiv(it, rcp_nbr), i = it - g * nbr;
    const int blk = fdiv(i, rcp_ns), j = i - blk * Ns;
    const int base = blk * R * Ns + j;
    cplx<double> w[R];
    if (j > 0) {
#pragma unroll
      for (int q = 1; q < R; ++q) {
        const double2 t = __ldg(&tw[q * j * step]);
        w[q] = {t.x, INV ? -t.y : t.y};
      }
    }
    for (int row = g; row < nrows; row += G) {
      cplx<double>* x = buf + row * S;
      cplx<double> v[R];
#pragma unroll
      for (int q = 0; q < R; ++q) v[q] = x[anel_slot(base + q * Ns, sw)];
      if (!DIF && j > 0) {
#pragma unroll
        for (int q = 1; q < R; ++q) v[q] = cmul(v[q], w[q]);
      }
      dft_small<R, INV>(v);
      if (DIF && j > 0) {
#pragma unroll
        for (int q = 1; q < R; ++q) v[q] = cmul(v[q], w[q]);
      }
#pragma unroll
      for (int q = 0; q < R; ++q) x[anel_slot(base + q * Ns, sw)] = v[q];
    }
  }
  __syncthreads();
}

// All stages of the rows: DIF (INV, synthesis) or DIT (forward, analysis) with
// the plan's radices rad[0..nst) (span of stage s = rad[0] ... rad[s - 1]).
template <bool INV>
__device__ __forceinline__ void fft_rows_ip(cplx<double>* buf, int nrows, int H, int S, int sw,
                                            const int* rad, int nst,
                                            const double2* __restrict__ tw) {
  constexpr bool DIF = INV;
  int Ns = DIF ? H : 1;
  for (int u = 0; u < nst; ++u) {
    const int s = DIF ? nst - 1 - u : u;
    const int r = rad[s];
    if (DIF) Ns /= r;
    switch (r) {
      case 8: fft_stage_ip<8, INV, DIF>(buf, nrows, H, S, sw, Ns, tw); break;
      case 4: fft_stage_ip<4, INV, DIF>(buf, nrows, H, S, sw, Ns, tw); break;
      case 3: fft_stage_ip<3, INV, DIF>(buf, nrows, H, S, sw, Ns, tw); break;
      case 2: fft_stage_ip<2, INV, DIF>(buf, nrows, H, S, sw, Ns, tw); break;
      default: fft_stage_ip<5, INV, DIF>(buf, nrows, H, S, sw, Ns, tw); break;
    }
    if (!DIF) Ns *= r;
  }
}

// The phi stage of the digit-split anelastic radial loop.  One CTA (256
// threads) per (theta row, level): the synthesis wrote this hemisphere's
// Fourier rows of the grid fields in FP64 (NlAnelArgs::Fs64; field order of
// nl_point.cuh), the kernel inverse-transforms them in place (fft_rows_ip),
// evaluates get_nl_anel (magic_torch/get_nl_anel.py:63-136, viscous and Ohmic
// heating included) and the Courant maxima (magic_torch/courant.py:25-77) at
// every grid point in FP64, and forward-transforms the 10-13 products into the
// weighted rows the analysis reads (NlAnelArgs::G64).  Shared memory holds
// only the rows (max(nfi, nfo) x (H + 1) complex values; the odd row stride
// puts consecutive rows on different banks), so that two CTAs share an SM
// without magnetic field at n_phi = 1152.  Velocity, its derivatives and cvr
// are zero on the two boundary levels (radial_loop_anel synthesises them on
// the bulk levels only, magic_torch/step_time.py:1233-1316); the
// phi-derivative fields get their 1/sin^2(theta) factor here
// (torpol_to_dphspat, magic_torch/sht.py:725-743).
constexpr int kNlAnelThreads = 256;

template <bool MAG, bool CHEM>
__global__ void __launch_bounds__(kNlAnelThreads, 2) k_nl_anel_f64(NlAnelArgs a) {
  using F = AnelFields<MAG, CHEM>;
  constexpr int NFI = F::NFI, NFO = F::NFO, T = kNlAnelThreads;
  extern __shared__ double smem[];
  __shared__ double red[32];
  cplx<double>* buf = reinterpret_cast<cplx<double>*>(smem);
  const Tables& t = a.t;
  const int N = t.n_phi, H = N / 2, M = t.n_m, S = H + 1;
  const int row = blockIdx.x, r = blockIdx.y, tid = threadIdx.x;
  const int sw = (H & 7) ? 0 : 7;
  auto at = [&](int f, int i) -> cplx<double>& { return buf[f * S + anel_slot(i, sw)]; };
  const double* frow = a.Fs64 + (int64_t)(row & 1) * a.fs_c + (int64_t)(row >> 1) * a.fs_j +
                       (int64_t)r * 2 * NFI;
  // asynchronous 16-byte copies of the M wavenumbers (every thread keeps its
  // copies in flight), zeros above
  for (int e = tid; e < H * NFI; e += T) {
    const int k = e / NFI, f = e - k * NFI;
    if (k < M) cp_async16(&at(f, k), reinterpret_cast<const double2*>(frow + k * a.fs_m) + f);
    else at(f, k) = {0.0, 0.0};
  }
  cp_async_wait_all();
  __syncthreads();
  // real-row synthesis: Z[k], Z[H - k] from X[k], X[H - k] (c2r_pre)
  for (int e = tid; e < NFI * (H / 2 + 1); e += T) {
    const int f = e / (H / 2 + 1), k = e - f * (H / 2 + 1);
    const int kc = H - k;
    cplx<double> Xk = at(f, k);
    if (k == 0) {
      Xk.y = 0.0;
      at(f, 0) = c2r_pre(Xk, cplx<double>{0.0, 0.0}, 0, t.twiddle);
    } else {
      const cplx<double> Xc = at(f, kc);
      const cplx<double> Zk = c2r_pre(Xk, Xc, k, t.twiddle);
      const cplx<double> Zc = c2r_pre(Xc, Xk, kc, t.twiddle);
      at(f, k) = Zk;
      if (kc != k) at(f, kc) = Zc;
    }
  }
  __syncthreads();
  fft_rows_ip<true>(buf, NFI, H, S, sw, t.fft_radix, t.fft_nstages, t.twiddle);

  const bool bnd = r == 0 || r == a.n_r - 1;
  AnelLevel<double> L;
  L.R = a.r[r];
  L.or1 = a.or1[r];
  L.or2 = a.or2[r];
  L.or4 = a.or4[r];
  L.beta = a.beta[r];
  L.orho1 = a.orho1[r];
  L.otemp1 = a.otemp1[r];
  L.visc = a.visc[r];
  L.lam = a.lambda_[r];
  L.LF = a.LFfac;
  L.vhf = a.ViscHeatFac;
  L.ohm = a.OhmLossFac;
  const double ost2 = t.ost2[row], cosn = t.cosn[row], orho2 = a.orho2[r];
  const double valri2 = a.valfac / a.delxr2[r], valhi2 = a.valfac / a.delxh2[r];
  double mr = 0.0, mh = 0.0;
  for (int i = tid; i < H; i += T) {
    const int si = anel_slot(i, sw);
    cplx<double> zin[NFI];
#pragma unroll
    for (int f = 0; f < NFI; ++f) zin[f] = buf[f * S + si];
#pragma unroll
    for (int h = 0; h < 2; ++h) {  // the two real grid points of complex element i
      double v[NFI];
#pragma unroll
      for (int f = 0; f < NFI; ++f) v[f] = h ? zin[f].y : zin[f].x;
      if (bnd) {
#pragma unroll
        for (int f = 0; f <= 10; ++f) v[f] = 0.0;  // velocity, derivatives, cvr
      }
      v[8] *= ost2;  // dvtdp, dvpdp: torpol_to_dphspat's 1/sin^2
      v[9] *= ost2;
      double vr2, vh2;
      if constexpr (MAG)
        courant_point(a.cour_mode, v[0], v[1], v[2], v[F::IB], v[F::IB + 1], v[F::IB + 2], L.or2,
                      L.or4, L.orho1, orho2, ost2, L.LF, a.cf2, a.af2, valri2, valhi2, vr2, vh2);
      else
        courant_point(0, v[0], v[1], v[2], 0.0, 0.0, 0.0, L.or2, L.or4, L.orho1, orho2, ost2, L.LF,
                      a.cf2, a.af2, valri2, valhi2, vr2, vh2);
      mr = fmax(mr, vr2);
      mh = fmax(mh, vh2);
      if (!bnd) {
        double o[NFO];
        anel_point<double, MAG, CHEM>(v, L, ost2, cosn, o);
        // complex element i belongs to this thread alone
#pragma unroll
        for (int q = 0; q < NFO; ++q) {
          if (h) buf[q * S + si].y = o[q];
          else buf[q * S + si].x = o[q];
        }
      }
    }
  }
  const double vmr = block_max(mr, red);
  if (tid == 0) atomic_max_pos(&a.vr2max[r], vmr);
  const double vmh = block_max(mh, red);
  if (tid == 0) atomic_max_pos(&a.vh2max[r], vmh);
  if (bnd) return;  // boundary levels: Courant only
  __syncthreads();
  fft_rows_ip<false>(buf, NFO, H, S, sw, t.fft_radix, t.fft_nstages, t.twiddle);
  const double ws = t.wq[row] / N, wv = t.wq_v[row] / N;
  double* Gr = a.G64 + (int64_t)(row & 1) * a.g_h + (int64_t)(row >> 1) * a.g_j +
               (int64_t)(r - 1) * a.g_level;
  for (int e = tid; e < M * NFO; e += T) {
    const int k = e / NFO, o = e - k * NFO;
    const cplx<double> X = r2c_post(at(o, k), at(o, (H - k) % H), k, t.twiddle);
    const double w = F::radial(o) ? ws : wv;
    reinterpret_cast<double2*>(Gr + k * a.g_m)[o] = make_double2(w * X.x, w * X.y);
  }
}

size_t nl_anel_f64_smem(int n_phi, bool mag, bool chem) {
  const int nfi = 12 + (chem ? 1 : 0) + (mag ? 6 : 0), nfo = 7 + (mag ? 3 : 0) + (chem ? 3 : 0);
  const int NB = std::max(nfi, nfo);
  const size_t sm = (size_t)NB * (n_phi / 2 + 1) * sizeof(double2);
  return sm <= 227 * 1024 - 32 * sizeof(double) ? sm : 0;
}

template <bool MAG, bool CHEM>
static int launch_nl_anel_f64_t(const NlAnelArgs& a, cudaStream_t st) {
  const size_t sm = nl_anel_f64_smem(a.t.n_phi, MAG, CHEM);
  MT_REQUIRE(sm > 0, MT_ERR_UNSUPPORTED, "n_phi too large for the FP64 anelastic phi stage");
  auto kern = k_nl_anel_f64<MAG, CHEM>;
  MT_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  MT_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     cudaSharedmemCarveoutMaxShared));
  dim3 grid(a.t.n_theta, a.n_r);
  kern<<<grid, kNlAnelThreads, sm, st>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

int launch_nl_anel_f64(bool mag, bool chem, const NlAnelArgs& a, cudaStream_t st) {
  if (mag)
    return chem ? launch_nl_anel_f64_t<true, true>(a, st)
                : launch_nl_anel_f64_t<true, false>(a, st);
  return chem ? launch_nl_anel_f64_t<false, true>(a, st)
              : launch_nl_anel_f64_t<false, false>(a, st);
}

int launch_nl_bouss(bool mag, bool chem, const NlBoussArgs& a, cudaStream_t st) {
  return a.split_io ? launch_nl_bouss_io<true>(mag, chem, a, st)
                    : launch_nl_bouss_io<false>(mag, chem, a, st);
}

__global__ void k_courant_finish(int n_r, const unsigned long long* vr2, const unsigned long long* vh2,
                                 const double* delxr2, const double* delxh2, double* dtr,
                                 double* dth) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_r) return;
  double a = __longlong_as_double((long long)vr2[r]);
  double b = __longlong_as_double((long long)vh2[r]);
  dtr[r] = a > 0.0 ? sqrt(delxr2[r] / a) : 1e10;  // magic_torch/courant.py:122-125
  dth[r] = b > 0.0 ? sqrt(delxh2[r] / b) : 1e10;
}

int launch_courant_finish(int n_r, const unsigned long long* vr2, const unsigned long long* vh2,
                          const double* delxr2, const double* delxh2, double* dtr, double* dth,
                          cudaStream_t st) {
  k_courant_finish<<<(n_r + 127) / 128, 128, 0, st>>>(n_r, vr2, vh2, delxr2, delxh2, dtr, dth);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

// ---------------------------------------------------- grid-space drop-ins


__global__ void k_get_nl(GridNlArgs a) {
  int64_t total = (int64_t)a.n_r * a.nt * a.np;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    int r = (int)(i / ((int64_t)a.nt * a.np));
    int th = (int)((i / a.np) % a.nt);
    BoussIn f;
    f.vr = a.in[0][i]; f.vt = a.in[1][i]; f.vp = a.in[2][i];
    f.cvr = a.in[3][i]; f.cvt = a.in[4][i]; f.cvp = a.in[5][i];
    f.s = a.in[6][i];
    f.br = a.in[7][i]; f.bt = a.in[8][i]; f.bp = a.in[9][i];
    f.cbr = a.in[10][i]; f.cbt = a.in[11][i]; f.cbp = a.in[12][i];
    f.xi = a.in[13][i];
    BoussOut o;
    bouss_point(f, a.or2[r], a.or4[r], a.ost2[th], a.LFfac, true, o);
#pragma unroll
    for (int q = 0; q < 12; ++q) a.out[q][i] = o.o[q];
  }
}

// magic_torch/get_nl_anel.py:63-134
__global__ void k_get_nl_anel(GridNlArgs a) {
  int64_t total = (int64_t)a.n_r * a.nt * a.np;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    int r = (int)(i / ((int64_t)a.nt * a.np));
    int th = (int)((i / a.np) % a.nt);
    const double vr = a.in[0][i], vt = a.in[1][i], vp = a.in[2][i];
    const double dvrdr = a.in[3][i], dvtdr = a.in[4][i], dvpdr = a.in[5][i];
    const double dvrdt = a.in[6][i], dvrdp = a.in[7][i], dvtdp = a.in[8][i], dvpdp = a.in[9][i];
    const double cvr = a.in[10][i], s = a.in[11][i], xi = a.in[12][i];
    const double br = a.in[13][i], bt = a.in[14][i], bp = a.in[15][i];
    const double cbr = a.in[16][i], cbt = a.in[17][i], cbp = a.in[18][i];
    const double R = a.r[r], or1 = a.or1[r], or2 = a.or2[r], or4 = a.or4[r];
    const double beta = a.beta[r], orho1 = a.orho1[r], otemp1 = a.otemp1[r];
    const double visc = a.visc[r], lam = a.lambda_[r];
    const double ost2 = a.ost2[th], cosn = a.cosn[th], LF = a.LFfac;
    double LFr = LF * ost2 * (cbt * bp - cbp * bt);
    double LFt = LF * or4 * (cbp * br - cbr * bp);
    double LFp = LF * or4 * (cbr * bt - cbt * br);
    double Advr = -or2 * orho1 * (vr * (dvrdr - (2.0 * or1 + beta) * vr) +
                                  ost2 * (vt * (dvrdt - R * vt) + vp * (dvrdp - R * vp)));
    double Advt = or4 * orho1 * (-vr * (dvtdr - beta * vt) + vt * (cosn * vt + dvpdp + dvrdr) +
                                 vp * (cosn * vp - dvtdp));
    double Advp = or4 * orho1 * (-vr * (dvpdr - beta * vp) - vt * (dvtdp + cvr) - vp * dvpdp);
    a.out[0][i] = Advr + LFr;
    a.out[1][i] = Advt + LFt;
    a.out[2][i] = Advp + LFp;
    a.out[3][i] = vr * s;
    a.out[4][i] = or2 * vt * s;
    a.out[5][i] = or2 * vp * s;
    a.out[6][i] = orho1 * ost2 * (vt * bp - vp * bt);
    a.out[7][i] = orho1 * or4 * (vp * br - vr * bp);
    a.out[8][i] = orho1 * or4 * (vr * bt - vt * br);
    a.out[9][i] = vr * xi;
    a.out[10][i] = or2 * vt * xi;
    a.out[11][i] = or2 * vp * xi;
    double prefac = a.ViscHeatFac * or4 * orho1 * otemp1 * visc;
    double beta_r = beta * R;
    double e_rr = dvrdr - (2.0 * or1 + beta) * vr;
    double e_tt = cosn * vt + dvpdp + dvrdr - or1 * vr;
    double e_pp = dvpdp + cosn * vt + or1 * vr;
    double e_tp = 2.0 * dvtdp + cvr - 2.0 * cosn * vp;
    double e_rt = R * dvtdr - (2.0 + beta_r) * vt + or1 * dvrdt;
    double e_rp = R * dvpdr - (2.0 + beta_r) * vp + or1 * dvrdp;
    double bv = beta * vr;
    double heat = prefac * (2.0 * e_rr * e_rr + 2.0 * e_tt * e_tt + 2.0 * e_pp * e_pp +
                            e_tp * e_tp + ost2 * (e_rt * e_rt + e_rp * e_rp) -
                            2.0 * (1.0 / 3.0) * bv * bv);
    if (a.l_mag && a.OhmLossFac != 0.0)
      heat += a.OhmLossFac * lam * or2 * otemp1 * (or2 * cbr * cbr + ost2 * (cbt * cbt + cbp * cbp));
    a.out[12][i] = heat;
  }
}

int launch_get_nl_grid(bool anel, const GridNlArgs& a, cudaStream_t st) {
  int64_t total = (int64_t)a.n_r * a.nt * a.np;
  int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
  if (blocks < 1) blocks = 1;
  if (anel) k_get_nl_anel<<<blocks, 256, 0, st>>>(a);
  else k_get_nl<<<blocks, 256, 0, st>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}


// one CTA per (level, slab of theta rows)
__global__ void k_courant_grid(CourantGridArgs a) {
  __shared__ double red[32];
  const int r = blockIdx.y;
  const int64_t per = (int64_t)a.nt * a.np;
  const int64_t base = (int64_t)r * per;
  const double valri2 = a.valfac / a.delxr2[r], valhi2 = a.valfac / a.delxh2[r];
  double mr = 0.0, mh = 0.0;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < per;
       j += (int64_t)gridDim.x * blockDim.x) {
    int th = (int)(j / a.np);
    int64_t i = base + j;
    double br = 0.0, bt = 0.0, bp = 0.0;
    if (a.mode != 0) { br = a.br[i]; bt = a.bt[i]; bp = a.bp[i]; }
    double vr2, vh2;
    courant_point(a.mode, a.vr[i], a.vt[i], a.vp[i], br, bt, bp, a.or2[r], a.or4[r], a.orho1[r],
                  a.orho2[r], a.ost2[th], a.LFfac, a.cf2, a.af2, valri2, valhi2, vr2, vh2);
    mr = fmax(mr, vr2);
    mh = fmax(mh, vh2);
  }
  double v = block_max(mr, red);
  if (threadIdx.x == 0) atomic_max_pos(&a.vr2max[r], v);
  v = block_max(mh, red);
  if (threadIdx.x == 0) atomic_max_pos(&a.vh2max[r], v);
}

int launch_courant_grid(const CourantGridArgs& a, cudaStream_t st) {
  int64_t per = (int64_t)a.nt * a.np;
  int bx = (int)std::min<int64_t>((per + 255) / 256, 32);
  dim3 grid(bx, a.n_r);
  k_courant_grid<<<grid, 256, 0, st>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

}  // namespace mt
