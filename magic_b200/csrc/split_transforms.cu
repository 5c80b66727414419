// phi stage of the split-precision drop-in transforms (FP32).
//
// Rows are (column b, field f) pairs, row r = b * nf + f, matching the row
// order of the split Legendre kernels (row program q = 2 f + re/im of column
// b).  Synthesis: the Legendre GEMM leaves equatorially symmetric and
// antisymmetric Fourier rows (FP32); this kernel forms north = sym + asym or
// south = sym - asym, runs irfft(norm="forward") and writes the FP64 grid
// row.  Analysis: rfft(norm="forward") of the FP64 grid row in FP32, scaled
// by 1/N and by the row's quadrature weight (2 pi w, or 2 pi w / sin^2 for
// vector components), written as north/south Fourier rows for the analysis
// packing kernel.  One CTA = (theta row, up to kPhiRows rows); the FFT is the
// half-warp one (fft_hw.cuh) for n_phi = 256, 384, 512, 768 (Q > 0) and the
// block-wide mixed-radix one (fft.cuh) otherwise (Q = 0).
#include "fft.cuh"
#include "fft_hw.cuh"
#include "split_kernels.cuh"

namespace mt {

constexpr int kPhiRows = 14;
constexpr int kPhiThreads = kPhiRows * 16;

template <int Q>
struct PhiLayout {
  // shared-memory index of value i of a row and the row pitch
  __device__ static int idx(int i) {
    if constexpr (Q > 0) return hw_swz<Q>(i);
    else return pad16(i);
  }
  __host__ __device__ static int pitch(int H) { return Q > 0 ? H + 1 : padded_len(H); }
};

// shared memory (in complex floats) of one CTA
template <int Q>
static size_t phi_smem_cplx(int H) {
  if constexpr (Q > 0) return (size_t)kPhiRows * (H + 1) + 15 * Q + H;
  else return (size_t)(kPhiRows + kFftRowBatch) * padded_len(H) + H;
}

template <int Q>
__global__ void __launch_bounds__(kPhiThreads) k_split_to_grid(SplitPhiArgs a) {
  extern __shared__ __align__(16) float smemf[];
  cplx<float>* buf = reinterpret_cast<cplx<float>*>(smemf);
  const Tables& t = a.t;
  const int N = t.n_phi, H = N / 2, M = t.n_m, nt = t.n_theta;
  const int S = PhiLayout<Q>::pitch(H);
  const int row = blockIdx.x, j = row >> 1;
  const float hs = (row & 1) ? -1.f : 1.f;  // north = sym + asym, south = sym - asym
  const int r0 = blockIdx.y * kPhiRows, nrow = min(kPhiRows, a.nrows - r0);
  const int tid = threadIdx.x;
  cplx<float>* tw2 = buf + kPhiRows * S;  // half-warp FFT tables (Q > 0)
  cplx<float>* tw3 = tw2 + 3 * Q;
  cplx<float>* twN = tw3 + 12 * Q;
  cplx<float>* tws = buf + (kPhiRows + kFftRowBatch) * S;  // block FFT table (Q = 0)
  if constexpr (Q > 0) hw_twiddles_to_smem<Q>(tw2, tw3, twN, t.twiddle, tid, kPhiThreads);
  else fft_twiddles_to_smem(tws, H, t.twiddle, t.fft_radix, t.fft_nstages);
  // rows r0 .. r0 + nrow of wavenumber k are contiguous in the synthesis output
  const float* fs = a.Fs + (int64_t)j * a.fs_j + 2 * r0;
  const float rcp = 1.0f / (float)nrow;
  for (int e = tid; e < nrow * M; e += kPhiThreads) {
    const int k = fdiv(e, rcp), q = e - k * nrow;
    const float2 sy = __ldg(reinterpret_cast<const float2*>(fs + k * a.fs_m) + q);
    const float2 as = __ldg(reinterpret_cast<const float2*>(fs + k * a.fs_m + a.fs_c) + q);
    buf[q * S + PhiLayout<Q>::idx(k)] = {sy.x + hs * as.x, sy.y + hs * as.y};
  }
  for (int e = tid; e < nrow * (H - M); e += kPhiThreads) {
    const int q = e / (H - M), k = M + e % (H - M);
    buf[q * S + PhiLayout<Q>::idx(k)] = {0.f, 0.f};
  }
  __syncthreads();
  if constexpr (Q > 0) {
    const int hw = tid >> 4, lane = tid & 15;
    if (hw < nrow) hw_row_fft<Q, true, true>(buf + hw * S, lane, 0xFFFFu << (16 * (hw & 1)), tw2,
                                              tw3, twN);
  } else {
    // half spectrum -> Z in place (fft.cuh, c2r_pre), then the block FFT
    for (int e = tid; e < nrow * (H / 2 + 1); e += kPhiThreads) {
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
    fft_rows<true>(buf, buf + kPhiRows * S, nrow, H, S, t.fft_radix, t.fft_nstages, tws);
  }
  __syncthreads();
  // one warp per row: z[n] carries grid values 2n, 2n+1 (one 16-byte store)
  const int warp = tid >> 5, l32 = tid & 31;
  for (int q = warp; q < nrow; q += kPhiThreads / 32) {
    const int r = r0 + q, b = r / a.nf, f = r - b * a.nf;
    double2* dst = reinterpret_cast<double2*>(a.out[f] + ((int64_t)b * nt + row) * N);
    for (int n = l32; n < H; n += 32) {
      const cplx<float> z = buf[q * S + PhiLayout<Q>::idx(n)];
      dst[n] = make_double2((double)z.x, (double)z.y);
    }
  }
}

template <int Q>
__global__ void __launch_bounds__(kPhiThreads) k_split_to_fourier(SplitPhiArgs a) {
  extern __shared__ __align__(16) float smemf[];
  cplx<float>* buf = reinterpret_cast<cplx<float>*>(smemf);
  const Tables& t = a.t;
  const int N = t.n_phi, H = N / 2, M = t.n_m, nt = t.n_theta;
  const int S = PhiLayout<Q>::pitch(H);
  const int row = blockIdx.x, j = row >> 1;
  const int r0 = blockIdx.y * kPhiRows, nrow = min(kPhiRows, a.nrows - r0);
  const int tid = threadIdx.x;
  cplx<float>* tw2 = buf + kPhiRows * S;
  cplx<float>* tw3 = tw2 + 3 * Q;
  cplx<float>* twN = tw3 + 12 * Q;
  cplx<float>* tws = buf + (kPhiRows + kFftRowBatch) * S;
  if constexpr (Q > 0) hw_twiddles_to_smem<Q>(tw2, tw3, twN, t.twiddle, tid, kPhiThreads);
  else fft_twiddles_to_smem(tws, H, t.twiddle, t.fft_radix, t.fft_nstages);
  const int warp = tid >> 5, l32 = tid & 31;
  for (int q = warp; q < nrow; q += kPhiThreads / 32) {
    const int r = r0 + q, b = r / a.nf, f = r - b * a.nf;
    const double2* src = reinterpret_cast<const double2*>(a.in[f] + ((int64_t)b * nt + row) * N);
    for (int n = l32; n < H; n += 32) {
      const double2 v = __ldg(src + n);
      buf[q * S + PhiLayout<Q>::idx(n)] = {(float)v.x, (float)v.y};
    }
  }
  __syncthreads();
  if constexpr (Q > 0) {
    const int hw = tid >> 4, lane = tid & 15;
    if (hw < nrow) hw_row_fft<Q, false, false>(buf + hw * S, lane, 0xFFFFu << (16 * (hw & 1)),
                                                tw2, tw3, twN);
  } else {
    fft_rows<false>(buf, buf + kPhiRows * S, nrow, H, S, t.fft_radix, t.fft_nstages, tws);
  }
  __syncthreads();
  const float ws = (float)(t.wq[row] / N), wv = (float)(t.wq_v[row] / N);
  float* G = a.G + (int64_t)(row & 1) * a.g_h + (int64_t)j * a.g_j;
  const float rcp = 1.0f / (float)nrow;
  for (int e = tid; e < M * nrow; e += kPhiThreads) {
    const int k = fdiv(e, rcp), q = e - k * nrow;
    const int r = r0 + q, b = r / a.nf, f = r - b * a.nf;
    const cplx<float>* z = buf + q * S;
    cplx<float> X;
    if constexpr (Q > 0)
      X = r2c_post_w(z[PhiLayout<Q>::idx(k)], z[PhiLayout<Q>::idx((H - k) % H)], twN[k]);
    else
      X = r2c_post(z[pad16(k)], z[pad16((H - k) % H)], k, t.twiddle);
    const float w = (a.vector_mask >> f) & 1 ? wv : ws;
    reinterpret_cast<float2*>(G + k * a.g_m + (int64_t)b * a.g_level)[f] =
        make_float2(w * X.x, w * X.y);
  }
}

template <int Q>
static int launch_phi(bool to_grid, const SplitPhiArgs& a, cudaStream_t st) {
  const size_t sm = phi_smem_cplx<Q>(a.t.n_phi / 2) * sizeof(cplx<float>);
  const dim3 grid(a.t.n_theta, (a.nrows + kPhiRows - 1) / kPhiRows);
  if (to_grid) {
    MT_CHECK_CUDA(cudaFuncSetAttribute(k_split_to_grid<Q>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_split_to_grid<Q><<<grid, kPhiThreads, sm, st>>>(a);
  } else {
    MT_CHECK_CUDA(cudaFuncSetAttribute(k_split_to_fourier<Q>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_split_to_fourier<Q><<<grid, kPhiThreads, sm, st>>>(a);
  }
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

int launch_split_phi(bool to_grid, const SplitPhiArgs& a, cudaStream_t st) {
  switch (a.t.n_phi) {
    case 256: return launch_phi<8>(to_grid, a, st);
    case 384: return launch_phi<12>(to_grid, a, st);
    case 512: return launch_phi<16>(to_grid, a, st);
    case 768: return launch_phi<24>(to_grid, a, st);
    default: return launch_phi<0>(to_grid, a, st);
  }
}

}  // namespace mt
