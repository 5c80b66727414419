// phi stage of the drop-in transforms: Fourier rows <-> grid rows.
//
// Every grid row is one real field: synthesis is irfft(norm="forward")
// (unnormalised, Im of mode 0 ignored), analysis rfft(norm="forward"), both
// through a half-length complex FFT (fft.cuh).  Analysis outputs are scaled
// by 1/N and by the row's quadrature weight (2 pi w, or 2 pi w/sin^2 for
// vector components), so the Legendre analysis needs only P and dP.
#include "fft.cuh"
#include "fourier.cuh"

namespace mt {

constexpr int kColsPerCta = 8;  // real columns (grid rows) per CTA
constexpr int kFftThreads = 256;

// Expand the half spectra staged at row[0..M) (zero above) into Z (in place).
template <typename R>
__device__ __forceinline__ void c2r_prepare(cplx<R>* row, int H, const double2* __restrict__ tw,
                                            int tid, int nthr) {
  for (int k = tid; k <= H / 2; k += nthr) {
    int kc = H - k;
    cplx<R> Xk = row[pad16(k)];
    if (k == 0) {
      Xk.y = 0;  // irfft ignores Im X[0]; X[H] is zero (2 (n_m - 1) < N)
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

__global__ void __launch_bounds__(kFftThreads) k_fourier_to_grid(ToGridArgs a) {
  extern __shared__ double smem[];
  cplx<double>* buf = reinterpret_cast<cplx<double>*>(smem);
  const Tables& t = a.t;
  const int N = t.n_phi, H = N / 2, M = t.n_m, nt = t.n_theta;
  const int stride = padded_len(H);
  const int row = blockIdx.y;
  const int col0 = blockIdx.x * kColsPerCta;
  const int ncol = min(kColsPerCta, a.ncols - col0);
  cplx<double>* tws = buf + (kColsPerCta + kFftRowBatch) * stride;
  fft_twiddles_to_smem(tws, H, t.twiddle, t.fft_radix, t.fft_nstages);
  for (int i = threadIdx.x; i < ncol * stride; i += blockDim.x) buf[i] = {0.0, 0.0};
  __syncthreads();
  const double2* Fr = a.F + (int64_t)row * a.f_row + col0;
  const float rcp = 1.0f / (float)ncol;
  for (int e = threadIdx.x; e < M * ncol; e += blockDim.x) {
    int k = fdiv(e, rcp), q = e - k * ncol;
    cp_async16(&buf[q * stride + pad16(k)], &Fr[k * a.f_m + q]);
  }
  cp_async_wait_all();
  __syncthreads();
  for (int q = threadIdx.x / 64; q < ncol; q += kFftThreads / 64)
    c2r_prepare(buf + q * stride, H, t.twiddle, threadIdx.x % 64, 64);
  __syncthreads();
  fft_rows<true>(buf, buf + kColsPerCta * stride, ncol, H, stride, t.fft_radix, t.fft_nstages, tws);
  const float rcpN = 1.0f / (float)N;
  for (int e = threadIdx.x; e < ncol * N; e += blockDim.x) {
    int q = fdiv(e, rcpN), n = e - q * N;
    cplx<double> z = buf[q * stride + pad16(n >> 1)];
    int c = col0 + q;
    int f = c / a.B, b = c % a.B;
    a.out[f][((int64_t)b * nt + row) * N + n] = (n & 1) ? z.y : z.x;
  }
}

__global__ void __launch_bounds__(kFftThreads) k_grid_to_fourier(ToFourierArgs a) {
  extern __shared__ double smem[];
  cplx<double>* buf = reinterpret_cast<cplx<double>*>(smem);
  const Tables& t = a.t;
  const int N = t.n_phi, H = N / 2, M = t.n_m, nt = t.n_theta;
  const int stride = padded_len(H);
  const int row = blockIdx.y;
  const int col0 = blockIdx.x * kColsPerCta;
  const int ncol = min(kColsPerCta, a.ncols - col0);
  cplx<double>* tws = buf + (kColsPerCta + kFftRowBatch) * stride;
  fft_twiddles_to_smem(tws, H, t.twiddle, t.fft_radix, t.fft_nstages);
  const float rcpH = 1.0f / (float)H;
  for (int e = threadIdx.x; e < ncol * H; e += blockDim.x) {
    int q = fdiv(e, rcpH), h = e - q * H;
    int c = col0 + q;
    const double* src = a.in[c / a.B] + ((int64_t)(c % a.B) * nt + row) * N;
    double2 v = *reinterpret_cast<const double2*>(src + 2 * h);
    buf[q * stride + pad16(h)] = {v.x, v.y};
  }
  __syncthreads();
  fft_rows<false>(buf, buf + kColsPerCta * stride, ncol, H, stride, t.fft_radix, t.fft_nstages, tws);
  const double w = (a.vector ? t.wq_v[row] : t.wq[row]) / N;
  double2* Fr = a.F + (int64_t)row * a.f_row + col0;
  const float rcpc = 1.0f / (float)ncol;
  for (int e = threadIdx.x; e < M * ncol; e += blockDim.x) {
    int k = fdiv(e, rcpc), q = e - k * ncol;
    const cplx<double>* z = buf + q * stride;
    cplx<double> X = r2c_post(z[pad16(k)], z[pad16((H - k) % H)], k, t.twiddle);
    Fr[k * a.f_m + q] = make_double2(w * X.x, w * X.y);
  }
}

static size_t fft_smem(const Tables& t) {
  return ((size_t)(kColsPerCta + kFftRowBatch) * padded_len(t.n_phi / 2) + t.n_phi / 2) *
         sizeof(double2);
}

int launch_fourier_to_grid(const ToGridArgs& a, cudaStream_t st) {
  size_t sm = fft_smem(a.t);
  MT_CHECK_CUDA(cudaFuncSetAttribute(k_fourier_to_grid, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sm));
  dim3 grid((a.ncols + kColsPerCta - 1) / kColsPerCta, a.t.n_theta);
  k_fourier_to_grid<<<grid, kFftThreads, sm, st>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

int launch_grid_to_fourier(const ToFourierArgs& a, cudaStream_t st) {
  size_t sm = fft_smem(a.t);
  MT_CHECK_CUDA(cudaFuncSetAttribute(k_grid_to_fourier, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sm));
  dim3 grid((a.ncols + kColsPerCta - 1) / kColsPerCta, a.t.n_theta);
  k_grid_to_fourier<<<grid, kFftThreads, sm, st>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

// Largest n_phi the fused stage's shared memory holds: 14 field rows plus a
// 7-row scratch of H = n_phi/2 padded complex FP64 values and the H-point
// twiddle table within 227 KB.
int fft_max_nphi() { return 1168; }

}  // namespace mt
