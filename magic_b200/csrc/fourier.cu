// phi stage of the drop-in transforms: Fourier rows <-> grid rows.
//
// Two real rows a, b share one complex FFT of length n_phi (z = a + i b).
// Inverse (synthesis, irfft norm="forward"): the half spectra A, B (modes
// 0..n_m-1, zero above) are expanded to the full Hermitian spectrum of z,
//   Z[k] = A[k] + i B[k],  Z[N-k] = conj(A[k]) + i conj(B[k]),  k >= 1,
//   Z[0] = Re A[0] + i Re B[0]  (irfft ignores the imaginary part of mode 0),
// then a = Re ifft(Z), b = Im ifft(Z), unnormalised.
// Forward (analysis, rfft norm="forward"), for k < n_m:
//   A[k] = (Z[k] + conj Z[N-k]) / 2,  B[k] = (Z[k] - conj Z[N-k]) / (2i),
// scaled by 1/N and by the row's quadrature weight (2 pi w, or 2 pi w/sin^2
// for vector components), so the Legendre analysis needs only P and dP.
#include "fft.cuh"
#include "fourier.cuh"

namespace mt {

constexpr int kRowsPerCta = 4;  // complex rows = 8 real columns
constexpr int kFftThreads = 512;
constexpr int kFftCap = 10;  // complex values per thread and stage: 4 rows x 1280 / 512

__global__ void __launch_bounds__(kFftThreads) k_fourier_to_grid(ToGridArgs a) {
  extern __shared__ double smem[];
  cplx<double>* buf = reinterpret_cast<cplx<double>*>(smem);
  const Tables& t = a.t;
  const int N = t.n_phi, M = t.n_m, nt = t.n_theta;
  const int row = blockIdx.y;
  const int col0 = blockIdx.x * 2 * kRowsPerCta;
  for (int i = threadIdx.x; i < kRowsPerCta * N; i += blockDim.x) buf[i] = {0.0, 0.0};
  __syncthreads();
  const double2* Fr = a.F + (int64_t)row * a.f_row;
  for (int e = threadIdx.x; e < M * kRowsPerCta; e += blockDim.x) {
    int k = e / kRowsPerCta, q = e % kRowsPerCta;
    int c = col0 + 2 * q;
    double2 A = make_double2(0.0, 0.0), B = A;
    if (c < a.ncols) A = Fr[k * a.f_m + c];
    if (c + 1 < a.ncols) B = Fr[k * a.f_m + c + 1];
    cplx<double>* z = buf + q * N;
    if (k == 0) {
      z[0] = {A.x, B.x};
    } else {
      z[k] = {A.x - B.y, A.y + B.x};
      z[N - k] = {A.x + B.y, B.x - A.y};
    }
  }
  __syncthreads();
  fft_rows<true, kFftCap>(buf, kRowsPerCta, N, N, t.fft_radix, t.fft_nstages, t.twiddle);
  for (int e = threadIdx.x; e < kRowsPerCta * N; e += blockDim.x) {
    int q = e / N, n = e % N;
    cplx<double> z = buf[e];
    int c = col0 + 2 * q;
    if (c < a.ncols) {
      int f = c / a.B, b = c % a.B;
      a.out[f][((int64_t)b * nt + row) * N + n] = z.x;
    }
    if (c + 1 < a.ncols) {
      int f = (c + 1) / a.B, b = (c + 1) % a.B;
      a.out[f][((int64_t)b * nt + row) * N + n] = z.y;
    }
  }
}

__global__ void __launch_bounds__(kFftThreads) k_grid_to_fourier(ToFourierArgs a) {
  extern __shared__ double smem[];
  cplx<double>* buf = reinterpret_cast<cplx<double>*>(smem);
  const Tables& t = a.t;
  const int N = t.n_phi, M = t.n_m, nt = t.n_theta;
  const int row = blockIdx.y;
  const int col0 = blockIdx.x * 2 * kRowsPerCta;
  for (int e = threadIdx.x; e < kRowsPerCta * N; e += blockDim.x) {
    int q = e / N, n = e % N;
    int c = col0 + 2 * q;
    double x = 0.0, y = 0.0;
    if (c < a.ncols) x = a.in[c / a.B][((int64_t)(c % a.B) * nt + row) * N + n];
    if (c + 1 < a.ncols) y = a.in[(c + 1) / a.B][((int64_t)((c + 1) % a.B) * nt + row) * N + n];
    buf[e] = {x, y};
  }
  __syncthreads();
  fft_rows<false, kFftCap>(buf, kRowsPerCta, N, N, t.fft_radix, t.fft_nstages, t.twiddle);
  const double w = (a.vector ? t.wq_v[row] : t.wq[row]) / N;
  double2* Fr = a.F + (int64_t)row * a.f_row;
  for (int e = threadIdx.x; e < M * kRowsPerCta; e += blockDim.x) {
    int k = e / kRowsPerCta, q = e % kRowsPerCta;
    int c = col0 + 2 * q;
    const cplx<double>* z = buf + q * N;
    cplx<double> Z = z[k], Zc = z[(N - k) % N];
    // A = (Z + conj Zc)/2 ; B = (Z - conj Zc)/(2i)
    double ax = 0.5 * (Z.x + Zc.x), ay = 0.5 * (Z.y - Zc.y);
    double dx = Z.x - Zc.x, dy = Z.y + Zc.y;
    double bx = 0.5 * dy, by = -0.5 * dx;
    if (c < a.ncols) Fr[k * a.f_m + c] = make_double2(w * ax, w * ay);
    if (c + 1 < a.ncols) Fr[k * a.f_m + c + 1] = make_double2(w * bx, w * by);
  }
}

static size_t fft_smem(const Tables& t) { return (size_t)kRowsPerCta * t.n_phi * 16; }

int launch_fourier_to_grid(const ToGridArgs& a, cudaStream_t st) {
  size_t sm = fft_smem(a.t);
  MT_CHECK_CUDA(cudaFuncSetAttribute(k_fourier_to_grid, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sm));
  dim3 grid((a.ncols + 2 * kRowsPerCta - 1) / (2 * kRowsPerCta), a.t.n_theta);
  k_fourier_to_grid<<<grid, kFftThreads, sm, st>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

int launch_grid_to_fourier(const ToFourierArgs& a, cudaStream_t st) {
  size_t sm = fft_smem(a.t);
  MT_CHECK_CUDA(cudaFuncSetAttribute(k_grid_to_fourier, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sm));
  dim3 grid((a.ncols + 2 * kRowsPerCta - 1) / (2 * kRowsPerCta), a.t.n_theta);
  k_grid_to_fourier<<<grid, kFftThreads, sm, st>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

// Largest n_phi the fixed per-thread register budget supports (every radix:
// ceil(CAP/R) * R * threads >= rows * n_phi).
int fft_max_nphi() { return kFftCap * kFftThreads / kRowsPerCta; }

}  // namespace mt
