// Horizontal tables of a plan, built on the GPU in FP64.
//
// * Gauss-Legendre nodes/weights: Newton iteration on P_n from the guess
//   cos(pi (i - 1/4)/(n + 1/2)), stop when the update is <= 10 eps
//   (reference magic_torch/horizontal_data.py:16-50).  One thread per root.
// * P_l^m (fully normalised, 1/sqrt(4 pi), no Condon-Shortley phase) and
//   sin(theta) dP_l^m/dtheta by the three-term recurrences of
//   magic_torch/plms.py:21-155.  One thread per (m, northern theta): the
//   thread walks l = m .. l_max+1 keeping three consecutive P values.
// * Interleaved-row weights 2 pi w, 1/sin^2, cos/sin^2
//   (magic_torch/horizontal_data.py:59-84) and FFT twiddles.
#include <cmath>
#include <vector>

#include "common.cuh"

namespace mt {

__global__ void k_gauleg(int n, double* theta, double* gauss) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;  // root index, 0-based
  int half = (n + 1) / 2;
  if (i >= half) return;
  const double eps = 10.0 * 2.220446049250313e-16;
  double z = cos(M_PI * ((i + 1) - 0.25) / (n + 0.5));
  double z1 = z + 10.0 * eps;
  double pp = 0.0;
  for (int it = 0; it < 100 && fabs(z - z1) > eps; ++it) {
    double p1 = 1.0, p2 = 0.0;
    for (int j = 1; j <= n; ++j) {
      double p3 = p2;
      p2 = p1;
      p1 = ((2 * j - 1) * z * p2 - (j - 1) * p3) / j;
    }
    pp = n * (z * p1 - p2) / (z * z - 1.0);
    z1 = z;
    z = z1 - p1 / pp;
  }
  theta[i] = acos(z);
  theta[n - 1 - i] = acos(-z);
  double w = 2.0 / ((1.0 - z * z) * pp * pp);
  gauss[i] = w;
  gauss[n - 1 - i] = w;
}

__global__ void k_plm(int l_max, int minc, int n_m, int nhs, const int* __restrict__ lstart,
                      const double* __restrict__ theta, double* plm, double* dplm) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  int mc = blockIdx.y;
  if (j >= nhs || mc >= n_m) return;
  const double osq4pi = 0.28209479177387814347;  // 1/sqrt(4 pi)
  int m = mc * minc;
  double th = theta[j];
  double ct = cos(th), st = sin(th);
  double fac = 1.0;
  for (int q = 3; q <= 2 * m + 1; q += 2) fac = fac * q / (q - 1);
  double p = sqrt(fac);
  if (st != 0.0) p = p * pow(st, (double)m);
  else if (m != 0) p = 0.0;
  size_t base = (size_t)lstart[mc];
  // window of normalised values: pm1 = P_{l-1}, p0 = P_l, raw recurrence state
  double raw_prev = 0.0, raw = p;
  double nm1 = 0.0, n0 = osq4pi * raw;
  plm[base * nhs + j] = n0;
  for (int l = m + 1; l <= l_max + 1; ++l) {
    // integer products formed in double (exact below 2^53, as the reference's
    // Python integers rounded once)
    const double L = l, M = m;
    double a = sqrt(((2 * L - 1) * (2 * L + 1)) / ((L - M) * (L + M)));
    double b = sqrt(((2 * L + 1) * (L + M - 1) * (L - M - 1)) /
                    ((2 * L - 3) * (L - M) * (L + M)));
    double rn = ct * a * raw - b * raw_prev;
    raw_prev = raw;
    raw = rn;
    double n1 = osq4pi * raw;  // P_l, normalised
    // emit sin dP/dtheta for degree l-1 now that P_l is known
    int lp = l - 1;
    const double P = lp;
    double up = (lp == m) ? P / sqrt(2 * P + 3) * n1
                          : P * sqrt(((P + M + 1) * (P - M + 1)) / ((2 * P + 1) * (2 * P + 3))) * n1;
    double dn = (lp == m) ? 0.0
                          : (P + 1) * sqrt(((P + M) * (P - M)) / ((2 * P - 1) * (2 * P + 1))) * nm1;
    dplm[(base + (lp - m)) * nhs + j] = up - dn;
    if (l <= l_max) plm[(base + (l - m)) * nhs + j] = n1;
    nm1 = n0;
    n0 = n1;
  }
}

__global__ void k_rows(int n, const double* __restrict__ theta, const double* __restrict__ gauss,
                       double* wq, double* wq_v, double* ost2, double* cosn) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int nhs = n / 2;
  int geo = (i % 2 == 0) ? i / 2 : n - 1 - (i - 1) / 2;
  double th = theta[geo];
  double s = sin(th);
  double o = 1.0 / (s * s);
  double w = 2.0 * M_PI * gauss[geo];
  (void)nhs;
  wq[i] = w;
  ost2[i] = o;
  wq_v[i] = w * o;
  cosn[i] = cos(th) * o;
}

__global__ void k_lm(int l_max, int minc, int lm_max, double* dlh) {
  int lm = blockIdx.x * blockDim.x + threadIdx.x;
  if (lm >= lm_max) return;
  // invert lm -> (m, l) by walking the order blocks (lm_max is small)
  int pos = 0;
  for (int m = 0; m <= l_max; m += minc) {
    int n = l_max - m + 1;
    if (lm < pos + n) {
      double l = (double)(m + (lm - pos));
      dlh[lm] = l * (l + 1.0);
      return;
    }
    pos += n;
  }
}

__global__ void k_twiddle(int n, double2* tw) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s, c;
  sincospi(2.0 * i / n, &s, &c);
  tw[i] = make_double2(c, -s);
}

static int factor_radices(int n, int* out) {
  int ns = 0;
  while (n % 8 == 0 && ns < kMaxFftStages) { out[ns++] = 8; n /= 8; }
  while (n % 4 == 0 && ns < kMaxFftStages) { out[ns++] = 4; n /= 4; }
  while (n % 2 == 0 && ns < kMaxFftStages) { out[ns++] = 2; n /= 2; }
  while (n % 3 == 0 && ns < kMaxFftStages) { out[ns++] = 3; n /= 3; }
  while (n % 5 == 0 && ns < kMaxFftStages) { out[ns++] = 5; n /= 5; }
  return n == 1 ? ns : -1;
}

int build_tables(mt_plan* p) {
  const int nt = p->n_theta, nhs = p->nhs;
  std::vector<int> ls(p->n_m);
  int pos = 0;
  for (int mc = 0; mc < p->n_m; ++mc) {
    ls[mc] = pos;
    pos += p->l_max - mc * p->minc + 1;
  }
  MT_REQUIRE(pos == p->lm_max, MT_ERR_ARG, "lm_max mismatch");
  int radix[kMaxFftStages];
  MT_REQUIRE(p->n_phi % 2 == 0, MT_ERR_UNSUPPORTED, "n_phi_max must be even");
  int nst = factor_radices(p->n_phi / 2, radix);  // real FFTs run as half-length complex FFTs
  MT_REQUIRE(nst > 0, MT_ERR_UNSUPPORTED, "n_phi_max must factor into 2, 3, 5");

  size_t tsz = (size_t)p->lm_max * nhs * sizeof(double);
  MT_CHECK_CUDA(cudaMalloc(&p->d_lstart, p->n_m * sizeof(int)));
  MT_CHECK_CUDA(cudaMalloc(&p->d_theta, nt * sizeof(double)));
  MT_CHECK_CUDA(cudaMalloc(&p->d_gauss, nt * sizeof(double)));
  MT_CHECK_CUDA(cudaMalloc(&p->d_plm, tsz));
  MT_CHECK_CUDA(cudaMalloc(&p->d_dplm, tsz));
  MT_CHECK_CUDA(cudaMalloc(&p->d_dlh, p->lm_max * sizeof(double)));
  MT_CHECK_CUDA(cudaMalloc(&p->d_wq, nt * sizeof(double)));
  MT_CHECK_CUDA(cudaMalloc(&p->d_wq_v, nt * sizeof(double)));
  MT_CHECK_CUDA(cudaMalloc(&p->d_ost2, nt * sizeof(double)));
  MT_CHECK_CUDA(cudaMalloc(&p->d_cosn, nt * sizeof(double)));
  MT_CHECK_CUDA(cudaMalloc(&p->d_twiddle, p->n_phi * sizeof(double2)));
  MT_CHECK_CUDA(cudaMemcpy(p->d_lstart, ls.data(), p->n_m * sizeof(int), cudaMemcpyHostToDevice));

  k_gauleg<<<(nt / 2 + 127) / 128, 128>>>(nt, p->d_theta, p->d_gauss);
  dim3 gp((nhs + 127) / 128, p->n_m);
  k_plm<<<gp, 128>>>(p->l_max, p->minc, p->n_m, nhs, p->d_lstart, p->d_theta, p->d_plm,
                     p->d_dplm);
  k_rows<<<(nt + 127) / 128, 128>>>(nt, p->d_theta, p->d_gauss, p->d_wq, p->d_wq_v, p->d_ost2,
                                   p->d_cosn);
  k_lm<<<(p->lm_max + 255) / 256, 256>>>(p->l_max, p->minc, p->lm_max, p->d_dlh);
  k_twiddle<<<(p->n_phi + 255) / 256, 256>>>(p->n_phi, p->d_twiddle);
  MT_CHECK_CUDA(cudaGetLastError());
  MT_CHECK_CUDA(cudaDeviceSynchronize());

  Tables& t = p->tab;
  t.l_max = p->l_max;
  t.minc = p->minc;
  t.n_theta = nt;
  t.n_phi = p->n_phi;
  t.n_m = p->n_m;
  t.lm_max = p->lm_max;
  t.nhs = nhs;
  t.lstart = p->d_lstart;
  t.plm = p->d_plm;
  t.dplm = p->d_dplm;
  t.dlh = p->d_dlh;
  t.wq = p->d_wq;
  t.wq_v = p->d_wq_v;
  t.ost2 = p->d_ost2;
  t.cosn = p->d_cosn;
  t.twiddle = p->d_twiddle;
  t.fft_nstages = nst;
  for (int s = 0; s < kMaxFftStages; ++s) t.fft_radix[s] = s < nst ? radix[s] : 1;
  return MT_OK;
}

}  // namespace mt
