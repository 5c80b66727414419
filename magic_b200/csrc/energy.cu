// Kinetic and magnetic energy integrals of the outer core (FP64):
// magic_torch/output.py:101-180 (get_e_kin_full, get_e_mag_oc_full).
//
// Per (lm, r): poloidal density c(r) l(l+1) (l(l+1) or2(r) |a|^2 + |da|^2),
// toroidal density c(r) l(l+1) |t|^2, with |x|^2 the reference's cc2real
// (Re^2 for m = 0, 2 (Re^2 + Im^2) otherwise) and c = orho1 / 2 (kinetic) or
// LFfac / 2 (magnetic).  Each density is summed over lm under four masks
// (all, m = 0, equatorially symmetric, its m = 0 part) and integrated over r
// with the reference's radial rule (weights rint[r], built on the host as the
// rule applied to unit vectors).  The magnetic case adds the potential-field
// energy outside the shell, sum l^2 (l+1) |b(r_cmb)|^2 (all and m = 0; the
// caller scales it by LFfac / (2 r_cmb)).
//
// k_energy_part: CTA = (chunk of 64 rows l of one order m, which are
// contiguous in memory); thread = radial level(s) r, so a warp reads 32
// consecutive levels of a row.  Each CTA integrates its rows' densities over r
// and writes 10 partial sums; k_energy_sum adds the partials in a fixed
// order (results do not depend on scheduling).
#include "common.cuh"

namespace mt {
namespace {

constexpr int kEnRows = 64;
constexpr int kEnThreads = 128;
constexpr int kEnQ = 10;  // pol: all, m0, ES, EAS; tor: all, m0, ES, EAS; outside: all, m0

struct EnArgs {
  int n_r, l_max, minc, mag;
  const int* lstart;
  const double2 *a, *da, *t;
  int64_t ld;
  const double *or2, *cr, *rint;
  double* part;
};

__device__ __forceinline__ double cc2real(double2 c, bool m0) {
  return m0 ? c.x * c.x : 2.0 * (c.x * c.x + c.y * c.y);
}

// deterministic sum of v over the CTA (fixed shuffle tree, then warp order)
__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
  return s;
}

__global__ void __launch_bounds__(kEnThreads) k_energy_part(EnArgs a) {
  __shared__ double red[kEnThreads / 32];
  const int mc = blockIdx.y, m = mc * a.minc;
  const int l0 = m + blockIdx.x * kEnRows;
  const int chunk = blockIdx.y * gridDim.x + blockIdx.x;
  double acc[kEnQ];
#pragma unroll
  for (int q = 0; q < kEnQ; ++q) acc[q] = 0.0;
  const bool m0 = m == 0;
  if (l0 <= a.l_max) {
    const int nrow = min(kEnRows, a.l_max - l0 + 1);
    const int64_t lm0 = a.lstart[mc] + (l0 - m);
    for (int r = threadIdx.x; r < a.n_r; r += blockDim.x) {
      const double or2 = a.or2[r], wr = a.rint[r] * a.cr[r];
      double s[kEnQ];
#pragma unroll
      for (int q = 0; q < kEnQ; ++q) s[q] = 0.0;
      for (int rr = 0; rr < nrow; ++rr) {
        const int l = l0 + rr;
        const int64_t o = (lm0 + rr) * a.ld + r;
        const double dL = (double)l * (l + 1.0);
        const double ep = dL * (dL * or2 * cc2real(a.a[o], m0) + cc2real(a.da[o], m0));
        const double et = dL * cc2real(a.t[o], m0);
        const bool lpm_even = ((l + m) & 1) == 0, l_even = (l & 1) == 0;
        // kinetic: ES pol (l+m) even, tor (l+m) odd; EAS pol m = 0 l even, tor l odd.
        // magnetic: the opposite parities (output.py:121-131, 165-171).
        const bool es_p = a.mag ? !lpm_even : lpm_even;
        const bool eas_p = m0 && (a.mag ? !l_even : l_even);
        s[0] += ep;
        s[4] += et;
        if (m0) {
          s[1] += ep;
          s[5] += et;
        }
        if (es_p) s[2] += ep; else s[6] += et;
        if (m0) {
          if (eas_p) s[3] += ep; else s[7] += et;
        }
        if (a.mag && r == 0) {
          const double os = (double)l * l * (l + 1.0) * cc2real(a.a[o], m0);
          s[8] += os;
          if (m0) s[9] += os;
        }
      }
#pragma unroll
      for (int q = 0; q < 8; ++q) acc[q] += wr * s[q];
      acc[8] += s[8];
      acc[9] += s[9];
    }
  }
#pragma unroll
  for (int q = 0; q < kEnQ; ++q) {
    const double v = block_sum(acc[q], red);
    if (threadIdx.x == 0) a.part[(int64_t)chunk * kEnQ + q] = v;
  }
}

// out[q] = sum over chunks of part[chunk][q], one warp per q, fixed order
__global__ void k_energy_sum(const double* __restrict__ part, int nchunk, double* out) {
  const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (q >= kEnQ) return;
  double v = 0.0;
  for (int c = lane; c < nchunk; c += 32) v += part[(int64_t)c * kEnQ + q];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if (lane == 0) out[q] = v;
}

int energy_chunks(const mt_plan* p) { return ((p->l_max + kEnRows) / kEnRows) * p->n_m; }

}  // namespace
}  // namespace mt

using namespace mt;

extern "C" {

size_t mt_energy_workspace(const mt_plan* p) {
  if (!p) return 0;
  return (size_t)(energy_chunks(p) + 1) * kEnQ * sizeof(double);
}

int mt_energy(const mt_plan* p, int n_r, const mt_energy_args* e, double* out, void* work,
              size_t work_bytes, void* stream) {
  MT_REQUIRE(p && e && out, MT_ERR_ARG, "null argument");
  int dev = -1;
  MT_CHECK_CUDA(cudaGetDevice(&dev));
  MT_REQUIRE(dev == p->device, MT_ERR_ARG, "plan used on a different device than it was built on");
  MT_REQUIRE(n_r >= 2 && e->ld >= n_r, MT_ERR_ARG, "bad radial size or stride");
  MT_REQUIRE(e->pol && e->dpol && e->tor && e->or2 && e->cr && e->rint, MT_ERR_ARG,
             "null field or profile");
  MT_REQUIRE(work && work_bytes >= mt_energy_workspace(p), MT_ERR_ARG, "workspace too small");
  EnArgs a{};
  a.n_r = n_r;
  a.l_max = p->l_max;
  a.minc = p->minc;
  a.mag = e->magnetic ? 1 : 0;
  a.lstart = p->d_lstart;
  a.a = (const double2*)e->pol;
  a.da = (const double2*)e->dpol;
  a.t = (const double2*)e->tor;
  a.ld = e->ld;
  a.or2 = e->or2;
  a.cr = e->cr;
  a.rint = e->rint;
  a.part = (double*)work;
  const dim3 grid((p->l_max + kEnRows) / kEnRows, p->n_m);
  k_energy_part<<<grid, kEnThreads, 0, (cudaStream_t)stream>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  k_energy_sum<<<1, 32 * kEnQ, 0, (cudaStream_t)stream>>>(a.part, energy_chunks(p), out);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

}  // extern "C"
