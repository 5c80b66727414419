// Plan-time bf16x3 images of the Legendre tables for the tcgen05 kernels.
//
// Synthesis images (B operand: rows = northern theta, K = l of one parity):
//   [m][table P/dP][parity][theta tile] -> chunks c of 16 l values
//   (l - m = 2 (16 c + i) + parity), each 3 planes x wth rows x 16, core layout.
// Analysis images (B operand: rows = l of one parity, K = theta pairs):
//   [m][table][parity] -> chunks of 16 theta pairs, each 3 planes x wk x 16.
// Values outside the tables are zero, so ragged chunks need no special case.
#include <vector>

#include "split.cuh"

namespace mt {

__global__ void k_split_syn(const double* __restrict__ plm, const double* __restrict__ dplm,
                            const int* __restrict__ lstart, int l_max, int minc, int nhs, int wth,
                            int nthtile, uint8_t* img, const int64_t* __restrict__ off) {
  const int id = blockIdx.x;  // ((mc * 2 + t) * 2 + p) * nthtile + tau
  const int tau = id % nthtile;
  const int p = (id / nthtile) % 2;
  const int t = (id / nthtile / 2) % 2;
  const int mc = id / nthtile / 4;
  const int nlm = l_max - mc * minc + 1;
  const int nch = (split_nk(nlm, p) + kSplitKC - 1) / kSplitKC;
  const double* T = t == 0 ? plm : dplm;
  const int ls = lstart[mc];
  uint8_t* base = img + off[id];
  const int per = wth * kSplitKC;
  for (int e = threadIdx.x; e < nch * per; e += blockDim.x) {
    int c = e / per, rem = e - c * per;
    int r = rem / kSplitKC, kl = rem % kSplitKC;
    int k = 2 * (kSplitKC * c + kl) + p;
    int th = tau * wth + r;
    double v = (k < nlm && th < nhs) ? T[(int64_t)(ls + k) * nhs + th] : 0.0;
    __nv_bfloat16 q[3];
    split3(v, q[0], q[1], q[2]);
    uint8_t* cb = base + (int64_t)c * 3 * wth * 32;
#pragma unroll
    for (int s = 0; s < 3; ++s)
      *reinterpret_cast<__nv_bfloat16*>(cb + s * wth * 32 + core_off(r, kl)) = q[s];
  }
}

__global__ void k_split_ana(const double* __restrict__ plm, const double* __restrict__ dplm,
                            const int* __restrict__ lstart, int l_max, int minc, int nhs,
                            uint8_t* img, const int64_t* __restrict__ off,
                            const int* __restrict__ wks) {
  const int id = blockIdx.x;  // (mc * 2 + t) * 2 + p
  const int p = id % 2, t = (id / 2) % 2, mc = id / 4;
  const int nlm = l_max - mc * minc + 1;
  const int wk = wks[mc * 2 + p];
  const int nch = (nhs + kSplitKC - 1) / kSplitKC;
  const double* T = t == 0 ? plm : dplm;
  const int ls = lstart[mc];
  uint8_t* base = img + off[id];
  const int per = wk * kSplitKC;
  for (int e = threadIdx.x; e < nch * per; e += blockDim.x) {
    int c = e / per, rem = e - c * per;
    int r = rem / kSplitKC, jl = rem % kSplitKC;
    int k = 2 * r + p, j = kSplitKC * c + jl;
    double v = (k < nlm && j < nhs) ? T[(int64_t)(ls + k) * nhs + j] : 0.0;
    __nv_bfloat16 q[3];
    split3(v, q[0], q[1], q[2]);
    uint8_t* cb = base + (int64_t)c * 3 * wk * 32;
#pragma unroll
    for (int s = 0; s < 3; ++s)
      *reinterpret_cast<__nv_bfloat16*>(cb + s * wk * 32 + core_off(r, jl)) = q[s];
  }
}

struct SplitStore {
  SplitTables t;
  uint8_t *syn = nullptr, *ana = nullptr;
  int64_t *syn_off = nullptr, *ana_off = nullptr;
  int *ana_wk = nullptr, *syn_nch = nullptr, *syn_prefix = nullptr;
  std::vector<int64_t> h_syn_off, h_ana_off;
  std::vector<int> h_wk, h_syn_nch, h_syn_prefix;
};

int build_split_tables(mt_plan* p) {
  const int nhs = p->nhs;
  MT_REQUIRE(nhs <= 512 && p->l_max <= 511, MT_ERR_UNSUPPORTED,
             "split precision supports l_max <= 511 and n_theta_max <= 1024");
  SplitStore* S = new SplitStore();
  p->split = S;
  int nthtile = nhs <= 256 ? 1 : 2;
  int wth = round16((nhs + nthtile - 1) / nthtile);
  S->t.wth = wth;
  S->t.nthtile = nthtile;
  const int nm = p->n_m;
  S->h_syn_off.resize((size_t)nm * 4 * nthtile);
  int64_t pos = 0;
  for (int mc = 0; mc < nm; ++mc) {
    int nlm = p->l_max - mc * p->minc + 1;
    for (int t = 0; t < 2; ++t)
      for (int par = 0; par < 2; ++par)
        for (int tau = 0; tau < nthtile; ++tau) {
          S->h_syn_off[((mc * 2 + t) * 2 + par) * nthtile + tau] = pos;
          int nch = (split_nk(nlm, par) + kSplitKC - 1) / kSplitKC;
          pos += (int64_t)nch * 3 * wth * 32;
        }
  }
  int64_t syn_bytes = pos;
  S->h_ana_off.resize((size_t)nm * 4);
  S->h_wk.resize((size_t)nm * 2);
  pos = 0;
  const int nchj = (nhs + kSplitKC - 1) / kSplitKC;
  for (int mc = 0; mc < nm; ++mc) {
    int nlm = p->l_max - mc * p->minc + 1;
    for (int par = 0; par < 2; ++par) S->h_wk[mc * 2 + par] = round16(split_nk(nlm, par));
    for (int t = 0; t < 2; ++t)
      for (int par = 0; par < 2; ++par) {
        S->h_ana_off[(mc * 2 + t) * 2 + par] = pos;
        pos += (int64_t)nchj * 3 * S->h_wk[mc * 2 + par] * 32;
      }
  }
  int64_t ana_bytes = pos;
  S->h_syn_nch.resize((size_t)nm * 2);
  S->h_syn_prefix.resize((size_t)nm * 2 + 1);
  int acc = 0;
  for (int mc = 0; mc < nm; ++mc)
    for (int combo = 0; combo < 2; ++combo) {
      int n = syn_nchunks(p->l_max - mc * p->minc + 1, combo);
      S->h_syn_nch[mc * 2 + combo] = n;
      S->h_syn_prefix[mc * 2 + combo] = acc;
      acc += n;
    }
  S->h_syn_prefix[(size_t)nm * 2] = acc;
  MT_CHECK_CUDA(cudaMalloc(&S->syn, syn_bytes > 0 ? syn_bytes : 16));
  MT_CHECK_CUDA(cudaMalloc(&S->ana, ana_bytes > 0 ? ana_bytes : 16));
  MT_CHECK_CUDA(cudaMalloc(&S->syn_off, S->h_syn_off.size() * sizeof(int64_t)));
  MT_CHECK_CUDA(cudaMalloc(&S->ana_off, S->h_ana_off.size() * sizeof(int64_t)));
  MT_CHECK_CUDA(cudaMalloc(&S->ana_wk, S->h_wk.size() * sizeof(int)));
  MT_CHECK_CUDA(cudaMalloc(&S->syn_nch, S->h_syn_nch.size() * sizeof(int)));
  MT_CHECK_CUDA(cudaMalloc(&S->syn_prefix, S->h_syn_prefix.size() * sizeof(int)));
  MT_CHECK_CUDA(cudaMemcpy(S->syn_nch, S->h_syn_nch.data(), S->h_syn_nch.size() * sizeof(int),
                           cudaMemcpyHostToDevice));
  MT_CHECK_CUDA(cudaMemcpy(S->syn_prefix, S->h_syn_prefix.data(),
                           S->h_syn_prefix.size() * sizeof(int), cudaMemcpyHostToDevice));
  MT_CHECK_CUDA(cudaMemcpy(S->syn_off, S->h_syn_off.data(), S->h_syn_off.size() * sizeof(int64_t),
                           cudaMemcpyHostToDevice));
  MT_CHECK_CUDA(cudaMemcpy(S->ana_off, S->h_ana_off.data(), S->h_ana_off.size() * sizeof(int64_t),
                           cudaMemcpyHostToDevice));
  MT_CHECK_CUDA(cudaMemcpy(S->ana_wk, S->h_wk.data(), S->h_wk.size() * sizeof(int),
                           cudaMemcpyHostToDevice));
  k_split_syn<<<nm * 4 * nthtile, 256>>>(p->d_plm, p->d_dplm, p->d_lstart, p->l_max, p->minc, nhs,
                                         wth, nthtile, S->syn, S->syn_off);
  k_split_ana<<<nm * 4, 256>>>(p->d_plm, p->d_dplm, p->d_lstart, p->l_max, p->minc, nhs, S->ana,
                               S->ana_off, S->ana_wk);
  MT_CHECK_CUDA(cudaGetLastError());
  MT_CHECK_CUDA(cudaDeviceSynchronize());
  S->t.syn = S->syn;
  S->t.syn_off = S->syn_off;
  S->t.ana = S->ana;
  S->t.ana_off = S->ana_off;
  S->t.ana_wk = S->ana_wk;
  S->t.syn_nch = S->syn_nch;
  S->t.syn_chunk_prefix = S->syn_prefix;
  return MT_OK;
}

void free_split_tables(mt_plan* p) {
  SplitStore* S = (SplitStore*)p->split;
  if (!S) return;
  void* ptrs[] = {S->syn, S->ana, S->syn_off, S->ana_off, S->ana_wk, S->syn_nch, S->syn_prefix};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  delete S;
  p->split = nullptr;
}

const SplitTables& split_tables(const mt_plan* p) { return ((SplitStore*)p->split)->t; }
const std::vector<int64_t>& split_syn_off_host(const mt_plan* p) {
  return ((SplitStore*)p->split)->h_syn_off;
}
const std::vector<int>& split_wk_host(const mt_plan* p) { return ((SplitStore*)p->split)->h_wk; }
int split_syn_total_chunks(const mt_plan* p) {
  return ((SplitStore*)p->split)->h_syn_prefix.back();
}

}  // namespace mt
