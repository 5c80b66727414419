// Digit-split ("ozaki") Legendre stage of the fused Boussinesq radial loop:
// table digit images (plan time), the synthesis and analysis packing kernels
// and the two persistent tcgen05 kind::i8 GEMMs (ozaki.cuh has the scheme).
//
// Orientation as in the bf16x3 kernels (legendre_split.cu): the data operand
// is A (M = 128 rows per tile, one row per output real component), the table
// is B (N = kOzSynN theta rows for the synthesis, kOzAnaN l rows for the
// analysis), K runs over l (synthesis) or theta pairs (analysis) in chunks of
// 32.  Row scales of A are found by the packing kernels in a first pass over
// the whole K range of their block; column scales of B at plan time.
#include <algorithm>
#include <vector>

#include "ozaki.cuh"
#include "umma.cuh"

namespace mt {

// ------------------------------------------------------------- digits

// Exponent e with |x| < 2^e for the largest magnitude x of a row (0 for 0).
__device__ __forceinline__ int oz_exponent(double mx) {
  int e = 0;
  if (mx > 0.0) frexp(mx, &e);
  return e;
}

// Six signed digits of v at scale 2^e (|v| < 2^e): Y = rint(v 2^(41 - e)),
// |Y| <= 2^41, written in balanced base 128, Y = sum_i d_i 2^(7 (5 - i)) with
// d_0 in [-64, 64] and d_1..d_5 in [-64, 63], so v = 2^(e - 6) sum_i d_i 2^(-7 i)
// to 2^(e - 42).  Adding O = 64 sum_i 2^(7 (5 - i)) makes every base-128 digit
// of Y + O non-negative (d_i = digit_i(Y + O) - 64), so the six digits come
// from independent shifts of one integer.
constexpr unsigned long long kOzDigitOffset =
    64ull * ((1ull << 35) + (1ull << 28) + (1ull << 21) + (1ull << 14) + (1ull << 7) + 1ull);

__device__ __forceinline__ double oz_scale_up(double v, int s);
__device__ __forceinline__ double oz_pow2(int s);

__device__ __forceinline__ void oz_digits(double v, int e, int8_t (&d)[kOzDigits]) {
  const long long Y = __double2ll_rn(oz_scale_up(v, 41 - e));
  const unsigned long long U = (unsigned long long)Y + kOzDigitOffset;
  d[0] = (int8_t)((int)(U >> 35) - 64);
#pragma unroll
  for (int i = 1; i < kOzDigits; ++i) d[i] = (int8_t)((int)((U >> (7 * (5 - i))) & 127u) - 64);
}

// The pack kernels' form of the same digits, four values to a 32-bit word
// per digit plane.  One fma forms T = 1.5 2^52 + O + rint(v 2^(41 - e)): the
// product v 2^(41 - e) is exact, |rint(..)| <= 2^41, and the fma's single
// rounding to the integer grid of [2^52, 2^53) is rint's with ties to even,
// 1.5 2^52 + O being an even integer; the mantissa of T is then 2^51 + U
// (U = Y + O < 2^43): U mod 2^32 is T's low word and U / 2^32 the low bits of
// its high word, so the six base-128 fields x_i of U need only 32-bit shifts
// (x_0 <= 128 takes eight bits).  oz_put_digits puts byte b of w[i]:
// d_0 = x_0 - 64 directly, x_1 .. x_5 raw; oz_bias_bytes then subtracts 64 from
// each byte of a word of raw fields (all below 128) without borrows.
__device__ __forceinline__ double oz_digit_word(double v, int e) {
  constexpr double kC = 6755399441055744.0 + (double)kOzDigitOffset;
  const int s = 41 - e;
  if (s <= 1023) return fma(v, oz_pow2(s), kC);
  return fma(v * oz_pow2(min(s - 1023, 1023)), 0x1p1023, kC);
}

__device__ __forceinline__ void oz_put_digits(double v, int e, int b, uint32_t (&w)[kOzDigits]) {
  const double T = oz_digit_word(v, e);
  const uint32_t lo = (uint32_t)__double2loint(T), hi = (uint32_t)__double2hiint(T);
  const int sh = 8 * b;
  w[0] |= (((hi >> 3) + 192u) & 0xFFu) << sh;
  w[1] |= (__funnelshift_r(lo, hi, 28) & 127u) << sh;
  w[2] |= ((lo >> 21) & 127u) << sh;
  w[3] |= ((lo >> 14) & 127u) << sh;
  w[4] |= ((lo >> 7) & 127u) << sh;
  w[5] |= (lo & 127u) << sh;
}

__device__ __forceinline__ uint32_t oz_bias_bytes(uint32_t w) {
  return ((w | 0x80808080u) - 0x40404040u) ^ 0x80808080u;
}

// Digits of four values (scale 2^e each) as the six plane words of a 4-byte
// group: w[i] byte b = digit i of v[b].
__device__ __forceinline__ void oz_digit_words(const double (&v)[4], int e,
                                               uint32_t (&w)[kOzDigits]) {
#pragma unroll
  for (int s = 0; s < kOzDigits; ++s) w[s] = 0u;
#pragma unroll
  for (int b = 0; b < 4; ++b) oz_put_digits(v[b], e, b, w);
#pragma unroll
  for (int s = 1; s < kOzDigits; ++s) w[s] = oz_bias_bytes(w[s]);
}

// Instruction descriptor: kind::i8, s8 x s8 -> s32, A and B K-major.
__host__ __device__ constexpr uint32_t umma_idesc_s8(int M, int N) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_s8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
      : "memory");
}

// 16 consecutive int32 columns of this thread's TMEM lane, without the wait:
// several loads are issued, then one tmem_wait_ld() makes their registers valid.
__device__ __forceinline__ void tmem_ld16_i32_nowait(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

// 8 consecutive int32 columns of this thread's TMEM lane, without the wait.
__device__ __forceinline__ void tmem_ld8_i32_nowait(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}

// v 2^s rounded once, as ldexp rounds it, without a library call.  For
// -1022 <= s <= 1023 it is one multiplication by the exact power of two.  The
// epilogues' exponents never exceed 1023; below -1022, v 2^(s + 1022) is exact
// (v, an integer sum below 2^59, is far from the underflow range) and the
// multiplication by 2^-1022 rounds once into the subnormals (for s < -2044 the
// result is 0 either way).  The packs' exponents (41 - e for |v| < 2^e) are
// at least -982, and exceed 1023 only for values below 2^-982, scaled by two
// exact multiplications.
__device__ __forceinline__ double oz_pow2(int s) {  // s in [-1022, 1023]
  return __longlong_as_double((long long)(s + 1023) << 52);
}

__device__ __forceinline__ double oz_scale(double v, int s) {  // s <= 1023
  if (s >= -1022) return v * oz_pow2(s);
  return (v * oz_pow2(max(s + 1022, -1022))) * 0x1p-1022;
}

__device__ __forceinline__ double oz_scale_up(double v, int s) {  // s >= -1022
  if (s <= 1023) return v * oz_pow2(s);
  return (v * oz_pow2(min(s - 1023, 1023))) * 0x1p1023;
}

// Exact int32 -> double without a conversion instruction: the double whose
// high word is 0x43300000 and low word w + 2^31 is 2^52 + w + 2^31.
__device__ __forceinline__ double oz_i2d(uint32_t w) {
  return __hiloint2double(0x43300000, (int)(w ^ 0x80000000u)) - 4503601774854144.0;
}

// 2^35 sum_g 2^(-7 g) C_g for one accumulator column from raw TMEM words,
// rounded once to FP64: the halves P1 = (C0 2^7 + C1) 2^7 + C2 and
// P2 = (C3 2^7 + C4) 2^7 + C5 are integers below 2^38, exact in FP64, and the
// sum P1 2^21 + P2 (below 2^59) is rounded by the final fma alone; callers
// scale by 2^(e - 35).
template <int W>
__device__ __forceinline__ double oz_combine_u(const uint32_t (&c)[kOzGroups][W], int i) {
  static_assert(kOzGroups == 6, "two exact halves of three groups each");
  const double p1 = fma(fma(oz_i2d(c[0][i]), 128.0, oz_i2d(c[1][i])), 128.0, oz_i2d(c[2][i]));
  const double p2 = fma(fma(oz_i2d(c[3][i]), 128.0, oz_i2d(c[4][i])), 128.0, oz_i2d(c[5][i]));
  return fma(p1, 2097152.0, p2);
}

// Named barrier over `n` threads that also ANDs a predicate across them, so
// that all participants take the same branch afterwards.
__device__ __forceinline__ void named_bar_sync(int id, int n) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(n) : "memory");
}

__device__ __forceinline__ bool bar_and(int id, int n, bool v) {
  uint32_t r;
  asm volatile(
      "{\n.reg .pred p, q;\nsetp.ne.u32 p, %1, 0;\nbar.red.and.pred q, %2, %3, p;\n"
      "selp.u32 %0, 1, 0, q;\n}\n"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(id), "r"(n)
      : "memory");
  return r != 0;
}

// Issue the 21 digit-pair products of one K chunk: pair (i, j) accumulates
// into group g = i + j at tmem_acc + g * NP (NP: MMA columns per table digit
// plane).  The table's six digit planes lie one after another in shared
// memory (NP rows of 32 bytes each, 8-row core groups 256 bytes apart), so the
// planes j0 .. j0 + np - 1 form one operand of N = np * NP rows, and its
// product with data plane i lands in groups i + j0 .. i + j0 + np - 1: eight
// MMAs of up to 256 columns (NP = 64) or six (NP = 32) instead of 21, each
// data plane read once per chunk.  `first`: the first chunk of an item, whose
// i = 0 products (covering every group) overwrite the accumulators.
template <int NP>
__device__ __forceinline__ void oz_mma_chunk(uint32_t tmem_acc, uint32_t sa, uint32_t sb,
                                             bool first) {
  constexpr int kMaxPlanes = 256 / NP;
#pragma unroll
  for (int i = 0; i < kOzDigits; ++i) {
    const uint64_t da = umma_desc(sa + (uint32_t)i * kOzAPlane, 128, 256);
#pragma unroll
    for (int j0 = 0; j0 < kOzDigits - i; j0 += kMaxPlanes) {
      const int np = (kOzDigits - i - j0) < kMaxPlanes ? (kOzDigits - i - j0) : kMaxPlanes;
      const uint64_t db = umma_desc(sb + (uint32_t)(j0 * NP * kOzK), 128, 256);
      umma_s8(tmem_acc + (uint32_t)((i + j0) * NP), da, db, umma_idesc_s8(kOzRows, np * NP),
              (first && i == 0) ? 0u : 1u);
    }
  }
}

// ------------------------------------------------------ plan-time tables

// Synthesis column exponents: block (m, combo), thread per theta: the largest
// |P| over l - m of parity combo and |dP| over the other parity.
__global__ void k_oz_syn_fexp(const double* __restrict__ plm, const double* __restrict__ dplm,
                              const int* __restrict__ lstart, int l_max, int minc, int nhs,
                              int nthw, int* fexp) {
  const int mc = blockIdx.x >> 1, combo = blockIdx.x & 1;
  const int nlm = l_max - mc * minc + 1;
  const int ls = lstart[mc];
  for (int th = threadIdx.x; th < nthw; th += blockDim.x) {
    double mx = 0.0;
    if (th < nhs)
      for (int k = 0; k < nlm; ++k) {
        const bool p_par = ((k & 1) == combo);  // P rows of parity combo, dP rows of the other
        const double v = p_par ? plm[(int64_t)(ls + k) * nhs + th] : dplm[(int64_t)(ls + k) * nhs + th];
        mx = fmax(mx, fabs(v));
      }
    fexp[((int64_t)mc * 2 + combo) * nthw + th] = oz_exponent(mx);
  }
}

// Synthesis table digits: block ((m * 2 + q) * 2 + p) * nthtile + tau.
__global__ void k_oz_syn_img(const double* __restrict__ plm, const double* __restrict__ dplm,
                             const int* __restrict__ lstart, int l_max, int minc, int nhs,
                             int nthtile, const int* __restrict__ fexp, int8_t* img,
                             const int64_t* __restrict__ off) {
  const int id = blockIdx.x;
  const int tau = id % nthtile;
  const int p = (id / nthtile) % 2;
  const int q = (id / nthtile / 2) % 2;
  const int mc = id / nthtile / 4;
  const int nlm = l_max - mc * minc + 1;
  const int nch = (split_nk(nlm, p) + kOzK - 1) / kOzK;
  const int combo = q == 0 ? p : 1 - p;
  const double* T = q == 0 ? plm : dplm;
  const int ls = lstart[mc];
  const int nthw = nthtile * kOzSynN;
  int8_t* base = img + off[id];
  const int per = kOzSynN * kOzK;
  for (int e = threadIdx.x; e < nch * per; e += blockDim.x) {
    const int c = e / per, rem = e - c * per;
    const int r = rem / kOzK, kl = rem % kOzK;
    const int k = 2 * (kOzK * c + kl) + p;
    const int th = tau * kOzSynN + r;
    const double v = (k < nlm && th < nhs) ? T[(int64_t)(ls + k) * nhs + th] : 0.0;
    int8_t d[kOzDigits];
    oz_digits(v, fexp[((int64_t)mc * 2 + combo) * nthw + th], d);
    int8_t* cb = base + (int64_t)c * kOzSynBChunk;
#pragma unroll
    for (int s = 0; s < kOzDigits; ++s) cb[s * kOzSynBPlane + oz_off(r, kl)] = d[s];
  }
}

// Analysis row exponents: block (m * 2 + q) * 2 + p, thread per l row: the
// largest |T_l| over the theta pairs.
__global__ void k_oz_ana_fexp(const double* __restrict__ plm, const double* __restrict__ dplm,
                              const int* __restrict__ lstart, int l_max, int minc, int nhs,
                              int nlt, int* fexp) {
  const int id = blockIdx.x;
  const int p = id % 2, q = (id / 2) % 2, mc = id / 4;
  const int nlm = l_max - mc * minc + 1;
  const double* T = q == 0 ? plm : dplm;
  const int ls = lstart[mc];
  for (int kk = threadIdx.x; kk < nlt * kOzAnaN; kk += blockDim.x) {
    const int k = 2 * kk + p;
    double mx = 0.0;
    if (k < nlm)
      for (int j = 0; j < nhs; ++j) mx = fmax(mx, fabs(T[(int64_t)(ls + k) * nhs + j]));
    fexp[(int64_t)id * nlt * kOzAnaN + kk] = oz_exponent(mx);
  }
}

// Analysis table digits: block ((m * 2 + q) * 2 + p) * nlt + lt.
__global__ void k_oz_ana_img(const double* __restrict__ plm, const double* __restrict__ dplm,
                             const int* __restrict__ lstart, int l_max, int minc, int nhs, int nlt,
                             const int* __restrict__ fexp, int8_t* img,
                             const int64_t* __restrict__ off) {
  const int id = blockIdx.x;
  const int lt = id % nlt;
  const int tp = id / nlt;  // (m * 2 + q) * 2 + p
  const int p = tp % 2, q = (tp / 2) % 2, mc = tp / 4;
  const int nlm = l_max - mc * minc + 1;
  const double* T = q == 0 ? plm : dplm;
  const int ls = lstart[mc];
  const int nchj = (nhs + kOzK - 1) / kOzK;
  int8_t* base = img + off[id];
  const int per = kOzAnaN * kOzK;
  for (int e = threadIdx.x; e < nchj * per; e += blockDim.x) {
    const int c = e / per, rem = e - c * per;
    const int r = rem / kOzK, jl = rem % kOzK;
    const int kk = lt * kOzAnaN + r, k = 2 * kk + p, j = kOzK * c + jl;
    const double v = (k < nlm && j < nhs) ? T[(int64_t)(ls + k) * nhs + j] : 0.0;
    int8_t d[kOzDigits];
    oz_digits(v, fexp[(int64_t)tp * nlt * kOzAnaN + kk], d);
    int8_t* cb = base + (int64_t)c * kOzAnaBChunk;
#pragma unroll
    for (int s = 0; s < kOzDigits; ++s) cb[s * kOzAnaBPlane + oz_off(r, jl)] = d[s];
  }
}

struct OzStore {
  OzTables t;
  int8_t *syn = nullptr, *ana = nullptr;
  int64_t *syn_off = nullptr, *ana_off = nullptr;
  int *syn_fexp = nullptr, *ana_fexp = nullptr, *syn_prefix = nullptr;
  std::vector<int> h_prefix;
};

int build_ozaki_tables(mt_plan* p) {
  const int nhs = p->nhs, nm = p->n_m;
  OzStore* S = new OzStore();
  p->ozaki = S;
  const int nthtile = (nhs + kOzSynN - 1) / kOzSynN;
  const int nthw = nthtile * kOzSynN;
  const int nlt = (split_nk(p->l_max + 1, 0) + kOzAnaN - 1) / kOzAnaN;
  const int nchj = (nhs + kOzK - 1) / kOzK;
  std::vector<int64_t> so((size_t)nm * 4 * nthtile), ao((size_t)nm * 4 * nlt);
  int64_t pos = 0;
  for (int mc = 0; mc < nm; ++mc) {
    const int nlm = p->l_max - mc * p->minc + 1;
    for (int q = 0; q < 2; ++q)
      for (int par = 0; par < 2; ++par)
        for (int tau = 0; tau < nthtile; ++tau) {
          so[((mc * 2 + q) * 2 + par) * nthtile + tau] = pos;
          pos += (int64_t)((split_nk(nlm, par) + kOzK - 1) / kOzK) * kOzSynBChunk;
        }
  }
  const int64_t syn_bytes = pos;
  pos = 0;
  for (int mc = 0; mc < nm; ++mc)
    for (int q = 0; q < 2; ++q)
      for (int par = 0; par < 2; ++par)
        for (int lt = 0; lt < nlt; ++lt) {
          ao[((mc * 2 + q) * 2 + par) * nlt + lt] = pos;
          pos += (int64_t)nchj * kOzAnaBChunk;
        }
  const int64_t ana_bytes = pos;
  S->h_prefix.resize((size_t)nm * 2 + 1);
  int acc = 0;
  for (int mc = 0; mc < nm; ++mc)
    for (int combo = 0; combo < 2; ++combo) {
      S->h_prefix[mc * 2 + combo] = acc;
      acc += oz_syn_nch(p->l_max - mc * p->minc + 1, combo);
    }
  S->h_prefix[(size_t)nm * 2] = acc;
  MT_CHECK_CUDA(cudaMalloc(&S->syn, syn_bytes > 0 ? syn_bytes : 16));
  MT_CHECK_CUDA(cudaMalloc(&S->ana, ana_bytes > 0 ? ana_bytes : 16));
  MT_CHECK_CUDA(cudaMalloc(&S->syn_off, so.size() * sizeof(int64_t)));
  MT_CHECK_CUDA(cudaMalloc(&S->ana_off, ao.size() * sizeof(int64_t)));
  MT_CHECK_CUDA(cudaMalloc(&S->syn_fexp, (size_t)nm * 2 * nthw * sizeof(int)));
  MT_CHECK_CUDA(cudaMalloc(&S->ana_fexp, (size_t)nm * 4 * nlt * kOzAnaN * sizeof(int)));
  MT_CHECK_CUDA(cudaMalloc(&S->syn_prefix, S->h_prefix.size() * sizeof(int)));
  MT_CHECK_CUDA(cudaMemcpy(S->syn_off, so.data(), so.size() * sizeof(int64_t),
                           cudaMemcpyHostToDevice));
  MT_CHECK_CUDA(cudaMemcpy(S->ana_off, ao.data(), ao.size() * sizeof(int64_t),
                           cudaMemcpyHostToDevice));
  MT_CHECK_CUDA(cudaMemcpy(S->syn_prefix, S->h_prefix.data(), S->h_prefix.size() * sizeof(int),
                           cudaMemcpyHostToDevice));
  k_oz_syn_fexp<<<nm * 2, 256>>>(p->d_plm, p->d_dplm, p->d_lstart, p->l_max, p->minc, nhs, nthw,
                                 S->syn_fexp);
  k_oz_syn_img<<<nm * 4 * nthtile, 256>>>(p->d_plm, p->d_dplm, p->d_lstart, p->l_max, p->minc,
                                          nhs, nthtile, S->syn_fexp, S->syn, S->syn_off);
  k_oz_ana_fexp<<<nm * 4, 256>>>(p->d_plm, p->d_dplm, p->d_lstart, p->l_max, p->minc, nhs, nlt,
                                 S->ana_fexp);
  k_oz_ana_img<<<nm * 4 * nlt, 256>>>(p->d_plm, p->d_dplm, p->d_lstart, p->l_max, p->minc, nhs,
                                      nlt, S->ana_fexp, S->ana, S->ana_off);
  MT_CHECK_CUDA(cudaGetLastError());
  MT_CHECK_CUDA(cudaDeviceSynchronize());
  S->t.nthtile = nthtile;
  S->t.nlt = nlt;
  S->t.syn = S->syn;
  S->t.syn_off = S->syn_off;
  S->t.syn_fexp = S->syn_fexp;
  S->t.ana = S->ana;
  S->t.ana_off = S->ana_off;
  S->t.ana_fexp = S->ana_fexp;
  S->t.syn_prefix = S->syn_prefix;
  return MT_OK;
}

void free_ozaki_tables(mt_plan* p) {
  OzStore* S = (OzStore*)p->ozaki;
  if (!S) return;
  void* ptrs[] = {S->syn, S->ana, S->syn_off, S->ana_off, S->syn_fexp, S->ana_fexp,
                  S->syn_prefix};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  delete S;
  p->ozaki = nullptr;
}

const OzTables& ozaki_tables(const mt_plan* p) { return ((OzStore*)p->ozaki)->t; }
int ozaki_syn_total_chunks(const mt_plan* p) { return ((OzStore*)p->ozaki)->h_prefix.back(); }

// ------------------------------------------------------------ synthesis

constexpr int kOzPackThreads = 256;

__host__ __device__ inline int oz_stage_pitch(int stg_lev) { return 2 * kOzK * stg_lev + 1; }
__host__ __device__ inline size_t oz_syn_pack_smem(int narr, int stg_lev) {
  return (size_t)narr * oz_stage_pitch(stg_lev) * 16 + 2 * kOzRows * sizeof(int);
}

__host__ __device__ inline int64_t oz_syn_img_chunk(int64_t total_chunks, int rt, int prefix, int c,
                                                    int q) {
  return (((int64_t)rt * total_chunks + prefix + c) * 2 + q);
}

__device__ __forceinline__ double oz_coef(int code, double m) {
  switch (code) {
    case 1: return 1.0;
    case 2: return -1.0;
    case 3: return m;
    case 4: return -m;
    case 5: return -m * m;
    default: return 0.0;
  }
}

__device__ __forceinline__ void cp16_zfill(void* dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_commit_wait_all() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// k_oz_syn_pack: block (row tile rt, order m).  Thread = (table q, parity p,
// row pair): rows 2 pr, 2 pr + 1 are the real and imaginary rows of one field.
// Pass 0 walks every chunk of 2 kOzK values of l - m and finds the largest
// |value| of each (row, combo); pass 1 walks them again and writes the six
// digit planes of every chunk at the row's scale.
__global__ void __launch_bounds__(kOzPackThreads, 2) k_oz_syn_pack(OzSynArgs a) {
  extern __shared__ __align__(128) uint8_t smem[];
  const Tables& t = a.t;
  const int rt = blockIdx.x, mc = blockIdx.y;
  const int m = mc * t.minc;
  const int nlm = t.l_max - m + 1;
  const int ls = t.lstart[mc];
  const int tid = threadIdx.x;
  const int lev0 = (rt * kOzRows) / a.row_per_level;
  const int nlev = min(a.stg_lev, a.n_lev - lev0);
  const int pitch = oz_stage_pitch(a.stg_lev);
  double2* d = reinterpret_cast<double2*>(smem);
  int* rexp_s = reinterpret_cast<int*>(smem + (size_t)a.narr * pitch * 16);  // [combo][row]
  const int qp = tid >> 6, row0 = 2 * (tid & 63);
  const int q = qp >> 1, p = qp & 1;
  const int combo = q == 0 ? p : 1 - p;
  const int nch_all = (nlm + 2 * kOzK - 1) / (2 * kOzK);
  const int nch_combo = oz_syn_nch(nlm, combo);
  const double dm = (double)m;
  struct RowSrc {
    int ia, ib, cpart;
    double f, dl, o2, cw;
    bool live;
  } rs[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int R = rt * kOzRows + row0 + h;
    rs[h].live = R < a.nrows;
    const int lev = rs[h].live ? R / a.row_per_level : lev0;
    const int qf = rs[h].live ? R - lev * a.row_per_level : 0;
    const RowOp op = a.ops[qf];
    const TermIx tm = a.term[q ? op.tD : op.tP];
    rs[h].cpart = q ? op.cD : op.cP;
    rs[h].f = rs[h].live ? oz_coef(q ? op.kD : op.kP, dm) : 0.0;
    rs[h].dl = tm.recipe == kRaw ? 0.0 : 1.0;
    rs[h].o2 = (tm.recipe == kCurlT && a.or2) ? a.or2[lev] : 1.0;
    rs[h].cw = tm.recipe == kCurlT ? 1.0 : 0.0;
    rs[h].ia = tm.ia * pitch + (lev - lev0);
    rs[h].ib = tm.ib * pitch + (lev - lev0);
  }
  // value of row h at the i-th l - m of parity p in chunk c (staged)
  auto value = [&](int h, int c, int i) -> double {
    const int kk = 2 * i + p;  // l - m offset inside the staged chunk
    const double l = (double)(m + 2 * kOzK * c + kk);
    const double2 x = d[rs[h].ia + kk * a.stg_lev];
    const double2 w = rs[h].cw != 0.0 ? d[rs[h].ib + kk * a.stg_lev] : make_double2(0.0, 0.0);
    const double mul = rs[h].o2 * (1.0 + rs[h].dl * (l * (l + 1.0) - 1.0));
    const double xa = rs[h].cpart ? x.y : x.x, xb = rs[h].cpart ? w.y : w.x;
    return rs[h].f * (mul * xa - rs[h].cw * xb);
  };
  auto stage = [&](int c) {
    __syncthreads();  // the staging buffer is free
    for (int e = tid; e < 2 * kOzK * a.stg_lev; e += kOzPackThreads) {
      const int kk = e / a.stg_lev, lvv = e - kk * a.stg_lev;
      if (lvv >= nlev) continue;
      const int k = 2 * kOzK * c + kk;
      const int64_t off = (int64_t)(ls + min(k, nlm - 1)) * a.ld + lev0 + lvv;
      const uint32_t bytes = k < nlm ? 16u : 0u;
      for (int ia = 0; ia < a.narr; ++ia)
        cp16_zfill(&d[ia * pitch + kk * a.stg_lev + lvv], a.arr[ia] + off, bytes);
    }
    cp_commit_wait_all();
    __syncthreads();
  };
  // pass 0: row maxima per combo; each (row, combo) gets contributions from
  // two threads (P of one parity, dP of the other), merged through shared memory
  double mx[2] = {0.0, 0.0};
  for (int c = 0; c < nch_all; ++c) {
    stage(c);
#pragma unroll 4
    for (int i = 0; i < kOzK; ++i) {
      mx[0] = fmax(mx[0], fabs(value(0, c, i)));
      mx[1] = fmax(mx[1], fabs(value(1, c, i)));
    }
  }
  unsigned long long* rmax = reinterpret_cast<unsigned long long*>(smem);  // reuses staging
  __syncthreads();
  for (int e = tid; e < 2 * kOzRows; e += kOzPackThreads) rmax[e] = 0ull;
  __syncthreads();
#pragma unroll
  for (int h = 0; h < 2; ++h)
    atomicMax(&rmax[combo * kOzRows + row0 + h], (unsigned long long)__double_as_longlong(mx[h]));
  __syncthreads();
  for (int e = tid; e < 2 * kOzRows; e += kOzPackThreads) {
    const int e_ = oz_exponent(__longlong_as_double((long long)rmax[e]));
    rexp_s[e] = e_;
    const int cb = e / kOzRows, row = e % kOzRows;
    a.rexp[((int64_t)mc * 2 + cb) * a.rows_pad + (int64_t)rt * kOzRows + row] = e_;
  }
  __syncthreads();
  const int ex[2] = {rexp_s[combo * kOzRows + row0], rexp_s[combo * kOzRows + row0 + 1]};
  // pass 1: digit planes
  for (int c = 0; c < nch_all; ++c) {
    stage(c);
    if (c >= nch_combo) continue;
    uint8_t* dst = a.aimg + oz_syn_img_chunk(a.total_chunks, rt,
                                             a.z.syn_prefix[mc * 2 + combo], c, q) * kOzAChunk;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
#pragma unroll 1
      for (int half = 0; half < 2; ++half) {
        uint32_t w[4][kOzDigits];
#pragma unroll
        for (int i4 = 0; i4 < 4; ++i4) {
          double v4[4];
#pragma unroll
          for (int b = 0; b < 4; ++b) v4[b] = value(h, c, 16 * half + 4 * i4 + b);
          oz_digit_words(v4, ex[h], w[i4]);
        }
#pragma unroll
        for (int s = 0; s < kOzDigits; ++s)
          *reinterpret_cast<uint4*>(dst + s * kOzAPlane + oz_off(row0 + h, 16 * half)) =
              make_uint4(w[0][s], w[1][s], w[2][s], w[3][s]);
      }
    }
  }
}

constexpr int kOzStages = 4;     // analysis ring
// Synthesis: one CTA per SM, six accumulator groups of kOzSynN = 64 columns
// (384 of 512 TMEM columns), a 4-stage ring, and a shared-memory stash that
// holds an item's symmetric half until its antisymmetric half is formed, so
// that the epilogue writes the north (sym + asym) and south (sym - asym) rows.
constexpr int kOzSynStages = 4;
constexpr int kOzSynEpiWarps = 16;  // four per TMEM lane quarter, 16 columns each
constexpr int kOzSynEpiCols = kOzSynN / (kOzSynEpiWarps / 4);
constexpr int kOzSynThreads = 64 + 32 * kOzSynEpiWarps;
constexpr int kOzSynTmemCols = 512;

struct OzSynSmem {
  static constexpr uint32_t stage_bytes = kOzAChunk + kOzSynBChunk;
  static constexpr uint32_t stash_off = kOzSynStages * stage_bytes;
  static constexpr uint32_t stash_bytes = kOzRows * kOzSynN * 8;  // [column][row] doubles
  static constexpr uint32_t bar_off = stash_off + stash_bytes;
  // full/empty per stage, tfull, tempty, done, tmem slot, abort flag
  static constexpr size_t total = bar_off + 8 * (2 * kOzSynStages + 3) + 16;
};

// Persistent synthesis GEMM: one CTA per SM walks the items (tile, theta tile,
// m) with a stride of gridDim.x; an item is two accumulations, the symmetric
// (combo 0: P of even l - m, dP of odd) and the antisymmetric (combo 1) half.
// Warp 0 lane 0 bulk-copies the A digit chunk and the table digit chunk of
// every K step into the ring, warp 1 lane 0 issues the MMAs of every step
// (oz_mma_chunk: eight MMAs covering the 21 digit pairs) into the six group
// accumulators (TMEM columns 64 g) and commits at the end of each half, warps
// 2-9 drain the accumulators (one TMEM lane and 32 columns per thread): the
// symmetric half into the stash, then with the antisymmetric half the north
// and south rows into Fs, handing the accumulators back after each half.
__global__ void __launch_bounds__(kOzSynThreads, 1) k_oz_synth_gemm(OzSynArgs a) {
  extern __shared__ __align__(128) uint8_t smem[];
  const Tables& t = a.t;
  const OzTables& z = a.z;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + OzSynSmem::bar_off);
  uint64_t* empty = full + kOzSynStages;
  uint64_t* tfull = empty + kOzSynStages;
  uint64_t* tempty = tfull + 1;
  uint64_t* done = tempty + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  double* stash = reinterpret_cast<double*>(smem + OzSynSmem::stash_off);

  if (*(volatile int*)a.err) return;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ntiles = (a.nrows + kOzRows - 1) / kOzRows;
  const int nitems = ntiles * z.nthtile * t.n_m;
  const int nthw = z.nthtile * kOzSynN;
  struct Item {
    int rt, tau, mc, nlm;
  };
  auto decode = [&](int item) {
    Item it;
    it.rt = item % ntiles;
    const int r = item / ntiles;
    it.tau = r % z.nthtile;
    it.mc = r / z.nthtile;
    it.nlm = t.l_max - it.mc * t.minc + 1;
    return it;
  };
  // K chunks of the table of kind q (0: P, 1: dP) in half `combo` of an item
  auto nch_of = [&](const Item& it, int combo, int q) {
    return (split_nk(it.nlm, q ? 1 - combo : combo) + kOzK - 1) / kOzK;
  };

  if (tid == 0) {
    for (int s = 0; s < kOzSynStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(tfull, 1);
    mbar_init(tempty, 32 * kOzSynEpiWarps);
    mbar_init(done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 1) tmem_alloc(tmem_slot, kOzSynTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      int g = 0;
      bool ok = true;
      for (int item = blockIdx.x; item < nitems && ok; item += gridDim.x) {
        const Item it = decode(item);
        for (int combo = 0; combo < 2 && ok; ++combo) {
          const uint8_t* aimg =
              a.aimg + oz_syn_img_chunk(a.total_chunks, it.rt, z.syn_prefix[it.mc * 2 + combo],
                                        0, 0) * kOzAChunk;
          const int8_t* img[2];
          for (int q = 0; q < 2; ++q)
            img[q] = z.syn + z.syn_off[((it.mc * 2 + q) * 2 + (q ? 1 - combo : combo)) *
                                           z.nthtile + it.tau];
          const int nq[2] = {nch_of(it, combo, 0), nch_of(it, combo, 1)};
          const int nch = max(nq[0], nq[1]);
          for (int c = 0; c < nch && ok; ++c) {
            for (int q = 0; q < 2; ++q) {
              if (c >= nq[q]) continue;
              const int s = g % kOzSynStages;
              if (g >= kOzSynStages &&
                  !mbar_wait(&empty[s], ((g / kOzSynStages) - 1) & 1, abort_flag, a.err, 23)) {
                ok = false;
                break;
              }
              uint8_t* stg = smem + s * OzSynSmem::stage_bytes;
              mbar_expect_tx(&full[s], OzSynSmem::stage_bytes);
              bulk_g2s(stg, aimg + (int64_t)(2 * c + q) * kOzAChunk, kOzAChunk, &full[s]);
              bulk_g2s(stg + kOzAChunk, img[q] + (int64_t)c * kOzSynBChunk, kOzSynBChunk,
                       &full[s]);
              ++g;
            }
          }
        }
      }
      for (int k = max(0, g - kOzSynStages); k < g; ++k)
        mbar_drain(&full[k % kOzSynStages], (k / kOzSynStages) & 1);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int g = 0, n = 0;
      bool ok = true;
      for (int item = blockIdx.x; item < nitems && ok; item += gridDim.x) {
        const Item it = decode(item);
        for (int combo = 0; combo < 2 && ok; ++combo, ++n) {
          if (n >= 1 && !mbar_wait(tempty, (n - 1) & 1, abort_flag, a.err, 26)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const int nq[2] = {nch_of(it, combo, 0), nch_of(it, combo, 1)};
          const int nch = max(nq[0], nq[1]);
          bool first = true;
          for (int c = 0; c < nch && ok; ++c) {
            for (int q = 0; q < 2; ++q) {
              if (c >= nq[q]) continue;
              const int s = g % kOzSynStages;
              if (!mbar_wait(&full[s], (g / kOzSynStages) & 1, abort_flag, a.err, 24)) {
                ok = false;
                break;
              }
              tc_fence_after();
              const uint32_t sa = smem_u32(smem + s * OzSynSmem::stage_bytes);
              oz_mma_chunk<kOzSynN>(tbase, sa, sa + kOzAChunk, first);
              first = false;
              umma_commit(&empty[s]);
              ++g;
            }
          }
          if (ok) umma_commit(tfull);
        }
      }
      umma_commit(done);
    }
  } else {
    // epilogue: warps 2 .. 2 + kOzSynEpiWarps - 1; warp w owns TMEM lane
    // quarter w % 4 and the kOzSynEpiCols accumulator columns of slice (w - 2) / 4
    const int quarter = warp & 3, half = (warp - 2) >> 2;
    const int R0 = quarter * 32 + lane;
    int n = 0;
    bool live = true;
    for (int item = blockIdx.x; item < nitems && live; item += gridDim.x) {
      const Item it = decode(item);
      const int R = it.rt * kOzRows + R0;
      double* north = a.Fs + (int64_t)it.mc * a.fs_m;
      double* south = north + a.fs_c;
      for (int combo = 0; combo < 2; ++combo, ++n) {
        // the row and column exponents do not depend on the MMAs: their loads
        // are issued before the wait for the accumulators
        const int er =
            R < a.nrows ? a.rexp[((int64_t)it.mc * 2 + combo) * a.rows_pad + R] : 0;
        // column exponents of this warp's columns, one per lane, shared by shuffles
        const int fe_l = __ldg(z.syn_fexp + ((int64_t)it.mc * 2 + combo) * nthw +
                               it.tau * kOzSynN + kOzSynEpiCols * half +
                               (lane % kOzSynEpiCols));
        const bool ok = mbar_wait(tfull, n & 1, abort_flag, a.err, 22);
        if (!__all_sync(0xffffffffu, ok && !*abort_flag)) {
          live = false;
          break;
        }
        tc_fence_after();
        const uint32_t taddr =
            tbase + ((uint32_t)(32 * quarter) << 16) + kOzSynEpiCols * half;
#pragma unroll 1
        for (int c0 = 0; c0 < kOzSynEpiCols; c0 += 8) {
          uint32_t cg[kOzGroups][8];
#pragma unroll
          for (int g = 0; g < kOzGroups; ++g)
            tmem_ld8_i32_nowait(taddr + g * kOzSynN + c0, cg[g]);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const int fe = __shfl_sync(0xffffffffu, fe_l, c0 + i);
            const int col = kOzSynEpiCols * half + c0 + i;
            const double v = oz_scale(oz_combine_u(cg, i), er + fe - 12 - 35);
            double* st = stash + col * kOzRows + R0;  // this thread's own entry
            if (combo == 0) {
              *st = v;
            } else {
              const int th = it.tau * kOzSynN + col;
              if (R < a.nrows && th < t.nhs) {
                const double sy = *st;
                north[(int64_t)th * a.fs_j + R] = sy + v;
                south[(int64_t)th * a.fs_j + R] = sy - v;
              }
            }
          }
        }
        tc_fence_before();
        mbar_arrive(tempty);
      }
    }
  }
  __syncwarp();
  if (warp == 1) mbar_drain(done, 0);  // no MMA may still write TMEM at dealloc
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tbase, kOzSynTmemCols);
  }
}

size_t oz_syn_image_bytes(int nrows, int64_t total_chunks) {
  return (size_t)((nrows + kOzRows - 1) / kOzRows) * (size_t)total_chunks * 2 * kOzAChunk;
}

int launch_oz_synth(const OzSynArgs& a, cudaStream_t st) {
  const int ntiles = (a.nrows + kOzRows - 1) / kOzRows;
  const size_t pack_sm = std::max(oz_syn_pack_smem(a.narr, a.stg_lev),
                                  (size_t)2 * kOzRows * 8 + 2 * kOzRows * sizeof(int));
  MT_REQUIRE(pack_sm <= 220 * 1024, MT_ERR_UNSUPPORTED, "digit pack staging too large");
  MT_CHECK_CUDA(cudaFuncSetAttribute(k_oz_syn_pack, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)pack_sm));
  k_oz_syn_pack<<<dim3(ntiles, a.t.n_m), kOzPackThreads, pack_sm, st>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  const size_t sm = OzSynSmem::total;
  MT_CHECK_CUDA(cudaFuncSetAttribute(k_oz_synth_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sm));
  int dev = 0, nsm = 148;
  MT_CHECK_CUDA(cudaGetDevice(&dev));
  MT_CHECK_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int nitems = ntiles * a.z.nthtile * a.t.n_m;
  k_oz_synth_gemm<<<std::min(nitems, nsm), kOzSynThreads, sm, st>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

// -------------------------------------------------------------- analysis
//
// k_oz_ana_pack<RB>: block (RB rows of tile rt, order m).  The block's raw
// Fourier values (north and south, every theta pair) are read from HBM once
// into shared memory, [hemisphere][theta pair][row]; each row then yields
// both folds, fold 0 north + south and fold 1 north - south: pass 0 finds
// each (row, fold)'s largest |value| over all theta pairs, pass 1 writes the
// digit planes of every chunk of kOzK pairs from shared memory.
// k_oz_anal_gemm (persistent; item = tile, output parity, l tile, m)
// accumulates acc0 = fold_par . P and acc1 = fold_(1-par) . dP in six groups
// each, and its epilogue forms each output component as
// coef(kP) acc0[colP] + coef(kD) acc1[colD] (the row program) through an
// FP64 exchange buffer in shared memory.

__host__ __device__ inline int64_t oz_ana_img_chunk(int n_m, int nchj, int rt, int mc, int fold,
                                                    int c) {
  return (((int64_t)rt * n_m + mc) * 2 + fold) * nchj + c;
}

// rows per analysis-pack block: the largest of 32, 16, 8 whose staging buffer
// (2 x nhs x RB doubles) lets two blocks share an SM
inline int oz_ana_pack_rows(int nhs) {
  for (int rb = 32; rb > 8; rb >>= 1)
    if ((size_t)2 * nhs * rb * 8 <= 110 * 1024) return rb;
  return 8;
}
inline size_t oz_ana_pack_smem(int nhs, int rb) {
  return (size_t)2 * nhs * rb * 8 + (size_t)2 * (kOzPackThreads + rb) * 8;
}

template <int RB>
__global__ void __launch_bounds__(kOzPackThreads, 2) k_oz_ana_pack(OzAnaArgs a) {
  extern __shared__ __align__(16) double stg[];  // [hemisphere][theta pair][row]
  constexpr int NG = kOzPackThreads / RB;        // theta-pair groups of the load pass
  const Tables& t = a.t;
  const int nhs = t.nhs;
  const int rt = blockIdx.x / (kOzRows / RB), rq = blockIdx.x % (kOzRows / RB);
  const int mc = blockIdx.y;
  const int nchj = (nhs + kOzK - 1) / kOzK;
  const int tid = threadIdx.x;
  double* red = stg + (size_t)2 * nhs * RB;  // [fold][group][row] partial maxima
  double* exs = red + 2 * kOzPackThreads;    // [fold][row] exponents (as doubles)
  const int lev0 = rt * a.lev_tile;
  const int nlev = min(a.lev_tile, a.n_lev - lev0);
  // load pass: thread (row rr, group g) reads theta pairs g, g + NG, ...;
  // consecutive threads read consecutive rows of one theta pair
  {
    const int rr = tid % RB, g = tid / RB;
    const int R = rq * RB + rr, lv = R / a.cols, col = R - lv * a.cols;
    const bool live = lv < nlev;
    const double* nb = a.G + (int64_t)mc * a.g_m + (int64_t)(lev0 + (live ? lv : 0)) * a.g_level +
                       col;
    double m0 = 0.0, m1 = 0.0;
    constexpr int kB = 8;
    for (int j0 = g; j0 < nhs; j0 += kB * NG) {
      double vn[kB], vs[kB];
#pragma unroll
      for (int u = 0; u < kB; ++u) {
        const int j = j0 + u * NG;
        vn[u] = vs[u] = 0.0;
        if (live && j < nhs) {
          vn[u] = __ldg(nb + (int64_t)j * a.g_j);
          vs[u] = __ldg(nb + a.g_h + (int64_t)j * a.g_j);
        }
      }
#pragma unroll
      for (int u = 0; u < kB; ++u) {
        const int j = j0 + u * NG;
        if (j < nhs) {
          stg[(size_t)j * RB + rr] = vn[u];
          stg[(size_t)(nhs + j) * RB + rr] = vs[u];
        }
        m0 = fmax(m0, fabs(vn[u] + vs[u]));
        m1 = fmax(m1, fabs(vn[u] - vs[u]));
      }
    }
    red[g * RB + rr] = m0;
    red[(NG + g) * RB + rr] = m1;
  }
  __syncthreads();
  if (tid < 2 * RB) {
    const int fold = tid / RB, rr = tid % RB;
    double mx = 0.0;
    for (int g = 0; g < NG; ++g) mx = fmax(mx, red[(fold * NG + g) * RB + rr]);
    const int ex = oz_exponent(mx);
    exs[tid] = (double)ex;
    a.rexp[((int64_t)mc * 2 + fold) * a.rows_pad + (int64_t)rt * kOzRows + rq * RB + rr] = ex;
  }
  __syncthreads();
  // digit pass: task (row rr, fold, half chunk hc of 16 theta pairs)
  const int ntask = RB * 2 * 2 * nchj;
  for (int task = tid; task < ntask; task += kOzPackThreads) {
    const int rr = task % RB, rest = task / RB;
    const int fold = rest & 1, hc = rest >> 1;
    const double sg = fold ? -1.0 : 1.0;
    const int ex = (int)exs[fold * RB + rr];
    uint32_t w[4][kOzDigits];
#pragma unroll
    for (int i4 = 0; i4 < 4; ++i4) {
      double v4[4];
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int j = 16 * hc + 4 * i4 + b;
        v4[b] = j < nhs ? stg[(size_t)j * RB + rr] + sg * stg[(size_t)(nhs + j) * RB + rr] : 0.0;
      }
      oz_digit_words(v4, ex, w[i4]);
    }
    uint8_t* dst =
        a.aimg + oz_ana_img_chunk(t.n_m, nchj, rt, mc, fold, hc >> 1) * kOzAChunk;
#pragma unroll
    for (int s = 0; s < kOzDigits; ++s)
      *reinterpret_cast<uint4*>(dst + s * kOzAPlane + oz_off(rq * RB + rr, 16 * (hc & 1))) =
          make_uint4(w[0][s], w[1][s], w[2][s], w[3][s]);
  }
}

constexpr int kOzAnaEpiWarps = 16;  // four per TMEM lane quarter: (table kind, 16 columns)
constexpr int kOzAnaEpiThreads = 32 * kOzAnaEpiWarps;
constexpr int kOzAnaThreads = 64 + kOzAnaEpiThreads;
constexpr int kOzXS = kOzAnaN + 1;  // padded exchange row (doubles)

struct OzAnaSmem {
  static constexpr uint32_t stage_bytes = kOzAChunk + kOzAnaBChunk;
  static constexpr uint32_t xch_off = kOzStages * stage_bytes;
  static constexpr uint32_t xch_bytes = 2 * kOzRows * kOzXS * 8;
  static constexpr uint32_t tab_off = xch_off + xch_bytes;  // row-program tables
  static constexpr uint32_t tab_bytes = 64 * 8 + 64 * 4 + kOzAnaN * 8 + 16;
  static constexpr uint32_t bar_off = (tab_off + tab_bytes + 15) & ~15u;
  static constexpr size_t total = bar_off + 8 * (2 * kOzStages + 3) + 16;
};

__global__ void __launch_bounds__(kOzAnaThreads, 1) k_oz_anal_gemm(OzAnaArgs a) {
  extern __shared__ __align__(128) uint8_t smem[];
  const Tables& t = a.t;
  const OzTables& z = a.z;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + OzAnaSmem::bar_off);
  uint64_t* empty = full + kOzStages;
  uint64_t* tfull = empty + kOzStages;
  uint64_t* tempty = tfull + 1;
  uint64_t* done = tempty + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  if (*(volatile int*)a.err) return;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nchj = (t.nhs + kOzK - 1) / kOzK;
  const int ntiles = (a.n_lev + a.lev_tile - 1) / a.lev_tile;
  const int ny = 2 * z.nlt;
  const int nitems = ntiles * ny * t.n_m;
  struct Item {
    int rt, par, lt, mc, nk;
    bool live;
  };
  auto decode = [&](int item) {
    Item it;
    it.rt = item % ntiles;
    const int r = item / ntiles, y = r % ny;
    it.mc = r / ny;
    it.par = y & 1;
    it.lt = y >> 1;
    const int nlm = t.l_max - it.mc * t.minc + 1;
    it.nk = split_nk(nlm, it.par);
    it.live = it.lt * kOzAnaN < it.nk;
    return it;
  };

  if (tid == 0) {
    for (int s = 0; s < kOzStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(tfull, 1);
    mbar_init(tempty, kOzAnaEpiThreads);
    mbar_init(done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 1) tmem_alloc(tmem_slot, 512);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      int g = 0;
      bool ok = true;
      for (int item = blockIdx.x; item < nitems && ok; item += gridDim.x) {
        const Item it = decode(item);
        if (!it.live) continue;
        const uint8_t* aimg[2];
        const int8_t* img[2];
        for (int q = 0; q < 2; ++q) {
          const int fold = q ? 1 - it.par : it.par;
          aimg[q] = a.aimg + oz_ana_img_chunk(t.n_m, nchj, it.rt, it.mc, fold, 0) * kOzAChunk;
          img[q] = z.ana + z.ana_off[((it.mc * 2 + q) * 2 + it.par) * z.nlt + it.lt];
        }
        for (int c = 0; c < nchj && ok; ++c) {
          for (int q = 0; q < 2; ++q) {
            const int s = g % kOzStages;
            if (g >= kOzStages &&
                !mbar_wait(&empty[s], ((g / kOzStages) - 1) & 1, abort_flag, a.err, 33)) {
              ok = false;
              break;
            }
            uint8_t* stg = smem + s * OzAnaSmem::stage_bytes;
            mbar_expect_tx(&full[s], OzAnaSmem::stage_bytes);
            bulk_g2s(stg, aimg[q] + (int64_t)c * kOzAChunk, kOzAChunk, &full[s]);
            bulk_g2s(stg + kOzAChunk, img[q] + (int64_t)c * kOzAnaBChunk, kOzAnaBChunk, &full[s]);
            ++g;
          }
        }
      }
      for (int k = max(0, g - kOzStages); k < g; ++k)
        mbar_drain(&full[k % kOzStages], (k / kOzStages) & 1);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int g = 0, n = 0;
      bool ok = true;
      for (int item = blockIdx.x; item < nitems && ok; item += gridDim.x) {
        const Item it = decode(item);
        if (!it.live) continue;
        if (n >= 1 && !mbar_wait(tempty, (n - 1) & 1, abort_flag, a.err, 36)) break;
        tc_fence_after();
        for (int c = 0; c < nchj && ok; ++c) {
          for (int q = 0; q < 2; ++q) {
            const int s = g % kOzStages;
            if (!mbar_wait(&full[s], (g / kOzStages) & 1, abort_flag, a.err, 34)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t sa = smem_u32(smem + s * OzAnaSmem::stage_bytes);
            oz_mma_chunk<kOzAnaN>(tbase + (uint32_t)(q * kOzGroups * kOzAnaN), sa,
                                  sa + kOzAChunk, c == 0);
            umma_commit(&empty[s]);
            ++g;
          }
        }
        if (ok) umma_commit(tfull);
        ++n;
      }
      umma_commit(done);
    }
  } else {
    // epilogue: warps 2 .. 2 + kOzAnaEpiWarps - 1, thread e = tid - 64; warp w
    // owns TMEM lane quarter w % 4 (R0 = 32 (w % 4) + lane) and, for slice
    // sl = (w - 2) / 4, the 16 columns 16 (sl & 1) .. of table kind q = sl / 2
    const int e = tid - 64;
    const int quarter = warp & 3, sl = (warp - 2) >> 2;
    const int qs = sl >> 1, cs = 16 * (sl & 1);
    const int R0 = quarter * 32 + lane;
    const int lv_e = e % a.lev_tile, rest_e = e / a.lev_tile;
    const int ddq = kOzAnaEpiThreads / a.lev_tile, ddr = kOzAnaEpiThreads - ddq * a.lev_tile;
    double* xch = reinterpret_cast<double*>(smem + OzAnaSmem::xch_off);  // [2][128][kOzXS]
    double* cf = reinterpret_cast<double*>(smem + OzAnaSmem::tab_off);   // [64]
    int* colx = reinterpret_cast<int*>(cf + 64);                        // [64]
    double* osc = reinterpret_cast<double*>(colx + 64);                 // [kOzAnaN]
    int n = 0;
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
      const Item it = decode(item);
      if (!it.live) continue;
      // the row exponent and this warp's 16 column exponents (one per lane,
      // shared by shuffles), loaded before the wait for the accumulators
      // (they do not depend on the MMAs)
      const int Rg = it.rt * kOzRows + R0;
      const int fold = qs ? 1 - it.par : it.par;
      const int er = a.rexp[((int64_t)it.mc * 2 + fold) * a.rows_pad + Rg];
      const int fe_l = __ldg(z.ana_fexp +
                             ((int64_t)(it.mc * 2 + qs) * 2 + it.par) * z.nlt * kOzAnaN +
                             it.lt * kOzAnaN + cs + (lane & 15));
      const bool ok = mbar_wait(tfull, n & 1, abort_flag, a.err, 32);
      ++n;
      // all epilogue warps agree, since they meet at named barriers below
      if (!bar_and(1, kOzAnaEpiThreads, ok && !*abort_flag)) break;
      tc_fence_after();
      const int m = it.mc * t.minc;
      const int nlm = t.l_max - m + 1;
      const int ls = t.lstart[it.mc];
      const uint32_t taddr = tbase + ((uint32_t)(32 * quarter) << 16);
#pragma unroll 1
      for (int c0 = 0; c0 < 16; c0 += 8) {
        uint32_t cg[kOzGroups][8];
#pragma unroll
        for (int g = 0; g < kOzGroups; ++g)
          tmem_ld8_i32_nowait(taddr + (uint32_t)((qs * kOzGroups + g) * kOzAnaN + cs + c0), cg[g]);
        tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int fe = __shfl_sync(0xffffffffu, fe_l, c0 + i);
          xch[(qs * kOzRows + R0) * kOzXS + cs + c0 + i] =
              oz_scale(oz_combine_u(cg, i), er + fe - 12 - 35);
        }
      }
      tc_fence_before();
      mbar_arrive(tempty);  // the accumulators are free for the next item's MMAs
      // row-program tables of this item
      const double dm = (double)m;
      for (int r = e; r < 2 * a.n_out; r += kOzAnaEpiThreads) {
        const RowOp op = a.ops[r];
        cf[2 * r] = oz_coef(op.kP, dm);
        cf[2 * r + 1] = oz_coef(op.kD, dm);
        colx[2 * r] = 2 * op.tP + op.cP;
        colx[2 * r + 1] = kOzRows + 2 * op.tD + op.cD;
      }
      for (int i = e; i < kOzAnaN; i += kOzAnaEpiThreads) {
        const double l = (double)(m + 2 * (it.lt * kOzAnaN + i) + it.par);
        osc[i] = l > 0.0 ? 1.0 / (l * (l + 1.0)) : 0.0;
      }
      named_bar_sync(1, kOzAnaEpiThreads);
      const int lev0 = it.rt * a.lev_tile;
      const int nlev = min(a.lev_tile, a.n_lev - lev0);
      const int nel = a.n_out * a.lev_tile * kOzAnaN;
      // x = lv + lev_tile (i + kOzAnaN o) advances by the thread count: (lv,
      // rest) step by (ddr, ddq) with a carry, no division in the loop
      int lv = lv_e, rest = rest_e;
      for (int x = e; x < nel; x += kOzAnaEpiThreads) {
        const int i = rest % kOzAnaN, o = rest / kOzAnaN;
        const int lv_x = lv;
        lv += ddr;
        rest += ddq;
        if (lv >= a.lev_tile) {
          lv -= a.lev_tile;
          ++rest;
        }
        const int kk = it.lt * kOzAnaN + i, k = 2 * kk + it.par;
        if (lv_x >= nlev || kk >= it.nk || k >= nlm) continue;
        const int base = lv_x * a.cols;
        const int r4 = 4 * o;
        const double re = cf[r4] * xch[(base + colx[r4]) * kOzXS + i] +
                          cf[r4 + 1] * xch[(base + colx[r4 + 1]) * kOzXS + i];
        const double im = cf[r4 + 2] * xch[(base + colx[r4 + 2]) * kOzXS + i] +
                          cf[r4 + 3] * xch[(base + colx[r4 + 3]) * kOzXS + i];
        const double sc = a.ops[2 * o].scale ? osc[i] : 1.0;
        a.out[o][(int64_t)(ls + k) * a.ld + a.out_col0 + lev0 + lv_x] =
            make_double2(sc * re, sc * im);
      }
      named_bar_sync(1, kOzAnaEpiThreads);  // exchange buffer free again
    }
  }
  __syncwarp();
  if (warp == 1) mbar_drain(done, 0);
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tbase, 512);
  }
}

size_t oz_ana_image_bytes(int n_m, int nhs, int n_lev, int lev_tile) {
  const int ntiles = (n_lev + lev_tile - 1) / lev_tile;
  return (size_t)ntiles * n_m * 2 * ((nhs + kOzK - 1) / kOzK) * kOzAChunk;
}

int launch_oz_anal(const OzAnaArgs& a, cudaStream_t st) {
  const int ntiles = (a.n_lev + a.lev_tile - 1) / a.lev_tile;
  MT_REQUIRE(a.cols * a.lev_tile <= kOzRows && a.g_level % 2 == 0, MT_ERR_ARG,
             "analysis tile layout");
  const int rb = oz_ana_pack_rows(a.t.nhs);
  const size_t psm = oz_ana_pack_smem(a.t.nhs, rb);
  auto pack = rb == 32 ? k_oz_ana_pack<32> : rb == 16 ? k_oz_ana_pack<16> : k_oz_ana_pack<8>;
  MT_CHECK_CUDA(cudaFuncSetAttribute(pack, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psm));
  pack<<<dim3(ntiles * (kOzRows / rb), a.t.n_m), kOzPackThreads, psm, st>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  const size_t sm = OzAnaSmem::total;
  MT_CHECK_CUDA(cudaFuncSetAttribute(k_oz_anal_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sm));
  int dev = 0, nsm = 148;
  MT_CHECK_CUDA(cudaGetDevice(&dev));
  MT_CHECK_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int nitems = ntiles * 2 * a.z.nlt * a.t.n_m;
  k_oz_anal_gemm<<<std::min(nitems, nsm), kOzAnaThreads, sm, st>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

}  // namespace mt
