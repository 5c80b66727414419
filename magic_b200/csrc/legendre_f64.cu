// FP64 Legendre contractions on the FP64 tensor pipe (mma.sync m8n8k4 f64).
//
// Synthesis, per order m (grid z), 32 northern theta (grid y) and R columns
// (grid x, fastest so that consecutive CTAs reuse the same table tile in L2):
//   K loop over l in chunks of 16 rows (8 even + 8 odd l-m), register
//   prefetch of the next chunk; every warp owns one 8-row theta tile and
//   R/8 column tiles and accumulates BOTH parities of EVERY product of the
//   operation, so the north/south unfolding and the product combination
//   happen in registers.
// Analysis, per order m, 64 rows l (8 warps = 8 row tiles of one parity
// each) and R columns: K loop over theta pairs in chunks of 16; the B
// operand is folded on load (north +/- south) according to the row parity
// and the table parity.
#include "legendre.cuh"

namespace mt {

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

__device__ __forceinline__ double2 load_term(const TermSrc& s, int64_t row, int64_t ld, int col,
                                             double dlh, const double* or2) {
  int64_t o = row * ld + col;
  switch (s.recipe) {
    case kRaw: return __ldg(&s.a[o]);
    case kDlh: {
      double2 v = __ldg(&s.a[o]);
      return make_double2(dlh * v.x, dlh * v.y);
    }
    case kCurlT: {
      double2 v = __ldg(&s.a[o]);
      double2 w = __ldg(&s.b[o]);
      double f = __ldg(&or2[col]) * dlh;
      return make_double2(f * v.x - w.x, f * v.y - w.y);
    }
    default: return make_double2(0.0, 0.0);
  }
}

template <class OP, int R>
struct SynthCfg {
  static constexpr int TH = 32, KC = 16;
  static constexpr int SA = 36;         // sA row stride (doubles): 16*SA = 64 mod 128 B
  static constexpr int SB = 2 * R + 4;  // sB row stride (doubles)
  static constexpr int WC = R / 8;      // column tiles per warp
  static constexpr int NA = OP::NT * KC * TH / 256;                 // A elems / thread
  static constexpr int NB = (OP::NX * KC * R + 255) / 256;          // B elems / thread
  static constexpr size_t smem = (size_t)(OP::NT * KC * SA + OP::NX * KC * SB) * 8;
};

template <class OP, int R>
__global__ void __launch_bounds__(256, 2) k_synth_f64(SynthArgs<OP::NX> a) {
  using C = SynthCfg<OP, R>;
  constexpr int NX = OP::NX, NP = OP::NP, NT = OP::NT, NO = OP::NO;
  constexpr int TH = C::TH, KC = C::KC, SA = C::SA, SB = C::SB, WC = C::WC;
  extern __shared__ double smem[];
  double* sA = smem;                 // [NT][KC][SA]
  double* sB = smem + NT * KC * SA;  // [NX][KC][SB]

  const Tables& t = a.t;
  const int c0 = blockIdx.x * R;
  const int th0 = blockIdx.y * TH;
  const int mc = blockIdx.z;
  const int m = mc * t.minc;
  const int nlm = t.l_max - m + 1;
  const int ls = t.lstart[mc];
  const int nhs = t.nhs;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t4 = lane & 3;
  const int rt = warp & 3, ctg = warp >> 2;

  double ra[C::NA];
  double2 rb[C::NB];
  auto load = [&](int k0) {
#pragma unroll
    for (int i = 0; i < C::NA; ++i) {
      int e = tid + 256 * i;
      int tb = e / (KC * TH), r = e % (KC * TH);
      int kk = r / TH, jj = r % TH;
      int k = k0 + kk, th = th0 + jj;
      const double* T = (NT == 2) ? (tb == 0 ? t.plm : t.dplm)
                                  : (OP::table(0) == kP ? t.plm : t.dplm);
      ra[i] = (k < nlm && th < nhs) ? __ldg(&T[(int64_t)(ls + k) * nhs + th]) : 0.0;
    }
#pragma unroll
    for (int i = 0; i < C::NB; ++i) {
      int e = tid + 256 * i;
      double2 v = make_double2(0.0, 0.0);
      if (e < NX * KC * R) {
        int x = e / (KC * R), r = e % (KC * R);
        int kk = r / R, cc = r % R;
        int k = k0 + kk, col = c0 + cc;
        if (k < nlm && col < a.ncols) {
          double l = (double)(m + k);
          v = load_term(a.src[x], ls + k, a.ld, col, l * (l + 1.0), a.or2);
        }
      }
      rb[i] = v;
    }
  };
  auto store = [&]() {
#pragma unroll
    for (int i = 0; i < C::NA; ++i) {
      int e = tid + 256 * i;
      int tb = e / (KC * TH), r = e % (KC * TH);
      sA[(tb * KC + r / TH) * SA + r % TH] = ra[i];
    }
#pragma unroll
    for (int i = 0; i < C::NB; ++i) {
      int e = tid + 256 * i;
      if (e < NX * KC * R) {
        int x = e / (KC * R), r = e % (KC * R);
        double* d = &sB[(x * KC + r / R) * SB + 2 * (r % R)];
        d[0] = rb[i].x;
        d[1] = rb[i].y;
      }
    }
  };

  double acc[2][NP][WC][2];
#pragma unroll
  for (int p = 0; p < 2; ++p)
#pragma unroll
    for (int q = 0; q < NP; ++q)
#pragma unroll
      for (int w = 0; w < WC; ++w) acc[p][q][w][0] = acc[p][q][w][1] = 0.0;

  load(0);
  for (int k0 = 0; k0 < nlm; k0 += KC) {
    store();
    __syncthreads();
    if (k0 + KC < nlm) load(k0 + KC);
#pragma unroll
    for (int par = 0; par < 2; ++par) {
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const int kk = par + 2 * (4 * s + t4);
        double fa[NT];
#pragma unroll
        for (int tb = 0; tb < NT; ++tb) fa[tb] = sA[(tb * KC + kk) * SA + 8 * rt + g];
        double fb[NX][WC];
#pragma unroll
        for (int x = 0; x < NX; ++x)
#pragma unroll
          for (int w = 0; w < WC; ++w) fb[x][w] = sB[(x * KC + kk) * SB + 8 * (ctg * WC + w) + g];
#pragma unroll
        for (int q = 0; q < NP; ++q) {
          const int tb = (NT == 2) ? OP::table(q) : 0;
#pragma unroll
          for (int w = 0; w < WC; ++w) dmma(acc[par][q][w], fa[tb], fb[OP::term(q)][w]);
        }
      }
    }
    __syncthreads();
  }

  const int th = th0 + 8 * rt + g;
  if (th >= nhs) return;
  const double dm = (double)m;
#pragma unroll
  for (int w = 0; w < WC; ++w) {
    const int col = c0 + 4 * (ctg * WC + w) + t4;
    if (col >= a.ncols) continue;
    dcx hN[NP], hS[NP];
#pragma unroll
    for (int q = 0; q < NP; ++q) {
      dcx E = {acc[0][q][w][0], acc[0][q][w][1]};
      dcx O = {acc[1][q][w][0], acc[1][q][w][1]};
      hN[q] = E + O;
      hS[q] = (OP::table(q) == kP) ? E - O : O - E;
    }
    dcx oN[NO], oS[NO];
    OP::combine(hN, dm, oN);
    OP::combine(hS, dm, oS);
    double2* FN = a.F + mc * a.f_m + (int64_t)(2 * th) * a.f_row + col * a.col_c;
    double2* FS = FN + a.f_row;
#pragma unroll
    for (int f = 0; f < NO; ++f) {
      FN[f * a.col_f] = make_double2(oN[f].x, oN[f].y);
      FS[f * a.col_f] = make_double2(oS[f].x, oS[f].y);
    }
  }
}

template <class OP, int R>
struct AnalCfg {
  static constexpr int TK = 64, KC = 16;
  static constexpr int SA = 18;         // sA row stride: rows 2 apart -> 32 B bank step
  static constexpr int SB = 2 * R + 8;  // sB row stride: 8*SB = 64 mod 128 B
  static constexpr int WC = R / 4;
  static constexpr int NA = OP::NT * TK * KC / 256;
  static constexpr int NB = (OP::NX * KC * R + 255) / 256;
  static constexpr size_t smem = (size_t)(OP::NT * TK * SA + OP::NX * 2 * KC * SB) * 8;
};

template <class OP, int R>
__global__ void __launch_bounds__(256, 2) k_anal_f64(AnalArgs<OP::NX, OP::NO> a) {
  using C = AnalCfg<OP, R>;
  constexpr int NX = OP::NX, NP = OP::NP, NT = OP::NT, NO = OP::NO;
  constexpr int TK = C::TK, KC = C::KC, SA = C::SA, SB = C::SB, WC = C::WC;
  extern __shared__ double smem[];
  double* sA = smem;                 // [NT][TK][SA]
  double* sB = smem + NT * TK * SA;  // [NX][2][KC][SB]

  const Tables& t = a.t;
  const int c0 = blockIdx.x * R;
  const int k0 = blockIdx.y * TK;
  const int mc = blockIdx.z;
  const int m = mc * t.minc;
  const int nlm = t.l_max - m + 1;
  if (k0 >= nlm) return;
  const int ls = t.lstart[mc];
  const int nhs = t.nhs;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t4 = lane & 3;
  const int par = warp & 1;
  const int rowi = par + 2 * (8 * (warp >> 1) + g);  // row inside the 64-row tile

  double ra[C::NA];
  double2 rbN[C::NB], rbS[C::NB];
  const double2* Fm = a.F + mc * a.f_m;
  auto load = [&](int j0) {
#pragma unroll
    for (int i = 0; i < C::NA; ++i) {
      int e = tid + 256 * i;
      int tb = e / (TK * KC), r = e % (TK * KC);
      int kr = r / KC, jj = r % KC;
      int k = k0 + kr, j = j0 + jj;
      const double* T = (NT == 2) ? (tb == 0 ? t.plm : t.dplm) : t.plm;
      ra[i] = (k < nlm && j < nhs) ? __ldg(&T[(int64_t)(ls + k) * nhs + j]) : 0.0;
    }
#pragma unroll
    for (int i = 0; i < C::NB; ++i) {
      int e = tid + 256 * i;
      double2 vn = make_double2(0.0, 0.0), vs = vn;
      if (e < NX * KC * R) {
        int x = e / (KC * R), r = e % (KC * R);
        int jj = r / R, cc = r % R;
        int j = j0 + jj, col = c0 + cc;
        if (j < nhs && col < a.ncols) {
          const double2* p = Fm + (int64_t)(2 * j) * a.f_row + x * a.col_x + col * a.col_c;
          vn = __ldg(p);
          vs = __ldg(p + a.f_row);
        }
      }
      rbN[i] = vn;
      rbS[i] = vs;
    }
  };
  auto store = [&]() {
#pragma unroll
    for (int i = 0; i < C::NA; ++i) {
      int e = tid + 256 * i;
      int tb = e / (TK * KC), r = e % (TK * KC);
      sA[(tb * TK + r / KC) * SA + r % KC] = ra[i];
    }
#pragma unroll
    for (int i = 0; i < C::NB; ++i) {
      int e = tid + 256 * i;
      if (e < NX * KC * R) {
        int x = e / (KC * R), r = e % (KC * R);
        int jj = r / R, cc = r % R;
        double* dp = &sB[((x * 2 + 0) * KC + jj) * SB + 2 * cc];
        double* dm = &sB[((x * 2 + 1) * KC + jj) * SB + 2 * cc];
        dp[0] = rbN[i].x + rbS[i].x;
        dp[1] = rbN[i].y + rbS[i].y;
        dm[0] = rbN[i].x - rbS[i].x;
        dm[1] = rbN[i].y - rbS[i].y;
      }
    }
  };

  double acc[NP][WC][2];
#pragma unroll
  for (int q = 0; q < NP; ++q)
#pragma unroll
    for (int w = 0; w < WC; ++w) acc[q][w][0] = acc[q][w][1] = 0.0;

  load(0);
  for (int j0 = 0; j0 < nhs; j0 += KC) {
    store();
    __syncthreads();
    if (j0 + KC < nhs) load(j0 + KC);
#pragma unroll
    for (int s = 0; s < KC / 4; ++s) {
      const int jj = 4 * s + t4;
      double fa[NT];
#pragma unroll
      for (int tb = 0; tb < NT; ++tb) fa[tb] = sA[(tb * TK + rowi) * SA + jj];
#pragma unroll
      for (int q = 0; q < NP; ++q) {
        const int tb = (NT == 2) ? OP::table(q) : 0;
        // P rows: even -> north+south, odd -> north-south; dP the reverse
        const int sign = (OP::table(q) == kP) ? par : 1 - par;
        const double* b = &sB[((OP::term(q) * 2 + sign) * KC + jj) * SB + g];
#pragma unroll
        for (int w = 0; w < WC; ++w) dmma(acc[q][w], fa[tb], b[8 * w]);
      }
    }
    __syncthreads();
  }

  // C fragment: row g of this warp's tile = k, complex column 4w + t4
  const int k = k0 + par + 2 * (8 * (warp >> 1) + g);
  if (k >= nlm) return;
  const double l = (double)(m + k);
  const double inv = (m + k) > 0 ? 1.0 / (l * (l + 1.0)) : 0.0;
  const double dm = (double)m;
#pragma unroll
  for (int w = 0; w < WC; ++w) {
    const int col = c0 + 4 * w + t4;
    if (col >= a.ncols) continue;
    dcx h[NP];
#pragma unroll
    for (int q = 0; q < NP; ++q) h[q] = {acc[q][w][0], acc[q][w][1]};
    dcx o[NO];
    OP::finish(h, dm, inv, o);
    const int64_t off = (int64_t)(ls + k) * a.ld + a.out_col0 + col;
#pragma unroll
    for (int f = 0; f < NO; ++f)
      if (a.out[f]) a.out[f][off] = make_double2(o[f].x, o[f].y);
  }
}

// ----------------------------------------------------------------- launchers

template <class OP, int R>
int launch_synth_f64(const SynthArgs<OP::NX>& a, cudaStream_t st) {
  using C = SynthCfg<OP, R>;
  static_assert(C::smem <= 200 * 1024, "synthesis tile too large");
  auto kern = k_synth_f64<OP, R>;
  MT_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)C::smem));
  dim3 grid((a.ncols + R - 1) / R, (a.t.nhs + C::TH - 1) / C::TH, a.t.n_m);
  kern<<<grid, 256, C::smem, st>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

template <class OP, int R>
int launch_anal_f64(const AnalArgs<OP::NX, OP::NO>& a, cudaStream_t st) {
  using C = AnalCfg<OP, R>;
  static_assert(C::smem <= 200 * 1024, "analysis tile too large");
  auto kern = k_anal_f64<OP, R>;
  MT_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)C::smem));
  dim3 grid((a.ncols + R - 1) / R, (a.t.l_max + 1 + C::TK - 1) / C::TK, a.t.n_m);
  kern<<<grid, 256, C::smem, st>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

template int launch_synth_f64<SynScalar, 16>(const SynthArgs<1>&, cudaStream_t);
template int launch_synth_f64<SynGrad, 16>(const SynthArgs<1>&, cudaStream_t);
template int launch_synth_f64<SynTorpol, 8>(const SynthArgs<3>&, cudaStream_t);
template int launch_synth_f64<SynGroups<2, 0>, 8>(const SynthArgs<6>&, cudaStream_t);
template int launch_synth_f64<SynGroups<2, 1>, 8>(const SynthArgs<7>&, cudaStream_t);
template int launch_synth_f64<SynGroups<2, 2>, 8>(const SynthArgs<8>&, cudaStream_t);
template int launch_anal_f64<AnaScalar, 8>(const AnalArgs<1, 1>&, cudaStream_t);
template int launch_anal_f64<AnaSphtor, 8>(const AnalArgs<2, 2>&, cudaStream_t);
template int launch_anal_f64<AnaGroups<1, 2>, 8>(const AnalArgs<6, 5>&, cudaStream_t);
template int launch_anal_f64<AnaGroups<1, 0>, 8>(const AnalArgs<3, 3>&, cudaStream_t);
template int launch_anal_f64<AnaGroups<2, 0>, 8>(const AnalArgs<3, 2>&, cudaStream_t);

}  // namespace mt
