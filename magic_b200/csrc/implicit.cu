// Implicit (IMEX) updates with a per-degree solve (FP64): entropy,
// composition, toroidal velocity, magnetic field (k_update_field) and the
// double-curl poloidal velocity with the l = 0 pressure (k_update_poloidal).
//
// Replaces magic_torch/update_s.py:213-271 (updateS; updateXi,
// update_xi.py:208-262, has the same form) and update_z.py:333-505 (updateZ
// without inner-core rotation or angular-momentum correction) with the CNAB2
// right-hand side of time_scheme.py:82-96 and the history rotation of
// time_scheme.py:130-143.
//
// The per-degree solve is an operator set (mt_lop): one dense n_r x n_r
// matrix per l, built on the host as the inverse of the reference's
// preconditioned LHS (update_s.py:67-134); for the Chebyshev scheme the
// DCT-I back to grid values and the Chebyshev truncation are folded in
// (M_l = C T A_l^-1).  Matrices are stored transposed, MT[l][k][j], with the
// j stride rounded up to even, so consecutive threads read consecutive
// 16-byte level pairs (j, j + 1).
//
// k_update_field: CTA = (16 orders m of one degree l); thread = (group of 4
// orders, pair of output levels j, j + 1), a 4 x 2 complex register tile:
//   rhs = w_old old + w_impl impl + w_expl0 expl0 + w_expl1 expl1, rows 0 and
//   n_r - 1 replaced by the boundary values; expl1 <- expl0 (rotation);
//   x = M_l rhs, imaginary part dropped for m = 0; dx = D1 x, d2x = D2 x
//   (d2x stored when requested);
//   old <- so_l so_r x; impl <- ia_l ia_r (d2x + ib_r dx - (ic_r + ic_l ic_r2) x).
// M_l streams through shared memory in chunks of 16 rows k (double-buffered
// cp.async, overlapping the right-hand-side loads and the products), each
// coefficient pair feeding 16 FMAs.  For n_r > 256 a wide variant (4 orders
// per CTA, coefficients read from L2) keeps shared memory bounded.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "radial_op.cuh"

struct mt_lop {
  int n_l = 0, n_r = 0, ldm = 0, device = 0;  // ldm: j stride (>= n_r, multiple of 8)
  double* mt = nullptr;  // (n_l, n_r, ldm) transposed: mt[(l * n_r + k) * ldm + j] = M_l[j][k]
  // banded form (mt null): pivoted LU factors of the preconditioned matrices in
  // band storage, (n_l, 2 kl + ku + 1, n_r) row-major, 1-based pivots (n_l, n_r),
  // and the row / column scalings (n_l, n_r) of the solve (fc may be null)
  int kl = 0, ku = 0;
  double* abd = nullptr;
  int* piv = nullptr;
  double *fr = nullptr, *fc = nullptr;
};

namespace mt {

namespace {

constexpr int kRows = 4;           // orders m per thread
constexpr int kKc = 16;            // solve-matrix rows k per staged chunk
constexpr int kStagedMaxR = 256;   // largest n_r on the shared-memory path
constexpr int kStagedThreads = 256;
constexpr int kWideThreads = 512;  // one group of up to 512 level pairs

// staged: up to 4 row groups within 256 threads, kMinBlocks resident CTAs
// per SM (the register cap); wide: one group
template <bool kStaged, int kMinBlocks>
struct Bounds {
  static constexpr int kThreads = kStaged ? kStagedThreads : kWideThreads;
  static constexpr int kBlocks = kStaged ? kMinBlocks : 1;
};

__device__ __forceinline__ void dmma_f64(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

// thread = (row group rg: rows rg * kRows .. + kRows - 1, level pair jp: j = 2 jp, 2 jp + 1)
struct Slot {
  int rg, jp;
  bool active;
};
__device__ __forceinline__ Slot slot_of(int n_r, int groups) {
  const int n_jp = (n_r + 1) >> 1;
  Slot s;
  s.jp = threadIdx.x % n_jp;
  s.rg = threadIdx.x / n_jp;
  s.active = s.rg < groups;
  return s;
}

__device__ __forceinline__ void cpa16(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpa_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// rows k of chunk c of M_l (row stride ldm, even, so every 16-byte piece is
// aligned) into a shared buffer of kKc x ldm doubles; one commit group
__device__ __forceinline__ void stage_chunk(const double* Ml, int n_r, int ldm, int c,
                                            double* buf) {
  const int k0 = c * kKc, nk = min(kKc, n_r - k0);
  const int nv = nk * ldm / 2;
  const double2* src = (const double2*)(Ml + (int64_t)k0 * ldm);
  for (int i = threadIdx.x; i < nv; i += blockDim.x) cpa16(buf + 2 * i, src + i);
  cpa_commit();
}

// acc[r][h] += m.h * f_r[k] for the thread's 4 rows (row stride fs, broadcast
// from shared memory)
__device__ __forceinline__ void fma_rows(double2 m, const double2* fr, int fs, int k,
                                         double2 (&acc)[kRows][2]) {
#pragma unroll
  for (int r = 0; r < kRows; ++r) {
    const double2 v = fr[r * fs + k];
    acc[r][0].x = fma(m.x, v.x, acc[r][0].x);
    acc[r][0].y = fma(m.x, v.y, acc[r][0].y);
    acc[r][1].x = fma(m.y, v.x, acc[r][1].x);
    acc[r][1].y = fma(m.y, v.y, acc[r][1].y);
  }
}

// Wide tiling: acc[r][h] = (M_l f_{rg kRows + r})[2 jp + h], M_l read from
// global memory (L2) as 16-byte level pairs.
__device__ __forceinline__ void solve_tile_wide(const double* __restrict__ Ml, int n_r, int ldm,
                                                int fs, const double2* f, const Slot& s,
                                                double2 (&acc)[kRows][2]) {
#pragma unroll
  for (int r = 0; r < kRows; ++r) acc[r][0] = acc[r][1] = double2{0.0, 0.0};
  if (!s.active) return;
  const double2* fr = f + s.rg * kRows * fs;
  const double* mp = Ml + 2 * s.jp;
#pragma unroll 8
  for (int k = 0; k < n_r; ++k)
    fma_rows(__ldg((const double2*)(mp + (int64_t)k * ldm)), fr, fs, k, acc);
}

// Staged tiling on the FP64 tensor pipe (mma.sync m8n8k4 f64): the CTA's
// right-hand sides as real rows (row 2 o + p = part p of order o; m-tile t =
// row group t = orders 4 t .. 4 t + 3) times M_l^T (n-tile = 8 output levels),
// K = the levels k in 4-wide steps.  M_l streams through shared memory in
// chunks of kKc rows (chunk 0 issued by the caller before the right-hand
// sides; double-buffered cp.async); warp w owns n-tiles w, w + nwarps, ...
// (at most kNt) for every m-tile, so each B fragment feeds all m-tiles and each
// A fragment all of the warp's n-tiles.  Padding: A is zero for k >= n_r, B for
// rows past the chunk; M_l's columns past n_r are stored as zeros.  Every
// thread of the CTA calls this (barriers inside).  The new field is written
// back over the right-hand sides in f (row stride fs), imaginary parts of
// m = 0 dropped.
//
// Fragments (PTX m8n8k4 .f64): A row-major 8x4, lane holds A[lane/4][lane%4];
// B col-major 4x8, lane holds B[lane%4][lane/4]; C/D 8x8, lane holds
// D[lane/4][2 (lane%4) + h], h = 0, 1.
template <int kNt>
__device__ __forceinline__ void solve_tile_dmma(const double* __restrict__ Ml, int n_r, int ldm,
                                                int fs, double2* f, double* mbuf, int groups,
                                                int mc0) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int nt_n = (n_r + 7) >> 3;
  const int ar = lane >> 2, ac = lane & 3;
  double acc[kNt][4][2];
#pragma unroll
  for (int i = 0; i < kNt; ++i)
#pragma unroll
    for (int t = 0; t < 4; ++t) acc[i][t][0] = acc[i][t][1] = 0.0;
  double* fd = reinterpret_cast<double*>(f);
  // A element of m-tile t at k: order 4 t + ar / 2, part ar % 2
  const int a_off = (ar >> 1) * fs * 2 + (ar & 1);
  const int nch = (n_r + kKc - 1) / kKc;
  for (int c = 0; c < nch; ++c) {
    if (c + 1 < nch) {
      stage_chunk(Ml, n_r, ldm, c + 1, mbuf + ((c + 1) & 1) * kKc * ldm);
      cpa_wait<1>();
    } else {
      cpa_wait<0>();
    }
    __syncthreads();
    const double* mb = mbuf + (c & 1) * kKc * ldm;
    const int k0 = c * kKc;
#pragma unroll
    for (int q = 0; q < kKc / 4; ++q) {
      const int kk = 4 * q + ac, k = k0 + kk;
      const bool kin = k < n_r;
      double av[4];
#pragma unroll
      for (int t = 0; t < 4; ++t)
        av[t] = (t < groups && kin) ? fd[a_off + (4 * t * fs + k) * 2] : 0.0;
#pragma unroll
      for (int i = 0; i < kNt; ++i) {
        const int nt = warp + i * nwarp;
        if (nt < nt_n) {
          const double bv = kin ? mb[kk * ldm + 8 * nt + ar] : 0.0;
#pragma unroll
          for (int t = 0; t < 4; ++t)
            if (t < groups) dmma_f64(acc[i][t], av[t], bv);
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < kNt; ++i) {
    const int nt = warp + i * nwarp;
    if (nt >= nt_n) continue;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      if (t >= groups) continue;
      const int o = 4 * t + (ar >> 1), p = ar & 1;
      const bool drop = p && mc0 + o == 0;  // m = 0: real
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int j = 8 * nt + 2 * ac + h;
        if (j < n_r) fd[(o * fs + j) * 2 + p] = drop ? 0.0 : acc[i][t][h];
      }
    }
  }
}

// acc[r] = (D f_r)[j] for a banded radial operator, coefficients shared by the
// rows (row stride fs)
__device__ __forceinline__ void op_rows(const OpView& op, const double2* f, int fs, int j,
                                        double2 (&acc)[kRows]) {
  const int k0 = __ldg(op.k0 + j);
#pragma unroll
  for (int r = 0; r < kRows; ++r) acc[r] = double2{0.0, 0.0};
  for (int kk = 0; kk < op.W; ++kk) {
    const double c = __ldg(op.vals + (int64_t)kk * op.n_r + j);
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      const double2 v = f[r * fs + k0 + kk];
      acc[r].x = fma(c, v.x, acc[r].x);
      acc[r].y = fma(c, v.y, acc[r].y);
    }
  }
}

// (A f_r)[j] and (B f_r)[j] in one sweep when both operators share level j's
// window (same width and first level: the dense Chebyshev operators), so that
// each staged value feeds both; per output the same FMA chain as op_rows.
// Falls back to two op_rows sweeps otherwise.
__device__ __forceinline__ void op_rows2(const OpView& A, const OpView& B, const double2* f,
                                         int fs, int j, double2 (&a)[kRows],
                                         double2 (&b)[kRows]) {
  const int k0 = __ldg(A.k0 + j);
  if (A.W != B.W || __ldg(B.k0 + j) != k0) {
    op_rows(A, f, fs, j, a);
    op_rows(B, f, fs, j, b);
    return;
  }
#pragma unroll
  for (int r = 0; r < kRows; ++r) a[r] = b[r] = double2{0.0, 0.0};
#pragma unroll 4
  for (int kk = 0; kk < A.W; ++kk) {
    const double ca = __ldg(A.vals + (int64_t)kk * A.n_r + j);
    const double cb = __ldg(B.vals + (int64_t)kk * B.n_r + j);
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      const double2 v = f[r * fs + k0 + kk];
      a[r].x = fma(ca, v.x, a[r].x);
      a[r].y = fma(ca, v.y, a[r].y);
      b[r].x = fma(cb, v.x, b[r].x);
      b[r].y = fma(cb, v.y, b[r].y);
    }
  }
}

// The derivatives of the (w, p) update in one sweep where D1, D2, D3 share
// level j's window: D1 w, D2 w, D3 w from the rows fw and D1 p from fp.
__device__ __forceinline__ void op_rows_wp(const OpView& D1, const OpView& D2, const OpView& D3,
                                           const double2* fw, const double2* fp, int fs, int j,
                                           double2 (&d1)[kRows], double2 (&d2)[kRows],
                                           double2 (&d3)[kRows], double2 (&dp)[kRows]) {
  const int k0 = __ldg(D1.k0 + j);
  if (D1.W != D2.W || D1.W != D3.W || __ldg(D2.k0 + j) != k0 || __ldg(D3.k0 + j) != k0) {
    op_rows(D1, fw, fs, j, d1);
    op_rows(D2, fw, fs, j, d2);
    op_rows(D3, fw, fs, j, d3);
    op_rows(D1, fp, fs, j, dp);
    return;
  }
#pragma unroll
  for (int r = 0; r < kRows; ++r) d1[r] = d2[r] = d3[r] = dp[r] = double2{0.0, 0.0};
#pragma unroll 4
  for (int kk = 0; kk < D1.W; ++kk) {
    const double c1 = __ldg(D1.vals + (int64_t)kk * D1.n_r + j);
    const double c2 = __ldg(D2.vals + (int64_t)kk * D2.n_r + j);
    const double c3 = __ldg(D3.vals + (int64_t)kk * D3.n_r + j);
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      const double2 v = fw[r * fs + k0 + kk];
      const double2 u = fp[r * fs + k0 + kk];
      d1[r].x = fma(c1, v.x, d1[r].x);
      d1[r].y = fma(c1, v.y, d1[r].y);
      d2[r].x = fma(c2, v.x, d2[r].x);
      d2[r].y = fma(c2, v.y, d2[r].y);
      d3[r].x = fma(c3, v.x, d3[r].x);
      d3[r].y = fma(c3, v.y, d3[r].y);
      dp[r].x = fma(c1, u.x, dp[r].x);
      dp[r].y = fma(c1, u.y, dp[r].y);
    }
  }
}

// Band factors of a banded per-degree operator set (null abd: dense form).
struct BandView {
  const double* abd;
  const int* piv;
  const double *fr, *fc;
  int kl, ku;
  const double* rd;  // 1 / U's diagonal (staged copies only)
};

// Pivoted banded LU solve of the CTA's rows in shared memory (the reference's
// solve_band_real, magic_torch/algebra.py:460-510, LINPACK dgbsl order, with
// the row and column scalings of banded_solve_by_l, :672-728): thread t <
// 2 nrow solves part t % 2 of row t / 2 in place (row stride fs); products and
// sums are rounded separately (no contraction), as the reference computes
// them.  m = 0 keeps only the real part.  Ends with a barrier.
__device__ __forceinline__ void band_solve_rows(const BandView& b, int l, int n_r, int fs,
                                                double2* f, int nrow, int mc0) {
  const int t = threadIdx.x;
  if (t < 2 * nrow) {
    const int row = t >> 1, part = t & 1;
    double* x = reinterpret_cast<double*>(f + row * fs) + part;  // level k at x[2 k]
    const int kl = b.kl, ku = b.ku, m = kl + ku + 1;
    const double* abd = b.abd;  // degree l's factors (stage_band), abd[i n_r + j]
    const int* piv = b.piv;
    const double* fr = b.fr;
    for (int k = 0; k < n_r; ++k) x[2 * k] = __dmul_rn(fr[k], x[2 * k]);
    for (int k = 1; k <= n_r - 1 && kl != 0; ++k) {  // L y = P (fr rhs), 1-based k
      const int lm = min(kl, n_r - k), lp = piv[k - 1];
      if (lp != k) {
        const double tv = x[2 * (k - 1)];
        x[2 * (k - 1)] = x[2 * (lp - 1)];
        x[2 * (lp - 1)] = tv;
      }
      const double xk = x[2 * (k - 1)];
      for (int i = 1; i <= lm; ++i)
        x[2 * (k - 1 + i)] =
            __dadd_rn(x[2 * (k - 1 + i)], __dmul_rn(xk, abd[(m - 1 + i) * n_r + (k - 1)]));
    }
    for (int k = n_r; k >= 1; --k) {  // U x = y
      x[2 * (k - 1)] = __ddiv_rn(x[2 * (k - 1)], abd[(m - 1) * n_r + (k - 1)]);
      const int lm = min(k, m) - 1, la = m - lm, lb = k - lm;
      const double tv = -x[2 * (k - 1)];
      for (int i = 0; i < lm; ++i)
        x[2 * (lb - 1 + i)] =
            __dadd_rn(x[2 * (lb - 1 + i)], __dmul_rn(tv, abd[(la - 1 + i) * n_r + (k - 1)]));
    }
    if (b.fc)
      for (int k = 0; k < n_r; ++k) x[2 * k] = __dmul_rn(b.fc[k], x[2 * k]);
    if (part == 1 && mc0 + row == 0)
      for (int k = 0; k < n_r; ++k) x[2 * k] = 0.0;
  }
  __syncthreads();
}

// Shared-memory bytes of one degree's band factors: abd ((2 kl + ku + 1) x n_r),
// fr, fc and the reciprocals of U's diagonal (n_r each), piv (n_r ints),
// 16-byte aligned.
__host__ __device__ inline size_t band_smem_bytes(int kl, int ku, int n_r) {
  const size_t d = (size_t)(2 * kl + ku + 1 + 3) * n_r * sizeof(double);
  return (d + (size_t)n_r * sizeof(int) + 15) / 16 * 16;
}

// Copy degree l's band factors into shared memory (all threads; the caller
// synchronises before the solve reads them) and return a view of the copy,
// so that the sequential solve reads shared memory instead of global memory.
__device__ __forceinline__ BandView stage_band(const BandView& b, int l, int n_r, double* sm) {
  const int nb = (2 * b.kl + b.ku + 1) * n_r;
  double* abd = sm;
  double* fr = abd + nb;
  double* fc = fr + n_r;
  double* rd = fc + n_r;
  int* piv = reinterpret_cast<int*>(rd + n_r);
  const double* gabd = b.abd + (int64_t)l * nb;
  const int dg = (b.kl + b.ku) * n_r;  // row of U's diagonal
  for (int i = threadIdx.x; i < nb; i += blockDim.x) abd[i] = gabd[i];
  for (int i = threadIdx.x; i < n_r; i += blockDim.x) {
    fr[i] = b.fr[(int64_t)l * n_r + i];
    if (b.fc) fc[i] = b.fc[(int64_t)l * n_r + i];
    piv[i] = b.piv[(int64_t)l * n_r + i];
    rd[i] = 1.0 / gabd[dg + i];
  }
  return BandView{abd, piv, fr, b.fc ? fc : nullptr, b.kl, b.ku, rd};
}

// x / d for U's diagonal entry d with r = 1/d: the product x r refined by one
// residual step (Markstein's correction, q' = q + (x - q d) r), which gives the
// correctly rounded quotient but in rare double-rounding cases; the refinement
// replaces a full division on the solve's dependence chain.
__device__ __forceinline__ double band_div(double x, double d, double r) {
  const double q = __dmul_rn(x, r);
  return fma(fma(-q, d, x), r, q);
}

// The solve of band_solve_rows for fixed half-bandwidths KL, KU with the
// working entries of each row in registers: the forward sweep touches only
// x[k-1 .. k-1+KL] at step k (the pivot row lies in that window), the
// backward sweep only x[k-1-KL-KU .. k-1]; both windows slide along the row,
// each entry read from and written to shared memory once per sweep.  Same
// operations and order as band_solve_rows, except the division (band_div).
template <int KL, int KU>
__device__ __forceinline__ void band_solve_rows_w(const BandView& b, int n_r, int fs, double2* f,
                                                  int nrow, int mc0) {
  constexpr int M = KL + KU + 1, M1 = KL + KU;
  const int t = threadIdx.x;
  if (t < 2 * nrow) {
    const int row = t >> 1, part = t & 1;
    double* x = reinterpret_cast<double*>(f + row * fs) + part;  // level k at x[2 k]
    const double* abd = b.abd;
    double W[KL + 1];
#pragma unroll
    for (int q = 0; q <= KL; ++q) W[q] = q < n_r ? __dmul_rn(b.fr[q], x[2 * q]) : 0.0;
    // unrolled so that the loads of later steps (factors, pivots, incoming
    // entries: independent of the running window) issue ahead of the chain
#pragma unroll 4
    for (int k = 1; k <= n_r - 1; ++k) {  // L y = P (fr rhs), 1-based k
      const int d = b.piv[k - 1] - k;     // 0 .. KL
#pragma unroll
      for (int q = 1; q <= KL; ++q)
        if (d == q) {
          const double tv = W[0];
          W[0] = W[q];
          W[q] = tv;
        }
      const double xk = W[0];
      const int lm = min(KL, n_r - k);
#pragma unroll
      for (int i = 1; i <= KL; ++i)
        if (i <= lm) W[i] = __dadd_rn(W[i], __dmul_rn(xk, abd[(M - 1 + i) * n_r + (k - 1)]));
      x[2 * (k - 1)] = W[0];
#pragma unroll
      for (int q = 0; q < KL; ++q) W[q] = W[q + 1];
      const int nx = k + KL;  // next entry entering the window
      W[KL] = nx < n_r ? __dmul_rn(b.fr[nx], x[2 * nx]) : 0.0;
    }
    x[2 * (n_r - 1)] = W[0];
    // U x = y: V[q] = x[k-1-M1+q], V[M1] the current entry
    double V[M1 + 1];
#pragma unroll
    for (int q = 0; q <= M1; ++q) {
      const int j = n_r - 1 - M1 + q;
      V[q] = j >= 0 ? x[2 * j] : 0.0;
    }
#pragma unroll 4
    for (int k = n_r; k >= 1; --k) {
      V[M1] = band_div(V[M1], abd[(M - 1) * n_r + (k - 1)], b.rd[k - 1]);
      // b(lb + i) += t abd(la + i, k), i < lm = min(k, M) - 1, la = M - lm,
      // lb = k - lm: entry x[k-1-lm+i] is V[q] with q = M1 - lm + i, and its
      // coefficient row la - 1 + i is q itself
      const int lm = min(k, M) - 1;
      const double tv = -V[M1];
#pragma unroll
      for (int q = 0; q < M1; ++q)
        if (q >= M1 - lm) V[q] = __dadd_rn(V[q], __dmul_rn(tv, abd[q * n_r + (k - 1)]));
      x[2 * (k - 1)] = V[M1];
#pragma unroll
      for (int q = M1; q > 0; --q) V[q] = V[q - 1];
      const int j = k - 2 - M1;
      V[0] = j >= 0 ? x[2 * j] : 0.0;
    }
    if (b.fc)
      for (int k = 0; k < n_r; ++k) x[2 * k] = __dmul_rn(b.fc[k], x[2 * k]);
    if (part == 1 && mc0 + row == 0)
      for (int k = 0; k < n_r; ++k) x[2 * k] = 0.0;
  }
  __syncthreads();
}

// dispatch on the half-bandwidths of the finite-difference operators
__device__ __forceinline__ void band_solve(const BandView& b, int l, int n_r, int fs, double2* f,
                                           int nrow, int mc0) {
  if (b.rd && b.kl == 2 && b.ku == 2) band_solve_rows_w<2, 2>(b, n_r, fs, f, nrow, mc0);
  else if (b.rd && b.kl == 3 && b.ku == 3) band_solve_rows_w<3, 3>(b, n_r, fs, f, nrow, mc0);
  else band_solve_rows(b, l, n_r, fs, f, nrow, mc0);
}

// the solved rows (band form) from shared memory to the field's global array
__device__ __forceinline__ void store_rows(const double2* f, int fs, int n_r, int nrow,
                                           const int* lm, double2* __restrict__ out, int64_t ld) {
  for (int e = threadIdx.x; e < nrow * n_r; e += blockDim.x) {
    const int row = e / n_r, j = e - row * n_r;
    out[(int64_t)lm[row] * ld + j] = f[row * fs + j];
  }
  __syncthreads();
}

struct UsArgs {
  int n_r, ldm, fs, l_max, minc, n_m, groups;
  BandView band;
  const int* lstart;
  double2 *x, *dx, *d2x, *old, *impl, *expl0, *expl1;
  const double2 *top, *bot;
  int64_t ld;
  double w_old, w_impl, w_expl0, w_expl1;
  const double *so_l, *so_r, *ia_l, *ia_r, *ib_r, *ic_r, *ic_l, *ic_r2;
  const double* mt;
  OpView D1, D2;
};

// number of valid rows of the CTA starting at order index mc0: mc < n_m, m <= l
__device__ __forceinline__ int cta_rows(int mc0, int rows, int l, int minc, int n_m) {
  int n = min(rows, n_m - mc0);
  if (n <= 0) return 0;
  return max(0, min(n, l / minc - mc0 + 1));
}

// CNAB2 right-hand sides of the CTA's rows into f ([rows][fs], zero for
// rows past nrow), with expl1 <- expl0.  kLd elements per thread are loaded
// before any store, so their HBM latencies overlap (the stores may alias the
// next loads as far as the compiler knows).  The poloidal form adds
// the buoyancy (and chemical) coupling and zeroes its boundary rows.
template <bool kPol, int kLd, class A>
__device__ __forceinline__ void build_rhs(const A& a, int l, int rows, int nrow,
                                          const int* lm_row, double2* f) {
  const int n_r = a.n_r;
  const double2 zero = {0.0, 0.0};
  const double dL = (double)l * (l + 1.0);
  // thread t takes elements t, t + T, ... of the rows x n_r block: (row, k)
  // advances by (T / n_r rows, T % n_r levels) with a carry, no division
  const int T = blockDim.x, dr = T / n_r, dk = T - dr * n_r;
  int row = threadIdx.x / n_r, k = threadIdx.x - row * n_r;
  while (row < rows) {
    double2 ol[kLd], im[kLd], e0[kLd], e1[kLd], cs[kLd], cx[kLd];
    int64_t off[kLd];
    int rr[kLd], kq[kLd];
#pragma unroll
    for (int u = 0; u < kLd; ++u) {
      rr[u] = row;
      kq[u] = k;
      off[u] = -1;
      ol[u] = im[u] = e0[u] = e1[u] = cs[u] = cx[u] = zero;
      if (row < nrow) {
        const int64_t o = (int64_t)lm_row[row] * a.ld + k;
        off[u] = o;
        ol[u] = a.old[o];
        im[u] = a.impl[o];
        e0[u] = a.expl0[o];
        e1[u] = a.expl1[o];
        if constexpr (kPol) {
          cs[u] = a.s[o];
          if (a.xi) cx[u] = a.xi[o];
        }
      }
      row += dr;
      k += dk;
      if (k >= n_r) {
        k -= n_r;
        ++row;
      }
    }
#pragma unroll
    for (int u = 0; u < kLd; ++u) {
      if (rr[u] >= rows) break;
      const int kk = kq[u];
      double2 v = zero;
      if (off[u] >= 0) {
        a.expl1[off[u]] = e0[u];
        v.x = a.w_old * ol[u].x + a.w_impl * im[u].x + a.w_expl0 * e0[u].x + a.w_expl1 * e1[u].x;
        v.y = a.w_old * ol[u].y + a.w_impl * im[u].y + a.w_expl0 * e0[u].y + a.w_expl1 * e1[u].y;
        if constexpr (kPol) {
          const double gb = a.wimp_lin0 * dL * a.or2[kk] * a.rgrav[kk];
          v.x += gb * a.BuoFac * cs[u].x;
          v.y += gb * a.BuoFac * cs[u].y;
          if (a.xi) {
            v.x += gb * a.ChemFac * cx[u].x;
            v.y += gb * a.ChemFac * cx[u].y;
          }
          if (kk < 2 || kk > n_r - 3 || l == 0) v = zero;
        } else {
          const int lm = lm_row[rr[u]];
          if (kk == 0) v = a.top ? a.top[lm] : zero;
          if (kk == n_r - 1) v = a.bot ? a.bot[lm] : zero;
        }
      }
      f[rr[u] * a.fs + kk] = v;
    }
  }
}

// the new field of the CTA's rows into f (row stride fs) and out: staged
// tiling on the tensor pipe, wide tiling with FMAs; returns after a barrier
template <bool kStaged, int kNt>
__device__ __forceinline__ void solve_rows_to(const double* __restrict__ Ml, int n_r, int ldm,
                                              int fs, double2* f, double* mbuf, int groups,
                                              int mc0, const Slot& s, int nrow,
                                              double2* __restrict__ out, int64_t ld,
                                              const int* lm) {
  if constexpr (kStaged) {
    solve_tile_dmma<kNt>(Ml, n_r, ldm, fs, f, mbuf, groups, mc0);
    __syncthreads();
    if (s.active) {
#pragma unroll
      for (int r = 0; r < kRows; ++r) {
        const int row = s.rg * kRows + r;
        if (row >= nrow) break;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int j = 2 * s.jp + h;
          if (j < n_r) out[(int64_t)lm[row] * ld + j] = f[row * fs + j];
        }
      }
    }
  } else {
    double2 acc[kRows][2];
    solve_tile_wide(Ml, n_r, ldm, fs, f, s, acc);
    __syncthreads();
    if (s.active) {
#pragma unroll
      for (int r = 0; r < kRows; ++r) {
        const int row = s.rg * kRows + r;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int j = 2 * s.jp + h;
          if (j >= n_r) continue;
          double2 v = acc[r][h];
          if (mc0 + row == 0) v.y = 0.0;  // m = 0
          f[row * fs + j] = v;
          if (row < nrow) out[(int64_t)lm[row] * ld + j] = v;
        }
      }
    }
  }
  __syncthreads();
}

template <bool kStaged, int kNt>
__global__ void __launch_bounds__(Bounds<kStaged, kNt == 2 ? 3 : 2>::kThreads,
                                  Bounds<kStaged, kNt == 2 ? 3 : 2>::kBlocks)
    k_update_field(UsArgs a) {
  extern __shared__ __align__(16) double2 usbuf[];
  __shared__ int lm_row[16];
  const int rows = a.groups * kRows;
  const int n_r = a.n_r, ldm = a.ldm, fs = a.fs, l = blockIdx.y, mc0 = blockIdx.x * rows;
  const int nrow = cta_rows(mc0, rows, l, a.minc, a.n_m);
  if (nrow == 0) return;
  double2* f = usbuf;                           // [rows][fs]: rhs, then x
  double* mbuf = (double*)(usbuf + rows * fs);  // staged: [2][kKc][ldm]
  const bool band = a.band.abd != nullptr;
  const double* Ml = band ? nullptr : a.mt + (int64_t)l * n_r * ldm;
  if constexpr (kStaged)
    if (!band) stage_chunk(Ml, n_r, ldm, 0, mbuf);
  const BandView bv = band ? stage_band(a.band, l, n_r, mbuf) : a.band;
  if (threadIdx.x < rows)
    lm_row[threadIdx.x] = threadIdx.x < nrow
        ? a.lstart[mc0 + threadIdx.x] + (l - (mc0 + threadIdx.x) * a.minc) : 0;
  __syncthreads();
  build_rhs<false, 3>(a, l, rows, nrow, lm_row, f);
  __syncthreads();
  const Slot s = slot_of(n_r, a.groups);
  if (band) {
    band_solve(bv, l, n_r, fs, f, nrow, mc0);
    store_rows(f, fs, n_r, nrow, lm_row, a.x, a.ld);
  } else {
    solve_rows_to<kStaged, kNt>(Ml, n_r, ldm, fs, f, mbuf, a.groups, mc0, s, nrow, a.x, a.ld,
                                lm_row);
  }
  if (!s.active) return;
  auto lm_of = [&](int row) { return lm_row[row]; };
  const double so_l = a.so_l ? a.so_l[l] : 1.0, ia_l = a.ia_l[l], ic_l = a.ic_l[l];
  const double2* fr = f + s.rg * kRows * fs;
#pragma unroll 1
  for (int h = 0; h < 2; ++h) {
    const int j = 2 * s.jp + h;
    if (j >= n_r) break;
    double2 d1[kRows], d2[kRows];
    op_rows2(a.D1, a.D2, fr, fs, j, d1, d2);
    const double so = so_l * (a.so_r ? a.so_r[j] : 1.0);
    const double c1 = a.ib_r[j], c0 = (a.ic_r ? a.ic_r[j] : 0.0) + ic_l * a.ic_r2[j];
    const double ia = ia_l * a.ia_r[j];
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      const int row = s.rg * kRows + r;
      if (row >= nrow) break;
      const int64_t o = (int64_t)lm_of(row) * a.ld + j;
      const double2 v = fr[r * fs + j];
      a.dx[o] = d1[r];
      if (a.d2x) a.d2x[o] = d2[r];
      a.old[o] = double2{so * v.x, so * v.y};
      a.impl[o] = double2{ia * (d2[r].x + c1 * d1[r].x - c0 * v.x),
                          ia * (d2[r].y + c1 * d1[r].y - c0 * v.y)};
    }
  }
}

struct PwArgs {
  int n_r, ldm, fs, l_max, minc, n_m, groups;
  BandView band;
  const int* lstart;
  double2 *w, *dw, *ddw, *old, *impl, *expl0, *expl1, *p;
  const double2 *s, *xi;
  int64_t ld;
  double w_old, w_impl, w_expl0, w_expl1, wimp_lin0, BuoFac, ChemFac;
  const double* hdif;
  const double *or2, *orho1, *beta, *visc, *rgrav, *rho0, *c3, *c2n, *c1n, *c1d, *c0n;
  const double* mt;
  OpView D1, D2, P0;
};

// Double-curl poloidal update (magic_torch/update_w_doublecurl.py:393-483):
// same tiling as k_update_field; the CTA holding (l, m) = (0, 0) also solves
// the l = 0 pressure (update_wp.py:173-194).
template <bool kStaged, int kNt>
__global__ void __launch_bounds__(Bounds<kStaged, 2>::kThreads, Bounds<kStaged, 2>::kBlocks)
    k_update_poloidal(PwArgs a) {
  extern __shared__ __align__(16) double2 pwbuf[];
  __shared__ int lm_row[16];
  const int rows = a.groups * kRows;
  const int n_r = a.n_r, ldm = a.ldm, fs = a.fs, l = blockIdx.y, mc0 = blockIdx.x * rows;
  const int nrow = cta_rows(mc0, rows, l, a.minc, a.n_m);
  if (nrow == 0) return;
  double2* f = pwbuf;                 // [rows][fs]: rhs, then w
  double2* dd = pwbuf + rows * fs;    // [rows][fs]: D2 w
  double* mbuf = (double*)(pwbuf + 2 * rows * fs);
  const bool band = a.band.abd != nullptr;
  const double* Ml = band ? nullptr : a.mt + (int64_t)l * n_r * ldm;
  if constexpr (kStaged)
    if (!band) stage_chunk(Ml, n_r, ldm, 0, mbuf);
  const BandView bv = band ? stage_band(a.band, l, n_r, mbuf) : a.band;
  const double2 zero = {0.0, 0.0};
  const double dL = (double)l * (l + 1.0);
  if (threadIdx.x < rows)
    lm_row[threadIdx.x] = threadIdx.x < nrow
        ? a.lstart[mc0 + threadIdx.x] + (l - (mc0 + threadIdx.x) * a.minc) : 0;
  auto lm_of = [&](int row) { return lm_row[row]; };
  __syncthreads();
  build_rhs<true, 2>(a, l, rows, nrow, lm_row, f);
  __syncthreads();
  const Slot s = slot_of(n_r, a.groups);
  if (band) {
    band_solve(bv, l, n_r, fs, f, nrow, mc0);
    store_rows(f, fs, n_r, nrow, lm_row, a.w, a.ld);
  } else {
    solve_rows_to<kStaged, kNt>(Ml, n_r, ldm, fs, f, mbuf, a.groups, mc0, s, nrow, a.w, a.ld,
                                lm_row);
  }
  const double2* fr = f + s.rg * kRows * fs;
  double2* dr = dd + s.rg * kRows * fs;
  if (s.active) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int j = 2 * s.jp + h;
      if (j >= n_r) break;
      double2 d2[kRows];
      op_rows(a.D2, fr, fs, j, d2);
#pragma unroll
      for (int r = 0; r < kRows; ++r) {
        const int row = s.rg * kRows + r;
        dr[r * fs + j] = d2[r];
        if (row < nrow) a.ddw[(int64_t)lm_of(row) * a.ld + j] = d2[r];
      }
    }
  }
  __syncthreads();
  if (s.active) {
    const double hd = a.hdif[l];
#pragma unroll 1
    for (int h = 0; h < 2; ++h) {
      const int j = 2 * s.jp + h;
      if (j >= n_r) break;
      double2 d1[kRows], d3[kRows], d4[kRows];
      op_rows(a.D1, fr, fs, j, d1);
      op_rows(a.D1, dr, fs, j, d3);
      op_rows(a.D2, dr, fs, j, d4);
      const bool bnd = j == 0 || j == n_r - 1;
      const double or2 = a.or2[j], orho1 = a.orho1[j], beta = a.beta[j];
      const double dLo = dL * or2, fo = -dLo * orho1;
      const double c3 = a.c3[j], c2 = a.c2n[j] - 2.0 * dLo, c1 = a.c1n[j] + dL * a.c1d[j];
      const double c0 = dLo * (a.c0n[j] + dLo);
      const double fd = -hd * dLo * a.visc[j] * orho1, gb = dLo * a.rgrav[j];
      // couplings of all rows loaded before the stores, so the loads overlap
      double2 cpl[kRows];
#pragma unroll
      for (int r = 0; r < kRows; ++r) {
        const int row = s.rg * kRows + r;
        cpl[r] = zero;
        if (row < nrow) {
          const int64_t o = (int64_t)lm_of(row) * a.ld + j;
          const double2 sv = a.s[o];
          cpl[r] = double2{a.BuoFac * gb * sv.x, a.BuoFac * gb * sv.y};
          if (a.xi) {
            const double2 xv = a.xi[o];
            cpl[r].x += a.ChemFac * gb * xv.x;
            cpl[r].y += a.ChemFac * gb * xv.y;
          }
        }
      }
#pragma unroll
      for (int r = 0; r < kRows; ++r) {
        const int row = s.rg * kRows + r;
        if (row >= nrow) break;
        const int64_t o = (int64_t)lm_of(row) * a.ld + j;
        const double2 v = fr[r * fs + j], e2 = dr[r * fs + j];
        a.dw[o] = d1[r];
        a.old[o] = bnd ? zero
                       : double2{fo * (e2.x - beta * d1[r].x - dLo * v.x),
                                 fo * (e2.y - beta * d1[r].y - dLo * v.y)};
        double2 im;
        im.x = fd * (d4[r].x + c3 * d3[r].x + c2 * e2.x + c1 * d1[r].x + c0 * v.x) + cpl[r].x;
        im.y = fd * (d4[r].y + c3 * d3[r].y + c2 * e2.y + c1 * d1[r].y + c0 * v.y) + cpl[r].y;
        a.impl[o] = bnd ? zero : im;
      }
    }
  }
  if (l != 0 || mc0 != 0 || !a.p) return;
  // l = 0 pressure: P0 (0, rho0 BuoFac rgrav Re s + Re expl0 [+ chemistry]); row (0, 0)
  __syncthreads();
  const int64_t row0 = (int64_t)lm_of(0) * a.ld;
  for (int k = threadIdx.x; k < n_r; k += blockDim.x) {
    double v = a.rho0[k] * a.BuoFac * a.rgrav[k] * a.s[row0 + k].x + a.expl0[row0 + k].x;
    if (a.xi) v += a.rho0[k] * a.ChemFac * a.rgrav[k] * a.xi[row0 + k].x;
    f[k] = double2{k == 0 ? 0.0 : v, 0.0};
  }
  __syncthreads();
  for (int j = threadIdx.x; j < n_r; j += blockDim.x)
    a.p[row0 + j] = double2{op_row(a.P0, f, j).x, 0.0};
}

// Launch shape of either tiling: threads = groups x level pairs (rounded to a
// warp), shared memory = row buffers (+ the two staged matrix chunks).
struct TileLaunch {
  bool staged;
  int groups, fs, nt;  // row groups, row stride of the shared rows, n-tiles per warp
  dim3 grid;
  int threads;
  size_t smem;
};
TileLaunch tile_launch(int n_r, int ldm, int l_max, int n_m, int row_buffers,
                       size_t band_bytes) {
  TileLaunch t;
  t.staged = n_r <= kStagedMaxR;
  const int n_jp = (n_r + 1) / 2;
  t.groups = t.staged ? std::min(4, kStagedThreads / n_jp) : 1;
  const int rows = t.groups * kRows;
  t.threads = (t.groups * n_jp + 31) / 32 * 32;
  t.grid = dim3((n_m + rows - 1) / rows, l_max + 1);
  // staged: rows 4 (mod 8) double2 apart, so the 8 rows x 4 levels of an A
  // fragment fall on distinct bank pairs (two wavefronts, the minimum)
  t.fs = t.staged ? n_r + ((4 - n_r) & 7) : n_r;
  const int nt_n = (n_r + 7) / 8, nwarp = t.threads / 32;
  t.nt = nt_n <= 2 * nwarp ? 2 : 4;
  // after the row buffers: the staged solve-matrix chunks, or a degree's band
  // factors (band_bytes, nonzero on the banded path)
  t.smem = (size_t)row_buffers * rows * t.fs * sizeof(double2) +
           (band_bytes ? band_bytes : t.staged ? (size_t)2 * kKc * ldm * sizeof(double) : 0);
  return t;
}

// ---------------------------------------------------------------------------
// Standard-form poloidal update (magic_torch/update_wp.py:387-531): the w and
// p equations are coupled through one 2 n_r x 2 n_r solve per degree.
// CTA = (kWpRows orders m of one degree l); the rows' right-hand sides and
// solutions sit in shared memory, each operator coefficient (read once per
// CTA from L2 as MT[l][k][j], consecutive j across threads) feeds kWpRows
// complex FMAs.  Derivatives with the radial operators D1, D2, D3.
constexpr int kWpRows = 8;
constexpr int kWpThreads = 256;

struct WpArgs {
  int n_r, ldm, l_max, minc, n_m;
  const int* lstart;
  double2 *w, *dw, *ddw, *p, *dp, *wo, *wi, *we0, *we1, *po, *pi, *pe0, *pe1;
  const double2 *s, *xi;
  int64_t ld;
  double w_old, w_impl, w_expl0, w_expl1, wimp_lin0, BuoFac, ChemFac;
  const double* hdif;
  const double *or1, *or2, *beta, *dbeta, *visc, *dLvisc, *rgrav, *rho0;
  int impl_interior;
  const double* p0_row0;
  const double* mt;
  OpView D1, D2, D3, P0;
};

// CNAB2 right-hand sides of element o (level k) of both equations, with the
// buoyancy coupling on the w rows and zero boundary rows, and the rotation
// expl1 <- expl0 of both histories
__device__ __forceinline__ void wp_rhs(const WpArgs& a, int64_t o, int k, double2& vw,
                                       double2& vp) {
  const double2 zero = {0.0, 0.0};
  const double2 ow = a.wo[o], iw = a.wi[o], e0w = a.we0[o], e1w = a.we1[o];
  const double2 op = a.po[o], ip = a.pi[o], e0p = a.pe0[o], e1p = a.pe1[o];
  const double2 sv = a.s[o];
  const double2 xv = a.xi ? a.xi[o] : zero;
  a.we1[o] = e0w;
  a.pe1[o] = e0p;
  vw = vp = zero;
  if (k > 0 && k < a.n_r - 1) {
    const double gb = a.wimp_lin0 * a.rho0[k] * a.rgrav[k];
    vw.x = a.w_old * ow.x + a.w_impl * iw.x + a.w_expl0 * e0w.x + a.w_expl1 * e1w.x +
           gb * (a.BuoFac * sv.x + a.ChemFac * xv.x);
    vw.y = a.w_old * ow.y + a.w_impl * iw.y + a.w_expl0 * e0w.y + a.w_expl1 * e1w.y +
           gb * (a.BuoFac * sv.y + a.ChemFac * xv.y);
    vp.x = a.w_old * op.x + a.w_impl * ip.x + a.w_expl0 * e0p.x + a.w_expl1 * e1p.x;
    vp.y = a.w_old * op.y + a.w_impl * ip.y + a.w_expl0 * e0p.y + a.w_expl1 * e1p.y;
  }
}

// right-hand side of the l = 0 pressure at level k (row (0, 0))
// (row 0: the anelastic integral constraint sum_r p0_row0[r] Re s00[r], or 0)
__device__ __forceinline__ double wp_p0_rhs(const WpArgs& a, int64_t row0, int k) {
  if (k == 0) {
    double c = 0.0;
    if (a.p0_row0)
      for (int j = 0; j < a.n_r; ++j) c += a.p0_row0[j] * a.s[row0 + j].x;
    return c;
  }
  double v = a.rho0[k] * a.BuoFac * a.rgrav[k] * a.s[row0 + k].x + a.we0[row0 + k].x;
  if (a.xi) v += a.rho0[k] * a.ChemFac * a.rgrav[k] * a.xi[row0 + k].x;
  return v;
}

// radial coefficients of the implicit terms at level j of degree l
struct WpCoef {
  double dLo, beta, fw, cw1, cw0, cp2, cp1, cp0, rg;
  bool zero_impl;
};
__device__ __forceinline__ WpCoef wp_coef(const WpArgs& a, int l, int j) {
  const double dL = (double)l * (l + 1.0);
  const double or1 = a.or1[j], or2 = a.or2[j], beta = a.beta[j], dbeta = a.dbeta[j];
  const double dLv = a.dLvisc[j];
  WpCoef c;
  c.dLo = dL * or2;
  c.beta = beta;
  c.fw = a.hdif[l] * c.dLo * a.visc[j];
  c.cw1 = 2.0 * dLv - beta / 3.0;
  c.cw0 = c.dLo + 4.0 / 3.0 * (dbeta + dLv * beta + (3.0 * dLv + beta) * or1);
  c.cp2 = beta - dLv;
  c.cp1 = c.dLo + dLv * beta + dbeta + 2.0 * (dLv + beta) * or1;
  c.cp0 = c.dLo * (2.0 * or1 + 2.0 / 3.0 * beta + dLv);
  c.rg = a.rho0[j] * a.rgrav[j];
  c.zero_impl = a.impl_interior && (l == 0 || j == 0 || j == a.n_r - 1);
  return c;
}

// new fields, derivatives, old and implicit terms of element o
__device__ __forceinline__ void wp_store(const WpArgs& a, const WpCoef& c, int64_t o, double2 w,
                                         double2 p, double2 d1, double2 d2, double2 d3,
                                         double2 dp) {
  const double2 zero = {0.0, 0.0};
  const double2 sv = a.s[o];
  const double2 xv = a.xi ? a.xi[o] : zero;
  a.w[o] = w;
  a.dw[o] = d1;
  a.ddw[o] = d2;
  a.p[o] = p;
  a.dp[o] = dp;
  a.wo[o] = double2{c.dLo * w.x, c.dLo * w.y};
  a.po[o] = double2{-c.dLo * d1.x, -c.dLo * d1.y};
  double2 iw, ip;
  iw.x = -dp.x + c.beta * p.x + c.fw * (d2.x + c.cw1 * d1.x - c.cw0 * w.x) +
         c.rg * (a.BuoFac * sv.x + a.ChemFac * xv.x);
  iw.y = -dp.y + c.beta * p.y + c.fw * (d2.y + c.cw1 * d1.y - c.cw0 * w.y) +
         c.rg * (a.BuoFac * sv.y + a.ChemFac * xv.y);
  ip.x = c.dLo * p.x + c.fw * (-d3.x + c.cp2 * d2.x + c.cp1 * d1.x - c.cp0 * w.x);
  ip.y = c.dLo * p.y + c.fw * (-d3.y + c.cp2 * d2.y + c.cp1 * d1.y - c.cp0 * w.y);
  if (c.zero_impl) iw = ip = zero;
  a.wi[o] = iw;
  a.pi[o] = ip;
}

__global__ void __launch_bounds__(kWpThreads) k_update_wp(WpArgs a) {
  extern __shared__ __align__(16) double2 wpbuf[];
  __shared__ int lm_row[kWpRows];
  const int n_r = a.n_r, n2 = 2 * n_r, l = blockIdx.y, mc0 = blockIdx.x * kWpRows;
  const int nrow = cta_rows(mc0, kWpRows, l, a.minc, a.n_m);
  if (nrow == 0) return;
  double2* f = wpbuf;                  // [kWpRows][n2]: right-hand sides
  double2* x = wpbuf + kWpRows * n2;   // [kWpRows][n2]: w (0..n_r-1), p (n_r..)
  if (threadIdx.x < kWpRows)
    lm_row[threadIdx.x] = threadIdx.x < nrow
        ? a.lstart[mc0 + threadIdx.x] + (l - (mc0 + threadIdx.x) * a.minc) : 0;
  __syncthreads();
  const double2 zero = {0.0, 0.0};
  for (int e = threadIdx.x; e < kWpRows * n_r; e += blockDim.x) {
    const int r = e / n_r, k = e - r * n_r;
    double2 vw = zero, vp = zero;
    if (r < nrow) wp_rhs(a, (int64_t)lm_row[r] * a.ld + k, k, vw, vp);
    f[r * n2 + k] = vw;
    f[r * n2 + n_r + k] = vp;
  }
  __syncthreads();
  if (l == 0) {
    // degree 0 (one row, (l, m) = (0, 0)): w = 0; the l = 0 pressure from its
    // own right-hand side, built in f's first n_r entries
    const int64_t row0 = (int64_t)lm_row[0] * a.ld;
    for (int k = threadIdx.x; k < n_r; k += blockDim.x) f[k] = double2{wp_p0_rhs(a, row0, k), 0.0};
    __syncthreads();
    for (int j = threadIdx.x; j < n_r; j += blockDim.x) {
      x[j] = zero;
      x[n_r + j] = double2{op_row(a.P0, f, j).x, 0.0};
    }
  } else {
    const double* Ml = a.mt + (int64_t)l * n2 * a.ldm;
    for (int j = threadIdx.x; j < n2; j += blockDim.x) {
      double2 acc[kWpRows];
#pragma unroll
      for (int r = 0; r < kWpRows; ++r) acc[r] = zero;
#pragma unroll 4
      for (int k = 0; k < n2; ++k) {
        const double c = __ldg(Ml + (int64_t)k * a.ldm + j);
#pragma unroll
        for (int r = 0; r < kWpRows; ++r) {
          const double2 v = f[r * n2 + k];
          acc[r].x = fma(c, v.x, acc[r].x);
          acc[r].y = fma(c, v.y, acc[r].y);
        }
      }
#pragma unroll
      for (int r = 0; r < kWpRows; ++r) {
        if (mc0 + r == 0) acc[r].y = 0.0;  // m = 0: real coefficients
        x[r * n2 + j] = acc[r];
      }
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nrow * n_r; e += blockDim.x) {
    const int r = e / n_r, j = e - r * n_r;
    const double2* xw = x + r * n2;
    const double2* xp = xw + n_r;
    wp_store(a, wp_coef(a, l, j), (int64_t)lm_row[r] * a.ld + j, xw[j], xp[j],
             op_row(a.D1, xw, j), op_row(a.D2, xw, j), op_row(a.D3, xw, j), op_row(a.D1, xp, j));
  }
}

// The same update with the coupled solve on the FP64 tensor pipe, for
// 2 n_r <= 64 kNt (kNt n-tiles of 8 levels per warp): CTA = 16 orders (4
// m-tiles) of one degree, 8 warps.  The rows' right-hand sides (w part, then p
// part, row stride fs) are the A operand of solve_tile_dmma with the
// 2 n_r x 2 n_r operator streamed through shared memory in 16-row chunks; the
// solution overwrites them.  Derivatives: thread = (4-row group, level), each
// D coefficient serving 4 rows.  kNt = 4 with 8 warps covers 2 n_r <= 256
// (two CTAs per SM by registers); kNt = 6 with 9 warps covers 2 n_r <= 432 and
// runs up to n_r = 192 (e.g. the 129 Chebyshev levels of the anelastic
// benchmark; its shared memory allows one CTA per SM anyway).
// The six-tile variant runs 9 warps: 129 levels give 33 n-tiles (at most four
// per warp) and 4 x 129 derivative items (two rounds of 288 threads, where 256
// threads would need a third round for four items).
constexpr int kWpDmmaMaxR = 128;
constexpr int kWpDmmaWideMaxR = 192;
__host__ __device__ constexpr int wp_dmma_threads(int kNt) { return kNt == 4 ? 256 : 288; }

template <int kNt>
__global__ void __launch_bounds__(wp_dmma_threads(kNt), kNt == 4 ? 2 : 1)
    k_update_wp_dmma(WpArgs a, int fs) {
  extern __shared__ __align__(16) double2 wpd[];
  __shared__ int lm_row[4 * kRows];
  constexpr int rows = 4 * kRows;
  const int n_r = a.n_r, n2 = 2 * n_r, l = blockIdx.y, mc0 = blockIdx.x * rows;
  const int nrow = cta_rows(mc0, rows, l, a.minc, a.n_m);
  if (nrow == 0) return;
  double2* f = wpd;                               // [rows][fs]
  double* mbuf = (double*)(wpd + rows * fs);      // 2 staged chunks of the operator
  const double* Ml = a.mt + (int64_t)l * n2 * a.ldm;
  if (l > 0) stage_chunk(Ml, n2, a.ldm, 0, mbuf);
  if (threadIdx.x < rows)
    lm_row[threadIdx.x] = threadIdx.x < nrow
        ? a.lstart[mc0 + threadIdx.x] + (l - (mc0 + threadIdx.x) * a.minc) : 0;
  __syncthreads();
  const double2 zero = {0.0, 0.0};
  for (int e = threadIdx.x; e < rows * n_r; e += blockDim.x) {
    const int r = e / n_r, k = e - r * n_r;
    double2 vw = zero, vp = zero;
    if (r < nrow) wp_rhs(a, (int64_t)lm_row[r] * a.ld + k, k, vw, vp);
    f[r * fs + k] = vw;
    f[r * fs + n_r + k] = vp;
  }
  __syncthreads();
  if (l == 0) {
    // degree 0, one row: w = 0, the l = 0 pressure from its own right-hand side
    // (built in the row's p half, then solved into the w half and copied)
    const int64_t row0 = (int64_t)lm_row[0] * a.ld;
    for (int k = threadIdx.x; k < n_r; k += blockDim.x)
      f[n_r + k] = double2{wp_p0_rhs(a, row0, k), 0.0};
    __syncthreads();
    for (int j = threadIdx.x; j < n_r; j += blockDim.x)
      f[j] = double2{op_row(a.P0, f + n_r, j).x, 0.0};
    __syncthreads();
    for (int j = threadIdx.x; j < n_r; j += blockDim.x) {
      f[n_r + j] = f[j];
      f[j] = zero;
    }
  } else {
    solve_tile_dmma<kNt>(Ml, n2, a.ldm, fs, f, mbuf, 4, mc0);
  }
  __syncthreads();
  const int groups = (nrow + kRows - 1) / kRows;
  for (int e = threadIdx.x; e < groups * n_r; e += blockDim.x) {
    const int rg = e / n_r, j = e - rg * n_r;
    const double2* xw = f + rg * kRows * fs;
    double2 d1[kRows], d2[kRows], d3[kRows], dp[kRows];
    op_rows_wp(a.D1, a.D2, a.D3, xw, xw + n_r, fs, j, d1, d2, d3, dp);
    const WpCoef c = wp_coef(a, l, j);
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      const int row = rg * kRows + r;
      if (row >= nrow) break;
      wp_store(a, c, (int64_t)lm_row[row] * a.ld + j, xw[r * fs + j], xw[r * fs + n_r + j],
               d1[r], d2[r], d3[r], dp[r]);
    }
  }
}

// Angular-momentum corrections after the toroidal update (update_z.py:446-475).
struct AmArgs {
  int n_r;
  int lm10, lm11;          // rows of (l, m) = (1, 0) and (1, 1); lm11 < 0: no m = 1
  double2 *x, *dx, *d2x, *old, *impl;
  int64_t ld;
  const double *so_l, *so_r, *ia_l, *ia_r, *ib_r, *ic_r, *ic_l, *ic_r2;
  const double *rint, *r, *am_z, *am_dz, *am_d2z;
  double c_moi_oc, am_start;
  int axial, equatorial;
};

constexpr int kAmThreads = 256;

// sum over the block of (a, b); every thread gets the totals
__device__ __forceinline__ double2 am_block_sum(double a, double b, double2* red) {
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[warp] = double2{a, b};
  __syncthreads();
  double2 t{0.0, 0.0};
  for (int w = 0; w < kAmThreads / 32; ++w) {
    t.x += red[w].x;
    t.y += red[w].y;
  }
  return t;
}

// subtract corr * (am_z, am_dz, am_d2z) from row lm of x, dx, d2x and the
// matching change from its old and implicit terms (degree l = 1)
__device__ void am_apply(const AmArgs& a, int lm, double2 corr) {
  const double so_l = a.so_l ? a.so_l[1] : 1.0;
  const double ia_l = a.ia_l[1], ic_l = a.ic_l[1];
  for (int j = threadIdx.x; j < a.n_r; j += kAmThreads) {
    const int64_t o = (int64_t)lm * a.ld + j;
    const double pz = a.am_z[j], pd = a.am_dz[j], pdd = a.am_d2z[j];
    a.x[o].x -= pz * corr.x;
    a.x[o].y -= pz * corr.y;
    a.dx[o].x -= pd * corr.x;
    a.dx[o].y -= pd * corr.y;
    if (a.d2x) {
      a.d2x[o].x -= pdd * corr.x;
      a.d2x[o].y -= pdd * corr.y;
    }
    const double so = so_l * (a.so_r ? a.so_r[j] : 1.0);
    const double ic = (a.ic_r ? a.ic_r[j] : 0.0) + ic_l * a.ic_r2[j];
    const double im = ia_l * a.ia_r[j] * (pdd + a.ib_r[j] * pd - ic * pz);
    a.old[o].x -= so * pz * corr.x;
    a.old[o].y -= so * pz * corr.y;
    a.impl[o].x -= im * corr.x;
    a.impl[o].y -= im * corr.y;
  }
}

// one CTA: the axial correction of (1, 0), then the equatorial one of (1, 1)
__global__ void __launch_bounds__(kAmThreads) k_correct_am(AmArgs a) {
  __shared__ double2 red[kAmThreads / 32];
  const double pi = 3.14159265358979323846;
  const double fac = 8.0 / 3.0 * pi;                 // update_z.py:322
  const double y10 = 0.5 * sqrt(3.0 / pi);           // pre_calculations.py:63
  const double y11 = 0.5 * sqrt(1.5 / pi);           // pre_calculations.py:92
  if (a.axial) {
    double s = 0.0;
    for (int j = threadIdx.x; j < a.n_r; j += kAmThreads)
      s += a.rint[j] * a.r[j] * a.r[j] * a.x[(int64_t)a.lm10 * a.ld + j].x;
    const double tot = am_block_sum(s, 0.0, red).x;
    const double am_z = fac * y10 * tot;
    am_apply(a, a.lm10, double2{(am_z - a.am_start) / (a.c_moi_oc * y10), 0.0});
  }
  if (a.equatorial && a.lm11 >= 0) {
    __syncthreads();
    double sr = 0.0, si = 0.0;
    for (int j = threadIdx.x; j < a.n_r; j += kAmThreads) {
      const double w = a.rint[j] * a.r[j] * a.r[j];
      const double2 z = a.x[(int64_t)a.lm11 * a.ld + j];
      sr += w * z.x;
      si += w * z.y;
    }
    const double2 tot = am_block_sum(sr, si, red);
    const double am_x = 2.0 * fac * y11 * tot.x, am_y = -2.0 * fac * y11 * tot.y;
    const double den = 2.0 * y11 * a.c_moi_oc;
    am_apply(a, a.lm11, double2{am_x / den, -am_y / den});
  }
}

int check_lop(const mt_lop* op) {
  MT_REQUIRE(op && (op->mt || op->abd), MT_ERR_ARG, "null per-degree operator");
  int dev = -1;
  MT_CHECK_CUDA(cudaGetDevice(&dev));
  MT_REQUIRE(dev == op->device, MT_ERR_ARG,
             "per-degree operator used on a different device than it was built on");
  return MT_OK;
}

}  // namespace

}  // namespace mt

using namespace mt;

extern "C" {

int mt_lop_create(int n_l, int n_r, const double* M, mt_lop** out) {
  MT_REQUIRE(out && M && n_l >= 1 && n_r >= 2 && n_r <= 1024, MT_ERR_ARG,
             "bad per-degree operator argument");
  *out = nullptr;
  const size_t per = (size_t)n_r * n_r;
  // j stride: a multiple of 8 (the tensor-pipe n-tiles read whole 8-level
  // groups), 8 (mod 16) so that the 4 k rows of a B fragment fall on distinct
  // bank halves
  int ldm = (n_r + 7) / 8 * 8;
  if (ldm % 16 == 0) ldm += 8;
  const size_t per_t = (size_t)n_r * ldm;
  std::vector<double> t(per_t * n_l, 0.0);
  for (int l = 0; l < n_l; ++l)
    for (int j = 0; j < n_r; ++j)
      for (int k = 0; k < n_r; ++k) {
        const double v = M[l * per + (size_t)j * n_r + k];
        MT_REQUIRE(std::isfinite(v), MT_ERR_ARG, "per-degree operator not finite");
        t[l * per_t + (size_t)k * ldm + j] = v;
      }
  mt_lop* op = new mt_lop();
  op->n_l = n_l;
  op->n_r = n_r;
  op->ldm = ldm;
  if (cudaGetDevice(&op->device) != cudaSuccess ||
      cudaMalloc(&op->mt, t.size() * sizeof(double)) != cudaSuccess ||
      cudaMemcpy(op->mt, t.data(), t.size() * sizeof(double), cudaMemcpyHostToDevice) !=
          cudaSuccess) {
    if (op->mt) cudaFree(op->mt);
    delete op;
    set_error("per-degree operator allocation or upload failed");
    return MT_ERR_CUDA;
  }
  *out = op;
  return MT_OK;
}

int mt_lop_destroy(mt_lop* op) {
  if (!op) return MT_OK;
  void* ptrs[] = {op->mt, op->abd, op->piv, op->fr, op->fc};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  delete op;
  return MT_OK;
}

// Pivoted banded LU factorisation of one band matrix in place (the reference's
// prepare_band, magic_torch/algebra.py:371-457, a port of LINPACK dgbfa with
// partial pivoting; 1-based indices as there): abd (nb x n, row-major, diagonal
// in row kl + ku), pivots 1-based.  Returns 0 or the 1-based singular column.
static int band_factor(double* abd, int n, int kl, int ku, int* pivot) {
  const double kZeroTol = 1.0e-15;
  const int m = kl + ku + 1;
  auto A = [&](int i, int j) -> double& { return abd[(size_t)(i - 1) * n + (j - 1)]; };
  int info = 0;
  const int j0 = ku + 2, j1 = std::min(n, m) - 1;
  for (int jz = j0; jz <= j1; ++jz)
    for (int i = m + 1 - jz; i <= kl; ++i) A(i, jz) = 0.0;
  int jz = j1, ju = 0;
  for (int k = 1; k <= n - 1; ++k) {
    const int kp1 = k + 1;
    ++jz;
    if (jz <= n)
      for (int i = 1; i <= kl; ++i) A(i, jz) = 0.0;
    const int lm = std::min(kl, n - k);
    int lrel = 0;
    double best = std::fabs(A(m, k));
    for (int i = 1; i <= lm; ++i)
      if (std::fabs(A(m + i, k)) > best) {
        best = std::fabs(A(m + i, k));
        lrel = i;
      }
    int l = lrel + m;
    pivot[k - 1] = l + k - m;
    if (std::fabs(A(l, k)) > kZeroTol) {
      if (l != m) std::swap(A(l, k), A(m, k));
      const double t = -1.0 / A(m, k);
      for (int i = 1; i <= lm; ++i) A(m + i, k) *= t;
      ju = std::min(std::max(ju, ku + pivot[k - 1]), n);
      int mm = m;
      for (int j = kp1; j <= ju; ++j) {
        --l;
        --mm;
        const double tt = A(l, j);
        if (l != mm) {
          A(l, j) = A(mm, j);
          A(mm, j) = tt;
        }
        for (int i = 1; i <= lm; ++i) A(mm + i, j) += tt * A(m + i, k);
      }
    } else {
      info = k;
    }
  }
  pivot[n - 1] = n;
  if (std::fabs(A(m, n)) <= kZeroTol) info = n;
  return info;
}

int mt_lop_create_band(int n_l, int n_r, int kl, int ku, const double* A, const double* fac_row,
                       const double* fac_col, mt_lop** out) {
  MT_REQUIRE(out && A && fac_row && n_l >= 1 && n_r >= 2 && n_r <= 1024 && kl >= 0 && ku >= 0 &&
                 kl < n_r && ku < n_r && kl <= 16 && ku <= 16,
             MT_ERR_ARG, "bad banded per-degree operator argument");
  *out = nullptr;
  const int nb = 2 * kl + ku + 1;
  const size_t per = (size_t)n_r * n_r, perb = (size_t)nb * n_r;
  std::vector<double> abd(perb * n_l, 0.0);
  std::vector<int> piv((size_t)n_l * n_r, 0);
  for (int l = 0; l < n_l; ++l) {
    const double* Al = A + l * per;
    double amax = 0.0;
    for (size_t e = 0; e < per; ++e) {
      MT_REQUIRE(std::isfinite(Al[e]), MT_ERR_ARG, "banded operator not finite");
      amax = std::max(amax, std::fabs(Al[e]));
    }
    double* b = abd.data() + l * perb;
    for (int j = 0; j < n_r; ++j)
      for (int i = 0; i < n_r; ++i) {
        const double v = Al[(size_t)i * n_r + j];
        if (i < j - ku || i > j + kl) {
          MT_REQUIRE(std::fabs(v) <= 1e-14 * amax, MT_ERR_ARG,
                     "banded operator has entries outside its band");
        } else {
          b[(size_t)(kl + ku + i - j) * n_r + j] = v;
        }
      }
    MT_REQUIRE(band_factor(b, n_r, kl, ku, piv.data() + (size_t)l * n_r) == 0, MT_ERR_ARG,
               "banded operator is singular");
  }
  mt_lop* op = new mt_lop();
  op->n_l = n_l;
  op->n_r = n_r;
  op->ldm = n_r;
  op->kl = kl;
  op->ku = ku;
  const size_t nf = (size_t)n_l * n_r;
  bool ok = cudaGetDevice(&op->device) == cudaSuccess &&
            cudaMalloc(&op->abd, abd.size() * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&op->piv, piv.size() * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&op->fr, nf * sizeof(double)) == cudaSuccess &&
            (!fac_col || cudaMalloc(&op->fc, nf * sizeof(double)) == cudaSuccess);
  ok = ok &&
       cudaMemcpy(op->abd, abd.data(), abd.size() * sizeof(double), cudaMemcpyHostToDevice) ==
           cudaSuccess &&
       cudaMemcpy(op->piv, piv.data(), piv.size() * sizeof(int), cudaMemcpyHostToDevice) ==
           cudaSuccess &&
       cudaMemcpy(op->fr, fac_row, nf * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess &&
       (!fac_col ||
        cudaMemcpy(op->fc, fac_col, nf * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess);
  if (!ok) {
    mt_lop_destroy(op);
    set_error("banded operator allocation or upload failed");
    return MT_ERR_CUDA;
  }
  *out = op;
  return MT_OK;
}

int mt_update_field(const mt_plan* p, int n_r, const mt_field_update* u, const mt_lop* solve,
                    const mt_radial_op* D1, const mt_radial_op* D2, void* stream) {
  MT_REQUIRE(p && u, MT_ERR_ARG, "null argument");
  int dev = -1;
  MT_CHECK_CUDA(cudaGetDevice(&dev));
  MT_REQUIRE(dev == p->device, MT_ERR_ARG, "plan used on a different device than it was built on");
  MT_TRY(check_lop(solve));
  MT_TRY(check_radial_op(D1));
  MT_TRY(check_radial_op(D2));
  MT_REQUIRE(solve->n_r == n_r && radial_op_size(D1) == n_r && radial_op_size(D2) == n_r,
             MT_ERR_ARG, "operator sizes differ from n_r");
  MT_REQUIRE(solve->n_l == p->l_max + 1, MT_ERR_ARG, "solve operators must cover l = 0..l_max");
  MT_REQUIRE(n_r >= 3 && u->ld >= n_r, MT_ERR_ARG, "bad radial size or stride");
  MT_REQUIRE(u->x && u->dx && u->old && u->impl && u->expl0 && u->expl1, MT_ERR_ARG,
             "null field or time array");
  MT_REQUIRE(u->ia_l && u->ia_r && u->ib_r && u->ic_l && u->ic_r2, MT_ERR_ARG,
             "null coefficient array");
  UsArgs a{};
  a.n_r = n_r;
  a.ldm = solve->ldm;
  a.l_max = p->l_max;
  a.minc = p->minc;
  a.n_m = p->n_m;
  a.lstart = p->d_lstart;
  auto d = [](double* x) { return (double2*)x; };
  a.x = d(u->x); a.dx = d(u->dx); a.d2x = d(u->d2x); a.old = d(u->old); a.impl = d(u->impl);
  a.expl0 = d(u->expl0); a.expl1 = d(u->expl1);
  a.top = (const double2*)u->top;
  a.bot = (const double2*)u->bot;
  a.ld = u->ld;
  a.w_old = u->w_old; a.w_impl = u->w_impl; a.w_expl0 = u->w_expl0; a.w_expl1 = u->w_expl1;
  a.so_l = u->so_l; a.so_r = u->so_r; a.ia_l = u->ia_l; a.ia_r = u->ia_r; a.ib_r = u->ib_r;
  a.ic_r = u->ic_r; a.ic_l = u->ic_l; a.ic_r2 = u->ic_r2;
  a.mt = solve->mt;
  a.band = BandView{solve->abd, solve->piv, solve->fr, solve->fc, solve->kl, solve->ku, nullptr};
  a.D1 = radial_op_view(D1);
  a.D2 = radial_op_view(D2);
  const TileLaunch t = tile_launch(n_r, a.ldm, p->l_max, p->n_m, 1,
                                   solve->abd ? band_smem_bytes(solve->kl, solve->ku, n_r) : 0);
  MT_REQUIRE(!t.staged || (n_r + 7) / 8 <= t.nt * (t.threads / 32), MT_ERR_ARG,
             "tile shape does not cover n_r");
  a.groups = t.groups;
  a.fs = t.fs;
  auto kern = !t.staged ? k_update_field<false, 2>
                        : (t.nt == 2 ? k_update_field<true, 2> : k_update_field<true, 4>);
  MT_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t.smem));
  kern<<<t.grid, t.threads, t.smem, (cudaStream_t)stream>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

int mt_correct_am(const mt_plan* p, int n_r, const mt_field_update* u, const mt_am_correction* c,
                  void* stream) {
  MT_REQUIRE(p && u && c, MT_ERR_ARG, "null argument");
  int dev = -1;
  MT_CHECK_CUDA(cudaGetDevice(&dev));
  MT_REQUIRE(dev == p->device, MT_ERR_ARG, "plan used on a different device than it was built on");
  MT_REQUIRE(p->l_max >= 1 && n_r >= 3 && u->ld >= n_r, MT_ERR_ARG, "bad size or stride");
  MT_REQUIRE(u->x && u->dx && u->old && u->impl && u->ia_l && u->ia_r && u->ib_r && u->ic_l &&
                 u->ic_r2,
             MT_ERR_ARG, "null field, time array or coefficient");
  MT_REQUIRE(c->rint && c->r && c->am_z && c->am_dz && c->am_d2z && c->c_moi_oc != 0.0,
             MT_ERR_ARG, "null radial profile or zero moment of inertia");
  if (!c->axial && !c->equatorial) return MT_OK;
  AmArgs a{};
  a.n_r = n_r;
  a.lm10 = 1;                                   // m = 0 block, l = 1
  a.lm11 = p->minc == 1 ? p->l_max + 1 : -1;    // m = 1 block starts after l = 0..l_max
  auto d = [](double* x) { return (double2*)x; };
  a.x = d(u->x); a.dx = d(u->dx); a.d2x = d(u->d2x); a.old = d(u->old); a.impl = d(u->impl);
  a.ld = u->ld;
  a.so_l = u->so_l; a.so_r = u->so_r; a.ia_l = u->ia_l; a.ia_r = u->ia_r; a.ib_r = u->ib_r;
  a.ic_r = u->ic_r; a.ic_l = u->ic_l; a.ic_r2 = u->ic_r2;
  a.rint = c->rint; a.r = c->r; a.am_z = c->am_z; a.am_dz = c->am_dz; a.am_d2z = c->am_d2z;
  a.c_moi_oc = c->c_moi_oc;
  a.am_start = c->am_start;
  a.axial = c->axial != 0;
  a.equatorial = c->equatorial != 0;
  k_correct_am<<<1, kAmThreads, 0, (cudaStream_t)stream>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

int mt_update_poloidal(const mt_plan* p, int n_r, const mt_poloidal_update* u,
                       const mt_lop* solve, const mt_radial_op* D1, const mt_radial_op* D2,
                       const mt_radial_op* P0, void* stream) {
  MT_REQUIRE(p && u, MT_ERR_ARG, "null argument");
  int dev = -1;
  MT_CHECK_CUDA(cudaGetDevice(&dev));
  MT_REQUIRE(dev == p->device, MT_ERR_ARG, "plan used on a different device than it was built on");
  MT_TRY(check_lop(solve));
  MT_TRY(check_radial_op(D1));
  MT_TRY(check_radial_op(D2));
  MT_TRY(check_radial_op(P0));
  MT_REQUIRE(solve->n_r == n_r && radial_op_size(D1) == n_r && radial_op_size(D2) == n_r &&
                 radial_op_size(P0) == n_r,
             MT_ERR_ARG, "operator sizes differ from n_r");
  MT_REQUIRE(solve->n_l == p->l_max + 1, MT_ERR_ARG, "solve operators must cover l = 0..l_max");
  MT_REQUIRE(n_r >= 5 && u->ld >= n_r, MT_ERR_ARG, "bad radial size or stride");
  MT_REQUIRE(u->w && u->dw && u->ddw && u->old && u->impl && u->expl0 && u->expl1 && u->s,
             MT_ERR_ARG, "null field or time array");
  MT_REQUIRE(u->hdif && u->or2 && u->orho1 && u->beta && u->visc && u->rgrav && u->rho0 &&
                 u->c3 && u->c2n && u->c1n && u->c1d && u->c0n,
             MT_ERR_ARG, "null coefficient array");
  PwArgs a{};
  a.n_r = n_r;
  a.ldm = solve->ldm;
  a.l_max = p->l_max;
  a.minc = p->minc;
  a.n_m = p->n_m;
  a.lstart = p->d_lstart;
  auto d = [](double* x) { return (double2*)x; };
  a.w = d(u->w); a.dw = d(u->dw); a.ddw = d(u->ddw); a.old = d(u->old); a.impl = d(u->impl);
  a.expl0 = d(u->expl0); a.expl1 = d(u->expl1); a.p = d(u->p);
  a.s = (const double2*)u->s;
  a.xi = (const double2*)u->xi;
  a.ld = u->ld;
  a.w_old = u->w_old; a.w_impl = u->w_impl; a.w_expl0 = u->w_expl0; a.w_expl1 = u->w_expl1;
  a.wimp_lin0 = u->wimp_lin0; a.BuoFac = u->BuoFac; a.ChemFac = u->ChemFac;
  a.hdif = u->hdif;
  a.or2 = u->or2; a.orho1 = u->orho1; a.beta = u->beta; a.visc = u->visc; a.rgrav = u->rgrav;
  a.rho0 = u->rho0; a.c3 = u->c3; a.c2n = u->c2n; a.c1n = u->c1n; a.c1d = u->c1d; a.c0n = u->c0n;
  a.mt = solve->mt;
  a.band = BandView{solve->abd, solve->piv, solve->fr, solve->fc, solve->kl, solve->ku, nullptr};
  a.D1 = radial_op_view(D1);
  a.D2 = radial_op_view(D2);
  a.P0 = radial_op_view(P0);
  const TileLaunch t = tile_launch(n_r, a.ldm, p->l_max, p->n_m, 2,
                                   solve->abd ? band_smem_bytes(solve->kl, solve->ku, n_r) : 0);
  MT_REQUIRE(!t.staged || (n_r + 7) / 8 <= t.nt * (t.threads / 32), MT_ERR_ARG,
             "tile shape does not cover n_r");
  a.groups = t.groups;
  a.fs = t.fs;
  auto kern = !t.staged ? k_update_poloidal<false, 2>
                        : (t.nt == 2 ? k_update_poloidal<true, 2> : k_update_poloidal<true, 4>);
  MT_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t.smem));
  kern<<<t.grid, t.threads, t.smem, (cudaStream_t)stream>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

int mt_update_wp(const mt_plan* p, int n_r, const mt_wp_update* u, const mt_lop* solve,
                 const mt_radial_op* D1, const mt_radial_op* D2, const mt_radial_op* D3,
                 const mt_radial_op* P0, void* stream) {
  MT_REQUIRE(p && u, MT_ERR_ARG, "null argument");
  int dev = -1;
  MT_CHECK_CUDA(cudaGetDevice(&dev));
  MT_REQUIRE(dev == p->device, MT_ERR_ARG, "plan used on a different device than it was built on");
  MT_TRY(check_lop(solve));
  MT_TRY(check_radial_op(D1));
  MT_TRY(check_radial_op(D2));
  MT_TRY(check_radial_op(D3));
  MT_TRY(check_radial_op(P0));
  MT_REQUIRE(solve->mt, MT_ERR_ARG, "the coupled (w, p) update takes a dense operator set");
  MT_REQUIRE(solve->n_r == 2 * n_r && radial_op_size(D1) == n_r && radial_op_size(D2) == n_r &&
                 radial_op_size(D3) == n_r && radial_op_size(P0) == n_r,
             MT_ERR_ARG, "operator sizes differ from n_r (solve operators: 2 n_r)");
  MT_REQUIRE(solve->n_l == p->l_max + 1, MT_ERR_ARG, "solve operators must cover l = 0..l_max");
  MT_REQUIRE(n_r >= 3 && u->ld >= n_r, MT_ERR_ARG, "bad radial size or stride");
  MT_REQUIRE(u->w && u->dw && u->ddw && u->p && u->dp && u->w_old && u->w_impl && u->w_expl0 &&
                 u->w_expl1 && u->p_old && u->p_impl && u->p_expl0 && u->p_expl1 && u->s,
             MT_ERR_ARG, "null field or time array");
  MT_REQUIRE(u->hdif && u->or1 && u->or2 && u->beta && u->dbeta && u->visc && u->dLvisc &&
                 u->rgrav && u->rho0,
             MT_ERR_ARG, "null coefficient array");
  const size_t smem = (size_t)2 * kWpRows * 2 * n_r * sizeof(double2);
  MT_REQUIRE(smem <= 227 * 1024, MT_ERR_ARG, "n_r too large for the coupled update");
  WpArgs a{};
  a.n_r = n_r;
  a.ldm = solve->ldm;
  a.l_max = p->l_max;
  a.minc = p->minc;
  a.n_m = p->n_m;
  a.lstart = p->d_lstart;
  auto d = [](double* x) { return (double2*)x; };
  a.w = d(u->w); a.dw = d(u->dw); a.ddw = d(u->ddw); a.p = d(u->p); a.dp = d(u->dp);
  a.wo = d(u->w_old); a.wi = d(u->w_impl); a.we0 = d(u->w_expl0); a.we1 = d(u->w_expl1);
  a.po = d(u->p_old); a.pi = d(u->p_impl); a.pe0 = d(u->p_expl0); a.pe1 = d(u->p_expl1);
  a.s = (const double2*)u->s;
  a.xi = (const double2*)u->xi;
  a.ld = u->ld;
  a.w_old = u->w_old_wt; a.w_impl = u->w_impl_wt; a.w_expl0 = u->w_expl0_wt;
  a.w_expl1 = u->w_expl1_wt; a.wimp_lin0 = u->wimp_lin0; a.BuoFac = u->BuoFac;
  a.ChemFac = u->ChemFac;
  a.hdif = u->hdif;
  a.or1 = u->or1; a.or2 = u->or2; a.beta = u->beta; a.dbeta = u->dbeta; a.visc = u->visc;
  a.dLvisc = u->dLvisc; a.rgrav = u->rgrav; a.rho0 = u->rho0;
  a.impl_interior = u->impl_interior;
  a.p0_row0 = u->p0_row0;
  a.mt = solve->mt;
  a.D1 = radial_op_view(D1);
  a.D2 = radial_op_view(D2);
  a.D3 = radial_op_view(D3);
  a.P0 = radial_op_view(P0);
  if (n_r <= kWpDmmaWideMaxR) {
    // tensor-pipe tiling: rows 4 (mod 8) double2 apart (conflict-free A
    // fragments), the operator's 16-row chunks double-buffered
    const int fs = 2 * n_r + ((4 - 2 * n_r) & 7);
    const size_t sm = (size_t)4 * kRows * fs * sizeof(double2) +
                      (size_t)2 * kKc * a.ldm * sizeof(double);
    const bool narrow = n_r <= kWpDmmaMaxR;
    auto kern = narrow ? k_update_wp_dmma<4> : k_update_wp_dmma<6>;
    MT_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    const dim3 grid((p->n_m + 4 * kRows - 1) / (4 * kRows), p->l_max + 1);
    kern<<<grid, wp_dmma_threads(narrow ? 4 : 6), sm, (cudaStream_t)stream>>>(a, fs);
    MT_CHECK_CUDA(cudaGetLastError());
    return MT_OK;
  }
  MT_CHECK_CUDA(cudaFuncSetAttribute(k_update_wp, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
  const dim3 grid((p->n_m + kWpRows - 1) / kWpRows, p->l_max + 1);
  k_update_wp<<<grid, kWpThreads, smem, (cudaStream_t)stream>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

}  // extern "C"
