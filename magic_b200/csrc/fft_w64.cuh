// Warp FFTs of the FP64 phi stage for row lengths H = 32 Q, Q in {4, 8, 12, 16}
// (n_phi = 256, 512, 768, 1024).
//
// One row belongs to one warp: lane l holds Q complex doubles in registers and
// the row goes through four Stockham passes with the butterfly map of
// fft_stage (fft.cuh):
//   radix Q (span 1), radix 4 (span Q), radix 4 (span 4 Q), radix 2 (span 16 Q),
// Q x 4 x 4 x 2 = H.  Between passes the row lives in shared memory at the
// padded positions pad16(i) and only the warp synchronises (__syncwarp), so
// rows of one CTA never wait for each other.  The radix-12 butterfly is a
// two-factor DFT (12 = 4 x 3) with literal inner twiddles.
#pragma once

#include "fft.cuh"

namespace mt {

// exp(-2 pi i e / 12) (forward) or its conjugate, e a compile-time constant
// after unrolling (cos/sin of multiples of 30 degrees).
template <bool INV>
__device__ __forceinline__ cplx<double> w12d(int e) {
  e %= 12;
  const double h = 0.86602540378443864676;  // sin(60 deg)
  double c, s;
  switch (e) {
    case 0: c = 1.0; s = 0.0; break;
    case 1: c = h; s = 0.5; break;
    case 2: c = 0.5; s = h; break;
    case 3: c = 0.0; s = 1.0; break;
    case 4: c = -0.5; s = h; break;
    case 5: c = -h; s = 0.5; break;
    case 6: c = -1.0; s = 0.0; break;
    case 7: c = -h; s = -0.5; break;
    case 8: c = -0.5; s = -h; break;
    case 9: c = 0.0; s = -1.0; break;
    case 10: c = 0.5; s = -h; break;
    default: c = h; s = -0.5; break;
  }
  return {c, INV ? s : -s};
}

// 12-point DFT in registers: n = 3 a + b (a < 4, b < 3), k = k1 + 4 k2.
template <bool INV>
__device__ __forceinline__ void dft12d(cplx<double> (&v)[12]) {
  cplx<double> t[3][4];
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    cplx<double> u[4] = {v[b], v[3 + b], v[6 + b], v[9 + b]};
    dft_small<4, INV>(u);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) t[b][k1] = (b && k1) ? cmul(u[k1], w12d<INV>(b * k1)) : u[k1];
  }
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) {
    cplx<double> u[3] = {t[0][k1], t[1][k1], t[2][k1]};
    dft_small<3, INV>(u);
#pragma unroll
    for (int k2 = 0; k2 < 3; ++k2) v[k1 + 4 * k2] = u[k2];
  }
}

template <int Q, bool INV>
__device__ __forceinline__ void dft_q_d(cplx<double> (&v)[Q]) {
  if constexpr (Q == 12) dft12d<INV>(v);
  else dft_small<Q, INV>(v);
}

// Z[k] of the real-row synthesis (c2r_pre in fft.cuh) with wN = exp(-2 pi i k / N).
__device__ __forceinline__ cplx<double> c2r_pre_d(cplx<double> Xk, cplx<double> Xc,
                                                  cplx<double> wN) {
  const cplx<double> cXc = conj(Xc);
  const cplx<double> F = cadd(Xk, cXc), D = csub(Xk, cXc);
  const cplx<double> G = cmul(D, conj(wN));
  return {F.x - G.y, F.y + G.x};
}

// X[k] of the real-row analysis (r2c_post in fft.cuh), wN = exp(-2 pi i k / N).
__device__ __forceinline__ cplx<double> r2c_post_d(cplx<double> Zk, cplx<double> Zc,
                                                   cplx<double> wN) {
  const cplx<double> cZc = conj(Zc);
  const cplx<double> F = cadd(Zk, cZc), D = csub(Zk, cZc);
  const cplx<double> t = cmul(D, wN);
  return {0.5 * (F.x + t.y), 0.5 * (F.y - t.x)};
}

// Twiddle tables of the passes in shared memory, each indexed by the
// butterfly's position inside its span so that consecutive lanes read
// consecutive entries (with w = exp(-2 pi i / H)):
//   t2[r-1][jm] = w^(8 r jm), jm < Q;  t3[r-1][jm] = w^(2 r jm), jm < 4 Q;
//   t4[j] = w^j, j < 16 Q;  twN[k] = exp(-2 pi i k / (2 H)), k < H.
template <int Q>
struct W64Tw {
  const cplx<double>* t2;
  const cplx<double>* t3;
  const cplx<double>* t4;
  const cplx<double>* twN;
  static constexpr int kEntries = 3 * Q + 12 * Q + 16 * Q + 32 * Q;
};

// Fill the tables from the plan's exp(-2 pi i n / (2 H)) table (n < 2 H) at
// `sm` (kEntries complex values); threads tid, tid + T, ... of the CTA.
template <int Q>
__device__ __forceinline__ W64Tw<Q> w64_twiddles(cplx<double>* sm, const double2* tw2h, int tid,
                                                 int T) {
  constexpr int H = 32 * Q;
  cplx<double>* t2 = sm;
  cplx<double>* t3 = t2 + 3 * Q;
  cplx<double>* t4 = t3 + 12 * Q;
  cplx<double>* tn = t4 + 16 * Q;
  auto wH = [&](int e) {  // w^e = exp(-2 pi i e / H)
    const double2 v = __ldg(&tw2h[(2 * e) % (2 * H)]);
    return cplx<double>{v.x, v.y};
  };
  for (int i = tid; i < 3 * Q; i += T) t2[i] = wH(8 * (i / Q + 1) * (i % Q));
  for (int i = tid; i < 12 * Q; i += T) t3[i] = wH(2 * (i / (4 * Q) + 1) * (i % (4 * Q)));
  for (int i = tid; i < 16 * Q; i += T) t4[i] = wH(i);
  for (int i = tid; i < H; i += T) {
    const double2 v = __ldg(&tw2h[i]);
    tn[i] = {v.x, v.y};
  }
  return W64Tw<Q>{t2, t3, t4, tn};
}

// In-place transform of one row (padded layout) by the calling warp, with the
// twiddle tables of w64_twiddles.
// PRE: the row holds the half spectrum X[0..H) of a real row of length 2 H and
// the transform input is Z[k] = c2r_pre(X[k], X[H - k]) (Im X[0] dropped,
// X[H] = 0); the result z[n] then carries x[2 n] + i x[2 n + 1].
template <int Q, bool INV, bool PRE>
__device__ __forceinline__ void w64_row_fft(cplx<double>* row, int lane, const W64Tw<Q>& T) {
  constexpr int H = 32 * Q;
  static_assert(Q % 4 == 0, "radix-4 passes need Q / 4 butterflies per lane");
  const cplx<double>* __restrict__ twN = T.twN;
  auto cj = [](cplx<double> w) {  // the inverse transform's conjugate twiddle
    if (INV) w.y = -w.y;
    return w;
  };
  cplx<double> v[Q];
  // pass 1: radix Q, span 1: butterfly `lane` reads x[lane + 32 r]
#pragma unroll
  for (int r = 0; r < Q; ++r) {
    const int k = lane + 32 * r;
    cplx<double> x = row[pad16(k)];
    if constexpr (PRE) {
      cplx<double> xc = row[pad16((H - k) % H)];
      if (k == 0) {
        x.y = 0.0;
        xc = {0.0, 0.0};
      }
      x = c2r_pre_d(x, xc, twN[k]);
    }
    v[r] = x;
  }
  __syncwarp();
  dft_q_d<Q, INV>(v);
#pragma unroll
  for (int r = 0; r < Q; ++r) row[pad16(lane * Q + r)] = v[r];
  __syncwarp();
  // pass 2: radix 4, span Q: butterfly j reads x[j + 8 Q r], twiddle w^(8 r (j % Q))
  constexpr int NB4 = Q / 4;
#pragma unroll
  for (int it = 0; it < NB4; ++it)
#pragma unroll
    for (int r = 0; r < 4; ++r) v[4 * it + r] = row[pad16(lane + 32 * it + 8 * Q * r)];
  __syncwarp();
#pragma unroll
  for (int it = 0; it < NB4; ++it) {
    const int j = lane + 32 * it, jm = j % Q;
    cplx<double> u[4] = {v[4 * it], v[4 * it + 1], v[4 * it + 2], v[4 * it + 3]};
#pragma unroll
    for (int r = 1; r < 4; ++r) u[r] = cmul(u[r], cj(T.t2[(r - 1) * Q + jm]));
    dft_small<4, INV>(u);
    const int d = (j - jm) * 4 + jm;
#pragma unroll
    for (int r = 0; r < 4; ++r) row[pad16(d + r * Q)] = u[r];
  }
  __syncwarp();
  // pass 3: radix 4, span 4 Q: butterfly j reads x[j + 8 Q r], twiddle w^(2 r (j % 4Q))
#pragma unroll
  for (int it = 0; it < NB4; ++it)
#pragma unroll
    for (int r = 0; r < 4; ++r) v[4 * it + r] = row[pad16(lane + 32 * it + 8 * Q * r)];
  __syncwarp();
#pragma unroll
  for (int it = 0; it < NB4; ++it) {
    const int j = lane + 32 * it, jm = j % (4 * Q);
    cplx<double> u[4] = {v[4 * it], v[4 * it + 1], v[4 * it + 2], v[4 * it + 3]};
#pragma unroll
    for (int r = 1; r < 4; ++r) u[r] = cmul(u[r], cj(T.t3[(r - 1) * 4 * Q + jm]));
    dft_small<4, INV>(u);
    const int d = (j - jm) * 4 + jm;
#pragma unroll
    for (int r = 0; r < 4; ++r) row[pad16(d + r * 4 * Q)] = u[r];
  }
  __syncwarp();
  // pass 4: radix 2, span 16 Q: butterfly j < 16 Q maps x[j], x[j + 16 Q] onto
  // themselves with twiddle w^j on the second input
#pragma unroll
  for (int it = 0; it < Q / 2; ++it) {
    const int j = lane + 32 * it;
    cplx<double> u[2] = {row[pad16(j)], cmul(row[pad16(j + 16 * Q)], cj(T.t4[j]))};
    dft_small<2, INV>(u);
    row[pad16(j)] = u[0];
    row[pad16(j + 16 * Q)] = u[1];
  }
  __syncwarp();
}

}  // namespace mt
