// Warp FFTs of the FP64 phi stage for row lengths H = 32 Q, Q in {4, 8, 12, 16}
// (n_phi = 256, 512, 768, 1024).
//
// One row belongs to one warp: lane l holds Q complex doubles in registers and
// the row goes through four Stockham passes with the butterfly map of
// fft_stage (fft.cuh):
//   radix Q (span 1), radix 4 (span Q), radix 4 (span 4 Q), radix 2 (span 16 Q),
// Q x 4 x 4 x 2 = H.  Between passes the row lives in shared memory and only
// the warp synchronises (__syncwarp), so rows of one CTA never wait for each
// other.  The radix-12 butterfly is a two-factor DFT (12 = 4 x 3) with
// literal inner twiddles.
//
// Shared-memory layout of a row: element i sits at w64_pos<Q>(i).  A warp's
// 16-byte accesses go to the banks a quarter warp at a time, eight slots per
// pass over the 32 banks.  For Q = 4, 8, 12 the slot of i within its group of
// eight is XORed with the group number (its low two bits; three for Q = 8),
// so that the stride-Q scatter of the first pass (eight lanes whose indices
// agree modulo 8 in pairs or all together) lands on distinct slots while every
// aligned run of eight (the other passes' reads and writes) stays
// conflict-free.  The pattern repeats every four groups (eight for Q = 8), so
// an index shift by a multiple of 32 (64) moves an element by the same amount
// and the strided reads use one per-lane base with constant offsets.  For
// Q = 16 the stride-16 scatter is conflict-free with one pad slot per 16
// (i + i / 16).
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

// Shared-memory position of element i (< H) of a row (see the file comment).
template <int Q>
__device__ __forceinline__ int w64_pos(int i) {
  if constexpr (Q == 16) return pad16(i);
  else if constexpr (Q == 8) return i ^ ((i >> 3) & 7);
  else return i ^ ((i >> 3) & 3);
}

// Whether an index shift by c moves every element by w64_disp<Q>(c), and by
// how much (c a compile-time constant after unrolling).
template <int Q>
__host__ __device__ constexpr bool w64_shift_ok(int c) {
  return Q == 16 ? c % 16 == 0 : Q == 8 ? c % 64 == 0 : c % 32 == 0;
}
template <int Q>
__host__ __device__ constexpr int w64_disp(int c) {
  return Q == 16 ? c + c / 16 : c;
}

// Element base + c of a row, base < 32 with position pb = w64_pos<Q>(base).
template <int Q>
__device__ __forceinline__ cplx<double>& w64_at(cplx<double>* row, int base, int pb, int c) {
  return w64_shift_ok<Q>(c) ? row[pb + w64_disp<Q>(c)] : row[w64_pos<Q>(base + c)];
}

// Slots of a row, plus one so that rows S apart start on different bank
// quads (the load and store phases touch several rows in one warp access).
template <int Q>
__host__ __device__ constexpr int w64_row_stride() {
  return Q == 16 ? padded_len(32 * Q) : 32 * Q + 1;
}

// exp(-2 pi i e / 16) (forward) or its conjugate, e < 8 a compile-time
// constant after unrolling (cos/sin of multiples of 22.5 degrees).
template <bool INV>
__device__ __forceinline__ cplx<double> w16d(int e) {
  const double c1 = 0.92387953251128675613, s1 = 0.38268343236508977173;  // 22.5 deg
  const double h = 0.70710678118654752440;
  double c, s;
  switch (e) {
    case 0: c = 1.0; s = 0.0; break;
    case 1: c = c1; s = s1; break;
    case 2: c = h; s = h; break;
    case 3: c = s1; s = c1; break;
    case 4: c = 0.0; s = 1.0; break;
    case 5: c = -s1; s = c1; break;
    case 6: c = -h; s = h; break;
    default: c = -c1; s = s1; break;
  }
  return {c, INV ? s : -s};
}

// exp(-2 pi i it / Q) (forward) for it < Q / 2: the factor between w^(lane)
// and w^(lane + 32 it), w = exp(-2 pi i / H).
template <int Q>
__device__ __forceinline__ cplx<double> w64_root(int it) {
  if constexpr (Q == 12) return w12d<false>(it);
  else return w16d<false>(it * (16 / Q));
}

// Twiddle tables in shared memory, each read so that the eight lanes of a
// quarter warp see eight distinct slots (w = exp(-2 pi i / H)):
//   t2[p] = w^(8 (p % Q)), p < Q + 8: pass 2's w^(8 jm), jm = j % Q, read at
//     p = (j & ~7) % Q + (j & 7) (the quarter's window of eight consecutive
//     jm, unwrapped);
//   t3[jm] = w^(2 jm), jm < 4 Q: pass 3's base twiddle;
//   wl[l] = w^l, l < 32: pass 4's w^j = wl[lane] exp(-2 pi i it / Q);
//   twN[k] = exp(-2 pi i k / (2 H)), k < H: the real-row pre/post-processing.
// The butterflies raise the base twiddle u to u^2 and u^3 by complex
// multiplication (one rounding each) instead of reading three tables.
template <int Q>
struct W64Tw {
  const cplx<double>* t2;
  const cplx<double>* t3;
  const cplx<double>* wl;
  const cplx<double>* twN;
  static constexpr int kEntries = (Q + 8) + 4 * Q + 32 + 32 * Q;
};

// Fill the tables from the plan's exp(-2 pi i n / (2 H)) table (n < 2 H) at
// `sm` (kEntries complex values) with asynchronous 16-byte copies issued by
// threads tid, tid + T, ... of the CTA; the caller waits for its copies
// (cp_async_wait_all) and synchronises the CTA before the tables are read.
template <int Q>
__device__ __forceinline__ W64Tw<Q> w64_twiddles(cplx<double>* sm, const double2* tw2h, int tid,
                                                 int T) {
  constexpr int H = 32 * Q;
  cplx<double>* t2 = sm;
  cplx<double>* t3 = t2 + (Q + 8);
  cplx<double>* wl = t3 + 4 * Q;
  cplx<double>* tn = wl + 32;
  auto wH = [&](int e) { return &tw2h[(2 * e) % (2 * H)]; };  // w^e = exp(-2 pi i e / H)
  for (int i = tid; i < Q + 8; i += T) cp_async16(&t2[i], wH(8 * (i % Q)));
  for (int i = tid; i < 4 * Q; i += T) cp_async16(&t3[i], wH(2 * i));
  for (int i = tid; i < 32; i += T) cp_async16(&wl[i], wH(i));
  for (int i = tid; i < H; i += T) cp_async16(&tn[i], &tw2h[i]);
  return W64Tw<Q>{t2, t3, wl, tn};
}

// u[r] *= w^r (forward) or conj(w)^r (inverse), r = 1, 2, 3, from the base
// twiddle w: the powers by complex multiplication, one rounding each.
template <bool INV>
__device__ __forceinline__ void twiddle3(cplx<double> (&u)[4], cplx<double> w) {
  if (INV) w.y = -w.y;
  u[1] = cmul(u[1], w);
  const cplx<double> w2 = cmul(w, w);
  u[2] = cmul(u[2], w2);
  u[3] = cmul(u[3], cmul(w2, w));
}

// In-place transform of one row (layout w64_pos) by the calling warp, with
// the twiddles of w64_twiddles.  The forward transform of the analysis takes
// z[n] = x[2 n] + i x[2 n + 1]; the inverse of the synthesis takes the
// pre-processed half spectrum Z[k] (c2r_pre_d), so that z[n] again carries
// x[2 n] + i x[2 n + 1].
template <int Q, bool INV>
__device__ __forceinline__ void w64_row_fft(cplx<double>* row, int lane, const W64Tw<Q>& T) {
  static_assert(Q % 4 == 0, "radix-4 passes need Q / 4 butterflies per lane");
  auto cj = [](cplx<double> w) {  // the inverse transform's conjugate twiddle
    if (INV) w.y = -w.y;
    return w;
  };
  cplx<double> v[Q];
  const int pl = w64_pos<Q>(lane);
  // pass 1: radix Q, span 1: butterfly `lane` reads x[lane + 32 r]
#pragma unroll
  for (int r = 0; r < Q; ++r) v[r] = w64_at<Q>(row, lane, pl, 32 * r);
  __syncwarp();
  dft_q_d<Q, INV>(v);
#pragma unroll
  for (int r = 0; r < Q; ++r) row[w64_pos<Q>(lane * Q + r)] = v[r];
  __syncwarp();
  // pass 2: radix 4, span Q: butterfly j reads x[j + 8 Q r], twiddle w^(8 r (j % Q))
  constexpr int NB4 = Q / 4;
#pragma unroll
  for (int it = 0; it < NB4; ++it)
#pragma unroll
    for (int r = 0; r < 4; ++r) v[4 * it + r] = w64_at<Q>(row, lane, pl, 32 * it + 8 * Q * r);
  __syncwarp();
#pragma unroll
  for (int it = 0; it < NB4; ++it) {
    const int j = lane + 32 * it, jm = j % Q;
    cplx<double> u[4] = {v[4 * it], v[4 * it + 1], v[4 * it + 2], v[4 * it + 3]};
    twiddle3<INV>(u, T.t2[(j & ~7) % Q + (j & 7)]);
    dft_small<4, INV>(u);
    const int d = (j - jm) * 4 + jm;
#pragma unroll
    for (int r = 0; r < 4; ++r) row[w64_pos<Q>(d + r * Q)] = u[r];
  }
  __syncwarp();
  // pass 3: radix 4, span 4 Q: butterfly j reads x[j + 8 Q r], twiddle w^(2 r (j % 4Q))
#pragma unroll
  for (int it = 0; it < NB4; ++it)
#pragma unroll
    for (int r = 0; r < 4; ++r) v[4 * it + r] = w64_at<Q>(row, lane, pl, 32 * it + 8 * Q * r);
  __syncwarp();
#pragma unroll
  for (int it = 0; it < NB4; ++it) {
    const int j = lane + 32 * it, jm = j % (4 * Q);
    cplx<double> u[4] = {v[4 * it], v[4 * it + 1], v[4 * it + 2], v[4 * it + 3]};
    twiddle3<INV>(u, T.t3[jm]);
    dft_small<4, INV>(u);
    const int d = (j - jm) * 4 + jm;
#pragma unroll
    for (int r = 0; r < 4; ++r) row[w64_pos<Q>(d + r * 4 * Q)] = u[r];
  }
  __syncwarp();
  // pass 4: radix 2, span 16 Q: butterfly j < 16 Q maps x[j], x[j + 16 Q] onto
  // themselves with twiddle w^j on the second input
  const cplx<double> wl = T.wl[lane];
#pragma unroll
  for (int it = 0; it < Q / 2; ++it) {
    const int j = lane + 32 * it;
    const cplx<double> w = cj(it ? cmul(wl, w64_root<Q>(it)) : wl);
    cplx<double>& x0 = w64_at<Q>(row, lane, pl, 32 * it);
    cplx<double>& x1 = w64_at<Q>(row, lane, pl, 32 * it + 16 * Q);
    cplx<double> u[2] = {x0, cmul(x1, w)};
    dft_small<2, INV>(u);
    x0 = u[0];
    x1 = u[1];
  }
  __syncwarp();
}

}  // namespace mt
