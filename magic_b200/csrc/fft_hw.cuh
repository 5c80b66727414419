// Half-warp FFTs of the phi stage for row lengths H = 16 Q, Q in {8, 12, 16, 24}
// (n_phi = 256, 384, 512, 768).
//
// One row belongs to one half-warp: lane l (0..15) holds Q values in
// registers and the row is transformed by three Stockham passes
//   radix Q (span 1), radix 4 (span Q), radix 4 (span 4 Q)
// with the same butterfly map as fft_stage (fft.cuh).  Between passes the row
// goes through shared memory and only the half-warp synchronises
// (__syncwarp), so rows of one CTA never wait for each other.  The radix-Q
// butterfly is itself a two-factor Cooley-Tukey DFT in registers (Q = A B,
// n = B a + b, k = k1 + A k2; inner twiddles W_Q^(b k1) are literals).
//
// Shared-memory layout of a row: value i at i ^ ((i >> s) & 15), s = 4 for
// Q = 8, 16 and 6 for Q = 12, 24 (two integer ops per address; for the
// pass-1 reads the xor term is a constant).  Enumerating the lane addresses of
// every access of the passes, the real-row pre/post steps and a warp reading
// 32 consecutive values gives 1.14 to 1.32 shared-memory wavefronts per
// half-warp access on average (1 is conflict-free); rows are H + 1 values
// apart so scatters across rows do not collide either.
#pragma once

#include "fft.cuh"

namespace mt {

template <int Q>
__device__ __forceinline__ int hw_swz(int i) {
  constexpr int sh = (Q == 8 || Q == 16) ? 4 : 6;
  return i ^ ((i >> sh) & 15);
}

// hw_swz(lane + 16 t) for lane < 16 and a compile-time t: the xor mask then
// depends on t only, so the address is (lane ^ const) + const.
template <int Q>
__device__ __forceinline__ int hw_swz16(int lane, int t) {
  constexpr int sh = (Q == 8 || Q == 16) ? 4 : 6;
  return (lane ^ ((t >> (sh - 4)) & 15)) + 16 * t;
}

// exp(-2 pi i e / 24) (forward) or its conjugate; e is a constant after
// unrolling, so the switch folds to literals (cos/sin of multiples of 15 deg).
template <bool INV>
__device__ __forceinline__ cplx<float> w24(int e) {
  e %= 24;
  const bool neg = e >= 12;
  if (neg) e -= 12;
  float c, s;
  switch (e) {
    case 0: c = 1.f; s = 0.f; break;
    case 1: c = 0.96592582628906829f; s = 0.25881904510252076f; break;
    case 2: c = 0.86602540378443865f; s = 0.5f; break;
    case 3: c = 0.70710678118654752f; s = 0.70710678118654752f; break;
    case 4: c = 0.5f; s = 0.86602540378443865f; break;
    case 5: c = 0.25881904510252076f; s = 0.96592582628906829f; break;
    case 6: c = 0.f; s = 1.f; break;
    case 7: c = -0.25881904510252076f; s = 0.96592582628906829f; break;
    case 8: c = -0.5f; s = 0.86602540378443865f; break;
    case 9: c = -0.70710678118654752f; s = 0.70710678118654752f; break;
    case 10: c = -0.86602540378443865f; s = 0.5f; break;
    default: c = -0.96592582628906829f; s = 0.25881904510252076f; break;
  }
  if (neg) { c = -c; s = -s; }
  return {c, INV ? s : -s};
}

template <int A, int B, bool INV>
__device__ __forceinline__ void dft_ab(cplx<float> (&v)[A * B]) {
  constexpr int Q = A * B;
  static_assert(24 % Q == 0, "inner twiddles are multiples of 2 pi / 24");
  cplx<float> t[B][A];
#pragma unroll
  for (int b = 0; b < B; ++b) {
    cplx<float> u[A];
#pragma unroll
    for (int a = 0; a < A; ++a) u[a] = v[B * a + b];
    dft_small<A, INV>(u);
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1)
      t[b][k1] = (b && k1) ? cmul(u[k1], w24<INV>((24 / Q) * b * k1)) : u[k1];
  }
#pragma unroll
  for (int k1 = 0; k1 < A; ++k1) {
    cplx<float> u[B];
#pragma unroll
    for (int b = 0; b < B; ++b) u[b] = t[b][k1];
    dft_small<B, INV>(u);
#pragma unroll
    for (int k2 = 0; k2 < B; ++k2) v[k1 + A * k2] = u[k2];
  }
}

template <int Q, bool INV>
__device__ __forceinline__ void dft_q(cplx<float> (&v)[Q]) {
  if constexpr (Q == 8 || Q == 16) dft_small<Q, INV>(v);
  else if constexpr (Q == 12) dft_ab<4, 3, INV>(v);
  else dft_ab<8, 3, INV>(v);
}

// Z[k] of the real-row synthesis (fft.cuh, c2r_pre) with the twiddle
// wN = exp(-2 pi i k / N) already at hand.
__device__ __forceinline__ cplx<float> c2r_pre_w(cplx<float> Xk, cplx<float> Xc, cplx<float> wN) {
  const cplx<float> cXc = conj(Xc);
  const cplx<float> F = cadd(Xk, cXc), D = csub(Xk, cXc);
  const cplx<float> G = cmul(D, conj(wN));
  return {F.x - G.y, F.y + G.x};
}

// X[k] of the real-row analysis (fft.cuh, r2c_post), wN = exp(-2 pi i k / N).
__device__ __forceinline__ cplx<float> r2c_post_w(cplx<float> Zk, cplx<float> Zc, cplx<float> wN) {
  const cplx<float> cZc = conj(Zc);
  const cplx<float> F = cadd(Zk, cZc), D = csub(Zk, cZc);
  const cplx<float> t = cmul(D, wN);
  return {0.5f * (F.x + t.y), 0.5f * (F.y - t.x)};
}

// Twiddle tables of the two radix-4 passes, laid out [butterfly][r - 1] so
// that the 16 lanes read words 3 apart (no bank conflicts):
//   tw2[3 jm + r - 1] = w^(4 r jm), jm < Q;  tw3[3 j + r - 1] = w^(r j), j < 4 Q;
// w = exp(-2 pi i / H).  Filled from the N-point table tw_N (N = 2 H).
template <int Q>
__device__ __forceinline__ void hw_twiddles_to_smem(cplx<float>* tw2, cplx<float>* tw3,
                                                    cplx<float>* twN,
                                                    const double2* __restrict__ tw_N, int tid,
                                                    int nthreads) {
  constexpr int H = 16 * Q;
  for (int e = tid; e < 3 * Q + 12 * Q + H; e += nthreads) {
    int idx;
    cplx<float>* dst;
    if (e < 3 * Q) {
      idx = 2 * (4 * (e % 3 + 1) * (e / 3));
      dst = tw2 + e;
    } else if (e < 15 * Q) {
      const int q = e - 3 * Q;
      idx = 2 * ((q % 3 + 1) * (q / 3));
      dst = tw3 + q;
    } else {
      idx = e - 15 * Q;
      dst = twN + idx;
    }
    const double2 w = __ldg(&tw_N[idx]);
    *dst = {(float)w.x, (float)w.y};
  }
}

// In-place transform of one row (swizzled layout) by the 16 lanes in `mask`.
// tw2, tw3: hw_twiddles_to_smem; twN[k] = exp(-2 pi i k / (2 H)), k < H.
// PRE: the row holds the half spectrum X[0..H) of a real row of length 2 H and
// the transform input is Z[k] = c2r_pre(X[k], X[H - k]) (Im X[0] dropped,
// X[H] = 0); the result z[n] then carries x[2 n] + i x[2 n + 1].
template <int Q, bool INV, bool PRE>
__device__ __forceinline__ void hw_row_fft(cplx<float>* row, int lane, unsigned mask,
                                           const cplx<float>* __restrict__ tw2,
                                           const cplx<float>* __restrict__ tw3,
                                           const cplx<float>* __restrict__ twN) {
  constexpr int H = 16 * Q, NBF = Q / 4;
  static_assert(Q % 4 == 0, "two radix-4 passes of 4 Q butterflies over 16 lanes");
  cplx<float> v[Q];
  // pass 1: radix Q, span 1: butterfly `lane` reads x[lane + 16 r]
#pragma unroll
  for (int r = 0; r < Q; ++r) {
    const int k = lane + 16 * r;
    cplx<float> x = row[hw_swz16<Q>(lane, r)];
    if constexpr (PRE) {
      cplx<float> xc = row[hw_swz<Q>((H - k) % H)];
      if (k == 0) {
        x.y = 0.f;
        xc = {0.f, 0.f};
      }
      x = c2r_pre_w(x, xc, twN[k]);
    }
    v[r] = x;
  }
  __syncwarp(mask);
  dft_q<Q, INV>(v);
#pragma unroll
  for (int r = 0; r < Q; ++r) row[hw_swz<Q>(lane * Q + r)] = v[r];
  __syncwarp(mask);
  // pass 2: radix 4, span Q: butterfly j reads x[j + 4 Q r], twiddle w^(4 r (j % Q))
#pragma unroll
  for (int it = 0; it < NBF; ++it)
#pragma unroll
    for (int r = 0; r < 4; ++r) v[4 * it + r] = row[hw_swz16<Q>(lane, it + Q / 4 * r)];
  __syncwarp(mask);
#pragma unroll
  for (int it = 0; it < NBF; ++it) {
    const int j = lane + 16 * it, jm = j % Q;
    cplx<float> u[4] = {v[4 * it], v[4 * it + 1], v[4 * it + 2], v[4 * it + 3]};
#pragma unroll
    for (int r = 1; r < 4; ++r) {
      cplx<float> w = tw2[3 * jm + r - 1];
      if (INV) w.y = -w.y;
      u[r] = cmul(u[r], w);
    }
    dft_small<4, INV>(u);
    const int d = (j / Q) * 4 * Q + jm;
#pragma unroll
    for (int r = 0; r < 4; ++r) row[hw_swz<Q>(d + r * Q)] = u[r];
  }
  __syncwarp(mask);
  // pass 3: radix 4, span 4 Q: butterfly j reads x[j + 4 Q r], twiddle w^(r j)
#pragma unroll
  for (int it = 0; it < NBF; ++it)
#pragma unroll
    for (int r = 0; r < 4; ++r) v[4 * it + r] = row[hw_swz16<Q>(lane, it + Q / 4 * r)];
  __syncwarp(mask);
#pragma unroll
  for (int it = 0; it < NBF; ++it) {
    const int j = lane + 16 * it;
    cplx<float> u[4] = {v[4 * it], v[4 * it + 1], v[4 * it + 2], v[4 * it + 3]};
#pragma unroll
    for (int r = 1; r < 4; ++r) {
      cplx<float> w = tw3[3 * j + r - 1];
      if (INV) w.y = -w.y;
      u[r] = cmul(u[r], w);
    }
    dft_small<4, INV>(u);
#pragma unroll
    for (int r = 0; r < 4; ++r) row[hw_swz16<Q>(lane, it + Q / 4 * r)] = u[r];
  }
  __syncwarp(mask);
}

}  // namespace mt
