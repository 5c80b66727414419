// Shared-memory FFTs of the phi stage.
//
// Each real field row of length N = n_phi is transformed on its own through a
// complex FFT of half length H = N/2 (z_n = x_2n + i x_2n+1), so rounding of
// one field never leaks into another (packing two different fields into one
// complex FFT does: the smaller field inherits eps * |larger field|).
//
// Complex FFTs: mixed-radix (2, 3, 4, 5, 8) Stockham autosort, out of place
// between a row batch and a scratch buffer in shared memory.  Stage s with
// radix R and span Ns (product of the previous radices) maps butterfly j as
//   in : x[j + r H/R] * w^(r (j % Ns) H/(Ns R)),  r < R
//   out: y[(j/Ns) Ns R + j % Ns + r Ns] = DFT_R(in)[r]
// (Govindaraju et al., "High performance discrete Fourier transforms on
// graphics processors", SC08).  Shared-memory index i is stored at
// i + (i >> 4) (one pad slot per 16) so the stride-R scatters of the first
// stages do not serialise on banks.  Forward uses w = exp(-2 pi i/H);
// inverse the conjugate, unnormalised.
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

namespace mt {

template <typename R>
struct cplx {
  R x, y;
};

template <typename R>
__device__ __forceinline__ cplx<R> cmul(cplx<R> a, cplx<R> b) {
  return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename R>
__device__ __forceinline__ cplx<R> cadd(cplx<R> a, cplx<R> b) { return {a.x + b.x, a.y + b.y}; }
template <typename R>
__device__ __forceinline__ cplx<R> csub(cplx<R> a, cplx<R> b) { return {a.x - b.x, a.y - b.y}; }
template <typename R>
__device__ __forceinline__ cplx<R> conj(cplx<R> a) { return {a.x, -a.y}; }
// multiply by -i (forward) or +i (inverse)
template <bool INV, typename R>
__device__ __forceinline__ cplx<R> mul_mi(cplx<R> a) {
  return INV ? cplx<R>{-a.y, a.x} : cplx<R>{a.y, -a.x};
}

__device__ __forceinline__ int pad16(int i) { return i + (i >> 4); }
__host__ __device__ constexpr int padded_len(int n) { return n + (n >> 4) + 1; }

// exp(-+ 2 pi i q / 8), q in 1..3 (used inside radix-8 and radix-16)
template <bool INV, typename R>
__device__ __forceinline__ cplx<R> rot8(cplx<R> a, int q) {
  const R h = (R)0.70710678118654752440;
  if (q == 1) {  // w8^1 = (1 - i)/sqrt2 forward
    return INV ? cplx<R>{h * (a.x - a.y), h * (a.x + a.y)} : cplx<R>{h * (a.x + a.y), h * (a.y - a.x)};
  }
  if (q == 2) return mul_mi<INV>(a);
  // q == 3: w8^3 = (-1 - i)/sqrt2 forward
  return INV ? cplx<R>{-h * (a.x + a.y), h * (a.x - a.y)} : cplx<R>{h * (a.y - a.x), -h * (a.x + a.y)};
}

template <bool INV, typename R>
__device__ __forceinline__ void dft4(cplx<R>& a, cplx<R>& b, cplx<R>& c, cplx<R>& d) {
  cplx<R> s0 = cadd(a, c), d0 = csub(a, c);
  cplx<R> s1 = cadd(b, d), d1 = mul_mi<INV>(csub(b, d));
  a = cadd(s0, s1);
  b = cadd(d0, d1);
  c = csub(s0, s1);
  d = csub(d0, d1);
}

// exp(-+ i pi q / 8) * a for the radix-16 inner twiddles, q in {1,2,3,4,6,9}
template <bool INV, int Q, typename R>
__device__ __forceinline__ cplx<R> rot16(cplx<R> a) {
  const R c = (R)0.92387953251128675613, s = (R)0.38268343236508977173;  // cos/sin(pi/8)
  const R h = (R)0.70710678118654752440;
  R cr, si;
  if constexpr (Q == 1) { cr = c; si = s; }
  else if constexpr (Q == 2) { cr = h; si = h; }
  else if constexpr (Q == 3) { cr = s; si = c; }
  else if constexpr (Q == 4) { cr = 0; si = 1; }
  else if constexpr (Q == 6) { cr = -h; si = h; }
  else { cr = -c; si = -s; }  // Q == 9
  const R sg = INV ? si : -si;  // forward: exp(-i x) = cos x - i sin x
  return {a.x * cr - a.y * sg, a.x * sg + a.y * cr};
}

template <int RADIX, bool INV, typename R>
__device__ __forceinline__ void dft_small(cplx<R> (&v)[RADIX]) {
  if constexpr (RADIX == 2) {
    cplx<R> a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if constexpr (RADIX == 3) {
    const R s3 = (R)0.86602540378443864676;  // sin(2 pi / 3)
    cplx<R> a = v[0], b = v[1], c = v[2];
    cplx<R> sbc = cadd(b, c), dbc = csub(b, c);
    cplx<R> t = {a.x - (R)0.5 * sbc.x, a.y - (R)0.5 * sbc.y};
    cplx<R> u = mul_mi<INV>(cplx<R>{s3 * dbc.x, s3 * dbc.y});
    v[0] = cadd(a, sbc);
    v[1] = cadd(t, u);
    v[2] = csub(t, u);
  } else if constexpr (RADIX == 4) {
    dft4<INV>(v[0], v[1], v[2], v[3]);
  } else if constexpr (RADIX == 5) {
    const R c1 = (R)0.30901699437494742410;   // cos(2 pi/5)
    const R c2 = (R)-0.80901699437494742410;  // cos(4 pi/5)
    const R s1 = (R)0.95105651629515357212;   // sin(2 pi/5)
    const R s2 = (R)0.58778525229247312917;   // sin(4 pi/5)
    cplx<R> a = v[0];
    cplx<R> p1 = cadd(v[1], v[4]), m1 = csub(v[1], v[4]);
    cplx<R> p2 = cadd(v[2], v[3]), m2 = csub(v[2], v[3]);
    cplx<R> t1 = {a.x + c1 * p1.x + c2 * p2.x, a.y + c1 * p1.y + c2 * p2.y};
    cplx<R> t2 = {a.x + c2 * p1.x + c1 * p2.x, a.y + c2 * p1.y + c1 * p2.y};
    cplx<R> u1 = mul_mi<INV>(cplx<R>{s1 * m1.x + s2 * m2.x, s1 * m1.y + s2 * m2.y});
    cplx<R> u2 = mul_mi<INV>(cplx<R>{s2 * m1.x - s1 * m2.x, s2 * m1.y - s1 * m2.y});
    v[0] = {a.x + p1.x + p2.x, a.y + p1.y + p2.y};
    v[1] = cadd(t1, u1);
    v[4] = csub(t1, u1);
    v[2] = cadd(t2, u2);
    v[3] = csub(t2, u2);
  } else if constexpr (RADIX == 8) {
    // 8 = 2 x 4: y[k1 + 2 k2] from two radix-4 DFTs of even/odd inputs
    cplx<R> e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    cplx<R> o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4<INV>(e0, e1, e2, e3);
    dft4<INV>(o0, o1, o2, o3);
    o1 = rot8<INV>(o1, 1);
    o2 = rot8<INV>(o2, 2);
    o3 = rot8<INV>(o3, 3);
    v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
    v[1] = cadd(e1, o1); v[5] = csub(e1, o1);
    v[2] = cadd(e2, o2); v[6] = csub(e2, o2);
    v[3] = cadd(e3, o3); v[7] = csub(e3, o3);
  } else if constexpr (RADIX == 16) {
    // 16 = 4 x 4: inner DFT4 over n2 (stride 4), twiddle w16^(n1 k2), outer DFT4 over n1
#pragma unroll
    for (int n1 = 0; n1 < 4; ++n1) dft4<INV>(v[n1], v[n1 + 4], v[n1 + 8], v[n1 + 12]);
    // v[n1 + 4 k2] now holds T[n1][k2]
    v[5] = rot16<INV, 1>(v[5]);
    v[9] = rot16<INV, 2>(v[9]);
    v[13] = rot16<INV, 3>(v[13]);
    v[6] = rot16<INV, 2>(v[6]);
    v[10] = rot16<INV, 4>(v[10]);
    v[14] = rot16<INV, 6>(v[14]);
    v[7] = rot16<INV, 3>(v[7]);
    v[11] = rot16<INV, 6>(v[11]);
    v[15] = rot16<INV, 9>(v[15]);
    // outer DFT4 over n1 for each k2: inputs v[4 k2 + n1]; outputs y[k2 + 4 k1]
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) dft4<INV>(v[4 * k2], v[4 * k2 + 1], v[4 * k2 + 2], v[4 * k2 + 3]);
    // v[4 k2 + k1] holds y[k2 + 4 k1]: transpose 4x4 in registers
    cplx<R> t;
    t = v[1]; v[1] = v[4]; v[4] = t;
    t = v[2]; v[2] = v[8]; v[8] = t;
    t = v[3]; v[3] = v[12]; v[12] = t;
    t = v[6]; v[6] = v[9]; v[9] = t;
    t = v[7]; v[7] = v[13]; v[13] = t;
    t = v[11]; v[11] = v[14]; v[14] = t;
  }
}

// floor(n / d) for 0 <= n < 2^22 from a float reciprocal of d (exact in this
// range: the product is off by < 2^-24 relative, far below the 0.5/d margin).
__device__ __forceinline__ int fdiv(int n, float rcp) {
  return __float2int_rd(((float)n + 0.5f) * rcp);
}

// One out-of-place Stockham stage over `nrows` rows of length H: src rows at
// src + row * stride, dst rows at dst + row * stride (padded indexing).
// tw: this stage's twiddles in shared memory, tw[(r - 1) Ns + jm] =
// exp(-2 pi i r jm / (Ns RADIX)) (fft_twiddles_to_smem), so that threads with
// consecutive butterflies read consecutive entries.
template <int RADIX, bool INV, typename R>
__device__ __forceinline__ void fft_stage(const cplx<R>* __restrict__ src, cplx<R>* __restrict__ dst,
                                          int nrows, int H, int stride, int Ns,
                                          const cplx<R>* __restrict__ tw) {
  const int nbr = H / RADIX;
  const int total = nrows * nbr;
  const float rcp_nbr = 1.0f / (float)nbr, rcp_ns = 1.0f / (float)Ns;
  for (int b = threadIdx.x; b < total; b += blockDim.x) {
    const int row = fdiv(b, rcp_nbr), j = b - row * nbr;
    const cplx<R>* x = src + row * stride;
    const int jm = j - fdiv(j, rcp_ns) * Ns;
    cplx<R> v[RADIX];
#pragma unroll
    for (int r = 0; r < RADIX; ++r) v[r] = x[pad16(j + r * nbr)];
    if (jm > 0) {
#pragma unroll
      for (int r = 1; r < RADIX; ++r) {
        cplx<R> w = tw[(r - 1) * Ns + jm];
        if (INV) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    dft_small<RADIX, INV>(v);
    cplx<R>* y = dst + row * stride;
    const int d = (j - jm) * RADIX + jm;
#pragma unroll
    for (int r = 0; r < RADIX; ++r) y[pad16(d + r * Ns)] = v[r];
  }
  __syncthreads();
}

constexpr int kFftRowBatch = 7;  // rows per pass through the scratch buffer

// Full transform of `nrows` rows (in place), ping-ponging each batch of at
// most kFftRowBatch rows through `scratch` (kFftRowBatch * stride values).
// Radices come from the plan (product H, each of 2, 3, 4, 5, 8); tw holds the
// stages' twiddle tables one after another (fft_twiddles_to_smem, H - 1 values).
template <bool INV, typename R>
__device__ __forceinline__ void fft_rows(cplx<R>* buf, cplx<R>* scratch, int nrows, int H,
                                         int stride, const int* radix, int nstages,
                                         const cplx<R>* __restrict__ tw) {
  for (int r0 = 0; r0 < nrows; r0 += kFftRowBatch) {
    cplx<R>* a = buf + r0 * stride;
    cplx<R>* b = scratch;
    const int nr = min(kFftRowBatch, nrows - r0);
    int Ns = 1, off = 0;
    for (int s = 0; s < nstages; ++s) {
      int rad = radix[s];
      const cplx<R>* tws = tw + off;
      switch (rad) {
        case 8: fft_stage<8, INV>(a, b, nr, H, stride, Ns, tws); break;
        case 4: fft_stage<4, INV>(a, b, nr, H, stride, Ns, tws); break;
        case 3: fft_stage<3, INV>(a, b, nr, H, stride, Ns, tws); break;
        case 2: fft_stage<2, INV>(a, b, nr, H, stride, Ns, tws); break;
        default: fft_stage<5, INV>(a, b, nr, H, stride, Ns, tws); break;
      }
      off += (rad - 1) * Ns;
      Ns *= rad;
      cplx<R>* t = a;
      a = b;
      b = t;
    }
    if (a != buf + r0 * stride) {  // odd number of stages: result is in scratch
      cplx<R>* d = buf + r0 * stride;
      for (int i = threadIdx.x; i < nr * stride; i += blockDim.x) d[i] = a[i];
      __syncthreads();
    }
  }
}

// The stages' twiddle tables of fft_rows into shared memory, one after another
// (H - 1 values in all): stage s of radix R and span Ns (the product of the
// earlier radices) gets exp(-2 pi i r jm / (Ns R)) at (r - 1) Ns + jm, r < R,
// jm < Ns, read from the plan's table tw_N[n] = exp(-2 pi i n / (2 H)) at
// n = 2 r jm H / (Ns R).  Caller syncs.
template <typename R>
__device__ __forceinline__ void fft_twiddles_to_smem(cplx<R>* tws, int H,
                                                     const double2* __restrict__ tw_N,
                                                     const int* radix, int nstages) {
  int Ns = 1, off = 0;
  for (int s = 0; s < nstages; ++s) {
    const int rad = radix[s], n = (rad - 1) * Ns, step = H / (Ns * rad);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const int r = i / Ns + 1, jm = i - (r - 1) * Ns;
      const double2 w = __ldg(&tw_N[2 * r * jm * step]);
      tws[off + i] = {(R)w.x, (R)w.y};
    }
    off += n;
    Ns *= rad;
  }
}

// 16-byte global -> shared copy that does not hold a register (cp.async).
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src));
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::);
}

// ---- real rows through half-length complex FFTs --------------------------
//
// Synthesis (irfft, norm="forward", unnormalised): from the half spectrum X
// (X[k] for k < n_m, zero above, Im X[0] ignored) form, for k in [0, H),
//   Z[k] = (X[k] + conj X[H-k]) + i (X[k] - conj X[H-k]) exp(+2 pi i k/N)
// then z = ifft_H(Z) and x[2n] = Re z[n], x[2n+1] = Im z[n].
// Analysis (rfft, norm="forward"), for k < n_m, with Z = fft_H(z):
//   X[k] = (Z[k] + conj Z[H-k]) / 2 - (i/2) exp(-2 pi i k/N) (Z[k] - conj Z[H-k]).
// tw: exp(-2 pi i n/N), n < N.

// Z[k] for one k of a row whose half spectrum is Xk = X[k], Xc = X[H-k].
template <typename R>
__device__ __forceinline__ cplx<R> c2r_pre(cplx<R> Xk, cplx<R> Xc, int k,
                                           const double2* __restrict__ tw) {
  cplx<R> cXc = conj(Xc);
  cplx<R> F = cadd(Xk, cXc);
  cplx<R> D = csub(Xk, cXc);
  double2 w = __ldg(&tw[k]);
  cplx<R> e = {(R)w.x, (R)-w.y};  // exp(+2 pi i k/N)
  cplx<R> G = cmul(D, e);
  return {F.x - G.y, F.y + G.x};  // F + i G
}

template <typename R>
__device__ __forceinline__ cplx<R> r2c_post(cplx<R> Zk, cplx<R> Zc, int k,
                                            const double2* __restrict__ tw) {
  cplx<R> cZc = conj(Zc);
  cplx<R> F = cadd(Zk, cZc);   // 2 F
  cplx<R> D = csub(Zk, cZc);   // 2 i G
  double2 w = __ldg(&tw[k]);
  cplx<R> e = {(R)w.x, (R)w.y};  // exp(-2 pi i k/N)
  cplx<R> t = cmul(D, e);
  // X = F - (i/2) e D  with the factor 1/2 on both terms
  return {(R)0.5 * (F.x + t.y), (R)0.5 * (F.y - t.x)};
}

}  // namespace mt
