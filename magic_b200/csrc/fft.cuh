// Shared-memory mixed-radix (2, 3, 4, 5) complex FFT used by the phi stage.
//
// In-place Stockham autosort: every stage reads each element once into
// registers, the block synchronises, then writes each element once, so one
// buffer per row suffices.  Stage s with radix R and span Ns (product of the
// previous radices) maps butterfly j of a row as
//   in : x[j + r N/R] * w^(r (j % Ns) N/(Ns R)),  r < R
//   out: y[(j/Ns) Ns R + j % Ns + r Ns] = DFT_R(in)[r]
// (Govindaraju et al., "High performance discrete Fourier transforms on
// graphics processors", SC08).  Forward uses w = exp(-2 pi i/N); inverse the
// conjugate, unnormalised.
#pragma once

#include <cuda_runtime.h>

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
// multiply by -i (forward) or +i (inverse): INV=false -> -i
template <bool INV, typename R>
__device__ __forceinline__ cplx<R> mul_mi(cplx<R> a) {
  return INV ? cplx<R>{-a.y, a.x} : cplx<R>{a.y, -a.x};
}

template <int RADIX, bool INV, typename R>
__device__ __forceinline__ void dft_small(cplx<R>* v) {
  if constexpr (RADIX == 2) {
    cplx<R> a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if constexpr (RADIX == 3) {
    const R s3 = (R)0.86602540378443864676;  // sin(2 pi / 3)
    cplx<R> a = v[0], b = v[1], c = v[2];
    cplx<R> sbc = cadd(b, c), dbc = csub(b, c);
    cplx<R> t = {a.x - (R)0.5 * sbc.x, a.y - (R)0.5 * sbc.y};
    cplx<R> u = mul_mi<INV>(cplx<R>{s3 * dbc.x, s3 * dbc.y});  // -i s3 (b-c) fwd
    v[0] = cadd(a, sbc);
    v[1] = cadd(t, u);
    v[2] = csub(t, u);
  } else if constexpr (RADIX == 4) {
    cplx<R> a = v[0], b = v[1], c = v[2], d = v[3];
    cplx<R> s0 = cadd(a, c), d0 = csub(a, c);
    cplx<R> s1 = cadd(b, d), d1 = mul_mi<INV>(csub(b, d));
    v[0] = cadd(s0, s1);
    v[1] = cadd(d0, d1);
    v[2] = csub(s0, s1);
    v[3] = csub(d0, d1);
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
    // forward: y1 = t1 - i (s1 m1 + s2 m2), y2 = t2 - i (s2 m1 - s1 m2)
    cplx<R> u1 = mul_mi<INV>(cplx<R>{s1 * m1.x + s2 * m2.x, s1 * m1.y + s2 * m2.y});
    cplx<R> u2 = mul_mi<INV>(cplx<R>{s2 * m1.x - s1 * m2.x, s2 * m1.y - s1 * m2.y});
    v[0] = {a.x + p1.x + p2.x, a.y + p1.y + p2.y};
    v[1] = cadd(t1, u1);
    v[4] = csub(t1, u1);
    v[2] = cadd(t2, u2);
    v[3] = csub(t2, u2);
  }
}

// One Stockham stage of radix RADIX over `nrows` rows of length N stored at
// buf + row * stride.  CAP bounds the elements a thread holds (nrows * N <=
// CAP * blockDim.x, checked by the caller at plan time).
template <int RADIX, bool INV, int CAP, typename R>
__device__ __forceinline__ void fft_stage(cplx<R>* buf, int nrows, int N, int stride, int Ns,
                                          const double2* __restrict__ tw) {
  constexpr int MAXB = (CAP + RADIX - 1) / RADIX;
  const int nbr = N / RADIX;
  const int total = nrows * nbr;
  const int twstep = N / (Ns * RADIX);
  cplx<R> v[MAXB][RADIX];
#pragma unroll
  for (int i = 0; i < MAXB; ++i) {
    int b = threadIdx.x + i * blockDim.x;
    if (b < total) {
      int row = b / nbr, j = b - row * nbr;
      const cplx<R>* x = buf + row * stride;
      int jm = j % Ns;
#pragma unroll
      for (int r = 0; r < RADIX; ++r) {
        cplx<R> e = x[j + r * nbr];
        if (r > 0 && jm > 0) {
          double2 w = __ldg(&tw[r * jm * twstep]);
          cplx<R> ww = {(R)w.x, INV ? (R)-w.y : (R)w.y};
          e = cmul(e, ww);
        }
        v[i][r] = e;
      }
      dft_small<RADIX, INV>(v[i]);
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < MAXB; ++i) {
    int b = threadIdx.x + i * blockDim.x;
    if (b < total) {
      int row = b / nbr, j = b - row * nbr;
      cplx<R>* y = buf + row * stride;
      int jm = j % Ns;
      int d = (j - jm) * RADIX + jm;
#pragma unroll
      for (int r = 0; r < RADIX; ++r) y[d + r * Ns] = v[i][r];
    }
  }
  __syncthreads();
}

// Full transform; radices from the plan (product = N).
template <bool INV, int CAP, typename R>
__device__ void fft_rows(cplx<R>* buf, int nrows, int N, int stride, const int* radix,
                         int nstages, const double2* __restrict__ tw) {
  int Ns = 1;
  for (int s = 0; s < nstages; ++s) {
    int rad = radix[s];
    switch (rad) {
      case 2: fft_stage<2, INV, CAP>(buf, nrows, N, stride, Ns, tw); break;
      case 3: fft_stage<3, INV, CAP>(buf, nrows, N, stride, Ns, tw); break;
      case 4: fft_stage<4, INV, CAP>(buf, nrows, N, stride, Ns, tw); break;
      default: fft_stage<5, INV, CAP>(buf, nrows, N, stride, Ns, tw); break;
    }
    Ns *= rad;
  }
}

}  // namespace mt
