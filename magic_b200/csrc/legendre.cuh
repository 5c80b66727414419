// Legendre-stage operation descriptors shared by the FP64 (DMMA) kernels.
//
// A synthesis operation contracts, per order m, the tables P and
// dP = sin(theta) dP/dtheta (rows l, columns northern theta) with NX complex
// input terms per column (radial level / batch entry).  Products are (table,
// term) pairs; the epilogue turns products into NO output fields.
//
// Equatorial folding (reference magic_torch/sht.py:120-149): rows with
// (l - m) even (E) and odd (O) are summed separately; then
//   P-product:  north = E + O, south = E - O
//   dP-product: north = E + O, south = O - E
// For the vector transforms the S/T form is used:
//   v_theta = dP.S + i m P.T          v_phi = i m P.S - dP.T
//   S = wdP.V_theta - i m wP.V_phi    T = -wdP.V_phi - i m wP.V_theta
// (algebraically equal to the reference's G = S - iT, C = S + iT stacks,
// magic_torch/sht.py:432-463 and :626-661).
#pragma once

#include "common.cuh"

namespace mt {

enum Table : int { kP = 0, kDP = 1 };

// Term recipes applied while loading spectral inputs (radial-loop assembly,
// magic_torch/step_time.py:980-1013).
enum Recipe : int {
  kRaw = 0,    // X = A
  kDlh = 1,    // X = l(l+1) A
  kCurlT = 2,  // X = or2[col] l(l+1) A - B
  kZero = 3    // X = 0
};

struct TermSrc {
  const double2* a;
  const double2* b;
  int recipe;
};

struct dcx {
  double x, y;
};
__device__ __forceinline__ dcx operator+(dcx a, dcx b) { return {a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ dcx operator-(dcx a, dcx b) { return {a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ dcx operator-(dcx a) { return {-a.x, -a.y}; }
__device__ __forceinline__ dcx times_im(dcx a, double m) { return {-m * a.y, m * a.x}; }  // i m a
__device__ __forceinline__ dcx scale(dcx a, double s) { return {s * a.x, s * a.y}; }

// ---------------------------------------------------------------- synthesis

struct SynScalar {
  static constexpr int NX = 1, NP = 1, NO = 1, NT = 1;
  __host__ __device__ static constexpr int table(int) { return kP; }
  __host__ __device__ static constexpr int term(int) { return 0; }
  __device__ static void combine(const dcx* h, double, dcx* o) { o[0] = h[0]; }
};

struct SynGrad {  // (dP X, i m P X) -> (d/dtheta, 1/sin d/dphi), sin-weighted
  static constexpr int NX = 1, NP = 2, NO = 2, NT = 2;
  __host__ __device__ static constexpr int table(int p) { return p == 0 ? kDP : kP; }
  __host__ __device__ static constexpr int term(int) { return 0; }
  __device__ static void combine(const dcx* h, double m, dcx* o) {
    o[0] = h[0];
    o[1] = times_im(h[1], m);
  }
};

// torpol group: terms (Q, S, T) at x0..x0+2, products (P,Q) (P,S) (P,T)
// (dP,S) (dP,T) at p0..p0+4, outputs (r, theta, phi) at f0..f0+2.
__host__ __device__ constexpr int torpol_table(int q) { return q < 3 ? kP : kDP; }
__host__ __device__ constexpr int torpol_term(int q) {
  return q == 0 ? 0 : (q == 1 ? 1 : (q == 2 ? 2 : (q == 3 ? 1 : 2)));
}
__device__ __forceinline__ void torpol_combine(const dcx* h, double m, dcx* o) {
  o[0] = h[0];
  o[1] = h[3] + times_im(h[2], m);
  o[2] = times_im(h[1], m) - h[4];
}

struct SynTorpol {
  static constexpr int NX = 3, NP = 5, NO = 3, NT = 2;
  __host__ __device__ static constexpr int table(int p) { return torpol_table(p); }
  __host__ __device__ static constexpr int term(int p) { return torpol_term(p); }
  __device__ static void combine(const dcx* h, double m, dcx* o) { torpol_combine(h, m, o); }
};

// G torpol groups (terms Q, S, T each) followed by NS scalar terms.  Output
// fields: (r, theta, phi) per group, then one field per scalar.  The fused
// Boussinesq synthesis is two launches: (B, curl B) and (u, curl u, s [, xi]).
template <int G, int NS>
struct SynGroups {
  static constexpr int NX = 3 * G + NS;
  static constexpr int NP = 5 * G + NS;
  static constexpr int NO = NX, NT = 2;
  __host__ __device__ static constexpr int table(int p) {
    return p < 5 * G ? torpol_table(p % 5) : kP;
  }
  __host__ __device__ static constexpr int term(int p) {
    return p < 5 * G ? 3 * (p / 5) + torpol_term(p % 5) : 3 * G + (p - 5 * G);
  }
  __device__ static void combine(const dcx* h, double m, dcx* o) {
#pragma unroll
    for (int gi = 0; gi < G; ++gi) torpol_combine(h + 5 * gi, m, o + 3 * gi);
#pragma unroll
    for (int si = 0; si < NS; ++si) o[3 * G + si] = h[5 * G + si];
  }
};

// ----------------------------------------------------------------- analysis

struct AnaScalar {
  static constexpr int NX = 1, NP = 1, NO = 1, NT = 1;
  __host__ __device__ static constexpr int table(int) { return kP; }
  __host__ __device__ static constexpr int term(int) { return 0; }
  __device__ static void finish(const dcx* h, double, double, dcx* o) { o[0] = h[0]; }
};

// vector pair (theta field at x0, phi field at x0+1): products (dP,th) (P,ph)
// (dP,ph) (P,th); outputs S, T divided by l(l+1).
__host__ __device__ constexpr int sph_table(int q) { return (q % 2 == 0) ? kDP : kP; }
__host__ __device__ constexpr int sph_term(int q) { return (q == 0 || q == 3) ? 0 : 1; }
__device__ __forceinline__ void sph_finish(const dcx* h, double m, double inv, dcx* S, dcx* T) {
  *S = scale(h[0] - times_im(h[1], m), inv);
  *T = scale(-h[2] - times_im(h[3], m), inv);
}

struct AnaSphtor {
  static constexpr int NX = 2, NP = 4, NO = 2, NT = 2;
  __host__ __device__ static constexpr int table(int p) { return sph_table(p); }
  __host__ __device__ static constexpr int term(int p) { return sph_term(p); }
  __device__ static void finish(const dcx* h, double m, double inv, dcx* o) {
    sph_finish(h, m, inv, &o[0], &o[1]);
  }
};

// Analysis of up to two vector groups (r, theta, phi fields each).
// Kind 1 (full): outputs scalar(r), S, T; products (P,r) + sphtor (4).
// Kind 2 (S only): outputs scalar(r), S; products (P,r) (dP,theta) (P,phi).
// The fused Boussinesq analysis (magic_torch/step_time.py:1071-1124) is two
// launches: (Adv full, VS S-only) and (VxB full, VXi S-only).
__host__ __device__ constexpr int grp_np(int kind) { return kind == 1 ? 5 : (kind == 2 ? 3 : 0); }
__host__ __device__ constexpr int grp_no(int kind) { return kind == 1 ? 3 : (kind == 2 ? 2 : 0); }
__host__ __device__ constexpr int grp_nx(int kind) { return kind ? 3 : 0; }
__host__ __device__ constexpr int grp_table(int kind, int q) {
  return q == 0 ? kP : (kind == 1 ? sph_table(q - 1) : (q == 1 ? kDP : kP));
}
__host__ __device__ constexpr int grp_term(int kind, int q) {
  return q == 0 ? 0 : (kind == 1 ? 1 + sph_term(q - 1) : q);
}
template <int K0, int K1>
struct AnaGroups {
  static constexpr int NX = grp_nx(K0) + grp_nx(K1);
  static constexpr int NP = grp_np(K0) + grp_np(K1);
  static constexpr int NO = grp_no(K0) + grp_no(K1);
  static constexpr int NT = 2;
  __host__ __device__ static constexpr int table(int p) {
    return p < grp_np(K0) ? grp_table(K0, p) : grp_table(K1, p - grp_np(K0));
  }
  __host__ __device__ static constexpr int term(int p) {
    return p < grp_np(K0) ? grp_term(K0, p) : grp_nx(K0) + grp_term(K1, p - grp_np(K0));
  }
  __device__ static void finish_one(int kind, const dcx* h, double m, double inv, dcx* o) {
    o[0] = h[0];
    if (kind == 1) sph_finish(h + 1, m, inv, &o[1], &o[2]);
    else o[1] = scale(h[1] - times_im(h[2], m), inv);
  }
  __device__ static void finish(const dcx* h, double m, double inv, dcx* o) {
    if (K0) finish_one(K0, h, m, inv, o);
    if (K1) finish_one(K1, h + grp_np(K0), m, inv, o + grp_no(K0));
  }
};

// ------------------------------------------------------------ kernel args

template <int NX>
struct SynthArgs {
  Tables t;
  TermSrc src[NX];
  int64_t ld;         // row stride of the spectral sources (complex elements)
  int ncols;          // columns (levels / batch entries)
  const double* or2;  // (ncols) for kCurlT
  double2* F;         // Fourier output, F[m][theta_row][col]
  int64_t f_m, f_row;
  int64_t col_f, col_c;  // column of (output field f, input column c)
};

template <int NX, int NO>
struct AnalArgs {
  Tables t;
  const double2* F;  // Fourier input, F[m][theta_row][col], pre-weighted
  int64_t f_m, f_row;
  int64_t col_x, col_c;  // column of (input field x, column c)
  int ncols;
  double2* out[NO];  // (lm_max, ld) arrays
  int64_t ld;
  int out_col0;      // output column = out_col0 + c
};

}  // namespace mt
