// Digit-split ("ozaki") Legendre contractions on the tcgen05 integer pipe.
//
// Each FP64 operand value v of a contraction sum_k a_k b_k is written, with a
// power-of-two scale 2^e shared by its whole row of A (or column of B) over K,
// as six signed 7-bit digits:
//   v = 2^(e - 6) (d0 + d1 2^-7 + d2 2^-14 + ... + d5 2^-35) + O(2^(e - 42)),
//   |d_i| <= 64, obtained exactly in FP64 by repeated round-to-nearest.
// The products of digit planes are exact in int8 x int8 -> int32 tensor-core
// MMAs (tcgen05.mma kind::i8), and so are their sums over K (|d_i d_j| <=
// 2^12, so 2^19 terms fit before int32 overflow).  The 21 digit pairs
// (i, j) with i + j <= 5 are accumulated by weight group g = i + j into six
// int32 TMEM accumulators, and the epilogue forms
//   sum_k a_k b_k = 2^(eA + eB - 12) sum_g 2^(-7 g) C_g
// in FP64.  Truncation error is ~2^-41 of the row/column scales, so the
// contraction is accurate to ~1e-12 of the output's scale: the accumulation
// itself adds no rounding at all.  (The scheme is the splitting method of
// Ozaki, Ogita, Oishi and Rump, "Error-free transformations of matrix
// multiplication by using fast routines of matrix multiplication and its
// applications", Numer. Algorithms 59 (2012), run on integer tensor cores as in
// Ootomo, Ozaki and Yokota, "DGEMM on integer matrix multiplication unit",
// IJHPCA 2024.)
//
// Operand chunks in shared memory use the K-major, no-swizzle canonical layout
// of an 8-bit MMA: 8-row x 16-byte core matrices, K = 32 per MMA (two core
// matrices 128 B apart = LBO), 8-row groups 256 B apart (SBO).
#pragma once

#include "legendre.cuh"
#include "split_kernels.cuh"

namespace mt {

constexpr int kOzDigits = 6;  // int8 digits per operand value
constexpr int kOzGroups = 6;  // digit-weight groups kept: i + j <= 5
constexpr int kOzK = 32;      // K per MMA and per operand chunk
constexpr int kOzRows = 128;  // MMA M: data rows per tile
constexpr int kOzSynN = 64;   // theta rows per synthesis tile (MMA N per table digit plane)
constexpr int kOzAnaN = 32;   // l rows per analysis tile (MMA N)
constexpr uint32_t kOzAPlane = kOzRows * kOzK;               // 4 KiB
constexpr uint32_t kOzAChunk = kOzDigits * kOzAPlane;        // 24 KiB
constexpr uint32_t kOzSynBPlane = kOzSynN * kOzK;            // 2 KiB
constexpr uint32_t kOzSynBChunk = kOzDigits * kOzSynBPlane;  // 12 KiB
constexpr uint32_t kOzAnaBPlane = kOzAnaN * kOzK;            // 1 KiB
constexpr uint32_t kOzAnaBChunk = kOzDigits * kOzAnaBPlane;  // 6 KiB

// byte offset of element (row, k) in a (rows x 32) K-major no-swizzle int8 tile
__host__ __device__ constexpr uint32_t oz_off(int row, int k) {
  return (uint32_t)((row >> 3) * 256 + (k >> 4) * 128 + (row & 7) * 16 + (k & 15));
}

// Chunks (of kOzK values of one parity) of the synthesis K range of (m, combo):
// P over l - m of parity combo and dP over the other parity.
__host__ __device__ inline int oz_syn_nch(int nlm, int combo) {
  const int a = (split_nk(nlm, combo) + kOzK - 1) / kOzK;
  const int b = (split_nk(nlm, 1 - combo) + kOzK - 1) / kOzK;
  return a > b ? a : b;
}

// Plan-time digit images of the tables and their scale exponents.
struct OzTables {
  int nthtile;              // synthesis theta tiles of kOzSynN rows
  int nlt;                  // analysis l tiles of kOzAnaN rows (max over m, parity)
  const int8_t* syn;        // [m][table][parity][theta tile] -> chunks over l
  const int64_t* syn_off;   // byte offset of ((m * 2 + q) * 2 + p) * nthtile + tau
  const int* syn_fexp;      // [(m * 2 + combo) * nthtile * kOzSynN + theta]
  const int8_t* ana;        // [m][table][parity][l tile] -> chunks over theta pairs
  const int64_t* ana_off;   // byte offset of ((m * 2 + q) * 2 + p) * nlt + lt
  const int* ana_fexp;      // [((m * 2 + q) * 2 + p) * nlt * kOzAnaN + k], l - m = 2 k + p
  const int* syn_prefix;    // (n_m * 2 + 1) prefix sums of oz_syn_nch over (m, combo)
};

struct OzSynArgs {
  Tables t;
  OzTables z;
  const double2* arr[12];  // spectral source arrays, (lm_max, ld) complex over levels
  int narr;
  TermIx term[16];
  int64_t ld;
  const double* or2;       // per level, for kCurlT
  int n_lev, nrows, row_per_level, stg_lev;
  RowOp ops[40];           // per (field, re/im) of a level
  uint8_t* aimg;           // A-operand digit images (workspace)
  int64_t total_chunks;    // oz_syn_nch summed over (m, combo)
  int* rexp;               // row exponents [(m * 2 + combo) * rows_pad + row]
  int64_t rows_pad;        // tiles * kOzRows
  double* Fs;              // [m][north|south][theta pair][row]
  int64_t fs_m, fs_c, fs_j;
  int* err;
};

struct OzAnaArgs {
  Tables t;
  OzTables z;
  const double* G;         // [m][north|south][theta pair][level * g_level + column]
  int64_t g_m, g_h, g_j, g_level;  // g_level: doubles per level, even
  int n_lev, cols, lev_tile, n_out;
  RowOp ops[32];
  double2* out[16];
  int64_t ld;
  int out_col0;
  uint8_t* aimg;           // folded A-operand digit images (workspace)
  int* rexp;               // row exponents [(m * 2 + fold) * rows_pad + row]
  int64_t rows_pad;
  int* err;
};

int build_ozaki_tables(mt_plan* p);
void free_ozaki_tables(mt_plan* p);
const OzTables& ozaki_tables(const mt_plan* p);
int ozaki_syn_total_chunks(const mt_plan* p);
size_t oz_syn_image_bytes(int nrows, int64_t total_chunks);
size_t oz_ana_image_bytes(int n_m, int nhs, int n_lev, int lev_tile);
int launch_oz_synth(const OzSynArgs& a, cudaStream_t st);
int launch_oz_anal(const OzAnaArgs& a, cudaStream_t st);

}  // namespace mt
