// Split-precision Legendre stage: shared definitions.
//
// Each FP64 operand value v is carried as three bf16 planes
//   hi = bf16(v), mid = bf16(v - hi), lo = bf16(v - hi - mid)
// (24 significant bits), and a contraction sum_k a_k b_k is formed on the
// tcgen05 tensor pipe (kind::f16, bf16 x bf16 -> fp32 accumulate in TMEM) as
// the six plane products whose magnitude is >= 2^-16 of the leading term:
//   hi.hi + hi.mid + mid.hi + hi.lo + mid.mid + lo.hi.
// The dropped terms are <= 2^-24 relative; FP32 accumulation adds ~2^-24 per
// step.
//
// Operand tiles in shared memory use the K-major, no-swizzle canonical UMMA
// layout: 8-row x 16-byte core matrices, K-chunks of 16 bf16 (two core
// matrices, 128 B apart = LBO), 8-row groups 256 B apart (SBO).
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"

namespace mt {

constexpr int kSplitKC = 16;      // K elements per chunk (one MMA)
constexpr int kSplitRows = 128;   // MMA M (rows of the data operand per CTA)

__host__ __device__ constexpr uint32_t core_off(int row, int k) {
  // byte offset of element (row, k) in a (rows x 16) K-major no-swizzle tile
  return (uint32_t)((row >> 3) * 256 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ void split3(double v, __nv_bfloat16& h, __nv_bfloat16& m,
                                       __nv_bfloat16& l) {
  h = __double2bfloat16(v);
  double r = v - (double)__bfloat162float(h);
  m = __double2bfloat16(r);
  r -= (double)__bfloat162float(m);
  l = __double2bfloat16(r);
}

// Per-plan split tables (device pointers + host-side offsets copied to device).
struct SplitTables {
  int wth;             // theta-tile width (rows of the synthesis B operand), mult. of 16
  int nthtile;         // theta tiles covering nhs
  // synthesis images: [m][table][parity][theta tile] -> chunks of 3 planes x wth x 32 B
  const uint8_t* syn;
  const int64_t* syn_off;  // (n_m * 2 * 2 * nthtile) byte offsets
  // analysis images: [m][table][parity] -> chunks (over theta pairs) of 3 x wk x 32 B
  const uint8_t* ana;
  const int64_t* ana_off;  // (n_m * 2 * 2) byte offsets
  const int* ana_wk;       // (n_m * 2) row count (k of that parity) padded to 16
  // synthesis A-operand images: K chunks of (m, combo) = max over the two
  // tables; prefix sums over (m, combo) in that order ((n_m * 2 + 1) entries)
  const int* syn_nch;
  const int* syn_chunk_prefix;
};

__host__ __device__ inline int split_nk(int nlm, int parity) { return (nlm + 1 - parity) / 2; }
__host__ __device__ inline int round16(int n) { return (n + 15) & ~15; }

// K chunks of the synthesis CTA (m, combo): P over l - m of parity combo and
// dP over the other parity, 16 values of each per chunk.
__host__ __device__ inline int syn_nchunks(int nlm, int combo) {
  const int a = (split_nk(nlm, combo) + 15) / 16, b = (split_nk(nlm, 1 - combo) + 15) / 16;
  return a > b ? a : b;
}


int build_split_tables(mt_plan* p);
void free_split_tables(mt_plan* p);

}  // namespace mt
