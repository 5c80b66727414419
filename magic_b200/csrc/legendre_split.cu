// Split-precision (bf16x3, FP32 accumulate) Legendre contractions on tcgen05.
//
// Orientation: the data operand is A (M = 128 rows per CTA, one row per
// output real component), the Legendre table is B (N = theta rows for the
// synthesis, l rows for the analysis), K runs over l (synthesis) or theta
// pairs (analysis) in chunks of 16.  Each output row is a fixed linear
// combination "A_P . P + A_dP . dP": the row's A_P and A_dP entries are
// scaled source values (e.g. v_theta.re = (dP.S).re - m (P.T).im), so one
// fp32 TMEM accumulator holds the finished field component.
//
// Equatorial parity: the synthesis CTA for combo c in {sym, asym} contracts
// P over l - m of parity c and dP over the other parity; north = sym + asym,
// south = sym - asym (formed by the phi-stage kernel).  The analysis CTA for
// output parity p reads the folded Fourier data north + south (P rows of even
// parity, dP rows of odd) or north - south (the other two cases).
//
// Synthesis: a packing kernel writes the A operand as pre-split bf16x3 images,
// then a 4-warp GEMM kernel bulk-copies A and table chunks into a 3-stage
// ring and issues the plane products (two CTAs per SM).
// Analysis warp roles (192 threads): warps 0-3 build the A tiles (bf16x3
// split in registers, written in the canonical core-matrix layout) and run
// the epilogue (tcgen05.ld, one TMEM lane per thread); warp 4 owns TMEM and
// bulk-copies the pre-split table chunks; warp 5 lane 0 issues tcgen05.mma
// (6 plane products per table per chunk) and commits to the stage barriers.
#include "legendre.cuh"
#include "split.cuh"
#include "split_kernels.cuh"
#include "umma.cuh"

namespace mt {

// plane pairs (a, b) of the six retained products
__device__ __constant__ int8_t kPairA[6] = {0, 0, 1, 0, 1, 2};
__device__ __constant__ int8_t kPairB[6] = {0, 1, 0, 2, 1, 0};

__device__ __forceinline__ double coef_value(int code, double m) {
  switch (code) {
    case 1: return 1.0;
    case 2: return -1.0;
    case 3: return m;
    case 4: return -m;
    case 5: return -m * m;
    default: return 0.0;
  }
}

// Three bf16 planes of two floats (packed pairs, first value in the low
// half): hi = bf16(v), mid = bf16(v - hi), lo = bf16(v - hi - mid).  A float
// has 24 significant bits, so hi + mid + lo == v exactly (no underflow).
__device__ __forceinline__ void split3f2(float v0, float v1, uint32_t& h, uint32_t& m,
                                        uint32_t& l) {
  const __nv_bfloat162 bh = __floats2bfloat162_rn(v0, v1);
  const float2 fh = __bfloat1622float2(bh);
  const float r0 = v0 - fh.x, r1 = v1 - fh.y;
  const __nv_bfloat162 bm = __floats2bfloat162_rn(r0, r1);
  const float2 fm = __bfloat1622float2(bm);
  const __nv_bfloat162 bl = __floats2bfloat162_rn(r0 - fm.x, r1 - fm.y);
  h = *reinterpret_cast<const uint32_t*>(&bh);
  m = *reinterpret_cast<const uint32_t*>(&bm);
  l = *reinterpret_cast<const uint32_t*>(&bl);
}

// Write 16 consecutive K values of one row as 3 planes into an A tile.
__device__ __forceinline__ void put_row16(uint8_t* tile, int row, const float (&v)[16]) {
  uint32_t w[3][8];
#pragma unroll
  for (int i = 0; i < 8; ++i) split3f2(v[2 * i], v[2 * i + 1], w[0][i], w[1][i], w[2][i]);
#pragma unroll
  for (int s = 0; s < 3; ++s) {
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const uint4 q = make_uint4(w[s][4 * half], w[s][4 * half + 1], w[s][4 * half + 2],
                                 w[s][4 * half + 3]);
      *reinterpret_cast<uint4*>(tile + s * (kSplitRows * 32) + core_off(row, 8 * half)) = q;
    }
  }
}

// Write K values 8 half .. 8 half + 7 of one row as 3 planes into an A tile.
__device__ __forceinline__ void put_row8(uint8_t* tile, int row, int half, const float (&v)[8]) {
  uint32_t w[3][4];
#pragma unroll
  for (int i = 0; i < 4; ++i) split3f2(v[2 * i], v[2 * i + 1], w[0][i], w[1][i], w[2][i]);
#pragma unroll
  for (int s = 0; s < 3; ++s)
    *reinterpret_cast<uint4*>(tile + s * (kSplitRows * 32) + core_off(row, 8 * half)) =
        make_uint4(w[s][0], w[s][1], w[s][2], w[s][3]);
}

// 16-byte global -> shared copy; src_bytes = 0 zero-fills (no global read).
__device__ __forceinline__ void cp_async16_zfill(void* dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
// Staged source values of one synthesis chunk: array ia, l - m offset kk,
// level lv at double2 index ia * syn_stage_pitch + kk * stg_lev + lv.  The
// pitch is odd so lanes reading different arrays at one (kk, lv) hit
// different banks.
__host__ __device__ inline int syn_stage_pitch(int stg_lev) { return 32 * stg_lev + 1; }
__host__ __device__ inline uint32_t syn_staging_bytes(int narr, int stg_lev) {
  return (uint32_t)narr * syn_stage_pitch(stg_lev) * 16;
}

// ------------------------------------------------------------- synthesis
//
// Two kernels.  k_syn_pack builds the A operand: block (tile rt, chunk c, m)
// stages l - m in [32 c, 32 c + 32) of every source array at the tile's
// levels, assembles the rows of the four (table, parity) chunks and writes
// them as bf16x3 planes in the canonical layout (an image chunk is
// 3 planes x 128 rows x 16 K = 12 KiB).  Image order per (rt, m, combo):
// chunk c, then table (P, dP), so one K step reads one contiguous chunk.
// k_synth_gemm is then a pure bulk-copy-fed tcgen05 GEMM.

constexpr int kPackThreads = 256;
constexpr uint32_t kImgPlane = kSplitRows * 32;  // one bf16 plane of a 128 x 16 chunk
constexpr uint32_t kImgChunk = 3 * kImgPlane;

__host__ __device__ inline int64_t syn_img_chunk(int64_t total_chunks, int rt, int prefix, int c,
                                                 int q) {
  return (((int64_t)rt * total_chunks + prefix + c) * 2 + q);
}

__global__ void __launch_bounds__(kPackThreads, 4) k_syn_pack(SplitSynArgs a) {
  extern __shared__ __align__(16) uint8_t smem[];
  const Tables& t = a.t;
  const int rt = blockIdx.x, c = blockIdx.y, mc = blockIdx.z;
  const int m = mc * t.minc;
  const int nlm = t.l_max - m + 1;
  if (c >= syn_nchunks(nlm, 0)) return;
  const int ls = t.lstart[mc];
  const int tid = threadIdx.x;
  const int lev0 = (rt * kSplitRows) / a.row_per_level;
  const int nlev = min(a.stg_lev, a.n_lev - lev0);
  double2* d = reinterpret_cast<double2*>(smem);
  const int pitch = syn_stage_pitch(a.stg_lev);
  {
    // thread -> (kk, level) of the chunk, looping over the source arrays;
    // l - m beyond the spectrum is zero-filled (no global read)
    for (int e = tid; e < 32 * a.stg_lev; e += kPackThreads) {
      const int kk = e / a.stg_lev, lvv = e - kk * a.stg_lev;
      if (lvv >= nlev) continue;
      const int k = 32 * c + kk;
      const int64_t off = (int64_t)(ls + min(k, nlm - 1)) * a.ld + lev0 + lvv;
      const uint32_t bytes = k < nlm ? 16u : 0u;
      for (int ia = 0; ia < a.narr; ++ia)
        cp_async16_zfill(&d[ia * pitch + kk * a.stg_lev + lvv], a.arr[ia] + off, bytes);
    }
    cp_async_commit();
    cp_async_wait0();
    __syncthreads();
  }
  // task = (table q, parity p, row pair): rows 2 pr, 2 pr + 1 are the real and
  // imaginary rows of one field (rows per level are even), whose programs read
  // the same terms with the components swapped, so one 16-byte load serves both
#pragma unroll 1
  for (int task = tid; task < 2 * kSplitRows; task += kPackThreads) {
    const int qp = task / (kSplitRows / 2), row0 = 2 * (task % (kSplitRows / 2));
    const int q = qp >> 1, p = qp & 1;  // table (0 P, 1 dP), parity of l - m
    const int R0 = rt * kSplitRows + row0;
    const bool live = R0 < a.nrows;
    const int lev = live ? R0 / a.row_per_level : lev0;
    const int qf = live ? R0 - lev * a.row_per_level : 0;
    const int lv = lev - lev0;
    const float o2l = a.or2 ? (float)a.or2[lev] : 1.f;
    struct RowSrc {
      const double2 *xa, *xb;
      int cpart;
      float f, dl, o2, cw;
      int tix;
    } rs[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const RowOp op = a.ops[qf + h];
      const int tix = q ? op.tD : op.tP;
      const TermIx tm = a.term[tix];
      rs[h].tix = tix;
      rs[h].cpart = q ? op.cD : op.cP;
      // value = f * (mul(l) * src_a - cw * src_b), branch-free over the recipes:
      //   raw: mul = 1; dlh: mul = l(l+1); curl: mul = or2 l(l+1), cw = 1
      rs[h].f = live ? (float)coef_value(q ? op.kD : op.kP, (double)m) : 0.f;
      rs[h].dl = tm.recipe == kRaw ? 0.f : 1.f;
      rs[h].o2 = tm.recipe == kCurlT ? o2l : 1.f;
      rs[h].cw = tm.recipe == kCurlT ? 1.f : 0.f;
      rs[h].xa = d + tm.ia * pitch + lv;
      rs[h].xb = d + tm.ib * pitch + lv;
    }
    const bool same = rs[0].tix == rs[1].tix;
    const int combo = q == 0 ? p : 1 - p;
    uint8_t* dst = a.aimg + syn_img_chunk(a.total_chunks, rt, a.s.syn_chunk_prefix[mc * 2 + combo],
                                          c, q) * kImgChunk;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      float v0[8], v1[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int kk = 2 * (8 * half + i) + p;
        const float l = (float)(m + 32 * c + kk);
        const int off = kk * a.stg_lev;
        const double2 x0 = rs[0].xa[off];
        const double2 w0 = rs[0].cw != 0.f ? rs[0].xb[off] : make_double2(0.0, 0.0);
        const double2 x1 = same ? x0 : rs[1].xa[off];
        const double2 w1 = same ? w0 : (rs[1].cw != 0.f ? rs[1].xb[off] : make_double2(0.0, 0.0));
        const float mul0 = rs[0].o2 * (1.f + rs[0].dl * (l * (l + 1.f) - 1.f));
        const float mul1 = rs[1].o2 * (1.f + rs[1].dl * (l * (l + 1.f) - 1.f));
        const float a0 = (float)(rs[0].cpart ? x0.y : x0.x), b0 = (float)(rs[0].cpart ? w0.y : w0.x);
        const float a1 = (float)(rs[1].cpart ? x1.y : x1.x), b1 = (float)(rs[1].cpart ? w1.y : w1.x);
        v0[i] = rs[0].f != 0.f ? rs[0].f * (mul0 * a0 - b0) : 0.f;
        v1[i] = rs[1].f != 0.f ? rs[1].f * (mul1 * a1 - b1) : 0.f;
      }
      put_row8(dst, row0, half, v0);
      put_row8(dst, row0 + 1, half, v1);
    }
  }
}

constexpr int kGemmStages = 3;
constexpr int kGemmThreads = 128;

// Shared memory of one GEMM CTA: stages of [A chunk | B chunk], then barriers.
struct GemmSmem {
  uint32_t b_plane, stage_bytes, bar_off;
  __host__ __device__ explicit GemmSmem(int brows)
      : b_plane((uint32_t)brows * 32),
        stage_bytes(kImgChunk + 3 * (uint32_t)brows * 32),
        bar_off(kGemmStages * (kImgChunk + 3 * (uint32_t)brows * 32)) {}
  __host__ __device__ size_t total() const { return bar_off + 8 * (2 * kGemmStages + 1) + 16; }
};

// Persistent synthesis GEMM: one CTA per SM walks the work items
// (tile, sym/asym, theta tile, m) with a stride of gridDim.x.  Warp 0 lane 0
// bulk-copies the A image chunk and the table chunk of every K step into a
// kPStages ring, warp 1 lane 0 issues the six plane products per step into
// one of two TMEM accumulators (columns 0 and 256) and commits it when the
// item's K loop ends, warps 2-9 drain the other accumulator into Fs (warp w
// reads TMEM lanes 32 (w % 4) ..., warps w and w + 4 split the columns) and
// hand it back.  K steps of an item:
// chunk c of the P table (parity combo), then chunk c of the dP table (the
// other parity), skipping chunks a table does not have.
constexpr int kPStages = 5;
constexpr int kPEpiWarps = 8;  // two per TMEM lane quarter, each half of the columns
constexpr int kPThreads = 64 + 32 * kPEpiWarps;

struct PSmem {
  uint32_t stage_bytes, bar_off;
  __host__ __device__ explicit PSmem(int brows)
      : stage_bytes(kImgChunk + 3 * (uint32_t)brows * 32),
        bar_off(kPStages * (kImgChunk + 3 * (uint32_t)brows * 32)) {}
  // full/empty per stage, tfull/tempty per accumulator, done, tmem slot, abort flag
  __host__ __device__ size_t total() const { return bar_off + 8 * (2 * kPStages + 5) + 16; }
};

__global__ void __launch_bounds__(kPThreads, 1) k_synth_gemm(SplitSynArgs a) {
  extern __shared__ __align__(128) uint8_t smem[];
  const Tables& t = a.t;
  const SplitTables& st = a.s;
  const int wth = st.wth;
  const PSmem L(wth);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + L.bar_off);
  uint64_t* empty = full + kPStages;
  uint64_t* tfull = empty + kPStages;  // [2] accumulator ready
  uint64_t* tempty = tfull + 2;        // [2] accumulator drained
  uint64_t* done = tempty + 2;         // every MMA issued by this CTA finished
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  // an earlier CTA already timed out: skip the work so a fault costs one wait, not one per CTA
  if (*(volatile int*)a.err) return;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ntiles = (a.nrows + kSplitRows - 1) / kSplitRows, ny = 2 * st.nthtile;
  const int nitems = ntiles * ny * t.n_m;
  struct Item {
    int rt, combo, tau, mc, nlm, nch_t[2];
  };
  auto decode = [&](int item) {
    Item it;
    it.rt = item % ntiles;
    const int r = item / ntiles, y = r % ny;
    it.mc = r / ny;
    it.combo = y & 1;
    it.tau = y >> 1;
    it.nlm = t.l_max - it.mc * t.minc + 1;
    it.nch_t[0] = (split_nk(it.nlm, it.combo) + kSplitKC - 1) / kSplitKC;
    it.nch_t[1] = (split_nk(it.nlm, 1 - it.combo) + kSplitKC - 1) / kSplitKC;
    return it;
  };

  if (tid == 0) {
    for (int s = 0; s < kPStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 32 * kPEpiWarps);
    }
    mbar_init(done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 1) tmem_alloc(tmem_slot, 512);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tmem_slot;

  if (warp == 0) {
    // ---------------- loader ----------------
    if (lane == 0) {
      const uint32_t bchunk = 3 * (uint32_t)wth * 32;
      int g = 0;
      bool ok = true;
      for (int item = blockIdx.x; item < nitems && ok; item += gridDim.x) {
        const Item it = decode(item);
        const uint8_t* aimg =
            a.aimg + syn_img_chunk(a.total_chunks, it.rt,
                                   st.syn_chunk_prefix[it.mc * 2 + it.combo], 0, 0) * kImgChunk;
        const uint8_t* img[2];
        for (int q = 0; q < 2; ++q)
          img[q] = st.syn + st.syn_off[((it.mc * 2 + q) * 2 + (q ? 1 - it.combo : it.combo)) *
                                           st.nthtile + it.tau];
        const int nch = max(it.nch_t[0], it.nch_t[1]);
        for (int c = 0; c < nch && ok; ++c) {
          for (int q = 0; q < 2; ++q) {
            if (c >= it.nch_t[q]) continue;
            const int s = g % kPStages;
            if (g >= kPStages &&
                !mbar_wait(&empty[s], ((g / kPStages) - 1) & 1, abort_flag, a.err, 3)) {
              ok = false;
              break;
            }
            uint8_t* stage = smem + s * L.stage_bytes;
            mbar_expect_tx(&full[s], kImgChunk + bchunk);
            bulk_g2s(stage, aimg + (int64_t)(2 * c + q) * kImgChunk, kImgChunk, &full[s]);
            bulk_g2s(stage + kImgChunk, img[q] + (int64_t)c * bchunk, bchunk, &full[s]);
            ++g;
          }
        }
      }
      // every issued copy must land before the CTA may exit
      for (int k = max(0, g - kPStages); k < g; ++k)
        mbar_drain(&full[k % kPStages], (k / kPStages) & 1);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      const uint32_t idesc = umma_idesc_bf16(kSplitRows, wth);
      int g = 0, n = 0;
      bool ok = true;
      for (int item = blockIdx.x; item < nitems && ok; item += gridDim.x, ++n) {
        const Item it = decode(item);
        const int buf = n & 1;
        if (n >= 2 && !mbar_wait(&tempty[buf], ((n >> 1) - 1) & 1, abort_flag, a.err, 6)) break;
        tc_fence_after();
        const uint32_t acc_col = tbase + 256u * buf;
        uint32_t acc = 0;
        const int nch = max(it.nch_t[0], it.nch_t[1]);
        for (int c = 0; c < nch && ok; ++c) {
          for (int q = 0; q < 2; ++q) {
            if (c >= it.nch_t[q]) continue;
            const int s = g % kPStages;
            if (!mbar_wait(&full[s], (g / kPStages) & 1, abort_flag, a.err, 4)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t sa = smem_u32(smem + s * L.stage_bytes);
            const uint32_t sb = sa + kImgChunk;
#pragma unroll
            for (int pp = 0; pp < 6; ++pp) {
              const uint64_t da = umma_desc(sa + kPairA[pp] * kImgPlane, 128, 256);
              const uint64_t db = umma_desc(sb + kPairB[pp] * (uint32_t)wth * 32, 128, 256);
              umma_bf16(acc_col, da, db, idesc, acc);
              acc = 1;
            }
            umma_commit(&empty[s]);
            ++g;
          }
        }
        if (ok) umma_commit(&tfull[buf]);
      }
      umma_commit(done);  // arrives once every MMA above has finished
    }
  } else {
    // ---------------- epilogue (warps 2-9) ----------------
    const int quarter = warp & 3, half = (warp - 2) >> 2;
    int n = 0;
    for (int item = blockIdx.x; item < nitems; item += gridDim.x, ++n) {
      const int buf = n & 1;
      const bool ok = mbar_wait(&tfull[buf], (n >> 1) & 1, abort_flag, a.err, 2);
      if (!__all_sync(0xffffffffu, ok && !*abort_flag)) break;
      tc_fence_after();
      const Item it = decode(item);
      const int R = it.rt * kSplitRows + quarter * 32 + lane;
      float* out = a.Fs + (int64_t)it.mc * a.fs_m + (int64_t)it.combo * a.fs_c;
      const uint32_t taddr = tbase + ((uint32_t)(32 * quarter) << 16) + 256u * buf;
      for (int c0 = 16 * half; c0 < wth; c0 += 32) {
        float v[16];
        tmem_ld16(taddr + c0, v);
        if (R < a.nrows) {
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const int th = it.tau * wth + c0 + i;
            if (th < t.nhs) out[(int64_t)th * a.fs_j + R] = v[i];
          }
        }
      }
      tc_fence_before();
      mbar_arrive(&tempty[buf]);
    }
  }
  __syncwarp();
  if (warp == 1) mbar_drain(done, 0);  // no MMA may still write TMEM at dealloc
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tbase, 512);
  }
}

// -------------------------------------------------------------- analysis
//
// k_ana_pack folds the north/south Fourier rows of the phi stage into
// bf16x3 A-operand images: block (tile rt, theta-pair chunk c, m) stages 16
// theta pairs of both hemispheres at the tile's levels and writes, for
// fold 0 (north + south) and fold 1 (north - south), a 128 x 16 chunk whose
// rows are the raw Fourier columns (level lv, column col) of the tile.
// k_anal_gemm (CTA = tile, output parity, m) accumulates
//   acc0[col][l] = sum_j fold_par(col)[j] P_l(j),
//   acc1[col][l] = sum_j fold_(1-par)(col)[j] dP_l(j)
// in two TMEM accumulators and its epilogue forms each output component as
// coef(kP) acc0[colP] + coef(kD) acc1[colD] (the row program), exchanging
// accumulator rows through shared memory.

__host__ __device__ inline int64_t ana_img_chunk(int n_m, int nchj, int rt, int mc, int fold,
                                                 int c) {
  return (((int64_t)rt * n_m + mc) * 2 + fold) * nchj + c;
}

__global__ void __launch_bounds__(kPackThreads, 8) k_ana_pack(SplitAnaArgs a) {
  extern __shared__ __align__(16) uint8_t smem[];
  const Tables& t = a.t;
  const int rt = blockIdx.x, c = blockIdx.y, mc = blockIdx.z;
  const int nchj = gridDim.y;
  const int tid = threadIdx.x;
  const int lev0 = rt * a.lev_tile;
  const int nlev = min(a.lev_tile, a.n_lev - lev0);
  const int gl = (int)a.g_level;
  const int rowlen = a.lev_tile * gl;  // floats per staged (hemisphere, theta pair)
  float* d = reinterpret_cast<float*>(smem);
  {
    const float* gm = a.G + (int64_t)mc * a.g_m + (int64_t)lev0 * gl;
    // warp -> (hemisphere, theta pair) rows, lanes -> consecutive 16-byte pieces
    const int cpl = nlev * gl / 4;  // 16-byte pieces per (hemisphere, theta pair)
    for (int hj = tid >> 5; hj < 2 * kSplitKC; hj += kPackThreads / 32) {
      const int h = hj / kSplitKC, j = kSplitKC * c + hj % kSplitKC;
      const float* src = gm + (int64_t)h * a.g_h + (int64_t)min(j, t.nhs - 1) * a.g_j;
      const uint32_t bytes = j < t.nhs ? 16u : 0u;
      for (int p4 = tid & 31; p4 < cpl; p4 += 32)
        cp_async16_zfill(d + hj * rowlen + 4 * p4, src + 4 * p4, bytes);
    }
    cp_async_commit();
    cp_async_wait0();
    __syncthreads();
  }
#pragma unroll 1
  for (int task = tid; task < 2 * kSplitRows; task += kPackThreads) {
    const int fold = task / kSplitRows, row = task % kSplitRows;
    const int lv = row / a.cols, col = row - lv * a.cols;
    const bool live = lv < nlev;
    const float sg = fold ? -1.f : 1.f;
    const float* n = d + lv * gl + col;
    float v[16];
#pragma unroll
    for (int i = 0; i < 16; ++i)
      v[i] = live ? n[i * rowlen] + sg * n[(kSplitKC + i) * rowlen] : 0.f;
    uint8_t* dst = a.aimg + ana_img_chunk(t.n_m, nchj, rt, mc, fold, c) * kImgChunk;
    put_row16(dst, row, v);
  }
}

// Warp 0 lane 0 loads, warp 1 lane 0 issues the MMAs, warp 2 owns TMEM, all
// four warps run the epilogue.  K steps: theta-pair chunk c of the P table
// (into acc0), then of the dP table (into acc1).
__global__ void __launch_bounds__(kGemmThreads, 2) k_anal_gemm(SplitAnaArgs a) {
  extern __shared__ __align__(128) uint8_t smem[];
  const Tables& t = a.t;
  const SplitTables& st = a.s;
  const int rt = blockIdx.x, par = blockIdx.y, mc = blockIdx.z;
  const int wk = st.ana_wk[mc * 2 + par];
  if (wk == 0 || *(volatile int*)a.err) return;
  const GemmSmem L(a.wk_max);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + L.bar_off);
  uint64_t* empty = full + kGemmStages;
  uint64_t* accb = empty + kGemmStages;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accb + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m = mc * t.minc;
  const int nlm = t.l_max - m + 1;
  const int ls = t.lstart[mc];
  const int nchj = (t.nhs + kSplitKC - 1) / kSplitKC;
  // two accumulators of wk columns; 512 (all of TMEM) only above l_max = 255
  uint32_t tcols = 32;
  while (tcols < 2u * wk) tcols *= 2;
  const uint32_t b_plane = wk * 32, bchunk = 3 * b_plane;

  if (tid == 0) {
    for (int s = 0; s < kGemmStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(accb, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 2) tmem_alloc(tmem_slot, tcols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---------------- loader ----------------
    const uint8_t* aimg[2];
    const uint8_t* img[2];
    for (int q = 0; q < 2; ++q) {
      const int fold = q ? 1 - par : par;
      aimg[q] = a.aimg + ana_img_chunk(t.n_m, nchj, rt, mc, fold, 0) * kImgChunk;
      img[q] = st.ana + st.ana_off[(mc * 2 + q) * 2 + par];
    }
    int step = 0;
    bool ok = true;
    for (int c = 0; c < nchj && ok; ++c) {
      for (int q = 0; q < 2; ++q) {
        const int s = step % kGemmStages;
        if (step >= kGemmStages &&
            !mbar_wait(&empty[s], ((step / kGemmStages) - 1) & 1, abort_flag, a.err, 13)) {
          ok = false;
          break;
        }
        uint8_t* stage = smem + s * L.stage_bytes;
        mbar_expect_tx(&full[s], kImgChunk + bchunk);
        bulk_g2s(stage, aimg[q] + (int64_t)c * kImgChunk, kImgChunk, &full[s]);
        bulk_g2s(stage + kImgChunk, img[q] + (int64_t)c * bchunk, bchunk, &full[s]);
        ++step;
      }
    }
    for (int k = max(0, step - kGemmStages); k < step; ++k)
      mbar_drain(&full[k % kGemmStages], (k / kGemmStages) & 1);
  } else if (warp == 1 && lane == 0) {
    // ---------------- MMA issuer ----------------
    const uint32_t idesc = umma_idesc_bf16(kSplitRows, wk);
    int step = 0;
    bool ok = true;
    for (int c = 0; c < nchj && ok; ++c) {
      for (int q = 0; q < 2; ++q) {
        const int s = step % kGemmStages;
        if (!mbar_wait(&full[s], (step / kGemmStages) & 1, abort_flag, a.err, 14)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t sa = smem_u32(smem + s * L.stage_bytes);
        const uint32_t sb = sa + kImgChunk;
#pragma unroll
        for (int pp = 0; pp < 6; ++pp) {
          const uint64_t da = umma_desc(sa + kPairA[pp] * kImgPlane, 128, 256);
          const uint64_t db = umma_desc(sb + kPairB[pp] * b_plane, 128, 256);
          umma_bf16(tbase + q * wk, da, db, idesc, (c > 0 || pp > 0) ? 1u : 0u);
        }
        umma_commit(&empty[s]);
        ++step;
      }
    }
    umma_commit(accb);
  }
  __syncwarp();
  // ---------------- epilogue ----------------
  const bool ok = mbar_wait(accb, 0, abort_flag, a.err, 12);
  tc_fence_after();
  if (__syncthreads_and(ok && !*abort_flag)) {
    // every copy landed and every MMA finished: the stages are free for the
    // exchange buffer and the per-CTA tables of the row programs
    constexpr int XS = 17;  // padded row of 16 columns
    float* xch = reinterpret_cast<float*>(smem);  // [2][128][XS]
    double* cf = reinterpret_cast<double*>(smem + 2 * kSplitRows * XS * sizeof(float));
    int* colx = reinterpret_cast<int*>(cf + 64);  // exchange row of each term (acc1 rows + 128)
    double* osc = reinterpret_cast<double*>(colx + 64);  // 1/(l(l+1)) of l - m = 2 kk + par
    const int lev0 = rt * a.lev_tile;
    const int nlev = min(a.lev_tile, a.n_lev - lev0);
    const double dm = (double)m;
    for (int q = tid; q < 2 * a.n_out; q += kGemmThreads) {
      const RowOp op = a.ops[q];
      cf[2 * q] = coef_value(op.kP, dm);
      cf[2 * q + 1] = coef_value(op.kD, dm);
      colx[2 * q] = 2 * op.tP + op.cP;
      colx[2 * q + 1] = kSplitRows + 2 * op.tD + op.cD;
    }
    for (int kk = tid; kk < wk; kk += kGemmThreads) {
      const double l = (double)(m + 2 * kk + par);
      osc[kk] = l > 0.0 ? 1.0 / (l * (l + 1.0)) : 0.0;
    }
    // (output o, level slot lv) pairs, lv fastest, R threads per pair splitting
    // the 16 columns of a chunk: consecutive threads write consecutive levels of
    // one (output, l), and each thread reads its row-program tables once per chunk
    int lvs = 0;  // level slot: smallest power of two >= lev_tile
    while ((1 << lvs) < a.lev_tile) ++lvs;
    const int npair = a.n_out << lvs;
    int R = 1;
    while (R < 16 && npair * R * 2 <= kGemmThreads) R *= 2;
    const int ispan = 16 / R;
    for (int c0 = 0; c0 < wk; c0 += 16) {
      float v[16];
      tmem_ld16(tbase + ((uint32_t)(32 * warp) << 16) + c0, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) xch[tid * XS + i] = v[i];
      tmem_ld16(tbase + ((uint32_t)(32 * warp) << 16) + wk + c0, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) xch[(kSplitRows + tid) * XS + i] = v[i];
      __syncthreads();
      for (int pr = tid / R; pr < npair; pr += kGemmThreads / R) {
        const int lv = pr & ((1 << lvs) - 1), o = pr >> lvs;
        if (lv >= nlev) continue;
        const int q = 4 * o, base = lv * a.cols;
        const double fr0 = cf[q], fr1 = cf[q + 1], fi0 = cf[q + 2], fi1 = cf[q + 3];
        const float* xr0 = xch + (base + colx[q]) * XS;
        const float* xr1 = xch + (base + colx[q + 1]) * XS;
        const float* xi0 = xch + (base + colx[q + 2]) * XS;
        const float* xi1 = xch + (base + colx[q + 3]) * XS;
        const bool scaled = a.ops[2 * o].scale;
        double2* dst = a.out[o] + a.out_col0 + lev0 + lv;
        const int i0 = (tid & (R - 1)) * ispan;
        for (int ii = 0; ii < ispan; ++ii) {
          const int i = i0 + ii, kk = c0 + i, k = 2 * kk + par;
          if (k >= nlm) break;
          const double re = fr0 * (double)xr0[i] + fr1 * (double)xr1[i];
          const double im = fi0 * (double)xi0[i] + fi1 * (double)xi1[i];
          const double sc = scaled ? osc[kk] : 1.0;
          dst[(int64_t)(ls + k) * a.ld] = make_double2(sc * re, sc * im);
        }
      }
      __syncthreads();
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 2) {
    tc_fence_after();
    tmem_dealloc(tbase, tcols);
  }
}

int launch_synth_split(const SplitSynArgs& a, cudaStream_t st) {
  const int ntiles = (a.nrows + kSplitRows - 1) / kSplitRows;
  const size_t pack_sm = syn_staging_bytes(a.narr, a.stg_lev);
  MT_CHECK_CUDA(cudaFuncSetAttribute(k_syn_pack, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)pack_sm));
  dim3 pgrid(ntiles, syn_nchunks(a.t.l_max + 1, 0), a.t.n_m);
  k_syn_pack<<<pgrid, kPackThreads, pack_sm, st>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  const PSmem L(a.s.wth);
  const size_t sm = L.total();
  MT_CHECK_CUDA(cudaFuncSetAttribute(k_synth_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sm));
  int dev = 0, nsm = 148;
  MT_CHECK_CUDA(cudaGetDevice(&dev));
  MT_CHECK_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int nitems = ntiles * 2 * a.s.nthtile * a.t.n_m;
  k_synth_gemm<<<std::min(nitems, nsm), kPThreads, sm, st>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

size_t synth_split_image_bytes(int nrows, int64_t total_chunks) {
  return (size_t)((nrows + kSplitRows - 1) / kSplitRows) * (size_t)total_chunks * 2 * kImgChunk;
}

// Self-test of the bounded waits: every thread waits on a barrier that no one
// arrives on, gives up after `spins` polls, records code 99 and returns.
__global__ void k_selftest_wait(int* status, long spins) {
  __shared__ uint64_t bar;
  __shared__ int abort_flag;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  const bool ok = mbar_wait_n(&bar, 0, &abort_flag, status, 99, spins);
  __syncthreads();
  if (threadIdx.x == 0 && ok) atomicCAS(status, 0, -1);  // a wait that nothing ends returned true
}

int launch_selftest_wait(int* status, long spins, cudaStream_t st) {
  k_selftest_wait<<<1, 64, 0, st>>>(status, spins);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

int launch_anal_split(const SplitAnaArgs& a, cudaStream_t st) {
  const int ntiles = (a.n_lev + a.lev_tile - 1) / a.lev_tile;
  const int nchj = (a.t.nhs + kSplitKC - 1) / kSplitKC;
  const size_t pack_sm = (size_t)2 * kSplitKC * a.lev_tile * a.g_level * sizeof(float);
  MT_CHECK_CUDA(cudaFuncSetAttribute(k_ana_pack, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)pack_sm));
  k_ana_pack<<<dim3(ntiles, nchj, a.t.n_m), kPackThreads, pack_sm, st>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  const GemmSmem L(a.wk_max);
  const size_t sm = L.total();
  MT_CHECK_CUDA(cudaFuncSetAttribute(k_anal_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sm));
  k_anal_gemm<<<dim3(ntiles, 2, a.t.n_m), kGemmThreads, sm, st>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

size_t anal_split_image_bytes(int n_m, int nhs, int n_lev, int lev_tile) {
  const int ntiles = (n_lev + lev_tile - 1) / lev_tile;
  return (size_t)ntiles * n_m * 2 * ((nhs + kSplitKC - 1) / kSplitKC) * kImgChunk;
}

}  // namespace mt
