// Argument blocks of the split-precision stage kernels.
#pragma once

#include "legendre.cuh"
#include "split.cuh"

namespace mt {

// One output real component as a linear combination of two scaled sources:
// value = coef(kP) * src(tP, cP) contracted with P + coef(kD) * src(tD, cD)
// contracted with dP.  coef codes: 0 zero, 1 +1, 2 -1, 3 +m, 4 -m, 5 -m^2.
// cP/cD select the real (0) or imaginary (1) part; scale = 1 divides the
// analysis result by l(l+1) (0 for l = 0).
struct RowOp {
  int8_t tP, cP, kP, tD, cD, kD, scale, pad;
};

// A synthesis term: recipe (legendre.cuh) applied to source arrays ia, ib.
struct TermIx {
  int8_t ia, ib, recipe, pad;
};

struct SplitSynArgs {
  Tables t;
  SplitTables s;
  const double2* arr[12];  // spectral source arrays, (lm_max, ld) complex over levels
  int narr;
  TermIx term[16];
  int64_t ld;           // row stride of the spectral sources (complex)
  const double* or2;    // per level, for kCurlT
  int n_lev;            // levels (columns) of the sources
  int nrows;            // n_lev * row_per_level
  int row_per_level;    // 2 * fields
  int stg_lev;          // levels one 128-row tile can touch (staging width)
  RowOp ops[40];        // per (field, re/im) of a level
  float* Fs;            // [m][sym|asym][theta pair][row]
  int64_t fs_m, fs_c, fs_j;
  uint8_t* aimg;        // A-operand images (workspace), synth_split_image_bytes
  int64_t total_chunks; // K chunks summed over (m, combo)
  int* err;
};

struct SplitAnaArgs {
  Tables t;
  SplitTables s;
  int wk_max;           // max rows of the analysis table images
  const float* G;       // [m][north|south][theta pair][level * g_level + column]
  int64_t g_m, g_h, g_j, g_level;  // g_level: floats per level, multiple of 4
  int n_lev;            // levels of G
  int cols;             // Fourier columns per level (2 per grid output field)
  int lev_tile;         // levels per 128-row tile: floor(128 / cols)
  int n_out;            // spectral outputs; ops[2 o + re/im] is output o's row program
  RowOp ops[32];        // tP/tD name grid output fields (column 2 t + c)
  double2* out[16];     // (lm_max, ld) outputs
  int64_t ld;
  int out_col0;
  uint8_t* aimg;        // folded A-operand images (workspace), anal_split_image_bytes
  int* err;
};

int launch_synth_split(const SplitSynArgs& a, cudaStream_t st);
size_t synth_split_image_bytes(int nrows, int64_t total_chunks);
int launch_anal_split(const SplitAnaArgs& a, cudaStream_t st);
int launch_selftest_wait(int* status, long spins, cudaStream_t st);
size_t anal_split_image_bytes(int n_m, int nhs, int n_lev, int lev_tile);

struct NlSplitArgs {
  Tables t;
  int n_r;
  const float* Fs;      // synthesis output (sym/asym), row = level * 2 nfi + 2 f + re/im
  int64_t fs_m, fs_c, fs_j;
  float* G;             // products (north/south), row = (level-1) * g_level + 2 f + re/im
  int64_t g_m, g_h, g_j, g_level;
  const double *or2, *or4, *orho1, *orho2, *delxr2, *delxh2;
  double LFfac;
  const double* LFfac_r;  // per-level Lorentz factor, or null (LFfac everywhere)
  int cour_mode;
  double cf2, af2, valfac;
  unsigned long long *vr2max, *vh2max;
};

int launch_nl_bouss_split(bool mag, bool chem, const NlSplitArgs& a, cudaStream_t st);

// phi stage of the fused anelastic stage (nl_anel_split.cu); Fs/G as NlSplitArgs
struct NlAnelArgs {
  Tables t;
  int n_r;
  const float* Fs;
  int64_t fs_m, fs_c, fs_j;
  float* G;
  int64_t g_m, g_h, g_j, g_level;
  const double *r, *or1, *or2, *or4, *beta, *orho1, *orho2, *otemp1, *visc, *lambda_, *delxr2,
      *delxh2;
  double LFfac, ViscHeatFac, OhmLossFac;
  int cour_mode;
  double cf2, af2, valfac;
  unsigned long long *vr2max, *vh2max;
  // FP64 rows of the digit-split stage (k_nl_anel_f64), in place of Fs and G:
  //   Fs64[m][north|south][theta pair][level * 2 nfi + 2 f + re/im]
  //   G64[m][north|south][theta pair][(level - 1) * g_level + 2 o + re/im]
  const double* Fs64;
  double* G64;
};
int launch_nl_anel_split(bool mag, bool chem, const NlAnelArgs& a, cudaStream_t st);
// FP64 anelastic phi stage; its dynamic shared memory (0 where n_phi is too
// long for one CTA's buffers)
int launch_nl_anel_f64(bool mag, bool chem, const NlAnelArgs& a, cudaStream_t st);
size_t nl_anel_f64_smem(int n_phi, bool mag, bool chem);

// phi stage of the split drop-in transforms (split_transforms.cu); rows are
// (column b, field f), r = b * nf + f
struct SplitPhiArgs {
  Tables t;
  int nrows;            // B * nf
  int nf;               // fields per column
  int vector_mask;      // bit f: field f takes the vector weight 2 pi w / sin^2 (analysis)
  const float* Fs;      // synthesis output [m][sym|asym][theta pair][2 r + re/im]
  int64_t fs_m, fs_c, fs_j;
  float* G;             // analysis input [m][north|south][theta pair][b * g_level + 2 f + re/im]
  int64_t g_m, g_h, g_j, g_level;
  double* out[3];       // synthesis: grids (B, n_theta, n_phi) per field
  const double* in[3];  // analysis: grids per field
};
int launch_split_phi(bool to_grid, const SplitPhiArgs& a, cudaStream_t st);

}  // namespace mt
