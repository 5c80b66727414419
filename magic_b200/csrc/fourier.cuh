// Argument blocks of the phi-stage kernels (fourier.cu, nonlinear.cu).
#pragma once

#include "common.cuh"

namespace mt {

// Fourier array layout used everywhere: F[m][theta_row][col], complex FP64,
// strides f_m (between orders) and f_row (between interleaved theta rows).

struct ToGridArgs {
  Tables t;
  const double2* F;
  int64_t f_m, f_row;
  int ncols;        // columns = n_fields * B (column c -> field c / B, entry c % B)
  int B;
  double* out[4];   // per field grids (B, n_theta, n_phi)
};

struct ToFourierArgs {
  Tables t;
  const double* in[4];
  int ncols, B;
  int vector;       // weight 2 pi w / sin^2 (vector components) instead of 2 pi w
  double2* F;
  int64_t f_m, f_row;
};

int launch_fourier_to_grid(const ToGridArgs& a, cudaStream_t st);
int launch_grid_to_fourier(const ToFourierArgs& a, cudaStream_t st);
int fft_max_nphi();

struct NlBoussArgs {
  Tables t;
  int n_r;
  const double2* F;  // synthesis output, column = r * nfi + field
  int64_t f_m, f_row;
  double2* G;        // analysis input, column = (r - 1) * nfo + field
  int64_t g_m, g_row;
  const double *or2, *or4, *orho1, *orho2, *delxr2, *delxh2;
  double LFfac;
  const double* LFfac_r;  // per-level Lorentz factor, or null (LFfac everywhere)
  int cour_mode;     // 0 non-magnetic, 1 damped, 2 undamped
  double cf2, af2, valfac;  // courfac^2, alffac^2, (0.5 (1 + 1/Pm))^2
  unsigned long long *vr2max, *vh2max;  // (n_r) non-negative doubles as bits
  // Digit-split (ozaki) stage layout, used when split_io is set: the synthesis
  // delivers north / south FP64 rows
  //   Fs[m][north|south][theta pair][level * 2 nfi + 2 f + re/im]
  // and the analysis reads plain north / south FP64 rows
  //   Gs[m][north|south][theta pair][(level - 1) * g_level + 2 f + re/im].
  int split_io;
  const double* Fs;
  int64_t fs_m, fs_c, fs_j;
  double* Gs;
  int64_t g_m2, g_h, g_j, g_level;
};

int launch_nl_bouss(bool mag, bool chem, const NlBoussArgs& a, cudaStream_t st);
int launch_courant_finish(int n_r, const unsigned long long* vr2, const unsigned long long* vh2,
                          const double* delxr2, const double* delxh2, double* dtr, double* dth,
                          cudaStream_t st);

struct GridNlArgs {
  int n_r, nt, np;
  const double* in[19];
  double* out[13];
  const double *r, *or1, *or2, *or4, *beta, *orho1, *otemp1, *visc, *lambda_;
  const double *ost2, *cosn;
  double LFfac, ViscHeatFac, OhmLossFac;
  int l_mag;
};
int launch_get_nl_grid(bool anel, const GridNlArgs& a, cudaStream_t st);

struct CourantGridArgs {
  int n_r, nt, np, mode;
  const double *vr, *vt, *vp, *br, *bt, *bp;
  const double *or2, *or4, *orho1, *orho2, *delxr2, *delxh2, *ost2;
  double LFfac, cf2, af2, valfac;
  unsigned long long *vr2max, *vh2max;
};
int launch_courant_grid(const CourantGridArgs& a, cudaStream_t st);

}  // namespace mt
