// Shared definitions of the magic_b200 CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/magic_b200.h"

namespace mt {

// Thread-local error message behind mt_last_error().
void set_error(const std::string& msg);

#define MT_CHECK_CUDA(call)                                                        \
  do {                                                                             \
    cudaError_t _e = (call);                                                       \
    if (_e != cudaSuccess) {                                                       \
      ::mt::set_error(std::string(#call) + ": " + cudaGetErrorString(_e));         \
      return MT_ERR_CUDA;                                                          \
    }                                                                              \
  } while (0)

#define MT_REQUIRE(cond, code, msg)                                                \
  do {                                                                             \
    if (!(cond)) {                                                                 \
      ::mt::set_error(msg);                                                        \
      return (code);                                                               \
    }                                                                              \
  } while (0)

#define MT_TRY(expr)              \
  do {                            \
    int _rc = (expr);             \
    if (_rc != MT_OK) return _rc; \
  } while (0)

constexpr int kMaxFftStages = 24;

// Device-side view of the horizontal tables, passed by value to kernels.
struct Tables {
  int l_max, minc, n_theta, n_phi, n_m, lm_max, nhs;
  const int* lstart;       // (n_m) first lm of each order block
  const double* plm;       // (lm_max, nhs) P_l^m over northern Gauss points
  const double* dplm;      // (lm_max, nhs) sin(theta) dP_l^m/dtheta
  const double* dlh;       // (lm_max) l(l+1)
  const double* wq;        // (n_theta) interleaved rows: 2 pi w
  const double* wq_v;      // (n_theta) interleaved rows: 2 pi w / sin^2
  const double* ost2;      // (n_theta) interleaved rows: 1/sin^2
  const double* cosn;      // (n_theta) interleaved rows: cos/sin^2
  const double2* twiddle;  // (n_phi) exp(-2 pi i n / n_phi)
  int fft_nstages;
  int fft_radix[kMaxFftStages];
};

}  // namespace mt

struct mt_plan {
  mt_grid_desc desc;
  int device = 0;
  int l_max = 0, minc = 1, n_theta = 0, n_phi = 0, n_m = 0, lm_max = 0, nhs = 0;
  int precision = MT_PREC_FP64;
  int* d_lstart = nullptr;
  double* d_theta = nullptr;   // geographic order
  double* d_gauss = nullptr;
  double* d_plm = nullptr;
  double* d_dplm = nullptr;
  double* d_dlh = nullptr;
  double* d_wq = nullptr;
  double* d_wq_v = nullptr;
  double* d_ost2 = nullptr;
  double* d_cosn = nullptr;
  double2* d_twiddle = nullptr;
  mt::Tables tab;              // device pointers + sizes, ready for launches
  // split-precision operand planes (null in FP64 plans)
  void* split = nullptr;
  // digit-split table images (MT_PREC_OZAKI plans only)
  void* ozaki = nullptr;
};

namespace mt {

// Build all tables of a plan on the current device (tables.cu); the bf16x3
// table images of split-precision plans (split_tables.cu).
int build_tables(mt_plan* p);
int build_split_tables(mt_plan* p);
void free_split_tables(mt_plan* p);

// Transform launchers (legendre_f64.cu, fourier.cu).
enum class SynthOp { kScalar = 0, kTorpol = 1, kGrad = 2 };
enum class AnalOp { kScalar = 0, kSphtor = 1 };

}  // namespace mt
