// extern "C" entry points (include/magic_b200.h).
#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "fourier.cuh"
#include "legendre.cuh"
#include "ozaki.cuh"
#include "split_kernels.cuh"

namespace mt {

static thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }

// legendre_f64.cu
template <class OP, int R>
int launch_synth_f64(const SynthArgs<OP::NX>& a, cudaStream_t st);
template <class OP, int R>
int launch_anal_f64(const AnalArgs<OP::NX, OP::NO>& a, cudaStream_t st);

// split_tables.cu
const SplitTables& split_tables(const mt_plan* p);
const std::vector<int>& split_wk_host(const mt_plan* p);
int split_syn_total_chunks(const mt_plan* p);

static int prime_decomposition(int n) {
  // smallest 2^i 3^j 5^k >= n, i < 13, j < 7, k < 7 (magic_torch/params.py:12-24)
  long best = -1;
  for (int i = 0; i < 13; ++i)
    for (int j = 0; j < 7; ++j)
      for (int k = 0; k < 7; ++k) {
        long v = 1;
        for (int q = 0; q < i; ++q) v *= 2;
        for (int q = 0; q < j; ++q) v *= 3;
        for (int q = 0; q < k; ++q) v *= 5;
        if (v >= n && (best < 0 || v < best)) best = v;
      }
  return (int)best;
}

static int check_plan(const mt_plan* p) {
  MT_REQUIRE(p != nullptr, MT_ERR_ARG, "null plan");
  int dev = -1;
  MT_CHECK_CUDA(cudaGetDevice(&dev));
  MT_REQUIRE(dev == p->device, MT_ERR_ARG, "plan used on a different device than it was built on");
  return MT_OK;
}


static size_t fourier_bytes(const mt_plan* p, int64_t ncols) {
  return (size_t)p->n_m * p->n_theta * ncols * sizeof(double2);
}

}  // namespace mt

using namespace mt;

namespace mt {

// ---- split-precision drop-in transforms -----------------------------------
//
// Synthesis: packing + tcgen05 GEMM (legendre_split.cu) with the batch
// columns in place of radial levels, then the FP32 phi stage
// (split_transforms.cu) writes the FP64 grids.  Analysis: FP32 phi stage,
// then folding + tcgen05 GEMM.  Workspace: [error int | Fourier rows | operand
// images].

struct SplitTrWs {
  size_t f, img, total;
};

static RowOp rop(int tP, int cP, int kP, int tD = 0, int cD = 0, int kD = 0, int scale = 0);
static void syn_group_ops(RowOp* ops, int Q, int S, int T);
static int ana_scalar_ops(RowOp* ops, int x);
static int ana_s_ops(RowOp* ops, int a, int b);
static int ana_t_ops(RowOp* ops, int a, int b);

static SplitTrWs split_tr_ws(const mt_plan* p, int B, int nf) {
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t rows = (size_t)B * 2 * nf;
  const size_t gl = (size_t)((2 * nf + 3) & ~3);
  const size_t fs = (size_t)p->n_m * 2 * p->nhs * rows * sizeof(float);
  const size_t g = (size_t)p->n_m * 2 * p->nhs * B * gl * sizeof(float);
  const size_t img = std::max(synth_split_image_bytes((int)rows, split_syn_total_chunks(p)),
                              anal_split_image_bytes(p->n_m, p->nhs, B, 128 / (2 * nf)));
  SplitTrWs w;
  w.f = 256;
  w.img = w.f + al(std::max(fs, g));
  w.total = w.img + al(img);
  return w;
}

// Synthesis of nf grid fields per column from narr spectral arrays; terms and
// row programs (2 nf per column) as in the fused stage.
static int split_synth_tr(const mt_plan* p, int B, int nf, int narr, const double* const* arr,
                          int64_t ld, const TermIx* terms, int nterms, const RowOp* ops,
                          double* const* out, void* work, cudaStream_t st) {
  const SplitTrWs W = split_tr_ws(p, B, nf);
  char* w = (char*)work;
  int* err = (int*)w;
  MT_CHECK_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
  SplitSynArgs s{};
  s.t = p->tab;
  s.s = split_tables(p);
  for (int i = 0; i < narr; ++i) s.arr[i] = (const double2*)arr[i];
  s.narr = narr;
  for (int i = 0; i < nterms; ++i) s.term[i] = terms[i];
  s.ld = ld;
  s.or2 = nullptr;
  s.n_lev = B;
  s.row_per_level = 2 * nf;
  s.nrows = B * 2 * nf;
  s.stg_lev = std::min(B, 127 / s.row_per_level + 2);
  for (int i = 0; i < 2 * nf; ++i) s.ops[i] = ops[i];
  s.Fs = (float*)(w + W.f);
  s.fs_j = s.nrows;
  s.fs_c = (int64_t)p->nhs * s.fs_j;
  s.fs_m = 2 * s.fs_c;
  s.aimg = (uint8_t*)(w + W.img);
  s.total_chunks = split_syn_total_chunks(p);
  s.err = err;
  MT_TRY(launch_synth_split(s, st));
  SplitPhiArgs f{};
  f.t = p->tab;
  f.nrows = B * nf;
  f.nf = nf;
  f.Fs = s.Fs;
  f.fs_m = s.fs_m;
  f.fs_c = s.fs_c;
  f.fs_j = s.fs_j;
  for (int i = 0; i < nf; ++i) f.out[i] = out[i];
  return launch_split_phi(true, f, st);
}

// Analysis of nf grid fields per column into n_out spectral outputs.
static int split_anal_tr(const mt_plan* p, int B, int nf, int vector_mask,
                         const double* const* in, int n_out, const RowOp* ops, double* const* out,
                         int64_t ld, void* work, cudaStream_t st) {
  const SplitTrWs W = split_tr_ws(p, B, nf);
  char* w = (char*)work;
  int* err = (int*)w;
  MT_CHECK_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
  SplitPhiArgs f{};
  f.t = p->tab;
  f.nrows = B * nf;
  f.nf = nf;
  f.vector_mask = vector_mask;
  f.G = (float*)(w + W.f);
  f.g_level = (2 * nf + 3) & ~3;
  f.g_j = (int64_t)B * f.g_level;
  f.g_h = (int64_t)p->nhs * f.g_j;
  f.g_m = 2 * f.g_h;
  for (int i = 0; i < nf; ++i) f.in[i] = in[i];
  MT_TRY(launch_split_phi(false, f, st));
  SplitAnaArgs a{};
  a.t = p->tab;
  a.s = split_tables(p);
  {
    const std::vector<int>& wk = split_wk_host(p);
    a.wk_max = *std::max_element(wk.begin(), wk.end());
  }
  a.G = f.G;
  a.g_m = f.g_m;
  a.g_h = f.g_h;
  a.g_j = f.g_j;
  a.g_level = f.g_level;
  a.n_lev = B;
  a.cols = 2 * nf;
  a.lev_tile = 128 / a.cols;
  a.n_out = n_out;
  for (int i = 0; i < 2 * n_out; ++i) a.ops[i] = ops[i];
  for (int i = 0; i < n_out; ++i) a.out[i] = (double2*)out[i];
  a.ld = ld;
  a.out_col0 = 0;
  a.aimg = (uint8_t*)(w + W.img);
  a.err = err;
  return launch_anal_split(a, st);
}

static TermIx term_ix(int ia, int recipe) {
  TermIx x;
  x.ia = (int8_t)ia;
  x.ib = 0;
  x.recipe = (int8_t)recipe;
  x.pad = 0;
  return x;
}

}  // namespace mt

extern "C" {

const char* mt_last_error(void) { return g_err.c_str(); }

int mt_plan_create(const mt_grid_desc* desc, mt_plan** out) {
  MT_REQUIRE(desc && out, MT_ERR_ARG, "null argument");
  *out = nullptr;
  MT_REQUIRE(desc->l_max >= 1 && desc->minc >= 1 && desc->minc <= desc->l_max + 1, MT_ERR_ARG,
             "l_max >= 1 and 1 <= minc required");
  MT_REQUIRE(desc->precision == MT_PREC_FP64 || desc->precision == MT_PREC_SPLIT ||
                 desc->precision == MT_PREC_OZAKI,
             MT_ERR_UNSUPPORTED, "precision must be MT_PREC_FP64, MT_PREC_SPLIT or MT_PREC_OZAKI");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    set_error("no CUDA device");
    return MT_ERR_NO_DEVICE;
  }
  int dev = 0;
  MT_CHECK_CUDA(cudaGetDevice(&dev));
  cudaDeviceProp prop;
  MT_CHECK_CUDA(cudaGetDeviceProperties(&prop, dev));
  MT_REQUIRE(prop.major == 10, MT_ERR_NO_DEVICE, "an sm_100 (B200) device is required");

  mt_plan* p = new mt_plan();
  p->desc = *desc;
  p->device = dev;
  p->l_max = desc->l_max;
  p->minc = desc->minc;
  int n_phi_tot = prime_decomposition(2 * ((30 * desc->l_max) / 20));
  p->n_phi = desc->n_phi_max > 0 ? desc->n_phi_max : n_phi_tot / desc->minc;
  p->n_theta = desc->n_theta_max > 0 ? desc->n_theta_max : n_phi_tot / 2;
  p->n_m = desc->l_max / desc->minc + 1;
  p->lm_max = 0;
  for (int m = 0; m <= desc->l_max; m += desc->minc) p->lm_max += desc->l_max - m + 1;
  p->nhs = p->n_theta / 2;
  p->precision = desc->precision;
  auto fail = [&](int code, const char* msg) {
    set_error(msg);
    mt_plan_destroy(p);
    return code;
  };
  if (p->n_theta < 2 || p->n_theta % 2) return fail(MT_ERR_UNSUPPORTED, "n_theta_max must be even");
  if (p->n_phi > fft_max_nphi())
    return fail(MT_ERR_UNSUPPORTED, "n_phi_max above the shared-memory FFT limit (1170)");
  if (2 * (p->n_m - 1) >= p->n_phi)
    return fail(MT_ERR_UNSUPPORTED, "n_phi_max too small for l_max/minc (modes alias)");
  int rc = build_tables(p);
  if (rc == MT_OK && p->precision == MT_PREC_SPLIT) rc = build_split_tables(p);
  if (rc == MT_OK && p->precision == MT_PREC_OZAKI) rc = build_ozaki_tables(p);
  if (rc != MT_OK) {
    std::string keep = g_err;
    mt_plan_destroy(p);
    g_err = keep;
    return rc;
  }
  *out = p;
  return MT_OK;
}

int mt_plan_destroy(mt_plan* p) {
  if (!p) return MT_OK;
  void* ptrs[] = {p->d_lstart, p->d_theta, p->d_gauss, p->d_plm, p->d_dplm, p->d_dlh,
                  p->d_wq,     p->d_wq_v,  p->d_ost2,  p->d_cosn, p->d_twiddle};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  free_split_tables(p);
  free_ozaki_tables(p);
  delete p;
  return MT_OK;
}

int mt_plan_get_info(const mt_plan* p, mt_plan_info* info) {
  MT_REQUIRE(p && info, MT_ERR_ARG, "null argument");
  info->l_max = p->l_max;
  info->minc = p->minc;
  info->n_theta_max = p->n_theta;
  info->n_phi_max = p->n_phi;
  info->n_m_max = p->n_m;
  info->lm_max = p->lm_max;
  info->nhs = p->nhs;
  info->precision = p->precision;
  return MT_OK;
}

int mt_plan_copy_tables(const mt_plan* p, double* theta, double* gauss, double* plm, double* dplm,
                        void* stream) {
  MT_TRY(check_plan(p));
  cudaStream_t st = (cudaStream_t)stream;
  size_t tsz = (size_t)p->lm_max * p->nhs * sizeof(double);
  if (theta)
    MT_CHECK_CUDA(cudaMemcpyAsync(theta, p->d_theta, p->n_theta * 8, cudaMemcpyDeviceToDevice, st));
  if (gauss)
    MT_CHECK_CUDA(cudaMemcpyAsync(gauss, p->d_gauss, p->n_theta * 8, cudaMemcpyDeviceToDevice, st));
  if (plm) MT_CHECK_CUDA(cudaMemcpyAsync(plm, p->d_plm, tsz, cudaMemcpyDeviceToDevice, st));
  if (dplm) MT_CHECK_CUDA(cudaMemcpyAsync(dplm, p->d_dplm, tsz, cudaMemcpyDeviceToDevice, st));
  return MT_OK;
}

size_t mt_transform_workspace(const mt_plan* p, int B, int n_fields) {
  if (!p || B < 1 || n_fields < 1) return 0;
  if (p->precision == MT_PREC_SPLIT) return split_tr_ws(p, B, n_fields).total;
  return fourier_bytes(p, (int64_t)B * n_fields);
}

static int check_ws(const mt_plan* p, int B, int nf, size_t bytes, const void* work) {
  MT_REQUIRE(B >= 1, MT_ERR_ARG, "B >= 1 required");
  MT_REQUIRE(work != nullptr, MT_ERR_ARG, "null workspace");
  MT_REQUIRE(bytes >= mt_transform_workspace(p, B, nf), MT_ERR_WORKSPACE, "workspace too small");
  return MT_OK;
}

int mt_scal_to_spat(const mt_plan* p, const double* Slm, int64_t ld, int B, double* grid,
                    void* work, size_t work_bytes, void* stream) {
  MT_TRY(check_plan(p));
  MT_REQUIRE(Slm && grid && ld >= B, MT_ERR_ARG, "bad spectral/grid argument");
  MT_TRY(check_ws(p, B, 1, work_bytes, work));
  cudaStream_t st = (cudaStream_t)stream;
  if (p->precision == MT_PREC_SPLIT) {
    const TermIx tm[1] = {term_ix(0, kRaw)};
    const RowOp ops[2] = {rop(0, 0, 1), rop(0, 1, 1)};
    return split_synth_tr(p, B, 1, 1, &Slm, ld, tm, 1, ops, &grid, work, st);
  }
  double2* F = (double2*)work;
  SynthArgs<1> s{};
  s.t = p->tab;
  s.src[0] = {(const double2*)Slm, nullptr, kRaw};
  s.ld = ld;
  s.ncols = B;
  s.F = F;
  s.f_row = B;
  s.f_m = (int64_t)p->n_theta * B;
  s.col_f = B;
  s.col_c = 1;
  MT_TRY((launch_synth_f64<SynScalar, 16>(s, st)));
  ToGridArgs g{};
  g.t = p->tab;
  g.F = F;
  g.f_m = s.f_m;
  g.f_row = s.f_row;
  g.ncols = B;
  g.B = B;
  g.out[0] = grid;
  return launch_fourier_to_grid(g, st);
}

}  // extern "C"

namespace mt {

// Fixed scratch of mt_scal_to_spat_noalloc.  Host code must not pass the
// symbol itself to a kernel (on the host it names a stand-in, not device
// memory): its device address is looked up once per device with
// cudaGetSymbolAddress while that device is current.
static __device__ __align__(256) unsigned char g_noalloc_scratch[MT_NOALLOC_SCRATCH_BYTES];
static std::mutex g_noalloc_mu;
constexpr int kNoallocMaxDevices = 64;
static void* g_noalloc_ptr[kNoallocMaxDevices] = {};

static int noalloc_scratch(void** out) {
  int dev = -1;
  MT_CHECK_CUDA(cudaGetDevice(&dev));
  MT_REQUIRE(dev >= 0 && dev < kNoallocMaxDevices, MT_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* ptr = nullptr;
    MT_CHECK_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
    g_noalloc_ptr[dev] = ptr;
  }
  *out = g_noalloc_ptr[dev];
  return MT_OK;
}

}  // namespace mt

extern "C" {

int mt_scal_to_spat_noalloc(const mt_plan* p, const double* Slm, int64_t ld, int B, double* grid,
                            void* stream) {
  MT_TRY(check_plan(p));
  MT_REQUIRE(B >= 1, MT_ERR_ARG, "B >= 1 required");
  const size_t need = mt_transform_workspace(p, B, 1);
  MT_REQUIRE(need <= MT_NOALLOC_SCRATCH_BYTES, MT_ERR_WORKSPACE,
             "mt_scal_to_spat_noalloc: B too large for the fixed 16 MiB scratch "
             "(need mt_transform_workspace(plan, B, 1) bytes); use mt_scal_to_spat with a "
             "workspace");
  void* work = nullptr;
  MT_TRY(noalloc_scratch(&work));
  return mt_scal_to_spat(p, Slm, ld, B, grid, work, MT_NOALLOC_SCRATCH_BYTES, stream);
}

int mt_scal_to_grad_spat(const mt_plan* p, const double* Slm, int64_t ld, int B, int scale_dlh,
                         double* gt, double* gp, void* work, size_t work_bytes, void* stream) {
  MT_TRY(check_plan(p));
  MT_REQUIRE(Slm && gt && gp && ld >= B, MT_ERR_ARG, "bad spectral/grid argument");
  MT_TRY(check_ws(p, B, 2, work_bytes, work));
  cudaStream_t st = (cudaStream_t)stream;
  if (p->precision == MT_PREC_SPLIT) {
    // theta = dP.S, phi = i m P.S
    const TermIx tm[1] = {term_ix(0, scale_dlh ? kDlh : kRaw)};
    const RowOp ops[4] = {rop(0, 0, 0, 0, 0, 1), rop(0, 0, 0, 0, 1, 1), rop(0, 1, 4),
                          rop(0, 0, 3)};
    double* outs[2] = {gt, gp};
    return split_synth_tr(p, B, 2, 1, &Slm, ld, tm, 1, ops, outs, work, st);
  }
  double2* F = (double2*)work;
  SynthArgs<1> s{};
  s.t = p->tab;
  s.src[0] = {(const double2*)Slm, nullptr, scale_dlh ? kDlh : kRaw};
  s.ld = ld;
  s.ncols = B;
  s.F = F;
  s.f_row = 2 * (int64_t)B;
  s.f_m = (int64_t)p->n_theta * s.f_row;
  s.col_f = B;
  s.col_c = 1;
  MT_TRY((launch_synth_f64<SynGrad, 16>(s, st)));
  ToGridArgs g{};
  g.t = p->tab;
  g.F = F;
  g.f_m = s.f_m;
  g.f_row = s.f_row;
  g.ncols = 2 * B;
  g.B = B;
  g.out[0] = gt;
  g.out[1] = gp;
  return launch_fourier_to_grid(g, st);
}

int mt_torpol_to_spat(const mt_plan* p, const double* Q, const double* S, const double* T,
                      int64_t ld, int B, double* br, double* bt, double* bp, void* work,
                      size_t work_bytes, void* stream) {
  MT_TRY(check_plan(p));
  MT_REQUIRE(Q && S && T && br && bt && bp && ld >= B, MT_ERR_ARG, "bad spectral/grid argument");
  MT_TRY(check_ws(p, B, 3, work_bytes, work));
  cudaStream_t st = (cudaStream_t)stream;
  if (p->precision == MT_PREC_SPLIT) {
    const TermIx tm[3] = {term_ix(0, kRaw), term_ix(1, kRaw), term_ix(2, kRaw)};
    RowOp ops[6];
    syn_group_ops(ops, 0, 1, 2);
    const double* arrs[3] = {Q, S, T};
    double* outs[3] = {br, bt, bp};
    return split_synth_tr(p, B, 3, 3, arrs, ld, tm, 3, ops, outs, work, st);
  }
  double2* F = (double2*)work;
  SynthArgs<3> s{};
  s.t = p->tab;
  s.src[0] = {(const double2*)Q, nullptr, kRaw};
  s.src[1] = {(const double2*)S, nullptr, kRaw};
  s.src[2] = {(const double2*)T, nullptr, kRaw};
  s.ld = ld;
  s.ncols = B;
  s.F = F;
  s.f_row = 3 * (int64_t)B;
  s.f_m = (int64_t)p->n_theta * s.f_row;
  s.col_f = B;
  s.col_c = 1;
  MT_TRY((launch_synth_f64<SynTorpol, 8>(s, st)));
  ToGridArgs g{};
  g.t = p->tab;
  g.F = F;
  g.f_m = s.f_m;
  g.f_row = s.f_row;
  g.ncols = 3 * B;
  g.B = B;
  g.out[0] = br;
  g.out[1] = bt;
  g.out[2] = bp;
  return launch_fourier_to_grid(g, st);
}

int mt_scal_to_SH(const mt_plan* p, const double* grid, int B, double* Slm, int64_t ld,
                  void* work, size_t work_bytes, void* stream) {
  MT_TRY(check_plan(p));
  MT_REQUIRE(Slm && grid && ld >= B, MT_ERR_ARG, "bad spectral/grid argument");
  MT_TRY(check_ws(p, B, 1, work_bytes, work));
  cudaStream_t st = (cudaStream_t)stream;
  if (p->precision == MT_PREC_SPLIT) {
    RowOp ops[2];
    ana_scalar_ops(ops, 0);
    return split_anal_tr(p, B, 1, 0, &grid, 1, ops, &Slm, ld, work, st);
  }
  double2* F = (double2*)work;
  ToFourierArgs f{};
  f.t = p->tab;
  f.in[0] = grid;
  f.ncols = B;
  f.B = B;
  f.vector = 0;
  f.F = F;
  f.f_row = B;
  f.f_m = (int64_t)p->n_theta * B;
  MT_TRY(launch_grid_to_fourier(f, st));
  AnalArgs<1, 1> a{};
  a.t = p->tab;
  a.F = F;
  a.f_m = f.f_m;
  a.f_row = f.f_row;
  a.col_x = B;
  a.col_c = 1;
  a.ncols = B;
  a.out[0] = (double2*)Slm;
  a.ld = ld;
  a.out_col0 = 0;
  return launch_anal_f64<AnaScalar, 8>(a, st);
}

int mt_spat_to_sphertor(const mt_plan* p, const double* vt, const double* vp, int B, double* S,
                        double* T, int64_t ld, void* work, size_t work_bytes, void* stream) {
  MT_TRY(check_plan(p));
  MT_REQUIRE(vt && vp && S && T && ld >= B, MT_ERR_ARG, "bad spectral/grid argument");
  MT_TRY(check_ws(p, B, 2, work_bytes, work));
  cudaStream_t st = (cudaStream_t)stream;
  if (p->precision == MT_PREC_SPLIT) {
    RowOp ops[4];
    ana_s_ops(ops, 0, 1);
    ana_t_ops(ops + 2, 0, 1);
    const double* ins[2] = {vt, vp};
    double* outs[2] = {S, T};
    return split_anal_tr(p, B, 2, 3, ins, 2, ops, outs, ld, work, st);
  }
  double2* F = (double2*)work;
  ToFourierArgs f{};
  f.t = p->tab;
  f.in[0] = vt;
  f.in[1] = vp;
  f.ncols = 2 * B;
  f.B = B;
  f.vector = 1;
  f.F = F;
  f.f_row = 2 * (int64_t)B;
  f.f_m = (int64_t)p->n_theta * f.f_row;
  MT_TRY(launch_grid_to_fourier(f, st));
  AnalArgs<2, 2> a{};
  a.t = p->tab;
  a.F = F;
  a.f_m = f.f_m;
  a.f_row = f.f_row;
  a.col_x = B;
  a.col_c = 1;
  a.ncols = B;
  a.out[0] = (double2*)S;
  a.out[1] = (double2*)T;
  a.ld = ld;
  a.out_col0 = 0;
  return launch_anal_f64<AnaSphtor, 8>(a, st);
}

int mt_get_nl(const mt_plan* p, int n_r, const double* const* in, double* const* out,
              const double* or2, const double* or4, double LFfac, void* stream) {
  MT_TRY(check_plan(p));
  MT_REQUIRE(in && out && or2 && or4 && n_r >= 1, MT_ERR_ARG, "bad argument");
  GridNlArgs a{};
  a.n_r = n_r;
  a.nt = p->n_theta;
  a.np = p->n_phi;
  for (int i = 0; i < 14; ++i) {
    MT_REQUIRE(in[i], MT_ERR_ARG, "null input grid");
    a.in[i] = in[i];
  }
  for (int i = 0; i < 12; ++i) {
    MT_REQUIRE(out[i], MT_ERR_ARG, "null output grid");
    a.out[i] = out[i];
  }
  a.or2 = or2;
  a.or4 = or4;
  a.ost2 = p->d_ost2;
  a.cosn = p->d_cosn;
  a.LFfac = LFfac;
  a.l_mag = 1;
  return launch_get_nl_grid(false, a, (cudaStream_t)stream);
}

int mt_get_nl_anel(const mt_plan* p, int n_r, const double* const* in, double* const* out,
                   const mt_anel_params* q, void* stream) {
  MT_TRY(check_plan(p));
  MT_REQUIRE(in && out && q && n_r >= 1, MT_ERR_ARG, "bad argument");
  MT_REQUIRE(q->r && q->or1 && q->or2 && q->or4 && q->beta && q->orho1 && q->otemp1 && q->visc &&
                 q->lambda_,
             MT_ERR_ARG, "null radial profile");
  GridNlArgs a{};
  a.n_r = n_r;
  a.nt = p->n_theta;
  a.np = p->n_phi;
  for (int i = 0; i < 19; ++i) {
    MT_REQUIRE(in[i], MT_ERR_ARG, "null input grid");
    a.in[i] = in[i];
  }
  for (int i = 0; i < 13; ++i) {
    MT_REQUIRE(out[i], MT_ERR_ARG, "null output grid");
    a.out[i] = out[i];
  }
  a.r = q->r;
  a.or1 = q->or1;
  a.or2 = q->or2;
  a.or4 = q->or4;
  a.beta = q->beta;
  a.orho1 = q->orho1;
  a.otemp1 = q->otemp1;
  a.visc = q->visc;
  a.lambda_ = q->lambda_;
  a.ost2 = p->d_ost2;
  a.cosn = p->d_cosn;
  a.LFfac = q->LFfac;
  a.ViscHeatFac = q->ViscHeatFac;
  a.OhmLossFac = q->OhmLossFac;
  a.l_mag = q->l_mag;
  return launch_get_nl_grid(true, a, (cudaStream_t)stream);
}

size_t mt_courant_workspace(const mt_plan* p, int n_r) {
  (void)p;
  return n_r > 0 ? (size_t)2 * n_r * sizeof(unsigned long long) : 0;
}

int mt_courant(const mt_plan* p, int n_r, const double* vr, const double* vt, const double* vp,
               const double* br, const double* bt, const double* bp, const mt_courant_params* q,
               double* dtrkc, double* dthkc, void* work, size_t work_bytes, void* stream) {
  MT_TRY(check_plan(p));
  MT_REQUIRE(q && vr && vt && vp && dtrkc && dthkc && n_r >= 1, MT_ERR_ARG, "bad argument");
  MT_REQUIRE(q->mode >= 0 && q->mode <= 2, MT_ERR_ARG, "mode must be 0, 1 or 2");
  MT_REQUIRE(q->mode == 0 || (br && bt && bp), MT_ERR_ARG, "magnetic grids required");
  MT_REQUIRE(q->or2 && q->or4 && q->orho1 && q->orho2 && q->delxr2 && q->delxh2, MT_ERR_ARG,
             "null radial profile");
  MT_REQUIRE(work && work_bytes >= mt_courant_workspace(p, n_r), MT_ERR_WORKSPACE,
             "workspace too small");
  cudaStream_t st = (cudaStream_t)stream;
  unsigned long long* mx = (unsigned long long*)work;
  MT_CHECK_CUDA(cudaMemsetAsync(mx, 0, 2 * n_r * sizeof(unsigned long long), st));
  CourantGridArgs a{};
  a.n_r = n_r;
  a.nt = p->n_theta;
  a.np = p->n_phi;
  a.mode = q->mode;
  a.vr = vr;
  a.vt = vt;
  a.vp = vp;
  a.br = br;
  a.bt = bt;
  a.bp = bp;
  a.or2 = q->or2;
  a.or4 = q->or4;
  a.orho1 = q->orho1;
  a.orho2 = q->orho2;
  a.delxr2 = q->delxr2;
  a.delxh2 = q->delxh2;
  a.ost2 = p->d_ost2;
  a.LFfac = q->LFfac;
  a.cf2 = q->courfac * q->courfac;
  a.af2 = q->alffac * q->alffac;
  double h = 0.5 * (1.0 + q->opm);
  a.valfac = h * h;
  a.vr2max = mx;
  a.vh2max = mx + n_r;
  MT_TRY(launch_courant_grid(a, st));
  return launch_courant_finish(n_r, mx, mx + n_r, q->delxr2, q->delxh2, dtrkc, dthkc, st);
}

}  // extern "C"

namespace mt {

static int bouss_nfi(int mag, int chem) { return (mag ? 6 : 0) + 7 + (chem ? 1 : 0); }
static int bouss_nfo(int mag, int chem) { return 6 + (mag ? 3 : 0) + (chem ? 3 : 0); }

template <bool MAG, bool CHEM>
static int nl_bouss_t(const mt_plan* p, int n_r, const mt_bouss_in* in, const mt_bouss_out* out,
                      const mt_bouss_params* q, double* dtrkc, double* dthkc, void* work,
                      cudaStream_t st) {
  const int nfi = bouss_nfi(MAG, CHEM), nfo = bouss_nfo(MAG, CHEM);
  char* w = (char*)work;
  double2* F = (double2*)w;
  w += fourier_bytes(p, (int64_t)n_r * nfi);
  double2* G = (double2*)w;
  w += fourier_bytes(p, (int64_t)(n_r - 2) * nfo);
  unsigned long long* mx = (unsigned long long*)w;
  const int parts = q->parts ? q->parts : 7;
  auto c = [](const double* x) { return (const double2*)x; };
  const int64_t f_row = (int64_t)n_r * nfi, f_m = (int64_t)p->n_theta * f_row;

  // Legendre synthesis of the 14 grid fields, two launches
  // (magic_torch/step_time.py:980-1013 input assembly on load)
  if ((parts & 1) && MAG) {
    SynthArgs<6> s{};
    s.t = p->tab;
    s.src[0] = {c(in->b), nullptr, kDlh};
    s.src[1] = {c(in->db), nullptr, kRaw};
    s.src[2] = {c(in->aj), nullptr, kRaw};
    s.src[3] = {c(in->aj), nullptr, kDlh};
    s.src[4] = {c(in->dj), nullptr, kRaw};
    s.src[5] = {c(in->b), c(in->ddb), kCurlT};
    s.ld = in->ld;
    s.ncols = n_r;
    s.or2 = q->or2;
    s.F = F;
    s.f_row = f_row;
    s.f_m = f_m;
    s.col_f = 1;
    s.col_c = nfi;
    MT_TRY((launch_synth_f64<SynGroups<2, 0>, 8>(s, st)));
  }
  if (parts & 1) {
    using SO = SynGroups<2, CHEM ? 2 : 1>;
    SynthArgs<SO::NX> s{};
    s.t = p->tab;
    s.src[0] = {c(in->w), nullptr, kDlh};
    s.src[1] = {c(in->dw), nullptr, kRaw};
    s.src[2] = {c(in->z), nullptr, kRaw};
    s.src[3] = {c(in->z), nullptr, kDlh};
    s.src[4] = {c(in->dz), nullptr, kRaw};
    s.src[5] = {c(in->w), c(in->ddw), kCurlT};
    s.src[6] = {c(in->s), nullptr, kRaw};
    if (CHEM) s.src[SO::NX - 1] = {c(in->xi), nullptr, kRaw};
    s.ld = in->ld;
    s.ncols = n_r;
    s.or2 = q->or2;
    s.F = F + (MAG ? 6 : 0);
    s.f_row = f_row;
    s.f_m = f_m;
    s.col_f = 1;
    s.col_c = nfi;
    MT_TRY((launch_synth_f64<SO, 8>(s, st)));
  }

  NlBoussArgs nl{};
  nl.t = p->tab;
  nl.n_r = n_r;
  nl.F = F;
  nl.f_m = f_m;
  nl.f_row = f_row;
  nl.G = G;
  nl.g_row = (int64_t)(n_r - 2) * nfo;
  nl.g_m = (int64_t)p->n_theta * nl.g_row;
  nl.or2 = q->or2;
  nl.or4 = q->or4;
  nl.orho1 = q->orho1;
  nl.orho2 = q->orho2;
  nl.delxr2 = q->delxr2;
  nl.delxh2 = q->delxh2;
  nl.LFfac = q->LFfac;
  nl.LFfac_r = q->LFfac_r;
  nl.cour_mode = MAG ? q->cour_mode : 0;
  nl.cf2 = q->courfac * q->courfac;
  nl.af2 = q->alffac * q->alffac;
  double h = 0.5 * (1.0 + q->opm);
  nl.valfac = h * h;
  nl.vr2max = mx;
  nl.vh2max = mx + n_r;
  if (parts & 2) {
    MT_CHECK_CUDA(cudaMemsetAsync(mx, 0, 2 * n_r * sizeof(unsigned long long), st));
    MT_TRY(launch_nl_bouss(MAG, CHEM, nl, st));
  }
  if (!(parts & 4)) return MT_OK;

  // Legendre analysis of the products, two launches
  // (magic_torch/step_time.py:1066-1124)
  auto anal_args = [&](auto& a, int field0) {
    a.t = p->tab;
    a.F = G + field0;
    a.f_m = nl.g_m;
    a.f_row = nl.g_row;
    a.col_x = 1;
    a.col_c = nfo;
    a.ncols = n_r - 2;
    a.ld = out->ld;
    a.out_col0 = 1;
  };
  {
    AnalArgs<6, 5> a{};
    anal_args(a, 0);
    a.out[0] = (double2*)out->Advr;
    a.out[1] = (double2*)out->Advt;
    a.out[2] = (double2*)out->Advp;
    a.out[3] = (double2*)out->VSr;
    a.out[4] = (double2*)out->VSt;
    MT_TRY((launch_anal_f64<AnaGroups<1, 2>, 8>(a, st)));
  }
  if (MAG && CHEM) {
    AnalArgs<6, 5> a{};
    anal_args(a, 6);
    a.out[0] = (double2*)out->VxBr;
    a.out[1] = (double2*)out->VxBt;
    a.out[2] = (double2*)out->VxBp;
    a.out[3] = (double2*)out->VXir;
    a.out[4] = (double2*)out->VXit;
    MT_TRY((launch_anal_f64<AnaGroups<1, 2>, 8>(a, st)));
  } else if (MAG) {
    AnalArgs<3, 3> a{};
    anal_args(a, 6);
    a.out[0] = (double2*)out->VxBr;
    a.out[1] = (double2*)out->VxBt;
    a.out[2] = (double2*)out->VxBp;
    MT_TRY((launch_anal_f64<AnaGroups<1, 0>, 8>(a, st)));
  } else if (CHEM) {
    AnalArgs<3, 2> a{};
    anal_args(a, 6);
    a.out[0] = (double2*)out->VXir;
    a.out[1] = (double2*)out->VXit;
    MT_TRY((launch_anal_f64<AnaGroups<2, 0>, 8>(a, st)));
  }
  return launch_courant_finish(n_r, mx, mx + n_r, q->delxr2, q->delxh2, dtrkc, dthkc, st);
}

// ---- split-precision fused stage ------------------------------------------

struct SplitWs {
  size_t err, fs, gs, mx, aimg, total;
  int64_t rows_syn, rows_nl, g_level;
};

// Workspace of a split stage with nfi grid fields in and nfo products out.
static SplitWs split_stage_ws(const mt_plan* p, int n_r, int nfi, int nfo) {
  SplitWs w;
  w.rows_syn = (int64_t)n_r * 2 * nfi;
  w.g_level = (2 * nfo + 3) & ~3;  // floats per level, 16-byte multiple
  w.rows_nl = (int64_t)(n_r - 2) * w.g_level;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  w.err = 0;
  w.fs = 256;
  w.gs = w.fs + al((size_t)p->n_m * 2 * p->nhs * w.rows_syn * sizeof(float));
  w.mx = w.gs + al((size_t)p->n_m * 2 * p->nhs * w.rows_nl * sizeof(float));
  w.aimg = w.mx + al(2 * (size_t)n_r * sizeof(unsigned long long));
  // A-operand images: the synthesis ones are dead before the analysis writes its own
  const size_t syn = synth_split_image_bytes((int)w.rows_syn, split_syn_total_chunks(p));
  const size_t ana = anal_split_image_bytes(p->n_m, p->nhs, n_r - 2, 128 / (2 * nfo));
  w.total = w.aimg + al(std::max(syn, ana));
  return w;
}

static SplitWs split_ws(const mt_plan* p, int n_r, int mag, int chem) {
  return split_stage_ws(p, n_r, bouss_nfi(mag, chem), bouss_nfo(mag, chem));
}

// anelastic stage: grid fields in, products out (nl_anel_split.cu)
static int anel_nfi(int mag, int chem) { return 12 + (chem ? 1 : 0) + (mag ? 6 : 0); }
static int anel_nfo(int mag, int chem) { return 7 + (mag ? 3 : 0) + (chem ? 3 : 0); }

static RowOp rop(int tP, int cP, int kP, int tD, int cD, int kD, int scale) {
  RowOp o;
  o.tP = (int8_t)tP;
  o.cP = (int8_t)cP;
  o.kP = (int8_t)kP;
  o.tD = (int8_t)tD;
  o.cD = (int8_t)cD;
  o.kD = (int8_t)kD;
  o.scale = (int8_t)scale;
  o.pad = 0;
  return o;
}

// coef codes: 1 +1, 2 -1, 3 +m, 4 -m
static void syn_group_ops(RowOp* ops, int Q, int S, int T) {
  ops[0] = rop(Q, 0, 1);            // r.re = (P.Q).re
  ops[1] = rop(Q, 1, 1);            // r.im
  ops[2] = rop(T, 1, 4, S, 0, 1);   // theta.re = -m (P.T).im + (dP.S).re
  ops[3] = rop(T, 0, 3, S, 1, 1);   // theta.im = +m (P.T).re + (dP.S).im
  ops[4] = rop(S, 1, 4, T, 0, 2);   // phi.re = -m (P.S).im - (dP.T).re
  ops[5] = rop(S, 0, 3, T, 1, 2);   // phi.im = +m (P.S).re - (dP.T).im
}

static int ana_scalar_ops(RowOp* ops, int x) {
  ops[0] = rop(x, 0, 1);
  ops[1] = rop(x, 1, 1);
  return 2;
}
// S = dP.a - i m P.b ; T = -dP.b - i m P.a  (a = theta field, b = phi field), / l(l+1)
static int ana_s_ops(RowOp* ops, int a, int b) {
  ops[0] = rop(b, 1, 3, a, 0, 1, 1);
  ops[1] = rop(b, 0, 4, a, 1, 1, 1);
  return 2;
}
static int ana_t_ops(RowOp* ops, int a, int b) {
  ops[0] = rop(a, 1, 3, b, 0, 2, 1);
  ops[1] = rop(a, 0, 4, b, 1, 2, 1);
  return 2;
}

// Source arrays, terms (recipes over them, step_time.py:980-1013) and the row
// programs of the fused stage's synthesis, shared by the split and digit-split
// argument blocks (fields arr, narr, term, ops).
template <typename A>
static void fill_bouss_synth(A& s, const mt_bouss_in* in, bool mag, bool chem) {
  auto c = [](const double* x) { return (const double2*)x; };
  int na = 0;
  auto arr = [&](const double* ptr) {
    s.arr[na] = c(ptr);
    return na++;
  };
  int x = 0;
  auto term = [&](int ia, int ib, int recipe) {
    s.term[x].ia = (int8_t)ia;
    s.term[x].ib = (int8_t)ib;
    s.term[x].recipe = (int8_t)recipe;
    s.term[x].pad = 0;
    ++x;
  };
  if (mag) {
    const int ib = arr(in->b), idb = arr(in->db), iaj = arr(in->aj), idj = arr(in->dj),
              iddb = arr(in->ddb);
    term(ib, 0, kDlh);
    term(idb, 0, kRaw);
    term(iaj, 0, kRaw);
    term(iaj, 0, kDlh);
    term(idj, 0, kRaw);
    term(ib, iddb, kCurlT);
  }
  const int iw = arr(in->w), idw = arr(in->dw), iz = arr(in->z), idz = arr(in->dz),
            iddw = arr(in->ddw), is = arr(in->s);
  const int ixi = chem ? arr(in->xi) : 0;
  term(iw, 0, kDlh);
  term(idw, 0, kRaw);
  term(iz, 0, kRaw);
  term(iz, 0, kDlh);
  term(idz, 0, kRaw);
  term(iw, iddw, kCurlT);
  const int xs = x;
  term(is, 0, kRaw);
  if (chem) term(ixi, 0, kRaw);
  s.narr = na;
  const int G = mag ? 4 : 2;
  for (int g = 0; g < G; ++g) syn_group_ops(&s.ops[6 * g], 3 * g, 3 * g + 1, 3 * g + 2);
  ana_scalar_ops(&s.ops[6 * G], xs);
  if (chem) ana_scalar_ops(&s.ops[6 * G + 2], xs + 1);
}

// Spectral outputs of the fused stage and their row programs
// (magic_torch/step_time.py:1066-1124); returns the number of outputs.
template <typename A>
static int fill_bouss_anal(A& a, const mt_bouss_out* out, bool mag, bool chem) {
  int o = 0, r = 0;
  r += ana_scalar_ops(&a.ops[r], 0);
  a.out[o++] = (double2*)out->Advr;
  r += ana_s_ops(&a.ops[r], 1, 2);
  a.out[o++] = (double2*)out->Advt;
  r += ana_t_ops(&a.ops[r], 1, 2);
  a.out[o++] = (double2*)out->Advp;
  r += ana_scalar_ops(&a.ops[r], 3);
  a.out[o++] = (double2*)out->VSr;
  r += ana_s_ops(&a.ops[r], 4, 5);
  a.out[o++] = (double2*)out->VSt;
  if (mag) {
    r += ana_scalar_ops(&a.ops[r], 6);
    a.out[o++] = (double2*)out->VxBr;
    r += ana_s_ops(&a.ops[r], 7, 8);
    a.out[o++] = (double2*)out->VxBt;
    r += ana_t_ops(&a.ops[r], 7, 8);
    a.out[o++] = (double2*)out->VxBp;
  }
  if (chem) {
    const int x0 = mag ? 9 : 6;
    r += ana_scalar_ops(&a.ops[r], x0);
    a.out[o++] = (double2*)out->VXir;
    r += ana_s_ops(&a.ops[r], x0 + 1, x0 + 2);
    a.out[o++] = (double2*)out->VXit;
  }
  return o;
}

template <bool MAG, bool CHEM>
static int nl_bouss_split_t(const mt_plan* p, int n_r, const mt_bouss_in* in,
                            const mt_bouss_out* out, const mt_bouss_params* q, double* dtrkc,
                            double* dthkc, void* work, cudaStream_t st) {
  const int nfi = bouss_nfi(MAG, CHEM), nfo = bouss_nfo(MAG, CHEM);
  const SplitWs W = split_ws(p, n_r, MAG, CHEM);
  constexpr int kSplitRowsHost = 128;
  char* w = (char*)work;
  int* err = (int*)(w + W.err);
  float* Fs = (float*)(w + W.fs);
  float* Gs = (float*)(w + W.gs);
  unsigned long long* mx = (unsigned long long*)(w + W.mx);
  const int parts = q->parts ? q->parts : 7;
  const int64_t fs_j = W.rows_syn, fs_c = (int64_t)p->nhs * fs_j, fs_m = 2 * fs_c;
  const int64_t g_j = W.rows_nl, g_h = (int64_t)p->nhs * g_j, g_m = 2 * g_h;

  if (parts & 1) {
    MT_CHECK_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
    SplitSynArgs s{};
    s.t = p->tab;
    s.s = split_tables(p);
    fill_bouss_synth(s, in, MAG, CHEM);
    s.n_lev = n_r;
    s.ld = in->ld;
    s.or2 = q->or2;
    s.nrows = (int)W.rows_syn;
    s.row_per_level = 2 * nfi;
    s.stg_lev = std::min(n_r, 127 / s.row_per_level + 2);
    s.Fs = Fs;
    s.fs_m = fs_m;
    s.fs_c = fs_c;
    s.fs_j = fs_j;
    s.aimg = (uint8_t*)(w + W.aimg);
    s.total_chunks = split_syn_total_chunks(p);
    s.err = err;
    MT_TRY(launch_synth_split(s, st));
  }
  if (parts & 2) {
    MT_CHECK_CUDA(cudaMemsetAsync(mx, 0, 2 * n_r * sizeof(unsigned long long), st));
    NlSplitArgs nl{};
    nl.t = p->tab;
    nl.n_r = n_r;
    nl.Fs = Fs;
    nl.fs_m = fs_m;
    nl.fs_c = fs_c;
    nl.fs_j = fs_j;
    nl.G = Gs;
    nl.g_m = g_m;
    nl.g_h = g_h;
    nl.g_j = g_j;
    nl.g_level = W.g_level;
    nl.or2 = q->or2;
    nl.or4 = q->or4;
    nl.orho1 = q->orho1;
    nl.orho2 = q->orho2;
    nl.delxr2 = q->delxr2;
    nl.delxh2 = q->delxh2;
    nl.LFfac = q->LFfac;
    nl.LFfac_r = q->LFfac_r;
    nl.cour_mode = MAG ? q->cour_mode : 0;
    nl.cf2 = q->courfac * q->courfac;
    nl.af2 = q->alffac * q->alffac;
    double h = 0.5 * (1.0 + q->opm);
    nl.valfac = h * h;
    nl.vr2max = mx;
    nl.vh2max = mx + n_r;
    MT_TRY(launch_nl_bouss_split(MAG, CHEM, nl, st));
  }
  if (!(parts & 4)) return MT_OK;
  SplitAnaArgs a{};
  a.t = p->tab;
  a.s = split_tables(p);
  {
    const std::vector<int>& wk = split_wk_host(p);
    a.wk_max = *std::max_element(wk.begin(), wk.end());
  }
  a.G = Gs;
  a.g_m = g_m;
  a.g_h = g_h;
  a.g_j = g_j;
  a.g_level = W.g_level;
  a.n_lev = n_r - 2;
  a.n_out = fill_bouss_anal(a, out, MAG, CHEM);
  a.cols = 2 * nfo;
  a.lev_tile = kSplitRowsHost / a.cols;
  a.ld = out->ld;
  a.out_col0 = 1;
  a.aimg = (uint8_t*)(w + W.aimg);
  a.err = err;
  MT_TRY(launch_anal_split(a, st));
  return launch_courant_finish(n_r, mx, mx + n_r, q->delxr2, q->delxh2, dtrkc, dthkc, st);
}

// ---- digit-split (ozaki) fused stage ---------------------------------------

struct OzWs {
  size_t err, fs, gs, mx, rexs, rexa, aimg, total;
  int64_t rows_syn, rows_pad_s, g_level, rows_pad_a;
  int cols, lev_tile;
};

// Workspace of a digit-split stage with nfi grid fields and nfo products.
static OzWs oz_stage_ws(const mt_plan* p, int n_r, int nfi, int nfo) {
  OzWs w;
  w.rows_syn = (int64_t)n_r * 2 * nfi;
  w.rows_pad_s = (w.rows_syn + 127) / 128 * 128;
  w.g_level = 2 * nfo;  // doubles per level (even: 16-byte pieces)
  w.cols = 2 * nfo;
  w.lev_tile = 128 / w.cols;
  w.rows_pad_a = (int64_t)((n_r - 2 + w.lev_tile - 1) / w.lev_tile) * 128;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t nm2 = (size_t)p->n_m * 2;
  w.err = 0;
  w.fs = 256;
  w.gs = w.fs + al(nm2 * p->nhs * w.rows_syn * sizeof(double));
  w.mx = w.gs + al(nm2 * p->nhs * (size_t)(n_r - 2) * w.g_level * sizeof(double));
  w.rexs = w.mx + al(2 * (size_t)n_r * sizeof(unsigned long long));
  w.rexa = w.rexs + al(nm2 * w.rows_pad_s * sizeof(int));
  w.aimg = w.rexa + al(nm2 * w.rows_pad_a * sizeof(int));
  const size_t syn = oz_syn_image_bytes((int)w.rows_syn, ozaki_syn_total_chunks(p));
  const size_t ana = oz_ana_image_bytes(p->n_m, p->nhs, n_r - 2, w.lev_tile);
  w.total = w.aimg + al(std::max(syn, ana));
  return w;
}

static OzWs oz_ws(const mt_plan* p, int n_r, int mag, int chem) {
  return oz_stage_ws(p, n_r, bouss_nfi(mag, chem), bouss_nfo(mag, chem));
}

template <bool MAG, bool CHEM>
static int nl_bouss_ozaki_t(const mt_plan* p, int n_r, const mt_bouss_in* in,
                            const mt_bouss_out* out, const mt_bouss_params* q, double* dtrkc,
                            double* dthkc, void* work, cudaStream_t st) {
  const int nfi = bouss_nfi(MAG, CHEM);
  const OzWs W = oz_ws(p, n_r, MAG, CHEM);
  char* w = (char*)work;
  int* err = (int*)(w + W.err);
  double* Fs = (double*)(w + W.fs);
  double* Gs = (double*)(w + W.gs);
  unsigned long long* mx = (unsigned long long*)(w + W.mx);
  const int parts = q->parts ? q->parts : 7;
  const int64_t fs_j = W.rows_syn, fs_c = (int64_t)p->nhs * fs_j, fs_m = 2 * fs_c;
  const int64_t g_j = (int64_t)(n_r - 2) * W.g_level, g_h = (int64_t)p->nhs * g_j, g_m = 2 * g_h;
  if (parts & 1) {
    MT_CHECK_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
    OzSynArgs s{};
    s.t = p->tab;
    s.z = ozaki_tables(p);
    fill_bouss_synth(s, in, MAG, CHEM);
    s.n_lev = n_r;
    s.ld = in->ld;
    s.or2 = q->or2;
    s.nrows = (int)W.rows_syn;
    s.row_per_level = 2 * nfi;
    s.stg_lev = std::min(n_r, 127 / s.row_per_level + 2);
    s.aimg = (uint8_t*)(w + W.aimg);
    s.total_chunks = ozaki_syn_total_chunks(p);
    s.rexp = (int*)(w + W.rexs);
    s.rows_pad = W.rows_pad_s;
    s.Fs = Fs;
    s.fs_m = fs_m;
    s.fs_c = fs_c;
    s.fs_j = fs_j;
    s.err = err;
    MT_TRY(launch_oz_synth(s, st));
  }
  if (parts & 2) {
    MT_CHECK_CUDA(cudaMemsetAsync(mx, 0, 2 * n_r * sizeof(unsigned long long), st));
    NlBoussArgs nl{};
    nl.t = p->tab;
    nl.n_r = n_r;
    nl.split_io = 1;
    nl.Fs = Fs;
    nl.fs_m = fs_m;
    nl.fs_c = fs_c;
    nl.fs_j = fs_j;
    nl.Gs = Gs;
    nl.g_m2 = g_m;
    nl.g_h = g_h;
    nl.g_j = g_j;
    nl.g_level = W.g_level;
    nl.or2 = q->or2;
    nl.or4 = q->or4;
    nl.orho1 = q->orho1;
    nl.orho2 = q->orho2;
    nl.delxr2 = q->delxr2;
    nl.delxh2 = q->delxh2;
    nl.LFfac = q->LFfac;
    nl.LFfac_r = q->LFfac_r;
    nl.cour_mode = MAG ? q->cour_mode : 0;
    nl.cf2 = q->courfac * q->courfac;
    nl.af2 = q->alffac * q->alffac;
    double h = 0.5 * (1.0 + q->opm);
    nl.valfac = h * h;
    nl.vr2max = mx;
    nl.vh2max = mx + n_r;
    MT_TRY(launch_nl_bouss(MAG, CHEM, nl, st));
  }
  if (!(parts & 4)) return MT_OK;
  OzAnaArgs a{};
  a.t = p->tab;
  a.z = ozaki_tables(p);
  a.G = Gs;
  a.g_m = g_m;
  a.g_h = g_h;
  a.g_j = g_j;
  a.g_level = W.g_level;
  a.n_lev = n_r - 2;
  a.n_out = fill_bouss_anal(a, out, MAG, CHEM);
  a.cols = W.cols;
  a.lev_tile = W.lev_tile;
  a.ld = out->ld;
  a.out_col0 = 1;
  a.aimg = (uint8_t*)(w + W.aimg);
  a.rexp = (int*)(w + W.rexa);
  a.rows_pad = W.rows_pad_a;
  a.err = err;
  MT_TRY(launch_oz_anal(a, st));
  return launch_courant_finish(n_r, mx, mx + n_r, q->delxr2, q->delxh2, dtrkc, dthkc, st);
}

}  // namespace mt

namespace mt {

// Source arrays, terms and row programs of the anelastic stage's synthesis
// (the input assembly of radial_loop_anel, magic_torch/step_time.py:1233-1316),
// shared by the split and digit-split argument blocks; returns the rows per
// level (2 per grid field, in the field order of nl_point.cuh).
template <typename A>
static int fill_anel_synth(A& s, const mt_anel_in* in, bool mag, bool chem) {
  int na = 0;
  auto arr = [&](const double* ptr) {
    s.arr[na] = (const double2*)ptr;
    return na++;
  };
  int x = 0;
  auto term = [&](int ia, int ib, int recipe) {
    s.term[x].ia = (int8_t)ia;
    s.term[x].ib = (int8_t)ib;
    s.term[x].recipe = (int8_t)recipe;
    s.term[x].pad = 0;
    return x++;
  };
  const int iw = arr(in->w), idw = arr(in->dw), iddw = arr(in->ddw), iz = arr(in->z),
            idz = arr(in->dz), is = arr(in->s);
  const int tQv = term(iw, 0, kDlh), tdw = term(idw, 0, kRaw), tz = term(iz, 0, kRaw);
  const int tQd = term(idw, 0, kDlh), tddw = term(iddw, 0, kRaw), tdz = term(idz, 0, kRaw);
  const int tcv = term(iz, 0, kDlh), ts = term(is, 0, kRaw);
  RowOp* o = s.ops;
  syn_group_ops(o, tQv, tdw, tz);       // vr vt vp
  syn_group_ops(o + 6, tQd, tddw, tdz);  // dvrdr dvtdr dvpdr
  // dvrdt, dvrdp = grad of l(l+1) w: (dP X, i m P X)
  o[12] = rop(0, 0, 0, tQv, 0, 1);
  o[13] = rop(0, 0, 0, tQv, 1, 1);
  o[14] = rop(tQv, 1, 4);
  o[15] = rop(tQv, 0, 3);
  // dvtdp, dvpdp before 1/sin^2: theta = i m dP dw - m^2 P z, phi = -m^2 P dw - i m dP z
  o[16] = rop(tz, 0, 5, tdw, 1, 4);
  o[17] = rop(tz, 1, 5, tdw, 0, 3);
  o[18] = rop(tdw, 0, 5, tz, 1, 3);
  o[19] = rop(tdw, 1, 5, tz, 0, 4);
  ana_scalar_ops(o + 20, tcv);  // cvr = l(l+1) z
  ana_scalar_ops(o + 22, ts);   // s
  int rows = 24;
  if (chem) {
    const int ixi = arr(in->xi);
    ana_scalar_ops(o + rows, term(ixi, 0, kRaw));
    rows += 2;
  }
  if (mag) {
    const int ib = arr(in->b), idb = arr(in->db), iaj = arr(in->aj), idj = arr(in->dj),
              iddb = arr(in->ddb);
    const int tQb = term(ib, 0, kDlh), tdb = term(idb, 0, kRaw), taj = term(iaj, 0, kRaw);
    const int tQa = term(iaj, 0, kDlh), tdj = term(idj, 0, kRaw), tcT = term(ib, iddb, kCurlT);
    syn_group_ops(o + rows, tQb, tdb, taj);
    syn_group_ops(o + rows + 6, tQa, tdj, tcT);
    rows += 12;
  }
  s.narr = na;
  return rows;
}

// Row programs and outputs of the anelastic stage's analysis (the forward
// transforms of radial_loop_anel, magic_torch/step_time.py:1319-1370) over the
// products of nl_point.cuh; returns the number of outputs.
template <typename A>
static int fill_anel_anal(A& a, const mt_anel_out* out, bool mag, bool chem) {
  int o = 0, r = 0;
  r += ana_scalar_ops(&a.ops[r], 0);
  a.out[o++] = (double2*)out->Advr;
  r += ana_s_ops(&a.ops[r], 1, 2);
  a.out[o++] = (double2*)out->Advt;
  r += ana_t_ops(&a.ops[r], 1, 2);
  a.out[o++] = (double2*)out->Advp;
  r += ana_scalar_ops(&a.ops[r], 3);
  a.out[o++] = (double2*)out->VSr;
  r += ana_s_ops(&a.ops[r], 4, 5);
  a.out[o++] = (double2*)out->VSt;
  if (mag) {
    r += ana_scalar_ops(&a.ops[r], 6);
    a.out[o++] = (double2*)out->VxBr;
    r += ana_s_ops(&a.ops[r], 7, 8);
    a.out[o++] = (double2*)out->VxBt;
    r += ana_t_ops(&a.ops[r], 7, 8);
    a.out[o++] = (double2*)out->VxBp;
  }
  if (chem) {
    const int x0 = mag ? 9 : 6;
    r += ana_scalar_ops(&a.ops[r], x0);
    a.out[o++] = (double2*)out->VXir;
    r += ana_s_ops(&a.ops[r], x0 + 1, x0 + 2);
    a.out[o++] = (double2*)out->VXit;
  }
  r += ana_scalar_ops(&a.ops[r], anel_nfo(mag, chem) - 1);
  a.out[o++] = (double2*)out->heat;
  return o;
}

// Fused anelastic stage in split precision: synthesis (input assembly of
// radial_loop_anel, magic_torch/step_time.py:1233-1316), phi stage
// (nl_anel_split.cu), analysis of the bulk levels (:1329-1391), Courant steps.
template <bool MAG, bool CHEM>
static int nl_anel_split_t(const mt_plan* p, int n_r, const mt_anel_in* in,
                           const mt_anel_out* out, const mt_anel_stage_params* q, double* dtrkc,
                           double* dthkc, void* work, cudaStream_t st) {
  const int nfi = anel_nfi(MAG, CHEM), nfo = anel_nfo(MAG, CHEM);
  const SplitWs W = split_stage_ws(p, n_r, nfi, nfo);
  char* w = (char*)work;
  int* err = (int*)(w + W.err);
  float* Fs = (float*)(w + W.fs);
  float* Gs = (float*)(w + W.gs);
  unsigned long long* mx = (unsigned long long*)(w + W.mx);
  const int64_t fs_j = W.rows_syn, fs_c = (int64_t)p->nhs * fs_j, fs_m = 2 * fs_c;
  const int64_t g_j = W.rows_nl, g_h = (int64_t)p->nhs * g_j, g_m = 2 * g_h;
  MT_CHECK_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
  {
    SplitSynArgs s{};
    s.t = p->tab;
    s.s = split_tables(p);
    const int rows = fill_anel_synth(s, in, MAG, CHEM);
    s.n_lev = n_r;
    s.ld = in->ld;
    s.or2 = q->or2;
    s.row_per_level = rows;
    s.nrows = n_r * rows;
    s.stg_lev = std::min(n_r, 127 / rows + 2);
    s.Fs = Fs;
    s.fs_m = fs_m;
    s.fs_c = fs_c;
    s.fs_j = fs_j;
    s.aimg = (uint8_t*)(w + W.aimg);
    s.total_chunks = split_syn_total_chunks(p);
    s.err = err;
    MT_TRY(launch_synth_split(s, st));
  }
  {
    MT_CHECK_CUDA(cudaMemsetAsync(mx, 0, 2 * n_r * sizeof(unsigned long long), st));
    NlAnelArgs nl{};
    nl.t = p->tab;
    nl.n_r = n_r;
    nl.Fs = Fs;
    nl.fs_m = fs_m;
    nl.fs_c = fs_c;
    nl.fs_j = fs_j;
    nl.G = Gs;
    nl.g_m = g_m;
    nl.g_h = g_h;
    nl.g_j = g_j;
    nl.g_level = W.g_level;
    nl.r = q->r;
    nl.or1 = q->or1;
    nl.or2 = q->or2;
    nl.or4 = q->or4;
    nl.beta = q->beta;
    nl.orho1 = q->orho1;
    nl.orho2 = q->orho2;
    nl.otemp1 = q->otemp1;
    nl.visc = q->visc;
    nl.lambda_ = q->lambda_;
    nl.delxr2 = q->delxr2;
    nl.delxh2 = q->delxh2;
    nl.LFfac = q->LFfac;
    nl.ViscHeatFac = q->ViscHeatFac;
    nl.OhmLossFac = MAG ? q->OhmLossFac : 0.0;
    nl.cour_mode = MAG ? q->cour_mode : 0;
    nl.cf2 = q->courfac * q->courfac;
    nl.af2 = q->alffac * q->alffac;
    const double h = 0.5 * (1.0 + q->opm);
    nl.valfac = h * h;
    nl.vr2max = mx;
    nl.vh2max = mx + n_r;
    MT_TRY(launch_nl_anel_split(MAG, CHEM, nl, st));
  }
  SplitAnaArgs a{};
  a.t = p->tab;
  a.s = split_tables(p);
  {
    const std::vector<int>& wk = split_wk_host(p);
    a.wk_max = *std::max_element(wk.begin(), wk.end());
  }
  a.G = Gs;
  a.g_m = g_m;
  a.g_h = g_h;
  a.g_j = g_j;
  a.g_level = W.g_level;
  a.n_lev = n_r - 2;
  a.n_out = fill_anel_anal(a, out, MAG, CHEM);
  a.cols = 2 * nfo;
  a.lev_tile = 128 / a.cols;
  a.ld = out->ld;
  a.out_col0 = 1;
  a.aimg = (uint8_t*)(w + W.aimg);
  a.err = err;
  MT_TRY(launch_anal_split(a, st));
  return launch_courant_finish(n_r, mx, mx + n_r, q->delxr2, q->delxh2, dtrkc, dthkc, st);
}

// The digit-split anelastic stage runs where one CTA of its FP64 phi stage
// holds a (theta row, level)'s buffers in shared memory.
static bool anel_ozaki_fits(const mt_plan* p, int mag, int chem) {
  return nl_anel_f64_smem(p->n_phi, mag, chem) > 0;
}

// Fused anelastic stage in digit-split precision: the synthesis row programs
// of the split stage on the int8 digit-plane GEMMs (ozaki.cu), the FP64 phi
// stage k_nl_anel_f64, and the analysis row programs on the digit-plane GEMMs,
// with FP64 rows between them.
template <bool MAG, bool CHEM>
static int nl_anel_ozaki_t(const mt_plan* p, int n_r, const mt_anel_in* in,
                           const mt_anel_out* out, const mt_anel_stage_params* q, double* dtrkc,
                           double* dthkc, void* work, cudaStream_t st) {
  const OzWs W = oz_stage_ws(p, n_r, anel_nfi(MAG, CHEM), anel_nfo(MAG, CHEM));
  char* w = (char*)work;
  int* err = (int*)(w + W.err);
  double* Fs = (double*)(w + W.fs);
  double* Gs = (double*)(w + W.gs);
  unsigned long long* mx = (unsigned long long*)(w + W.mx);
  const int64_t fs_j = W.rows_syn, fs_c = (int64_t)p->nhs * fs_j, fs_m = 2 * fs_c;
  const int64_t g_j = (int64_t)(n_r - 2) * W.g_level, g_h = (int64_t)p->nhs * g_j, g_m = 2 * g_h;
  MT_CHECK_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
  {
    OzSynArgs s{};
    s.t = p->tab;
    s.z = ozaki_tables(p);
    const int rows = fill_anel_synth(s, in, MAG, CHEM);
    s.n_lev = n_r;
    s.ld = in->ld;
    s.or2 = q->or2;
    s.nrows = (int)W.rows_syn;
    s.row_per_level = rows;
    s.stg_lev = std::min(n_r, 127 / rows + 2);
    s.aimg = (uint8_t*)(w + W.aimg);
    s.total_chunks = ozaki_syn_total_chunks(p);
    s.rexp = (int*)(w + W.rexs);
    s.rows_pad = W.rows_pad_s;
    s.Fs = Fs;
    s.fs_m = fs_m;
    s.fs_c = fs_c;
    s.fs_j = fs_j;
    s.err = err;
    MT_TRY(launch_oz_synth(s, st));
  }
  {
    MT_CHECK_CUDA(cudaMemsetAsync(mx, 0, 2 * n_r * sizeof(unsigned long long), st));
    NlAnelArgs nl{};
    nl.t = p->tab;
    nl.n_r = n_r;
    nl.Fs64 = Fs;
    nl.fs_m = fs_m;
    nl.fs_c = fs_c;
    nl.fs_j = fs_j;
    nl.G64 = Gs;
    nl.g_m = g_m;
    nl.g_h = g_h;
    nl.g_j = g_j;
    nl.g_level = W.g_level;
    nl.r = q->r;
    nl.or1 = q->or1;
    nl.or2 = q->or2;
    nl.or4 = q->or4;
    nl.beta = q->beta;
    nl.orho1 = q->orho1;
    nl.orho2 = q->orho2;
    nl.otemp1 = q->otemp1;
    nl.visc = q->visc;
    nl.lambda_ = q->lambda_;
    nl.delxr2 = q->delxr2;
    nl.delxh2 = q->delxh2;
    nl.LFfac = q->LFfac;
    nl.ViscHeatFac = q->ViscHeatFac;
    nl.OhmLossFac = MAG ? q->OhmLossFac : 0.0;
    nl.cour_mode = MAG ? q->cour_mode : 0;
    nl.cf2 = q->courfac * q->courfac;
    nl.af2 = q->alffac * q->alffac;
    const double h = 0.5 * (1.0 + q->opm);
    nl.valfac = h * h;
    nl.vr2max = mx;
    nl.vh2max = mx + n_r;
    MT_TRY(launch_nl_anel_f64(MAG, CHEM, nl, st));
  }
  OzAnaArgs a{};
  a.t = p->tab;
  a.z = ozaki_tables(p);
  a.G = Gs;
  a.g_m = g_m;
  a.g_h = g_h;
  a.g_j = g_j;
  a.g_level = W.g_level;
  a.n_lev = n_r - 2;
  a.n_out = fill_anel_anal(a, out, MAG, CHEM);
  a.cols = W.cols;
  a.lev_tile = W.lev_tile;
  a.ld = out->ld;
  a.out_col0 = 1;
  a.aimg = (uint8_t*)(w + W.aimg);
  a.rexp = (int*)(w + W.rexa);
  a.rows_pad = W.rows_pad_a;
  a.err = err;
  MT_TRY(launch_oz_anal(a, st));
  return launch_courant_finish(n_r, mx, mx + n_r, q->delxr2, q->delxh2, dtrkc, dthkc, st);
}

}  // namespace mt

extern "C" {

size_t mt_nl_bouss_workspace(const mt_plan* p, int n_r, int l_mag, int l_chem) {
  if (!p || n_r < 3) return 0;
  if (p->precision == MT_PREC_SPLIT) return split_ws(p, n_r, l_mag, l_chem).total;
  if (p->precision == MT_PREC_OZAKI) return oz_ws(p, n_r, l_mag, l_chem).total;
  size_t f = fourier_bytes(p, (int64_t)n_r * bouss_nfi(l_mag, l_chem));
  size_t g = fourier_bytes(p, (int64_t)(n_r - 2) * bouss_nfo(l_mag, l_chem));
  return f + g + 2 * (size_t)n_r * sizeof(unsigned long long) + 256;
}

int mt_nl_bouss(const mt_plan* p, int n_r, const mt_bouss_in* in, const mt_bouss_out* out,
                const mt_bouss_params* q, double* dtrkc, double* dthkc, void* work,
                size_t work_bytes, void* stream) {
  MT_TRY(check_plan(p));
  MT_REQUIRE(in && out && q && dtrkc && dthkc && n_r >= 3, MT_ERR_ARG, "bad argument");
  MT_REQUIRE(in->w && in->dw && in->ddw && in->z && in->dz && in->s, MT_ERR_ARG,
             "null velocity/entropy input");
  MT_REQUIRE(!q->l_mag || (in->b && in->db && in->ddb && in->aj && in->dj), MT_ERR_ARG,
             "null magnetic input");
  MT_REQUIRE(!q->l_chem || in->xi, MT_ERR_ARG, "null composition input");
  MT_REQUIRE(in->ld >= n_r && out->ld >= n_r, MT_ERR_ARG, "ld >= n_r required");
  MT_REQUIRE(out->Advr && out->Advt && out->Advp && out->VSr && out->VSt, MT_ERR_ARG,
             "null output");
  MT_REQUIRE(q->or2 && q->or4 && q->orho1 && q->orho2 && q->delxr2 && q->delxh2, MT_ERR_ARG,
             "null radial profile");
  MT_REQUIRE(q->cour_mode >= 0 && q->cour_mode <= 2, MT_ERR_ARG, "bad cour_mode");
  MT_REQUIRE(q->parts >= 0 && q->parts <= 7, MT_ERR_ARG, "parts must be a mask of 1, 2, 4");
  MT_REQUIRE(work && work_bytes >= mt_nl_bouss_workspace(p, n_r, q->l_mag, q->l_chem),
             MT_ERR_WORKSPACE, "workspace too small");
  cudaStream_t st = (cudaStream_t)stream;
  if (p->precision == MT_PREC_SPLIT) {
    if (q->l_mag)
      return q->l_chem ? nl_bouss_split_t<true, true>(p, n_r, in, out, q, dtrkc, dthkc, work, st)
                       : nl_bouss_split_t<true, false>(p, n_r, in, out, q, dtrkc, dthkc, work, st);
    return q->l_chem ? nl_bouss_split_t<false, true>(p, n_r, in, out, q, dtrkc, dthkc, work, st)
                     : nl_bouss_split_t<false, false>(p, n_r, in, out, q, dtrkc, dthkc, work, st);
  }
  if (p->precision == MT_PREC_OZAKI) {
    if (q->l_mag)
      return q->l_chem ? nl_bouss_ozaki_t<true, true>(p, n_r, in, out, q, dtrkc, dthkc, work, st)
                       : nl_bouss_ozaki_t<true, false>(p, n_r, in, out, q, dtrkc, dthkc, work, st);
    return q->l_chem ? nl_bouss_ozaki_t<false, true>(p, n_r, in, out, q, dtrkc, dthkc, work, st)
                     : nl_bouss_ozaki_t<false, false>(p, n_r, in, out, q, dtrkc, dthkc, work, st);
  }
  if (q->l_mag)
    return q->l_chem ? nl_bouss_t<true, true>(p, n_r, in, out, q, dtrkc, dthkc, work, st)
                     : nl_bouss_t<true, false>(p, n_r, in, out, q, dtrkc, dthkc, work, st);
  return q->l_chem ? nl_bouss_t<false, true>(p, n_r, in, out, q, dtrkc, dthkc, work, st)
                   : nl_bouss_t<false, false>(p, n_r, in, out, q, dtrkc, dthkc, work, st);
}


size_t mt_nl_anel_workspace(const mt_plan* p, int n_r, int l_mag, int l_chem) {
  if (!p || n_r < 3) return 0;
  if (p->precision == MT_PREC_SPLIT)
    return split_stage_ws(p, n_r, anel_nfi(l_mag, l_chem), anel_nfo(l_mag, l_chem)).total;
  if (p->precision == MT_PREC_OZAKI && anel_ozaki_fits(p, l_mag, l_chem))
    return oz_stage_ws(p, n_r, anel_nfi(l_mag, l_chem), anel_nfo(l_mag, l_chem)).total;
  return 0;
}

int mt_nl_anel(const mt_plan* p, int n_r, const mt_anel_in* in, const mt_anel_out* out,
               const mt_anel_stage_params* q, double* dtrkc, double* dthkc, void* work,
               size_t work_bytes, void* stream) {
  MT_TRY(check_plan(p));
  MT_REQUIRE(p->precision == MT_PREC_SPLIT || p->precision == MT_PREC_OZAKI, MT_ERR_UNSUPPORTED,
             "mt_nl_anel needs a MT_PREC_SPLIT or MT_PREC_OZAKI plan (FP64 callers compose "
             "the drop-in transforms and mt_get_nl_anel as radial_loop_anel does)");
  MT_REQUIRE(p->precision != MT_PREC_OZAKI || !q || anel_ozaki_fits(p, q->l_mag, q->l_chem),
             MT_ERR_UNSUPPORTED,
             "n_phi too long for the digit-split anelastic stage's phi buffers (compose the "
             "drop-in transforms and mt_get_nl_anel instead)");
  MT_REQUIRE(in && out && q && dtrkc && dthkc && n_r >= 3, MT_ERR_ARG, "bad argument");
  MT_REQUIRE(in->w && in->dw && in->ddw && in->z && in->dz && in->s, MT_ERR_ARG,
             "null velocity/entropy input");
  MT_REQUIRE(!q->l_mag || (in->b && in->db && in->ddb && in->aj && in->dj), MT_ERR_ARG,
             "null magnetic input");
  MT_REQUIRE(!q->l_chem || in->xi, MT_ERR_ARG, "null composition input");
  MT_REQUIRE(in->ld >= n_r && out->ld >= n_r, MT_ERR_ARG, "ld >= n_r required");
  MT_REQUIRE(out->Advr && out->Advt && out->Advp && out->VSr && out->VSt && out->heat,
             MT_ERR_ARG, "null output");
  MT_REQUIRE(!q->l_mag || (out->VxBr && out->VxBt && out->VxBp), MT_ERR_ARG,
             "null magnetic output");
  MT_REQUIRE(!q->l_chem || (out->VXir && out->VXit), MT_ERR_ARG, "null composition output");
  MT_REQUIRE(q->r && q->or1 && q->or2 && q->or4 && q->beta && q->orho1 && q->orho2 && q->otemp1 &&
                 q->visc && q->lambda_ && q->delxr2 && q->delxh2,
             MT_ERR_ARG, "null radial profile");
  MT_REQUIRE(q->cour_mode >= 0 && q->cour_mode <= 2, MT_ERR_ARG, "bad cour_mode");
  MT_REQUIRE(work && work_bytes >= mt_nl_anel_workspace(p, n_r, q->l_mag, q->l_chem),
             MT_ERR_WORKSPACE, "workspace too small");
  cudaStream_t st = (cudaStream_t)stream;
  if (p->precision == MT_PREC_OZAKI) {
    if (q->l_mag)
      return q->l_chem ? nl_anel_ozaki_t<true, true>(p, n_r, in, out, q, dtrkc, dthkc, work, st)
                       : nl_anel_ozaki_t<true, false>(p, n_r, in, out, q, dtrkc, dthkc, work, st);
    return q->l_chem ? nl_anel_ozaki_t<false, true>(p, n_r, in, out, q, dtrkc, dthkc, work, st)
                     : nl_anel_ozaki_t<false, false>(p, n_r, in, out, q, dtrkc, dthkc, work, st);
  }
  if (q->l_mag)
    return q->l_chem ? nl_anel_split_t<true, true>(p, n_r, in, out, q, dtrkc, dthkc, work, st)
                     : nl_anel_split_t<true, false>(p, n_r, in, out, q, dtrkc, dthkc, work, st);
  return q->l_chem ? nl_anel_split_t<false, true>(p, n_r, in, out, q, dtrkc, dthkc, work, st)
                   : nl_anel_split_t<false, false>(p, n_r, in, out, q, dtrkc, dthkc, work, st);
}

int mt_selftest_wait_timeout(int* status, long long spins, void* stream) {
  MT_REQUIRE(status && spins > 0 && spins <= (1LL << 30), MT_ERR_ARG,
             "status pointer and 0 < spins <= 2^30 required");
  return launch_selftest_wait(status, (long)spins, (cudaStream_t)stream);
}

int mt_device_status(const void* work, int* code, void* stream) {
  MT_REQUIRE(work && code, MT_ERR_ARG, "work and code pointers required");
  cudaStream_t st = (cudaStream_t)stream;
  int v = 0;
  MT_CHECK_CUDA(cudaMemcpyAsync(&v, work, sizeof(int), cudaMemcpyDeviceToHost, st));
  MT_CHECK_CUDA(cudaStreamSynchronize(st));
  *code = v;
  return MT_OK;
}

int mt_noalloc_status(int* code, void* stream) {
  MT_REQUIRE(code, MT_ERR_ARG, "code pointer required");
  void* work = nullptr;
  MT_TRY(noalloc_scratch(&work));
  return mt_device_status(work, code, stream);
}

}  // extern "C"
