/*
 * magic_b200 — C ABI of the B200 (sm_100a) pseudo-spectral nonlinear stage.
 *
 * Replaces, for the spherical-shell dynamo code torch-magic, the Python
 * functions of its transform module (magic_torch/sht.py) and of its
 * nonlinear-term builders (magic_torch/get_nl.py, get_nl_anel.py,
 * courant.py).  Each entry point below names the reference function it
 * replaces (path:line inside the reference project).
 *
 * Conventions (identical to the reference):
 *   - spectral arrays: complex128 stored as interleaved (re, im) doubles,
 *     shape (lm_max, B) row-major with row stride `ld` complex elements
 *     (ld >= B), m-major lm order: lm = lStart[m/minc] + (l - m);
 *   - grid arrays: float64, shape (B, n_theta_max, n_phi_max) contiguous,
 *     theta rows interleaved [N0, S0, N1, S1, ...];
 *   - synthesis = irfft(norm="forward") (unscaled), analysis =
 *     rfft(norm="forward") (scaled by 1/n_phi); the FFT index is m/minc.
 *
 * All pointers except `mt_plan*` and the `*_desc`/`*_params` structs are
 * DEVICE pointers owned by the caller.  `work` is caller-owned device
 * scratch of at least the size the matching `mt_*_workspace` query returns.
 * No entry point synchronises the host; all work is enqueued on `stream`
 * (a cudaStream_t passed as void*).  Return value: 0 (MT_OK) or an
 * mt_status code; mt_last_error() gives a message (thread-local).
 *
 * Plans are read-only after creation: several host threads may use one plan
 * concurrently on different streams with different workspaces.
 */
#ifndef MAGIC_B200_H
#define MAGIC_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define MT_API __attribute__((visibility("default")))
#else
#define MT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mt_plan mt_plan;

enum mt_status {
  MT_OK = 0,
  MT_ERR_ARG = 1,         /* bad argument (null pointer, bad size, ...)     */
  MT_ERR_CUDA = 2,        /* a CUDA runtime call failed                     */
  MT_ERR_UNSUPPORTED = 3, /* grid or option this build does not handle      */
  MT_ERR_WORKSPACE = 4,   /* workspace smaller than the query returned      */
  MT_ERR_NO_DEVICE = 5    /* no sm_100 device visible                       */
};

enum mt_precision {
  MT_PREC_FP64 = 0,       /* plain FP64 Legendre contractions (DMMA)        */
  MT_PREC_SPLIT = 1,      /* split-BF16 tcgen05 contractions, FP32 accumulate */
  MT_PREC_OZAKI = 2       /* fused stage: int8 digit planes on tcgen05 with
                             exact int32 accumulation, FP64 phi stage (about
                             1e-12 of scale); transforms as MT_PREC_FP64     */
};

/* Grid description.  n_theta_max / n_phi_max = 0 derive the reference's
 * sizes from l_max (magic_torch/params.py:57-76). */
typedef struct {
  int l_max;
  int minc;
  int n_theta_max;
  int n_phi_max;          /* points per azimuthal sector (n_phi_tot / minc) */
  int precision;          /* enum mt_precision                               */
} mt_grid_desc;

typedef struct {
  int l_max, minc, n_theta_max, n_phi_max, n_m_max, lm_max, nhs, precision;
} mt_plan_info;

/* Build all horizontal tables on the current device: Gauss-Legendre nodes
 * and weights (replaces magic_torch/horizontal_data.py:16-50), P_l^m and
 * sin(theta) dP_l^m/dtheta in FP64 (replaces magic_torch/plms.py:21-186),
 * FFT twiddles.  Synchronous. */
MT_API int mt_plan_create(const mt_grid_desc* desc, mt_plan** plan);
MT_API int mt_plan_destroy(mt_plan* plan);
MT_API int mt_plan_get_info(const mt_plan* plan, mt_plan_info* info);

/* Copy the plan's FP64 tables to caller device buffers (any may be NULL):
 * theta_ord, gauss (n_theta_max, geographic order), Plm, dPlm (lm_max, nhs).
 * Used to check the tables against the oracle. */
MT_API int mt_plan_copy_tables(const mt_plan* plan, double* theta_ord, double* gauss,
                        double* plm, double* dplm, void* stream);

/* ---- transforms (magic_torch/sht.py) ------------------------------------ */

/* Workspace bytes for a transform over B columns (all four transforms and the
 * helpers below use the same query). */
MT_API size_t mt_transform_workspace(const mt_plan* plan, int B, int n_fields);

/* scal_to_spat (magic_torch/sht.py:298-348): Slm (lm_max, ld) -> grid. */
MT_API int mt_scal_to_spat(const mt_plan* plan, const double* Slm, int64_t ld, int B,
                    double* grid, void* work, size_t work_bytes, void* stream);

/* Allocation-free scal_to_spat, for callers that cannot allocate device
 * memory while they run: a host code linked through this C ABI that budgets
 * all GPU memory once at start-up, or a process whose device memory is held by
 * another allocator, cannot hand a fresh cudaMalloc'd workspace to every call.
 * No counterpart in the reference.  Same inputs, outputs and results as
 * mt_scal_to_spat, but the workspace is a fixed array of
 * MT_NOALLOC_SCRATCH_BYTES inside the library: every GPU that loads the
 * library holds it until the process exits.  B is limited to
 * mt_transform_workspace(plan, B, 1) <= MT_NOALLOC_SCRATCH_BYTES: for FP64
 * plans that is n_m_max * n_theta_max * B * 16 bytes (about 10 columns at
 * l_max = 255); split plans also keep their operand images there and allow
 * fewer columns.  Larger B returns MT_ERR_WORKSPACE before any launch.  The
 * first call on a device looks up the array's device address (no allocation);
 * make that first call before any stream capture.  The address is kept per
 * device ordinal for the life of the process, so a context reset on that
 * device (cudaDeviceReset) requires a process restart before the next call.
 * All calls on a device share the array: calls that can overlap on the GPU
 * (different streams, different host threads) race and must be serialised by
 * the caller.  With a split plan, a device-side wait that ran out is reported
 * only through mt_noalloc_status (the array is not the caller's to read). */
#define MT_NOALLOC_SCRATCH_BYTES ((size_t)16 << 20)
MT_API int mt_scal_to_spat_noalloc(const mt_plan* plan, const double* Slm, int64_t ld, int B,
                                   double* grid, void* stream);

/* scal_to_SH (magic_torch/sht.py:351-405): grid -> Slm (lm_max, ld). */
MT_API int mt_scal_to_SH(const mt_plan* plan, const double* grid, int B, double* Slm,
                  int64_t ld, void* work, size_t work_bytes, void* stream);

/* torpol_to_spat (magic_torch/sht.py:408-497): Q,S,T -> br, bt, bp. */
MT_API int mt_torpol_to_spat(const mt_plan* plan, const double* Q, const double* S,
                      const double* T, int64_t ld, int B, double* br, double* bt,
                      double* bp, void* work, size_t work_bytes, void* stream);

/* spat_to_sphertor (magic_torch/sht.py:575-667): (vt, vp) -> (S, T),
 * divided by l(l+1), l=0 set to zero. */
MT_API int mt_spat_to_sphertor(const mt_plan* plan, const double* vt, const double* vp,
                        int B, double* S, double* T, int64_t ld, void* work,
                        size_t work_bytes, void* stream);

/* scal_to_grad_spat (magic_torch/sht.py:500-567): Slm -> (dtheta, dphi)
 * sin-weighted gradient grids.  pol_to_grad_spat (sht.py:706-722) is this with
 * `scale_dlh` = 1 (input multiplied by l(l+1) on load). */
MT_API int mt_scal_to_grad_spat(const mt_plan* plan, const double* Slm, int64_t ld, int B,
                         int scale_dlh, double* gt, double* gp, void* work,
                         size_t work_bytes, void* stream);

/* ---- grid-space nonlinear terms ----------------------------------------- */

/* get_nl (magic_torch/get_nl.py:30-87) on grids of n_r levels:
 * in[14] = vr,vt,vp,cvr,cvt,cvp,s,br,bt,bp,cbr,cbt,cbp,xi (each n_r x n_theta
 * x n_phi); out[12] = Advr,Advt,Advp,VSr,VSt,VSp,VxBr,VxBt,VxBp,VXir,VXit,VXip;
 * or2, or4: (n_r); LFfac scalar. */
MT_API int mt_get_nl(const mt_plan* plan, int n_r, const double* const* in,
              double* const* out, const double* or2, const double* or4,
              double LFfac, void* stream);

typedef struct {
  const double *r, *or1, *or2, *or4, *beta, *orho1, *otemp1, *visc, *lambda_;
  double LFfac, ViscHeatFac, OhmLossFac;
  int l_mag;
} mt_anel_params;

/* get_nl_anel (magic_torch/get_nl_anel.py:41-136): in[19] = vr,vt,vp,dvrdr,
 * dvtdr,dvpdr,dvrdt,dvrdp,dvtdp,dvpdp,cvr,s,xi,br,bt,bp,cbr,cbt,cbp;
 * out[13] = the 12 of get_nl followed by heatTerms. */
MT_API int mt_get_nl_anel(const mt_plan* plan, int n_r, const double* const* in,
                   double* const* out, const mt_anel_params* p, void* stream);

typedef struct {
  const double *or2, *or4, *orho1, *orho2, *delxr2, *delxh2; /* (n_r) */
  double courfac, alffac, LFfac, opm;
  int mode;               /* 0 non-magnetic, 1 magnetic damped, 2 undamped */
} mt_courant_params;

/* courant_check (magic_torch/courant.py:80-127): per-level dtrkc, dthkc
 * (n_r) from grids vr,vt,vp[,br,bt,bp].  work: mt_courant_workspace bytes. */
MT_API size_t mt_courant_workspace(const mt_plan* plan, int n_r);
MT_API int mt_courant(const mt_plan* plan, int n_r, const double* vr, const double* vt,
               const double* vp, const double* br, const double* bt,
               const double* bp, const mt_courant_params* p, double* dtrkc,
               double* dthkc, void* work, size_t work_bytes, void* stream);

/* ---- fused nonlinear stage ---------------------------------------------- */

/* Spectral inputs of the Boussinesq radial loop (magic_torch/step_time.py:
 * 931-1213), each (lm_max, ld) complex over n_r levels (column = level).
 * b, db, ddb, aj, dj may be NULL when l_mag = 0; xi NULL when no composition. */
typedef struct {
  const double *w, *dw, *ddw, *z, *dz, *s, *b, *db, *ddb, *aj, *dj, *xi;
  int64_t ld;
} mt_bouss_in;

/* Spectral outputs over the bulk levels 1..n_r-2 (written at columns 1..n_r-2
 * of (lm_max, ld) arrays; columns 0 and n_r-1 are left untouched):
 * AdvrLM, AdvtLM, AdvpLM, dVSrLM, VStLM, VxBrLM, VxBtLM, VxBpLM, dVXirLM,
 * VXitLM (the last five may be NULL as their inputs). */
typedef struct {
  double *Advr, *Advt, *Advp, *VSr, *VSt, *VxBr, *VxBt, *VxBp, *VXir, *VXit;
  int64_t ld;
} mt_bouss_out;

typedef struct {
  const double *or2, *or4, *orho1, *orho2, *delxr2, *delxh2; /* (n_r) */
  double LFfac, courfac, alffac, opm;
  int l_mag, l_chem, cour_mode; /* cour_mode as mt_courant_params.mode      */
  int parts;  /* 0 = whole stage; else a mask run in order on the same work:
                 1 Legendre synthesis, 2 phi FFT + products + Courant maxima,
                 4 Legendre analysis + Courant steps (lets a caller time or
                 overlap the three launches individually)                     */
  const double* LFfac_r; /* (n_r) per-level Lorentz factor in place of LFfac, or
                            NULL; lets one call serve the levels of several runs
                            with different Ekman or magnetic Prandtl numbers    */
} mt_bouss_params;

MT_API size_t mt_nl_bouss_workspace(const mt_plan* plan, int n_r, int l_mag, int l_chem);

/* Whole nonlinear stage of one radial loop in four launches: Legendre
 * synthesis of the 14 grid fields (inputs assembled on load: Q = l(l+1) w,
 * T_curl = or2 l(l+1) w - ddw, ...), fused inverse phi-FFT + get_nl products
 * + Courant maxima + forward phi-FFT, Legendre analysis of the 12 products
 * (with the 1/l(l+1) division).  dtrkc, dthkc: (n_r) Courant steps. */
MT_API int mt_nl_bouss(const mt_plan* plan, int n_r, const mt_bouss_in* in,
                const mt_bouss_out* out, const mt_bouss_params* p, double* dtrkc,
                double* dthkc, void* work, size_t work_bytes, void* stream);

/* ---- fused anelastic nonlinear stage (split, digit-split precision) --------
 * The nonlinear part of radial_loop_anel (magic_torch/step_time.py:1215-1475):
 * Legendre synthesis of the 18 grid fields (19 with composition; velocity and
 * its derivatives zero on the two boundary levels as in the reference),
 * get_nl_anel products with viscous and Ohmic heating (get_nl_anel.py:41-136)
 * and Courant maxima in the phi stage, Legendre analysis of the bulk levels.
 * Requires a plan created with MT_PREC_SPLIT (tcgen05 bf16x3 GEMMs, FP32 phi
 * stage) or MT_PREC_OZAKI (int8 digit-plane GEMMs, FP64 phi stage, ~1e-12 of
 * scale); FP64 plans compose the drop-in transforms and mt_get_nl_anel
 * exactly as radial_loop_anel does.  The FP64 phi stage keeps the rows of
 * one (theta row, level) in shared memory; where they would not fit (no plan
 * within the n_phi limit of mt_plan_create) mt_nl_anel_workspace returns 0
 * and mt_nl_anel MT_ERR_UNSUPPORTED.
 * Inputs: spectral (lm_max, ld) complex over n_r levels; b .. dj NULL
 * without magnetic field, xi NULL without composition. */
typedef struct {
  const double *w, *dw, *ddw, *z, *dz, *s, *xi, *b, *db, *ddb, *aj, *dj;
  int64_t ld;
} mt_anel_in;

/* Outputs over the bulk levels (columns 1..n_r-2): AdvrLM, AdvtLM, AdvpLM,
 * dVSrLM, VStLM, VxBrLM, VxBtLM, VxBpLM, dVXirLM, VXitLM, heatTermsLM (the
 * magnetic and composition ones may be NULL when their inputs are). */
typedef struct {
  double *Advr, *Advt, *Advp, *VSr, *VSt, *VxBr, *VxBt, *VxBp, *VXir, *VXit, *heat;
  int64_t ld;
} mt_anel_out;

typedef struct {
  const double *r, *or1, *or2, *or4, *beta, *orho1, *orho2, *otemp1, *visc,
      *lambda_, *delxr2, *delxh2; /* (n_r) */
  double LFfac, ViscHeatFac, OhmLossFac, courfac, alffac, opm;
  int l_mag, l_chem, cour_mode; /* cour_mode as mt_courant_params.mode */
} mt_anel_stage_params;

MT_API size_t mt_nl_anel_workspace(const mt_plan* plan, int n_r, int l_mag, int l_chem);
MT_API int mt_nl_anel(const mt_plan* plan, int n_r, const mt_anel_in* in,
               const mt_anel_out* out, const mt_anel_stage_params* p, double* dtrkc,
               double* dthkc, void* work, size_t work_bytes, void* stream);

/* Self-test of the device-side failure detection (no reference counterpart):
 * one CTA waits on an mbarrier that nothing completes, gives up after
 * `spins` polls, writes 99 to the device int *status (which the caller zeroes
 * first) and returns, so the context stays usable.  The tensor-core kernels
 * use the same bounded wait (2^22 polls) and report their own codes in the
 * first int of their workspace. */
/* ---- radial operators ---------------------------------------------------
 * A real n_r x n_r matrix D applied along the radial axis of complex rows:
 * out[b][j] = sum_k D[j][k] in[b][k] for b < nrows, rows of n_r complex
 * values with strides ld_in / ld_out (complex units; the reference's
 * (lm_max, n_r_max) spectral arrays are nrows = lm_max rows, ld = n_r_max).
 * Replaces magic_torch/radial_derivatives.py:29-68 (get_dr, get_ddr, get_dddr:
 * dense Chebyshev or banded finite-difference matrices) and
 * magic_torch/cosine_transform.py:18-45 (costf, the self-inverse DCT-I).
 * mt_radial_op_create copies D (HOST pointer, row-major) to the current
 * device and keeps only each row's nonzero band, so a banded matrix costs its
 * band only.  Operators are read-only after creation. */
typedef struct mt_radial_op mt_radial_op;
MT_API int mt_radial_op_create(int n_r, const double* D_host, mt_radial_op** op);
MT_API int mt_radial_op_create_dct1(int n_r, mt_radial_op** op);
MT_API int mt_radial_op_destroy(mt_radial_op* op);
MT_API int mt_radial_op_bandwidth(const mt_radial_op* op);
MT_API int mt_radial_apply(const mt_radial_op* op, int nrows, const double* in, int64_t ld_in,
                           double* out, int64_t ld_out, void* stream);
/* two operators on one input in one pass (get_ddr: D1 and D2) */
MT_API int mt_radial_apply2(const mt_radial_op* op1, const mt_radial_op* op2, int nrows,
                            const double* in, int64_t ld_in, double* out1, double* out2,
                            int64_t ld_out, void* stream);

/* ---- explicit time-derivative terms ----------------------------------------
 * Step 4 of the radial loop (magic_torch/step_time.py:1139-1176): the
 * nonlinear and Coriolis terms of get_td (magic_torch/get_td.py:58-308:
 * get_dwdt or get_dwdt_double_curl, get_dzdt, get_dpdt, get_dsdt,
 * get_dxidt, get_dbdt) completed by the finish_exp radial derivatives
 * (update_wp.py:371-385, update_s.py:191-210, update_xi.py:183-202,
 * update_b.py:514-528) with the operator D1.  Inputs: the spectral
 * nonlinear products of the stage (mt_bouss_out / mt_anel_out names) and the
 * velocity potentials, all (lm_max, n_r) complex with row stride `ld`;
 * outputs likewise.  dpdt is written only without the double-curl form (may
 * be null); ddw and dz are read only with it.  Values at the boundary levels
 * are those of the reference (zero before finish_exp, then plus or2 D1 of
 * the auxiliary).  heat (may be NULL): the spectral viscous / Ohmic heating of
 * the anelastic stage (mt_anel_out heat), added to the entropy's partial term
 * before finish_exp (step_time.py:1452-1455, get_td.f90:485,499). */
typedef struct {
  const double *Advr, *Advt, *Advp, *VSr, *VSt, *VxBr, *VxBt, *VxBp, *VXir, *VXit;
  const double *w, *dw, *ddw, *z, *dz;
  int64_t ld;
  const double* heat;
} mt_td_in;

typedef struct {
  double *dwdt, *dzdt, *dpdt, *dsdt, *dxidt, *dbdt, *djdt;
  int64_t ld;
} mt_td_out;

typedef struct {
  const double *r, *or1, *or2, *or4, *orho1, *beta; /* (n_r) device */
  double CorFac;
  int l_double_curl, l_heat, l_mag, l_chem, l_anel;
} mt_td_params;

MT_API int mt_get_td(const mt_plan* plan, int n_r, const mt_td_in* in, const mt_td_out* out,
                     const mt_td_params* p, const mt_radial_op* D1, void* stream);

/* ---- implicit update of a field with a per-degree solve ------------------
 * One CNAB2 step of an equation whose implicit operator is a radial
 * operator per degree l: entropy (magic_torch/update_s.py:213-271 updateS),
 * composition (update_xi.py updateXi), toroidal velocity (update_z.py:333-505
 * updateZ without inner-core rotation or angular-momentum correction), the
 * poloidal and toroidal magnetic field with an insulating inner core
 * (update_b.py:98-635 updateB, b and j each one call):
 *   rhs = w_old old + w_impl impl + w_expl0 expl0 + w_expl1 expl1
 *         (time_scheme.py:82-96), rows 0 and n_r-1 = top / bot values;
 *   x = M_l rhs per degree l (m = 0 coefficients real), dx = D1 x,
 *   d2x = D2 x (stored when d2x is not NULL),
 *   expl1 <- expl0 (time_scheme.py:130-143),
 *   old  <- so_l[l] so_r[r] x,
 *   impl <- ia_l[l] ia_r[r] (D2 x + ib_r[r] dx - (ic_r[r] + ic_l[l] ic_r2[r]) x).
 * Entropy: so = 1, ia = opr hdif_l kappa, ib = beta + dLtemp0 + 2/r + dLkappa,
 * ic_r = 0, ic_l ic_r2 = l(l+1)/r^2; toroidal velocity: so = l(l+1)/r^2,
 * ia = hdif_l l(l+1)/r^2 visc, ib = dLvisc - beta, ic_r = the l-independent
 * part, ic_l ic_r2 = l(l+1)/r^2 (magic_b200.implicit builds both).
 * M_l: the per-degree solve operators (mt_lop: one dense n_r x n_r matrix per
 * l = 0..l_max, HOST pointer, row-major; the inverse of the reference's LHS,
 * with the DCT-I to grid values folded in for the Chebyshev scheme).  All
 * (lm_max, n_r) complex arrays share the row stride ld; top/bot are
 * (lm_max) complex or NULL (zero); the coefficient arrays are device arrays,
 * *_l of l_max+1 and *_r of n_r values; so_l/so_r NULL mean 1, ic_r NULL 0. */
typedef struct mt_lop mt_lop;
MT_API int mt_lop_create(int n_l, int n_r, const double* M_host, mt_lop** op);

/* Banded form of the per-degree solve (replaces the dense inverse where the
 * reference factorises: finite differences of order > 2, magic_torch/
 * update_s.py:95-104, update_z.py:119-127, update_b.py:127-131,
 * update_w_doublecurl.py:106-125): A_host holds, per l = 0..n_l-1, the
 * preconditioned n_r x n_r LHS (row-major, zero outside kl sub- and ku
 * super-diagonals); fac_row (and fac_col, or NULL) the scalings of the solve,
 * (n_l, n_r) row-major.  Each matrix is factored on the host with pivoted
 * banded LU (algebra.py:371-457, LINPACK dgbfa order) and the updates then
 * solve fac_col * U^-1 L^-1 P (fac_row * rhs) on the GPU in the reference's
 * dgbsl order (algebra.py:460-510).  Used by mt_update_field and
 * mt_update_poloidal; mt_update_wp needs the dense form. */
MT_API int mt_lop_create_band(int n_l, int n_r, int kl, int ku, const double* A_host,
                              const double* fac_row, const double* fac_col, mt_lop** op);
MT_API int mt_lop_destroy(mt_lop* op);

typedef struct {
  double *x, *dx, *d2x, *old, *impl, *expl0, *expl1; /* d2x may be NULL */
  const double *top, *bot;
  int64_t ld;
  double w_old, w_impl, w_expl0, w_expl1;
  const double *so_l, *so_r, *ia_l, *ia_r, *ib_r, *ic_r, *ic_l, *ic_r2;
} mt_field_update;

MT_API int mt_update_field(const mt_plan* plan, int n_r, const mt_field_update* u,
                           const mt_lop* solve, const mt_radial_op* D1,
                           const mt_radial_op* D2, void* stream);

/* ---- angular-momentum corrections of the toroidal velocity ---------------
 * With stress-free boundaries the reference removes, after each toroidal
 * solve, the outer core's axial (l_correct_AMz) and equatorial
 * (l_correct_AMe) angular momentum (magic_torch/update_z.py:446-475, with
 * get_angular_moment :301-331 and the constants of pre_calculations.py:
 * 60-101).  For the row (l, m) = (1, 0):
 *   AM_z = 8/3 pi y10 sum_r rint r^2 Re z,  y10 = sqrt(3/pi)/2,
 *   c = (AM_z - am_start) / (c_moi_oc y10);
 * then for (1, 1) (when the plan holds m = 1), from the corrected state:
 *   AM_x = 16/3 pi y11 sum_r rint r^2 Re z,  AM_y = -16/3 pi y11 sum_r rint r^2 Im z,
 *   c = (AM_x - i AM_y) / (2 y11 c_moi_oc),  y11 = sqrt(1.5/pi)/2;
 * each correction subtracts c am_z from z, c am_dz from dz and c am_d2z from
 * d2z (when stored), and the same linear change from the old and implicit
 * terms that mt_update_field wrote with the coefficients of u (so the result
 * equals recomputing them from the corrected fields).  u: the toroidal
 * velocity's mt_field_update of this step, already applied. */
typedef struct {
  const double* rint;                   /* (n_r) weights of the radial integral */
  const double* r;                      /* (n_r) radii */
  const double *am_z, *am_dz, *am_d2z;  /* (n_r) rho0 r^2, rho0 (2 r + beta r^2),
                                           rho0 (2 + 4 beta r + (dbeta + beta^2) r^2) */
  double c_moi_oc;                      /* 8/3 pi sum_r rint r^4 rho0 */
  double am_start;                      /* axial angular momentum to hold (0: fresh start) */
  int axial, equatorial;
} mt_am_correction;

MT_API int mt_correct_am(const mt_plan* plan, int n_r, const mt_field_update* u,
                         const mt_am_correction* c, void* stream);

/* ---- implicit update of the poloidal velocity, double-curl form ----------
 * One CNAB2 step of magic_torch/update_w_doublecurl.py:393-483 (updateW, the
 * finite-difference scheme) with the l = 0 pressure of update_wp.py:80-194:
 *   rhs = CNAB2 combination + wimp_lin0 BuoFac l(l+1) or2 rgrav s on rows
 *         2..n_r-3 (+ ChemFac ... xi), rows 0, 1, n_r-2, n_r-1 zero;
 *   w = M_l rhs (degree 0 zero, m = 0 real), dw = D1 w, ddw = D2 w,
 *   dddw = D1 ddw, ddddw = D2 ddw;
 *   old  <- -l(l+1) or2 orho1 (ddw - beta dw - l(l+1) or2 w),
 *   impl <- -hdif_l l(l+1) or2 visc orho1 (ddddw + c3 dddw + c2 ddw + c1 dw + c0 w)
 *           + BuoFac l(l+1) or2 rgrav s (+ ChemFac ... xi), both zero at r_0, r_N-1,
 *     c2 = c2n - 2 l(l+1) or2, c1 = c1n + l(l+1) c1d, c0 = l(l+1) or2 (c0n + l(l+1) or2);
 *   expl1 <- expl0;
 *   p(0,0) = P0 (0, rho0 BuoFac rgrav Re s00 + Re expl0_00 (+ chemistry), ...).
 * s / xi: the entropy / composition of this step (after their own update).
 * P0: the inverse of the l = 0 pressure matrix as a radial operator. */
typedef struct {
  double *w, *dw, *ddw, *old, *impl, *expl0, *expl1, *p; /* p: row (l, m) = (0, 0) only */
  const double *s, *xi;                                   /* xi may be NULL */
  int64_t ld;
  double w_old, w_impl, w_expl0, w_expl1, wimp_lin0, BuoFac, ChemFac;
  const double* hdif;                                     /* (l_max + 1) */
  const double *or2, *orho1, *beta, *visc, *rgrav, *rho0; /* (n_r) */
  const double *c3, *c2n, *c1n, *c1d, *c0n;               /* (n_r) */
} mt_poloidal_update;

MT_API int mt_update_poloidal(const mt_plan* plan, int n_r, const mt_poloidal_update* u,
                              const mt_lop* solve, const mt_radial_op* D1,
                              const mt_radial_op* D2, const mt_radial_op* P0, void* stream);

/* ---- implicit update of the poloidal velocity and pressure, standard form --
 * One CNAB2 step of magic_torch/update_wp.py:387-531 (updateWP, the form the
 * Chebyshev scheme uses) with the l = 0 pressure of update_wp.py:80-194:
 *   rhs_w = CNAB2 combination of the w equation's time arrays
 *           + wimp_lin0 BuoFac rho0 rgrav s (+ ChemFac ... xi) on rows 1..n_r-2,
 *   rhs_p = CNAB2 combination of the p equation's time arrays on rows 1..n_r-2,
 *   boundary rows zero; (w, p) = M_l (rhs_w, rhs_p) per degree l >= 1 (m = 0
 *   real); w = 0 at l = 0 and p(0,0) = P0 (0, rho0 BuoFac rgrav Re s00
 *   + Re expl0_w,00 (+ chemistry), ...);
 *   dw = D1 w, ddw = D2 w, dddw = D3 w, dp = D1 p;
 *   w:  old <- l(l+1) or2 w,
 *       impl <- -dp + beta p + hdif_l l(l+1) or2 visc (ddw + (2 dLvisc - beta/3) dw
 *               - (l(l+1) or2 + 4/3 (dbeta + dLvisc beta + (3 dLvisc + beta) or1)) w)
 *               + BuoFac rho0 rgrav s (+ ChemFac rho0 rgrav xi);
 *   p:  old <- -l(l+1) or2 dw,
 *       impl <- l(l+1) or2 p + hdif_l visc l(l+1) or2 (-dddw + (beta - dLvisc) ddw
 *               + (l(l+1) or2 + dLvisc beta + dbeta + 2 (dLvisc + beta) or1) dw
 *               - l(l+1) or2 (2 or1 + 2/3 beta + dLvisc) w);
 *   expl1 <- expl0 for both equations.
 * solve: per-degree operators of size 2 n_r (mt_lop with n_r' = 2 n_r): the
 * inverse of the reference's coupled 2n_r x 2n_r matrix (get_wpMat) with the
 * Chebyshev truncation and the DCT-I to grid values of each block folded in;
 * P0: the l = 0 pressure inverse likewise; s / xi: this step's entropy /
 * composition (after their own update). */
typedef struct {
  double *w, *dw, *ddw, *p, *dp;
  double *w_old, *w_impl, *w_expl0, *w_expl1;
  double *p_old, *p_impl, *p_expl0, *p_expl1;
  const double *s, *xi;                                    /* xi may be NULL */
  int64_t ld;
  double w_old_wt, w_impl_wt, w_expl0_wt, w_expl1_wt, wimp_lin0, BuoFac, ChemFac;
  const double* hdif;                                      /* (l_max + 1) */
  const double *or1, *or2, *beta, *dbeta, *visc, *dLvisc, *rgrav, *rho0; /* (n_r) */
  int impl_interior; /* nonzero: both implicit terms zero at l = 0 and at the two boundary
                        levels, as the reference's time step stores them (step_time.py:385-394,
                        :538-545); zero: every entry, as updateWP alone */
  const double* p0_row0; /* (n_r) or NULL: row 0 of the l = 0 pressure right-hand side is
                            sum_r p0_row0[r] Re s00[r] (the anelastic integral constraint,
                            update_wp.py:416-421, with P0 built to match); NULL: 0 */
} mt_wp_update;

MT_API int mt_update_wp(const mt_plan* plan, int n_r, const mt_wp_update* u, const mt_lop* solve,
                        const mt_radial_op* D1, const mt_radial_op* D2, const mt_radial_op* D3,
                        const mt_radial_op* P0, void* stream);

/* ---- energy integrals of the outer core (FP64) ---------------------------
 * magic_torch/output.py:101-180 (get_e_kin_full, get_e_mag_oc_full): with
 * |x|^2 = Re^2 (m = 0) or 2 |x|^2 (m > 0) and L = l(l+1),
 *   pol(lm, r) = cr[r] L (L or2[r] |pol|^2 + |dpol|^2),  tor(lm, r) = cr[r] L |tor|^2,
 * out[0..3] = integral over r (weights rint[r]) of the sum over lm of pol
 *             for all lm, m = 0, the equatorially symmetric lm, their m = 0 part;
 * out[4..7] = the same for tor (the complementary parities);
 * out[8..9] = sum over lm of l^2 (l+1) |pol(r = 0)|^2, all and m = 0 (magnetic
 *             only; the caller scales by LFfac / (2 r_cmb)).
 * Kinetic (magnetic = 0): pol = w, dpol = dw, tor = z, cr = orho1 / 2, symmetric
 * parities pol (l+m) even, tor (l+m) odd; magnetic: b, db, aj, cr = LFfac / 2,
 * the opposite parities.  rint: the radial rule as weights (n_r).  out: 10
 * device doubles; work: mt_energy_workspace bytes of device memory. */
typedef struct {
  const double *pol, *dpol, *tor; /* (lm_max, n_r) complex, row stride ld */
  int64_t ld;
  const double *or2, *cr, *rint;  /* (n_r) device arrays */
  int magnetic;
} mt_energy_args;

MT_API size_t mt_energy_workspace(const mt_plan* plan);
MT_API int mt_energy(const mt_plan* plan, int n_r, const mt_energy_args* e, double* out,
                     void* work, size_t work_bytes, void* stream);

MT_API int mt_selftest_wait_timeout(int* status, long long spins, void* stream);

/* ---- cross-run batching ------------------------------------------------- */

/* One block copy of complex (re, im double) columns: for every row i < n_rows,
 * dst[i * dst_ld + dst_col0 + j] = src[i * src_ld + src_col0 + j], j < n_cols
 * (strides and offsets in complex elements).  src and dst are device pointers;
 * the array of copies itself lives in device memory. */
typedef struct {
  const double* src;
  double* dst;
  int64_t src_ld, dst_ld;
  int src_col0, dst_col0, n_cols, pad;
} mt_level_copy;

/* All copies in one launch on `stream` (no counterpart in the reference, which
 * runs one simulation per process): gathers the radial levels of several runs
 * of one resolution into the batch arrays of one mt_nl_bouss call, and
 * scatters the outputs back.  Copies must not overlap each other. */
MT_API int mt_copy_levels(int n_rows, const mt_level_copy* copies, int n_copies, void* stream);

/* ---- device status of the split-precision kernels ----------------------- */

/* The tcgen05 kernels of split-precision plans bound every wait on the tensor
 * pipe and on their bulk copies.  A wait that runs out stops the CTA, and the
 * kernel records a non-zero code in the first 4 bytes of the call's `work`
 * buffer; the results of that call are then invalid (the entry point itself
 * returned MT_OK: it does not synchronise).  The code stays there until the
 * next call that reuses the buffer clears it.  mt_device_status copies it into
 * *code after the work enqueued on `stream` so far has finished (it
 * synchronises `stream`).  0 means every wait completed; FP64 plans never
 * write the word (their kernels have no such waits) and always read 0 when
 * the buffer was cleared by a split call or zero-initialised.  No counterpart
 * in the reference (its bmm path has no device-side waits). */
MT_API int mt_device_status(const void* work, int* code, void* stream);

/* The same for the fixed scratch of mt_scal_to_spat_noalloc (the caller has
 * no pointer to it): the code of the last allocation-free call on the current
 * device. */
MT_API int mt_noalloc_status(int* code, void* stream);

/* Thread-local message for the last non-zero status. */
MT_API const char* mt_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* MAGIC_B200_H */
