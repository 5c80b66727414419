// Radial operators and the spectral explicit terms of a time step (FP64).
//
// Radial operator: a real n_r x n_r matrix D applied along the radial axis of
// complex (row, n_r) arrays, out[row][j] = sum_k D[j][k] in[row][k]
// (magic_torch/radial_derivatives.py:29-68: get_dr / get_ddr / get_dddr with
// the dense Chebyshev or the banded finite-difference matrices;
// magic_torch/cosine_transform.py:18-45: the self-inverse DCT-I, which is the
// same operation with the DCT-I matrix).  Each matrix row keeps only its
// nonzero band: W values starting at column k0[j] (W = widest band, rows
// shifted left so k0[j] + W <= n_r, padding zero), stored band-transposed,
// vals[kk * n_r + j] = D[j][k0[j] + kk], so the 32 lanes of a warp (32
// consecutive output levels) read 32 consecutive values.  A dense Chebyshev
// matrix has W = n_r; the fourth-order finite-difference ones W = 5.
//
// Explicit terms: a CTA takes 8 consecutive lm rows of one m block (contiguous
// in memory) and its threads stride over their (row, level) elements: the
// Coriolis and nonlinear terms of get_td (magic_torch/get_td.py:58-308) go to
// the outputs, the enabled finish_exp auxiliaries (dVxVhLM, dVSrLM, dVXirLM,
// dVxBhLM) to shared memory; after one barrier the threads apply D1 along
// each row and add the derivative terms (update_wp.py:371-385, update_s.py:191-210,
// update_xi.py:183-202, update_b.py:514-528).  The l -+ 1 couplings read the
// neighbouring rows lm -+ 1 of the same m block (m-major order).
#include <algorithm>
#include <cmath>
#include <vector>

#include "radial_op.cuh"

namespace mt {

namespace {

__device__ __forceinline__ double2 c_add(double2 a, double2 b) { return {a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ double2 c_sub(double2 a, double2 b) { return {a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ double2 c_scale(double s, double2 a) { return {s * a.x, s * a.y}; }
// i m x
__device__ __forceinline__ double2 c_im(double m, double2 a) { return {-m * a.y, m * a.x}; }

struct ApplyArgs {
  OpView op[2];
  int nop, nrows;
  const double2* in;
  int64_t ld_in;
  double2* out[2];
  int64_t ld_out;
};

// one warp per row: stage the row, then every lane forms its output levels
__global__ void k_radial_apply(ApplyArgs a) {
  extern __shared__ double2 rowbuf[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int n_r = a.op[0].n_r;
  double2* f = rowbuf + (int64_t)wib * n_r;
  const int wpb = blockDim.x >> 5;
  for (int row = blockIdx.x * wpb + wib; row < a.nrows; row += gridDim.x * wpb) {
    const double2* src = a.in + (int64_t)row * a.ld_in;
    for (int j = lane; j < n_r; j += 32) f[j] = src[j];
    __syncwarp();
#pragma unroll
    for (int o = 0; o < 2; ++o) {
      if (o >= a.nop) break;
      double2* dst = a.out[o] + (int64_t)row * a.ld_out;
      for (int j = lane; j < n_r; j += 32) dst[j] = op_row(a.op[o], f, j);
    }
    __syncwarp();
  }
}

struct TdArgs {
  int n_r, l_max, minc, n_m;
  const int* lstart;
  const double2 *Advr, *Advt, *Advp, *VSr, *VSt, *VxBr, *VxBt, *VxBp, *VXir, *VXit;
  const double2 *w, *dw, *ddw, *z, *dz;
  const double2* heatTerms;  // anelastic viscous / Ohmic heating, or null
  int64_t ld_in;
  double2 *dwdt, *dzdt, *dpdt, *dsdt, *dxidt, *dbdt, *djdt;
  int64_t ld_out;
  const double *r, *or1, *or2, *or4, *orho1, *beta;
  double CorFac;
  int double_curl, heat, mag, chem, anel;
  int naux;  // enabled auxiliaries, in the order double curl, heat, chem, mag
  OpView D1;
};

// sqrt((l+m)(l-m)/((2l-1)(2l+1))) for l > 0 (magic_torch/horizontal_data.py:91-100)
__device__ __forceinline__ double clm_d(double l, double m) {
  return l > 0.0 ? sqrt((l + m) * (l - m) / ((2.0 * l - 1.0) * (2.0 * l + 1.0))) : 0.0;
}

constexpr int kTdRows = 8;       // consecutive lm rows (one m block) per CTA
constexpr int kTdThreads = 256;

// CTA (row block x, order mc): rows l = m + kTdRows x .. of the m block, which
// are contiguous in memory, so the threads stride over all (row, level)
// elements of the block with fully coalesced loads.  Pass 1 writes the
// partial terms and the enabled auxiliaries (shared memory); pass 2 adds
// or2 D1 (auxiliary) along each row.
__global__ void __launch_bounds__(kTdThreads, 4) k_get_td(TdArgs a) {
  extern __shared__ double2 tdbuf[];
  const int n_r = a.n_r;
  const int mc = blockIdx.y, m = mc * a.minc;
  const int l0 = m + blockIdx.x * kTdRows;
  if (l0 > a.l_max) return;
  const int nrow = min(kTdRows, a.l_max + 1 - l0);
  const int lm0 = a.lstart[mc] + (l0 - m);
  const int nel = nrow * n_r;
  const int span = kTdRows * n_r;  // one auxiliary array of the block
  double2* xVh = tdbuf;
  double2* xVS = xVh + (a.double_curl ? span : 0);
  double2* xVX = xVS + (a.heat ? span : 0);
  double2* xVB = xVX + (a.chem ? span : 0);
  const double mf = (double)m, cf2 = 2.0 * a.CorFac;
  const float rcp = 1.0f / (float)n_r;

  for (int e = threadIdx.x; e < nel; e += kTdThreads) {
    int rr = (int)((float)e * rcp);
    rr -= (rr * n_r > e);
    rr += ((rr + 1) * n_r <= e);
    const int j = e - rr * n_r, l = l0 + rr, lm = lm0 + rr;
    const bool bnd = j == 0 || j == n_r - 1;
    // horizontal coefficients of this (l, m) (magic_torch/horizontal_data.py:103-130)
    const double lf = (double)l;
    const double c_l = clm_d(lf, mf), c_lp1 = clm_d(lf + 1.0, mf);
    const double dLh = lf * (lf + 1.0);
    const double dTh1S = (lf + 1.0) * c_l, dTh1A = lf * c_lp1;
    const double dTh2S = (lf - 1.0) * c_l, dTh2A = (lf + 2.0) * c_lp1;
    const double dTh3S = (lf - 1.0) * (lf + 1.0) * c_l, dTh3A = lf * (lf + 2.0) * c_lp1;
    const double dTh4S = dTh1S * (lf - 1.0) * lf, dTh4A = dTh1A * (lf + 1.0) * (lf + 2.0);
    // l+1 neighbour (masked at l_max) and l-1 neighbour (self, zero coefficient, at l = m)
    const bool hasA = l < a.l_max;
    const int64_t row = (int64_t)lm * a.ld_in + j;
    const int64_t rowA = hasA ? row + a.ld_in : row;
    const int64_t rowS = l > m ? row - a.ld_in : row;
    const double mA = hasA ? 1.0 : 0.0;
    const int64_t o = (int64_t)lm * a.ld_out + j;
    const double or1 = a.or1[j], or2 = a.or2[j], or4 = a.or4[j], r = a.r[j];
    const double orho1 = a.orho1[j], beta = a.beta[j];
    const double2 w = a.w[row], dw = a.dw[row], z = a.z[row];
    const double2 zA = c_scale(mA, a.z[rowA]), zS = a.z[rowS];
    // toroidal velocity (get_td.py:151-181)
    {
      const double2 dwA = c_scale(mA, a.dw[rowA]), dwS = a.dw[rowS];
      const double2 wA = c_scale(mA, a.w[rowA]), wS = a.w[rowS];
      double2 cor = c_im(mf, z);
      cor = c_add(cor, c_scale(dTh3A, dwA));
      cor = c_add(cor, c_scale(or1 * dTh4A, wA));
      cor = c_add(cor, c_scale(dTh3S, dwS));
      cor = c_sub(cor, c_scale(or1 * dTh4S, wS));
      const double2 v = c_add(c_scale(dLh, a.Advp[row]), c_scale(cf2 * or2, cor));
      a.dzdt[o] = bnd ? double2{0.0, 0.0} : v;
    }
    if (a.double_curl) {
      // get_td.py:88-148
      double2 v;
      if (lm == 0) {
        v = c_add(c_scale(or2, a.Advr[row]), c_scale(cf2 * or1 * dTh2A, zA));
      } else {
        const double2 ddw = a.ddw[row];
        const double2 dzA = c_scale(mA, a.dz[rowA]), dzS = a.dz[rowS];
        double2 t = c_add(c_scale(-1.0, ddw), c_scale(beta, dw));
        t = c_add(t, c_scale((beta * or1 + or2) * dLh, w));
        double2 in = c_im(mf, t);
        in = c_add(in, c_scale(dTh3A, c_sub(dzA, c_scale(beta, zA))));
        in = c_add(in, c_scale(dTh3S, c_sub(dzS, c_scale(beta, zS))));
        in = c_add(in, c_scale(or1, c_sub(c_scale(dTh4A, zA), c_scale(dTh4S, zS))));
        v = c_add(c_scale(dLh * or4 * orho1, a.Advr[row]), c_scale(cf2 * or2 * orho1, in));
      }
      a.dwdt[o] = bnd ? double2{0.0, 0.0} : v;
      xVh[e] = bnd ? double2{0.0, 0.0} : c_scale(-orho1 * (r * r) * dLh, a.Advt[row]);
    } else {
      // get_td.py:58-85 and 184-213
      double2 cor = c_im(mf, dw);
      cor = c_add(cor, c_scale(dTh2A, zA));
      cor = c_sub(cor, c_scale(dTh2S, zS));
      const double2 v = c_add(c_scale(or2, a.Advr[row]), c_scale(cf2 * or1, cor));
      a.dwdt[o] = bnd ? double2{0.0, 0.0} : v;
      if (a.dpdt) {
        double2 cp = c_scale(-1.0, c_im(mf, c_add(dw, c_scale(or1 * dLh, w))));
        cp = c_add(cp, c_scale(dTh3A, zA));
        cp = c_add(cp, c_scale(dTh3S, zS));
        const double2 p = c_add(c_scale(-dLh, a.Advt[row]), c_scale(cf2 * or2, cp));
        a.dpdt[o] = bnd ? double2{0.0, 0.0} : p;
      }
    }
    if (a.heat) {
      double2 ds = c_scale(dLh, a.VSt[row]);
      if (a.heatTerms) ds = c_add(ds, a.heatTerms[row]);  // step_time.py:1452-1455
      a.dsdt[o] = bnd ? double2{0.0, 0.0} : ds;
      xVS[e] = bnd ? double2{0.0, 0.0} : a.VSr[row];
    }
    if (a.chem) {
      a.dxidt[o] = bnd ? double2{0.0, 0.0} : c_scale(dLh, a.VXit[row]);
      xVX[e] = bnd ? double2{0.0, 0.0} : a.VXir[row];
    }
    if (a.mag) {
      a.dbdt[o] = bnd ? double2{0.0, 0.0} : c_scale(dLh, a.VxBp[row]);
      a.djdt[o] = bnd ? double2{0.0, 0.0} : c_scale(dLh * or4, a.VxBr[row]);
      const double2 h = c_scale(-dLh, a.VxBt[row]);
      xVB[e] = (lm == 0 && bnd) ? double2{0.0, 0.0} : c_scale(r * r, h);
    }
  }
  if (a.naux == 0) return;
  __syncthreads();
  // finish_exp: the radial derivative of each auxiliary along its row, added to
  // the partial term this thread wrote above (same element, same thread)
  for (int e = threadIdx.x; e < nel; e += kTdThreads) {
    int rr = (int)((float)e * rcp);
    rr -= (rr * n_r > e);
    rr += ((rr + 1) * n_r <= e);
    const int j = e - rr * n_r;
    const int64_t o = (int64_t)(lm0 + rr) * a.ld_out + j;
    const int base = rr * n_r;
    const double or2 = a.or2[j], orho1 = a.orho1[j];
    if (a.double_curl) a.dwdt[o] = c_add(a.dwdt[o], c_scale(or2, op_row(a.D1, xVh + base, j)));
    if (a.heat) {
      double2 v = c_sub(a.dsdt[o], c_scale(or2, op_row(a.D1, xVS + base, j)));
      a.dsdt[o] = a.anel ? c_scale(orho1, v) : v;
    }
    if (a.chem) {
      double2 v = c_sub(a.dxidt[o], c_scale(or2, op_row(a.D1, xVX + base, j)));
      a.dxidt[o] = a.anel ? c_scale(orho1, v) : v;
    }
    if (a.mag) a.djdt[o] = c_add(a.djdt[o], c_scale(or2, op_row(a.D1, xVB + base, j)));
  }
}


constexpr size_t kRadialSmemBudget = 96 * 1024;

}  // namespace

int check_radial_op(const mt_radial_op* op) {
  MT_REQUIRE(op && op->vals, MT_ERR_ARG, "null radial operator");
  int dev = -1;
  MT_CHECK_CUDA(cudaGetDevice(&dev));
  MT_REQUIRE(dev == op->device, MT_ERR_ARG,
             "radial operator used on a different device than it was built on");
  return MT_OK;
}

}  // namespace mt

using namespace mt;

extern "C" {

int mt_radial_op_create(int n_r, const double* D, mt_radial_op** out) {
  MT_REQUIRE(out && D && n_r >= 2 && n_r <= 4096, MT_ERR_ARG, "bad radial operator argument");
  *out = nullptr;
  // band of every row: first and last nonzero column
  std::vector<int> first(n_r), last(n_r);
  int W = 1;
  for (int j = 0; j < n_r; ++j) {
    int f = -1, l = -1;
    for (int k = 0; k < n_r; ++k) {
      MT_REQUIRE(std::isfinite(D[(size_t)j * n_r + k]), MT_ERR_ARG, "radial operator not finite");
      if (D[(size_t)j * n_r + k] != 0.0) {
        if (f < 0) f = k;
        l = k;
      }
    }
    if (f < 0) f = l = std::min(j, n_r - 1);
    first[j] = f;
    last[j] = l;
    W = std::max(W, l - f + 1);
  }
  std::vector<int> k0(n_r);
  std::vector<double> vals((size_t)W * n_r, 0.0);
  for (int j = 0; j < n_r; ++j) {
    k0[j] = std::min(first[j], n_r - W);  // keep k0 + W <= n_r; the extra columns are zero
    for (int kk = 0; kk < W; ++kk) vals[(size_t)kk * n_r + j] = D[(size_t)j * n_r + k0[j] + kk];
  }
  mt_radial_op* op = new mt_radial_op();
  op->n_r = n_r;
  op->W = W;
  auto fail = [&](int rc) {
    if (op->k0) cudaFree(op->k0);
    if (op->vals) cudaFree(op->vals);
    delete op;
    return rc;
  };
  if (cudaGetDevice(&op->device) != cudaSuccess) return fail((set_error("cudaGetDevice failed"), MT_ERR_CUDA));
  if (cudaMalloc(&op->k0, n_r * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&op->vals, vals.size() * sizeof(double)) != cudaSuccess ||
      cudaMemcpy(op->k0, k0.data(), n_r * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(op->vals, vals.data(), vals.size() * sizeof(double), cudaMemcpyHostToDevice) !=
          cudaSuccess)
    return fail((set_error("radial operator allocation or upload failed"), MT_ERR_CUDA));
  *out = op;
  return MT_OK;
}

int mt_radial_op_create_dct1(int n_r, mt_radial_op** out) {
  MT_REQUIRE(n_r >= 2 && n_r <= 4096, MT_ERR_ARG, "bad DCT-I length");
  // y[k] = (f[0] + (-1)^k f[N] + 2 sum_{j=1}^{N-1} f[j] cos(j k pi / N)) / sqrt(2 N)
  const int N = n_r - 1;
  const double s = 1.0 / std::sqrt(2.0 * N);
  std::vector<double> C((size_t)n_r * n_r);
  for (int k = 0; k < n_r; ++k)
    for (int j = 0; j < n_r; ++j) {
      double v;
      if (j == 0) v = 1.0;
      else if (j == N) v = (k & 1) ? -1.0 : 1.0;
      else v = 2.0 * std::cos(M_PI * (double)((int64_t)j * k % (2 * N)) / N);
      C[(size_t)k * n_r + j] = v * s;
    }
  return mt_radial_op_create(n_r, C.data(), out);
}

int mt_radial_op_destroy(mt_radial_op* op) {
  if (!op) return MT_OK;
  if (op->k0) cudaFree(op->k0);
  if (op->vals) cudaFree(op->vals);
  delete op;
  return MT_OK;
}

int mt_radial_op_bandwidth(const mt_radial_op* op) { return op ? op->W : 0; }

static int radial_apply_n(const mt_radial_op* const* ops, int nop, int nrows, const double* in,
                          int64_t ld_in, double* const* out, int64_t ld_out, void* stream) {
  for (int o = 0; o < nop; ++o) {
    MT_TRY(check_radial_op(ops[o]));
    MT_REQUIRE(ops[o]->n_r == ops[0]->n_r, MT_ERR_ARG, "radial operators of different sizes");
    MT_REQUIRE(out[o], MT_ERR_ARG, "null radial output");
  }
  const int n_r = ops[0]->n_r;
  MT_REQUIRE(in && nrows >= 0 && ld_in >= n_r && ld_out >= n_r, MT_ERR_ARG,
             "bad radial apply argument");
  if (nrows == 0) return MT_OK;
  ApplyArgs a{};
  for (int o = 0; o < nop; ++o) {
    a.op[o] = radial_op_view(ops[o]);
    a.out[o] = (double2*)out[o];
  }
  a.nop = nop;
  a.nrows = nrows;
  a.in = (const double2*)in;
  a.ld_in = ld_in;
  a.ld_out = ld_out;
  const size_t per_warp = (size_t)n_r * sizeof(double2);
  const int wpb = (int)std::max<size_t>(1, std::min<size_t>(8, kRadialSmemBudget / per_warp));
  MT_REQUIRE(per_warp <= 200 * 1024, MT_ERR_UNSUPPORTED, "radial row too long for shared memory");
  const size_t sm = wpb * per_warp;
  MT_CHECK_CUDA(cudaFuncSetAttribute(k_radial_apply, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sm));
  int dev = 0, nsm = 148;
  MT_CHECK_CUDA(cudaGetDevice(&dev));
  MT_CHECK_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int blocks = (int)std::min<int64_t>((nrows + wpb - 1) / wpb, (int64_t)nsm * 16);
  k_radial_apply<<<blocks, 32 * wpb, sm, (cudaStream_t)stream>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

int mt_radial_apply(const mt_radial_op* op, int nrows, const double* in, int64_t ld_in,
                    double* out, int64_t ld_out, void* stream) {
  const mt_radial_op* ops[1] = {op};
  double* outs[1] = {out};
  return radial_apply_n(ops, 1, nrows, in, ld_in, outs, ld_out, stream);
}

int mt_radial_apply2(const mt_radial_op* op1, const mt_radial_op* op2, int nrows,
                     const double* in, int64_t ld_in, double* out1, double* out2,
                     int64_t ld_out, void* stream) {
  const mt_radial_op* ops[2] = {op1, op2};
  double* outs[2] = {out1, out2};
  return radial_apply_n(ops, 2, nrows, in, ld_in, outs, ld_out, stream);
}

int mt_get_td(const mt_plan* p, int n_r, const mt_td_in* in, const mt_td_out* out,
              const mt_td_params* q, const mt_radial_op* D1, void* stream) {
  MT_REQUIRE(p && in && out && q, MT_ERR_ARG, "null argument");
  int dev = -1;
  MT_CHECK_CUDA(cudaGetDevice(&dev));
  MT_REQUIRE(dev == p->device, MT_ERR_ARG, "plan used on a different device than it was built on");
  MT_REQUIRE(n_r >= 3 && in->ld >= n_r && out->ld >= n_r, MT_ERR_ARG, "bad radial size or stride");
  MT_REQUIRE(q->r && q->or1 && q->or2 && q->or4 && q->orho1 && q->beta, MT_ERR_ARG,
             "null radial profile");
  MT_REQUIRE(in->w && in->dw && in->z && in->Advr && in->Advt && in->Advp && out->dwdt &&
                 out->dzdt,
             MT_ERR_ARG, "null velocity field or output");
  const bool need_d1 = q->l_double_curl || q->l_heat || q->l_chem || q->l_mag;
  if (need_d1) {
    MT_TRY(check_radial_op(D1));
    MT_REQUIRE(D1->n_r == n_r, MT_ERR_ARG, "D1 size differs from n_r");
  }
  if (q->l_double_curl) MT_REQUIRE(in->ddw && in->dz, MT_ERR_ARG, "double curl needs ddw and dz");
  if (q->l_heat) MT_REQUIRE(in->VSr && in->VSt && out->dsdt, MT_ERR_ARG, "heat terms missing");
  if (q->l_chem) MT_REQUIRE(in->VXir && in->VXit && out->dxidt, MT_ERR_ARG, "composition terms missing");
  if (q->l_mag)
    MT_REQUIRE(in->VxBr && in->VxBt && in->VxBp && out->dbdt && out->djdt, MT_ERR_ARG,
               "induction terms missing");
  TdArgs a{};
  a.n_r = n_r;
  a.l_max = p->l_max;
  a.minc = p->minc;
  a.n_m = p->n_m;
  a.lstart = p->d_lstart;
  auto c = [](const double* x) { return (const double2*)x; };
  a.Advr = c(in->Advr); a.Advt = c(in->Advt); a.Advp = c(in->Advp);
  a.VSr = c(in->VSr); a.VSt = c(in->VSt);
  a.VxBr = c(in->VxBr); a.VxBt = c(in->VxBt); a.VxBp = c(in->VxBp);
  a.VXir = c(in->VXir); a.VXit = c(in->VXit);
  a.w = c(in->w); a.dw = c(in->dw); a.ddw = c(in->ddw); a.z = c(in->z); a.dz = c(in->dz);
  a.heatTerms = q->l_heat ? c(in->heat) : nullptr;
  a.ld_in = in->ld;
  auto d = [](double* x) { return (double2*)x; };
  a.dwdt = d(out->dwdt); a.dzdt = d(out->dzdt); a.dpdt = d(out->dpdt); a.dsdt = d(out->dsdt);
  a.dxidt = d(out->dxidt); a.dbdt = d(out->dbdt); a.djdt = d(out->djdt);
  a.ld_out = out->ld;
  a.r = q->r; a.or1 = q->or1; a.or2 = q->or2; a.or4 = q->or4; a.orho1 = q->orho1; a.beta = q->beta;
  a.CorFac = q->CorFac;
  a.double_curl = q->l_double_curl != 0;
  a.heat = q->l_heat != 0;
  a.chem = q->l_chem != 0;
  a.mag = q->l_mag != 0;
  a.anel = q->l_anel != 0;
  if (need_d1) a.D1 = radial_op_view(D1);
  else a.D1 = OpView{n_r, 0, nullptr, nullptr};
  a.naux = (int)a.double_curl + (int)a.heat + (int)a.chem + (int)a.mag;
  const size_t sm = (size_t)a.naux * kTdRows * n_r * sizeof(double2);
  MT_REQUIRE(sm <= 200 * 1024, MT_ERR_UNSUPPORTED, "n_r too large for the explicit-term kernel");
  MT_CHECK_CUDA(cudaFuncSetAttribute(k_get_td, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  const dim3 grid((p->l_max + 1 + kTdRows - 1) / kTdRows, p->n_m);
  k_get_td<<<grid, kTdThreads, sm, (cudaStream_t)stream>>>(a);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

}  // extern "C"
