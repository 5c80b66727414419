// Radial operator (mt_radial_op): device layout shared by the kernels that
// apply a real n_r x n_r matrix along r (radial_td.cu, implicit.cu).
#pragma once

#include "common.cuh"

struct mt_radial_op {
  int n_r = 0, W = 0, device = 0;
  int* k0 = nullptr;       // (n_r) first column of each row's band
  double* vals = nullptr;  // (W, n_r) band-transposed values: vals[kk * n_r + j] = D[j][k0[j] + kk]
};

namespace mt {

struct OpView {
  int n_r, W;
  const int* k0;
  const double* vals;
};

// (D f)[j] for one complex row f staged in shared memory
__device__ __forceinline__ double2 op_row(const OpView& op, const double2* f, int j) {
  const int k0 = __ldg(op.k0 + j);
  double2 acc = {0.0, 0.0};
  for (int kk = 0; kk < op.W; ++kk) {
    const double c = __ldg(op.vals + (int64_t)kk * op.n_r + j);
    const double2 v = f[k0 + kk];
    acc.x = fma(c, v.x, acc.x);
    acc.y = fma(c, v.y, acc.y);
  }
  return acc;
}

inline OpView radial_op_view(const mt_radial_op* op) {
  return OpView{op->n_r, op->W, op->k0, op->vals};
}
inline int radial_op_size(const mt_radial_op* op) { return op ? op->n_r : 0; }
// non-null and built on the current device (radial_td.cu)
int check_radial_op(const mt_radial_op* op);

}  // namespace mt
