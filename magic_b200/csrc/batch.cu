// Level (column) block copies between per-run spectral arrays and the batch
// arrays of the cross-run fused stage: runs of one resolution concatenate their
// radial levels, so one stage launch serves them all (serve.py).
#include "common.cuh"

namespace mt {

// one warp per (copy, row); lanes walk the row's columns (contiguous complex
// values, so each warp moves whole 16-byte elements in order)
__global__ void k_copy_levels(int n_rows, const mt_level_copy* __restrict__ cps) {
  const mt_level_copy c = cps[blockIdx.y];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int row = blockIdx.x * (blockDim.x >> 5) + warp; row < n_rows;
       row += gridDim.x * (blockDim.x >> 5)) {
    const double2* s = reinterpret_cast<const double2*>(c.src) + (int64_t)row * c.src_ld + c.src_col0;
    double2* d = reinterpret_cast<double2*>(c.dst) + (int64_t)row * c.dst_ld + c.dst_col0;
    for (int j = lane; j < c.n_cols; j += 32) d[j] = s[j];
  }
}

}  // namespace mt

extern "C" {

int mt_copy_levels(int n_rows, const mt_level_copy* copies, int n_copies, void* stream) {
  using namespace mt;
  MT_REQUIRE(n_rows >= 1 && n_copies >= 0 && n_copies <= 65535 && (copies || !n_copies),
             MT_ERR_ARG, "mt_copy_levels: bad row or copy count");
  if (n_copies == 0) return MT_OK;
  const int warps = 8;
  int blocks = (n_rows + warps - 1) / warps;
  if (blocks > 1024) blocks = 1024;
  k_copy_levels<<<dim3(blocks, n_copies), 32 * warps, 0, (cudaStream_t)stream>>>(n_rows, copies);
  MT_CHECK_CUDA(cudaGetLastError());
  return MT_OK;
}

}  // extern "C"
