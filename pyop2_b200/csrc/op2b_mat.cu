// Mat operations on device CSR values.
//
// zero_rows follows cuda.Mat.zero_rows (pyop2/cuda.py:289-297) and PETSc
// MatZeroRowsLocal with KEEP_NONZERO_PATTERN (pyop2/petsc_base.py:116-135):
// every stored entry of the listed rows becomes 0 and the diagonal entry, if
// the pattern stores one, becomes diag.
#include <cuda_runtime.h>

#include <vector>

#include "op2b_internal.h"

namespace op2b {

template <typename T>
__global__ void zero_rows_kernel(T *__restrict__ vals, const int32_t *__restrict__ rowptr,
                                 const int32_t *__restrict__ colidx, const int32_t *__restrict__ rows,
                                 int nrows, T diag) {
  // one warp per listed row
  const int lane = threadIdx.x & 31;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nrows;
       i += (gridDim.x * blockDim.x) >> 5) {
    const int r = rows[i];
    for (int k = rowptr[r] + lane; k < rowptr[r + 1]; k += 32) vals[k] = colidx[k] == r ? diag : T(0);
  }
}

}  // namespace op2b

using namespace op2b;

extern "C" int op2b_mat_zero_rows(uint64_t vals, uint64_t rowptr, uint64_t colidx,
                                  const int32_t *rows, int32_t nrows_zero, double diag,
                                  int32_t elem_bytes, uint64_t stream) {
  OP2B_REQUIRE_INIT();
  if (nrows_zero <= 0) return OP2B_OK;
  cudaStream_t s = stream_of(stream);
  int32_t *d_rows = nullptr;
  int rc = dev_alloc((void **)&d_rows, sizeof(int32_t) * nrows_zero, s);
  if (rc) return rc;
  cudaError_t e = cudaMemcpyAsync(d_rows, rows, sizeof(int32_t) * nrows_zero, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) {
    dev_free(d_rows, s);
    return check_cuda(e, "op2b_mat_zero_rows copy");
  }
  const int grid = std::max(1, std::min(op2b_div_up(nrows_zero, 8), sm_count() * 8));
  if (elem_bytes == 8)
    zero_rows_kernel<double><<<grid, 256, 0, s>>>((double *)vals, (const int32_t *)rowptr,
                                                  (const int32_t *)colidx, d_rows, nrows_zero, diag);
  else if (elem_bytes == 4)
    zero_rows_kernel<float><<<grid, 256, 0, s>>>((float *)vals, (const int32_t *)rowptr,
                                                 (const int32_t *)colidx, d_rows, nrows_zero, (float)diag);
  else {
    dev_free(d_rows, s);
    return set_error(OP2B_ERR_ARG, "op2b_mat_zero_rows: elem_bytes %d", elem_bytes);
  }
  e = cudaGetLastError();
  // The pinned/pageable host rows buffer may be released by the caller as
  // soon as this returns, so complete the copy first.
  cudaError_t e2 = cudaStreamSynchronize(s);
  dev_free(d_rows, s);
  if (e != cudaSuccess) return check_cuda(e, "zero_rows_kernel");
  if (e2 != cudaSuccess) return check_cuda(e2, "op2b_mat_zero_rows sync");
  return OP2B_OK;
}
