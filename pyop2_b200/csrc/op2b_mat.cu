// Mat operations on device CSR values.
//
// zero_rows follows cuda.Mat.zero_rows (pyop2/cuda.py:289-297) and PETSc
// MatZeroRowsLocal with KEEP_NONZERO_PATTERN (pyop2/petsc_base.py:116-135):
// every stored entry of the listed rows becomes 0 and the diagonal entry, if
// the pattern stores one, becomes diag.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
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

// Host-side checks shared by both zero_rows entry points, made before any
// allocation, copy or launch: the kernel indexes rowptr by every listed row,
// so a row outside [0, mat_rows) would read and write outside the CSR arrays.
// PETSc's MatZeroRowsLocal (pyop2/petsc_base.py:131-135) raises on such a row
// as well.
static int check_zero_rows_args(const char *who, int32_t mat_rows, const int32_t *rows,
                                int32_t nrows_zero, int32_t elem_bytes) {
  if (elem_bytes != 8 && elem_bytes != 4)
    return set_error(OP2B_ERR_ARG, "%s: elem_bytes %d", who, elem_bytes);
  if (mat_rows < 0) return set_error(OP2B_ERR_ARG, "%s: mat_rows %d", who, mat_rows);
  if (!rows) return set_error(OP2B_ERR_ARG, "%s: rows is NULL", who);
  for (int32_t i = 0; i < nrows_zero; ++i)
    if (rows[i] < 0 || rows[i] >= mat_rows)
      return set_error(OP2B_ERR_ARG, "%s: row %d (entry %d) outside [0, %d)", who, rows[i], i,
                       mat_rows);
  return OP2B_OK;
}

// ---- scratch of op2b_mat_zero_rows_static: the row list lives in a fixed
// device array instead of memory allocated per call.  Every GPU that loads
// this library holds OP2B_ZERO_ROWS_STATIC_MAX * 4 bytes (256 KiB) for it
// until the process exits.
static __device__ __align__(256) int32_t g_zero_rows_scratch[OP2B_ZERO_ROWS_STATIC_MAX];

// Device address of g_zero_rows_scratch per device.  In host code the array's
// name is only a host-side stand-in, never a device address, so the address is
// looked up with cudaGetSymbolAddress on the first call on each device.
constexpr int kMaxDevices = 64;
static int32_t *g_zero_rows_scratch_dev[kMaxDevices] = {nullptr};
static std::mutex g_zero_rows_scratch_mutex;

static int zero_rows_scratch(int32_t **out) {
  int dev = 0;
  OP2B_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return set_error(OP2B_ERR_STATE, "device %d", dev);
  std::lock_guard<std::mutex> lock(g_zero_rows_scratch_mutex);
  if (!g_zero_rows_scratch_dev[dev]) {
    void *p = nullptr;
    OP2B_CUDA(cudaGetSymbolAddress(&p, g_zero_rows_scratch));
    g_zero_rows_scratch_dev[dev] = static_cast<int32_t *>(p);
  }
  *out = g_zero_rows_scratch_dev[dev];
  return OP2B_OK;
}

}  // namespace op2b

using namespace op2b;

extern "C" int op2b_mat_zero_rows_static(uint64_t vals, uint64_t rowptr, uint64_t colidx,
                                         int32_t mat_rows, const int32_t *rows,
                                         int32_t nrows_zero, double diag, int32_t elem_bytes,
                                         uint64_t stream) {
  // Arguments are checked before anything touches the device (before the
  // initialisation check too, so the checks also run on a host with no GPU).
  if (nrows_zero <= 0) return OP2B_OK;
  if (nrows_zero > OP2B_ZERO_ROWS_STATIC_MAX)
    return set_error(OP2B_ERR_ARG,
                     "op2b_mat_zero_rows_static: %d rows exceed its fixed scratch of %d rows; "
                     "use op2b_mat_zero_rows or split the list", nrows_zero,
                     OP2B_ZERO_ROWS_STATIC_MAX);
  int rc = check_zero_rows_args("op2b_mat_zero_rows_static", mat_rows, rows, nrows_zero, elem_bytes);
  if (rc) return rc;
  OP2B_REQUIRE_INIT();
  int32_t *d_rows = nullptr;
  rc = zero_rows_scratch(&d_rows);
  if (rc) return rc;
  cudaStream_t s = stream_of(stream);
  // The whole list is overwritten before use: nothing in the scratch needs to
  // start at zero.
  OP2B_CUDA(cudaMemcpyAsync(d_rows, rows, sizeof(int32_t) * nrows_zero, cudaMemcpyHostToDevice, s));
  const int grid = std::max(1, std::min(op2b_div_up(nrows_zero, 8), sm_count() * 8));
  if (elem_bytes == 8)
    zero_rows_kernel<double><<<grid, 256, 0, s>>>((double *)vals, (const int32_t *)rowptr,
                                                  (const int32_t *)colidx, d_rows, nrows_zero, diag);
  else
    zero_rows_kernel<float><<<grid, 256, 0, s>>>((float *)vals, (const int32_t *)rowptr,
                                                 (const int32_t *)colidx, d_rows, nrows_zero, (float)diag);
  OP2B_CUDA(cudaGetLastError());
  // The caller may release or reuse the host row list as soon as this returns.
  OP2B_CUDA(cudaStreamSynchronize(s));
  return OP2B_OK;
}

extern "C" int op2b_mat_zero_rows(uint64_t vals, uint64_t rowptr, uint64_t colidx,
                                  int32_t mat_rows, const int32_t *rows, int32_t nrows_zero,
                                  double diag, int32_t elem_bytes, uint64_t stream) {
  // Arguments are checked before anything touches the device (before the
  // initialisation check too, so the checks also run on a host with no GPU).
  if (nrows_zero <= 0) return OP2B_OK;
  int rc = check_zero_rows_args("op2b_mat_zero_rows", mat_rows, rows, nrows_zero, elem_bytes);
  if (rc) return rc;
  OP2B_REQUIRE_INIT();
  cudaStream_t s = stream_of(stream);
  int32_t *d_rows = nullptr;
  rc = dev_alloc((void **)&d_rows, sizeof(int32_t) * nrows_zero, s);
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
  else
    zero_rows_kernel<float><<<grid, 256, 0, s>>>((float *)vals, (const int32_t *)rowptr,
                                                 (const int32_t *)colidx, d_rows, nrows_zero, (float)diag);
  e = cudaGetLastError();
  // The pinned/pageable host rows buffer may be released by the caller as
  // soon as this returns, so complete the copy first.
  cudaError_t e2 = cudaStreamSynchronize(s);
  dev_free(d_rows, s);
  if (e != cudaSuccess) return check_cuda(e, "zero_rows_kernel");
  if (e2 != cudaSuccess) return check_cuda(e2, "op2b_mat_zero_rows sync");
  return OP2B_OK;
}

// ---- scatter-slot table of a scalar Mat assembly.  For element e and map
// indices (r, c): slots[(r * ca + c) * nelem + e] = CSR position of
// (rmap[e][r], cmap[e][c]), or -1 if the Sparsity lacks that entry.  The
// element index runs fastest, so a stub reading the slot of one (r, c) for
// consecutive elements makes coalesced loads; the column search of every
// entry (done once here) leaves the assembly loop.
namespace op2b {
__global__ void mat_slots_kernel(const int32_t *__restrict__ rowptr,
                                 const int32_t *__restrict__ colidx,
                                 const int32_t *__restrict__ rmap, const int32_t *__restrict__ cmap,
                                 int64_t nelem, int ra, int ca, int32_t *__restrict__ slots) {
  const int64_t total = nelem * ra;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int r = static_cast<int>(t / nelem);
    const int64_t e = t - (int64_t)r * nelem;
    const int row = rmap[e * ra + r];
    const int lo0 = rowptr[row], hi0 = rowptr[row + 1];
    for (int c = 0; c < ca; ++c) {
      const int col = cmap[e * ca + c];
      int lo = lo0, hi = hi0;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (colidx[mid] < col)
          lo = mid + 1;
        else
          hi = mid;
      }
      slots[((int64_t)r * ca + c) * nelem + e] = (lo < hi0 && colidx[lo] == col) ? lo : -1;
    }
  }
}
}  // namespace op2b

// ---- compact scatter-slot table: for element e and local row r, one 64-bit
// word whose byte c is the position of (rmap[e][r], cmap[e][c]) within the
// CSR row, counted from rowptr[row] (255: the Sparsity lacks the entry).
// Rows of up to 254 stored entries and up to 8 columns per element.
namespace op2b {
__global__ void mat_slots_rel_kernel(const int32_t *__restrict__ rowptr,
                                     const int32_t *__restrict__ colidx,
                                     const int32_t *__restrict__ rmap,
                                     const int32_t *__restrict__ cmap, int64_t nelem, int ra,
                                     int ca, unsigned long long *__restrict__ out) {
  const int64_t total = nelem * ra;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int r = static_cast<int>(t / nelem);
    const int64_t e = t - (int64_t)r * nelem;
    const int row = rmap[e * ra + r];
    const int lo0 = rowptr[row], hi0 = rowptr[row + 1];
    unsigned long long w = ~0ull;
    for (int c = 0; c < ca; ++c) {
      const int col = cmap[e * ca + c];
      int lo = lo0, hi = hi0;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (colidx[mid] < col)
          lo = mid + 1;
        else
          hi = mid;
      }
      const unsigned long long off =
          (lo < hi0 && colidx[lo] == col && lo - lo0 < 255) ? (unsigned long long)(lo - lo0) : 255ull;
      w = (w & ~(0xffull << (8 * c))) | (off << (8 * c));
    }
    out[(int64_t)r * nelem + e] = w;
  }
}
}  // namespace op2b

extern "C" int op2b_mat_slots_rel_build(uint64_t rowptr, uint64_t colidx, uint64_t rmap,
                                        uint64_t cmap, int64_t nelem, int32_t ra, int32_t ca,
                                        uint64_t slots, uint64_t stream) {
  OP2B_REQUIRE_INIT();
  if (nelem < 0 || ra <= 0 || ca <= 0 || ca > 8 ||
      (nelem > 0 && (!rowptr || !colidx || !rmap || !cmap || !slots)))
    return set_error(OP2B_ERR_ARG, "op2b_mat_slots_rel_build: bad arguments (ca %d)", ca);
  if (nelem == 0) return OP2B_OK;
  const int64_t work = nelem * ra;
  const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256,
                                                                           (int64_t)sm_count() * 16)));
  mat_slots_rel_kernel<<<grid, 256, 0, stream_of(stream)>>>(
      (const int32_t *)rowptr, (const int32_t *)colidx, (const int32_t *)rmap, (const int32_t *)cmap,
      nelem, ra, ca, (unsigned long long *)slots);
  return check_cuda(cudaGetLastError(), "mat_slots_rel_kernel");
}

extern "C" int op2b_mat_slots_build(uint64_t rowptr, uint64_t colidx, uint64_t rmap, uint64_t cmap,
                                    int64_t nelem, int32_t ra, int32_t ca, uint64_t slots,
                                    uint64_t stream) {
  OP2B_REQUIRE_INIT();
  if (nelem < 0 || ra <= 0 || ca <= 0 || (nelem > 0 && (!rowptr || !colidx || !rmap || !cmap || !slots)))
    return set_error(OP2B_ERR_ARG, "op2b_mat_slots_build: bad arguments");
  if (nelem == 0) return OP2B_OK;
  const int64_t work = nelem * ra;
  const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256,
                                                                           (int64_t)sm_count() * 16)));
  mat_slots_kernel<<<grid, 256, 0, stream_of(stream)>>>(
      (const int32_t *)rowptr, (const int32_t *)colidx, (const int32_t *)rmap, (const int32_t *)cmap,
      nelem, ra, ca, (int32_t *)slots);
  return check_cuda(cudaGetLastError(), "mat_slots_kernel");
}
