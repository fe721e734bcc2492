// Halo rows of partitioned sets: a rank packs the owned rows a peer imports
// into one contiguous send buffer and unpacks the rows it receives into its
// halo rows (pyop2/base.py:797-835 did both with numpy fancy indexing on the
// host: send_buf = data[sends[dest]], data[receives[source]] = recv_buf).
//
// One thread per 4-byte word of the packed rows (rows whose size is not a
// multiple of 4 bytes go byte by byte); reads of the index list and of the
// packed buffer are coalesced, the Dat side is a row gather or scatter.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>

#include "op2b_internal.h"

namespace op2b {

template <typename W, bool kUnpack>
__global__ void halo_rows_kernel(W *__restrict__ rows, W *__restrict__ buf,
                                 const int32_t *__restrict__ index, int64_t n, int words) {
  const int64_t tot = n * words;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < tot;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = q / words;
    const int w = (int)(q - i * words);
    const int64_t r = (int64_t)index[i] * words + w;
    if (kUnpack)
      rows[r] = buf[q];
    else
      buf[q] = rows[r];
  }
}

template <bool kUnpack>
int halo_rows(uint64_t rows, uint64_t buf, uint64_t index, int64_t n, int32_t row_bytes,
              uint64_t stream, const char *who) {
  OP2B_REQUIRE_INIT();
  if (n < 0 || row_bytes <= 0 || (n > 0 && (!rows || !buf || !index)))
    return set_error(OP2B_ERR_ARG, "%s: n %lld row_bytes %d", who, (long long)n, row_bytes);
  if (n == 0) return OP2B_OK;
  const bool word = row_bytes % 4 == 0;
  const int words = word ? row_bytes / 4 : row_bytes;
  const int64_t tot = n * words;
  const int grid = std::max(1, std::min<int>((int)std::min<int64_t>((tot + 255) / 256, INT_MAX),
                                             sm_count() * 8));
  cudaStream_t s = stream_of(stream);
  const int32_t *idx = reinterpret_cast<const int32_t *>(index);
  if (word)
    halo_rows_kernel<uint32_t, kUnpack><<<grid, 256, 0, s>>>(
        reinterpret_cast<uint32_t *>(rows), reinterpret_cast<uint32_t *>(buf), idx, n, words);
  else
    halo_rows_kernel<uint8_t, kUnpack><<<grid, 256, 0, s>>>(
        reinterpret_cast<uint8_t *>(rows), reinterpret_cast<uint8_t *>(buf), idx, n, words);
  return check_cuda(cudaGetLastError(), who);
}

}  // namespace op2b

using namespace op2b;

extern "C" {

int op2b_halo_pack(uint64_t buf, uint64_t rows, uint64_t index, int64_t n, int32_t row_bytes,
                   uint64_t stream) {
  return halo_rows<false>(rows, buf, index, n, row_bytes, stream, "op2b_halo_pack");
}

int op2b_halo_unpack(uint64_t rows, uint64_t buf, uint64_t index, int64_t n, int32_t row_bytes,
                     uint64_t stream) {
  return halo_rows<true>(rows, buf, index, n, row_bytes, stream, "op2b_halo_unpack");
}

}  // extern "C"
