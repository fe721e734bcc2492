// Two-phase (local-matrix) INC: deterministic accumulation in the sequential
// backend's order.
//
// Phase 1 is a generated par_loop stub that writes every element's INC
// contribution to a local-contribution array instead of adding it: for the
// contribution of element e at map position k (a Dat row, cdim values) or at
// local Mat entry k = r * ca + c (one value),
//     lma[(k * nelem + e) * cdim + comp].
// Phase 2 (this file) reduces per target t -- a Dat row or a Mat CSR slot --
// walking t's incidence list (flat positions e * arity + k in increasing
// order, op2b_incidence.cu) and adding the contributions to the target's
// current value in that order: elements in order, then positions in order,
// which is the order pyop2/sequential.py:55-72 adds them.  Optionally the
// sum is compensated (Kahan) so FP64 targets fed by FP32 element kernels keep
// every contribution's bits.
//
// For a Mat the incidence is built over the element-major scatter-slot table
// (slot of (e, r, c) at e * ra * ca + r * ca + c), so its targets are the CSR
// positions.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>

#include "op2b_internal.h"

namespace op2b {

__global__ void mat_slots_em_kernel(const int32_t *__restrict__ rowptr,
                                    const int32_t *__restrict__ colidx,
                                    const int32_t *__restrict__ rmap,
                                    const int32_t *__restrict__ cmap, int64_t nelem, int ra, int ca,
                                    int32_t *__restrict__ slots) {
  const int64_t total = nelem * ra;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = t / ra;
    const int r = static_cast<int>(t - e * ra);
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
      slots[(e * ra + r) * ca + c] = (lo < hi0 && colidx[lo] == col) ? lo : -1;
    }
  }
}

template <int CDIM, bool KAHAN>
__global__ void lma_reduce_kernel(double *__restrict__ out, const int32_t *__restrict__ ptr,
                                  const int32_t *__restrict__ list, int32_t ntargets,
                                  const double *__restrict__ lma, int64_t nelem, int arity,
                                  uint64_t kmask) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntargets;
       t += (int64_t)gridDim.x * blockDim.x) {
    double acc[CDIM], cmp[CDIM];
#pragma unroll
    for (int c = 0; c < CDIM; ++c) {
      acc[c] = out[t * CDIM + c];
      cmp[c] = 0.0;
    }
    const int q1 = ptr[t + 1];
    for (int q = ptr[t]; q < q1; ++q) {
      const int pos = __ldg(list + q);
      const int64_t e = pos / arity;
      const int k = pos - static_cast<int>(e) * arity;
      if (!((kmask >> k) & 1ull)) continue;
      const double *src = lma + ((int64_t)k * nelem + e) * CDIM;
#pragma unroll
      for (int c = 0; c < CDIM; ++c) {
        const double v = __ldg(src + c);
        if (KAHAN) {
          // compensated sum (Kahan): the rounding error of each addition is
          // carried into the next one
          const double y = v - cmp[c];
          const double s = acc[c] + y;
          cmp[c] = (s - acc[c]) - y;
          acc[c] = s;
        } else {
          acc[c] += v;
        }
      }
    }
#pragma unroll
    for (int c = 0; c < CDIM; ++c) out[t * CDIM + c] = acc[c];
  }
}

template <int CDIM>
static int launch_reduce(double *out, const int32_t *ptr, const int32_t *list, int32_t ntargets,
                         const double *lma, int64_t nelem, int arity, uint64_t kmask, bool kahan,
                         cudaStream_t s) {
  const int grid = std::max(1, std::min(op2b_div_up(ntargets, 256), sm_count() * 16));
  if (kahan)
    lma_reduce_kernel<CDIM, true><<<grid, 256, 0, s>>>(out, ptr, list, ntargets, lma, nelem, arity,
                                                       kmask);
  else
    lma_reduce_kernel<CDIM, false><<<grid, 256, 0, s>>>(out, ptr, list, ntargets, lma, nelem,
                                                        arity, kmask);
  return check_cuda(cudaGetLastError(), "lma_reduce_kernel");
}

}  // namespace op2b

using namespace op2b;

extern "C" {

int op2b_mat_incidence_build(uint64_t rowptr, uint64_t colidx, uint64_t rmap, uint64_t cmap,
                             int32_t nelem, int32_t ra, int32_t ca, int32_t nnz, uint64_t stream,
                             uint64_t *incidence) {
  OP2B_REQUIRE_INIT();
  if (nelem < 0 || ra <= 0 || ca <= 0 || nnz < 0 || !incidence)
    return set_error(OP2B_ERR_ARG, "op2b_mat_incidence_build: bad arguments");
  const int64_t tot = (int64_t)nelem * ra * ca;
  if (tot > INT_MAX)
    return set_error(OP2B_ERR_ARG, "op2b_mat_incidence_build: %lld local entries", (long long)tot);
  cudaStream_t s = stream_of(stream);
  int32_t *slots = nullptr;
  int rc = dev_alloc((void **)&slots, sizeof(int32_t) * std::max<int64_t>(tot, 1), s);
  if (rc) return rc;
  if (nelem > 0) {
    const int64_t work = (int64_t)nelem * ra;
    const int grid = static_cast<int>(
        std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, (int64_t)sm_count() * 16)));
    mat_slots_em_kernel<<<grid, 256, 0, s>>>((const int32_t *)rowptr, (const int32_t *)colidx,
                                             (const int32_t *)rmap, (const int32_t *)cmap, nelem,
                                             ra, ca, slots);
    rc = check_cuda(cudaGetLastError(), "mat_slots_em_kernel");
  }
  if (!rc) {
    rc = op2b_incidence_build(reinterpret_cast<uint64_t>(slots), nelem, ra * ca, nnz, stream,
                              incidence);
    if (rc == OP2B_ERR_MAP)
      rc = set_error(OP2B_ERR_MAP, "a Mat entry of the assembly is not in the Sparsity pattern");
  }
  dev_free(slots, s);
  return rc;
}

int op2b_lma_reduce(uint64_t out, int32_t cdim, uint64_t ptr, uint64_t list, int32_t ntargets,
                    uint64_t lma, int64_t nelem, int32_t arity, uint64_t kmask, int32_t kahan,
                    uint64_t stream) {
  OP2B_REQUIRE_INIT();
  if (ntargets < 0 || nelem < 0 || arity <= 0 || arity > 64)
    return set_error(OP2B_ERR_ARG, "op2b_lma_reduce: bad arguments");
  if (ntargets == 0) return OP2B_OK;
  cudaStream_t s = stream_of(stream);
  double *o = reinterpret_cast<double *>(out);
  const int32_t *p = reinterpret_cast<const int32_t *>(ptr);
  const int32_t *l = reinterpret_cast<const int32_t *>(list);
  const double *v = reinterpret_cast<const double *>(lma);
  switch (cdim) {
    case 1: return launch_reduce<1>(o, p, l, ntargets, v, nelem, arity, kmask, kahan, s);
    case 2: return launch_reduce<2>(o, p, l, ntargets, v, nelem, arity, kmask, kahan, s);
    case 3: return launch_reduce<3>(o, p, l, ntargets, v, nelem, arity, kmask, kahan, s);
    case 4: return launch_reduce<4>(o, p, l, ntargets, v, nelem, arity, kmask, kahan, s);
    default:
      return set_error(OP2B_ERR_ARG, "op2b_lma_reduce: cdim %d (1 to 4 supported)", cdim);
  }
}

}  // extern "C"
