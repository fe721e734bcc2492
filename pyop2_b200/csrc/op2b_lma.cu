// Two-phase (local-matrix) INC: deterministic accumulation in the sequential
// backend's order.
//
// Phase 1 is a generated par_loop stub that writes every element's INC
// contribution to a local-contribution array instead of adding it: for the
// contribution of element e at map position k (a Dat row, cdim values) or at
// local Mat entry k = r * ca + c (one value), in tiles of 32 elements,
//     lma[((((e / 32) * K + k) * 32) + e % 32) * cdim + comp].
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
// positions; its list entries are then converted to contribution-array
// indices, so the Mat reduction needs no index arithmetic.
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
                                  const double *__restrict__ lma, int arity, uint64_t kmask,
                                  bool from_zero) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntargets;
       t += (int64_t)gridDim.x * blockDim.x) {
    double acc[CDIM], cmp[CDIM];
#pragma unroll
    for (int c = 0; c < CDIM; ++c) {
      acc[c] = from_zero ? 0.0 : out[t * CDIM + c];
      cmp[c] = 0.0;
    }
    const int q1 = ptr[t + 1];
    for (int q = ptr[t]; q < q1; ++q) {
      // positions are non-negative int32: 32-bit unsigned division
      const unsigned pos = static_cast<unsigned>(__ldg(list + q));
      const unsigned e = pos / static_cast<unsigned>(arity);
      const unsigned k = pos - e * static_cast<unsigned>(arity);
      if (!((kmask >> k) & 1ull)) continue;
      // tiles of 32 elements, position-major inside a tile (op2b_lma_index)
      const int64_t row = ((((int64_t)(e >> 5)) * arity + k) << 5) + (e & 31u);
      const double *src = lma + row * CDIM;
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

// Mat incidence lists hold contribution-array indices (op2b_mat_incidence_build
// converts the positions once), so the Mat reduction reads them directly;
// two contributions are fetched together to overlap their latencies (most
// CSR slots have one or two).  The additions stay in list (element) order.
template <bool KAHAN>
__global__ void lma_reduce_mat_kernel(double *__restrict__ out, const int32_t *__restrict__ ptr,
                                      const int32_t *__restrict__ list, int32_t ntargets,
                                      const double *__restrict__ lma, bool from_zero) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntargets;
       t += (int64_t)gridDim.x * blockDim.x) {
    double acc = from_zero ? 0.0 : out[t], cmp = 0.0;
    int q = ptr[t];
    const int q1 = ptr[t + 1];
    auto add = [&](double v) {
      if (KAHAN) {
        const double y = v - cmp;
        const double s = acc + y;
        cmp = (s - acc) - y;
        acc = s;
      } else {
        acc += v;
      }
    };
    for (; q + 1 < q1; q += 2) {
      const int i0 = __ldg(list + q), i1 = __ldg(list + q + 1);
      const double v0 = __ldg(lma + i0), v1 = __ldg(lma + i1);
      add(v0);
      add(v1);
    }
    if (q < q1) add(__ldg(lma + __ldg(list + q)));
    out[t] = acc;
  }
}

// positions e * K + k -> tiled contribution-array indices, in place
__global__ void lma_index_kernel(int32_t *__restrict__ list, int64_t n, int K) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const unsigned pos = static_cast<unsigned>(list[i]);
    const unsigned e = pos / static_cast<unsigned>(K);
    const unsigned k = pos - e * static_cast<unsigned>(K);
    list[i] = static_cast<int32_t>((((e >> 5) * K + k) << 5) + (e & 31u));
  }
}

template <int CDIM>
static int launch_reduce(double *out, const int32_t *ptr, const int32_t *list, int32_t ntargets,
                         const double *lma, int arity, uint64_t kmask, bool kahan, bool from_zero,
                         cudaStream_t s) {
  const int grid = std::max(1, std::min(op2b_div_up(ntargets, 256), sm_count() * 16));
  if (kahan)
    lma_reduce_kernel<CDIM, true><<<grid, 256, 0, s>>>(out, ptr, list, ntargets, lma, arity, kmask,
                                                       from_zero);
  else
    lma_reduce_kernel<CDIM, false><<<grid, 256, 0, s>>>(out, ptr, list, ntargets, lma, arity,
                                                        kmask, from_zero);
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
  // the tiled indices run up to ceil(nelem / 32) * 32 * ra * ca
  if (((int64_t)nelem + 31) / 32 * 32 * ra * ca > INT_MAX)
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
  if (!rc && tot > 0) {
    uint64_t p = 0, l = 0;
    int32_t md = 0;
    rc = op2b_incidence_arrays(*incidence, &p, &l, &md);
    if (!rc) {
      const int grid = static_cast<int>(
          std::max<int64_t>(1, std::min<int64_t>((tot + 255) / 256, (int64_t)sm_count() * 16)));
      lma_index_kernel<<<grid, 256, 0, s>>>(reinterpret_cast<int32_t *>(l), tot, ra * ca);
      rc = check_cuda(cudaGetLastError(), "lma_index_kernel");
    }
    if (rc) {
      op2b_incidence_free(*incidence);
      *incidence = 0;
    }
  }
  return rc;
}

int op2b_lma_reduce(uint64_t out, int32_t cdim, uint64_t ptr, uint64_t list, int32_t ntargets,
                    uint64_t lma, int64_t nelem, int32_t arity, uint64_t kmask, int32_t flags,
                    uint64_t stream) {
  OP2B_REQUIRE_INIT();
  const bool kahan = flags & OP2B_LMA_KAHAN, from_zero = flags & OP2B_LMA_FROM_ZERO;
  if (ntargets < 0 || nelem < 0)
    return set_error(OP2B_ERR_ARG, "op2b_lma_reduce: bad arguments");
  if (ntargets == 0) return OP2B_OK;
  cudaStream_t s = stream_of(stream);
  double *o = reinterpret_cast<double *>(out);
  const int32_t *p = reinterpret_cast<const int32_t *>(ptr);
  const int32_t *l = reinterpret_cast<const int32_t *>(list);
  const double *v = reinterpret_cast<const double *>(lma);
  if (flags & OP2B_LMA_MAT_INDEX) {
    // a Mat incidence (op2b_mat_incidence_build): list entries are indices
    if (cdim != 1)
      return set_error(OP2B_ERR_ARG, "op2b_lma_reduce: Mat reduction with cdim %d", cdim);
    const int grid = std::max(1, std::min(op2b_div_up(ntargets, 256), sm_count() * 16));
    if (kahan)
      lma_reduce_mat_kernel<true><<<grid, 256, 0, s>>>(o, p, l, ntargets, v, from_zero);
    else
      lma_reduce_mat_kernel<false><<<grid, 256, 0, s>>>(o, p, l, ntargets, v, from_zero);
    return check_cuda(cudaGetLastError(), "lma_reduce_mat_kernel");
  }
  if (arity <= 0 || arity > 64) return set_error(OP2B_ERR_ARG, "op2b_lma_reduce: arity %d", arity);
  switch (cdim) {
    case 1: return launch_reduce<1>(o, p, l, ntargets, v, arity, kmask, kahan, from_zero, s);
    case 2: return launch_reduce<2>(o, p, l, ntargets, v, arity, kmask, kahan, from_zero, s);
    case 3: return launch_reduce<3>(o, p, l, ntargets, v, arity, kmask, kahan, from_zero, s);
    case 4: return launch_reduce<4>(o, p, l, ntargets, v, arity, kmask, kahan, from_zero, s);
    default:
      return set_error(OP2B_ERR_ARG, "op2b_lma_reduce: cdim %d (1 to 4 supported)", cdim);
  }
}

}  // extern "C"
