// Target -> (element, map index) incidence of a Map, built on the GPU.
//
// For every target t of a Map [n][arity], the flat positions p = e*arity + k
// with map[p] == t, in increasing order (so in element order, then map index
// order).  Owner-computes stubs walk this list to evaluate, for one target,
// every contribution the sequential backend would add to it, in the order the
// sequential backend adds them (pyop2/sequential.py:55-72 runs elements in
// order and each element's map indices in order).
//
// Built like the Sparsity's row buckets: count per target, exclusive scan,
// scatter (atomic cursors, order not yet defined), then one warp per target
// sorts its bucket (rank sort in shared memory up to 256 entries, repeated
// warp-minimum selection above that).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>

#include "op2b_internal.h"
#include "op2b_scan.cuh"

namespace op2b {

struct Incidence {
  int32_t ntargets = 0;
  int64_t nentries = 0;
  int32_t *ptr = nullptr, *list = nullptr;
  int32_t max_degree = 0;
};

__global__ void inc_count_kernel(const int32_t *__restrict__ map, int64_t tot, int32_t ntargets,
                                 int32_t *__restrict__ count, int32_t *__restrict__ err) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot;
       i += (int64_t)gridDim.x * blockDim.x) {
    int t = map[i];
    if (t < 0 || t >= ntargets) {
      atomicExch(err, 1);
      continue;
    }
    atomicAdd(&count[t], 1);
  }
}

__global__ void inc_fill_kernel(const int32_t *__restrict__ map, int64_t tot, int32_t ntargets,
                                const int32_t *__restrict__ ptr, int32_t *__restrict__ cursor,
                                int32_t *__restrict__ list) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot;
       i += (int64_t)gridDim.x * blockDim.x) {
    int t = map[i];
    if (t < 0 || t >= ntargets) continue;
    list[ptr[t] + atomicAdd(&cursor[t], 1)] = (int32_t)i;
  }
}

constexpr int kIncWarps = 8;
constexpr int kIncBuf = 256;

__global__ void __launch_bounds__(kIncWarps * 32)
inc_sort_kernel(const int32_t *__restrict__ ptr, int32_t *__restrict__ list, int32_t ntargets,
                int32_t *__restrict__ max_deg) {
  __shared__ int buf[kIncWarps][kIncBuf];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int local_max = 0;
  for (int64_t t = (int64_t)blockIdx.x * kIncWarps + w; t < ntargets;
       t += (int64_t)gridDim.x * kIncWarps) {
    const int p0 = ptr[t], k = ptr[t + 1] - p0;
    local_max = max(local_max, k);
    if (k <= 1) continue;
    if (k <= kIncBuf) {
      for (int i = lane; i < k; i += 32) buf[w][i] = list[p0 + i];
      __syncwarp();
      // entries are distinct flat positions: rank = number of smaller ones
      for (int i = lane; i < k; i += 32) {
        const int v = buf[w][i];
        int rank = 0;
        for (int j = 0; j < k; ++j) rank += buf[w][j] < v;
        list[p0 + rank] = v;
      }
      __syncwarp();
    } else {
      // long bucket: selection of successive minima (in place is unsafe while
      // other lanes read, so select into the sorted prefix one at a time)
      for (int out = 0; out < k; ++out) {
        int mn = INT_MAX, at = -1;
        for (int i = out + lane; i < k; i += 32) {
          int v = list[p0 + i];
          if (v < mn) {
            mn = v;
            at = i;
          }
        }
        for (int o = 16; o > 0; o >>= 1) {
          int omn = __shfl_xor_sync(0xffffffffu, mn, o);
          int oat = __shfl_xor_sync(0xffffffffu, at, o);
          if (omn < mn) {
            mn = omn;
            at = oat;
          }
        }
        if (lane == 0) {
          int tmp = list[p0 + out];
          list[p0 + out] = mn;
          list[p0 + at] = tmp;
        }
        __syncwarp();
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) local_max = max(local_max, __shfl_xor_sync(0xffffffffu, local_max, o));
  if (lane == 0) atomicMax(max_deg, local_max);
}

// ---- first-use order of a Map's targets along an element order.
// Position q = pos * arity + k stands for map row k of element order[pos]
// (order == nullptr: element pos).  first[t] = the smallest q whose target
// is t; a target is listed at the rank of its first use among all first
// uses, and targets no element uses follow in increasing id.
__global__ void fu_first_kernel(const int32_t *__restrict__ map, int arity, int64_t nelem,
                                const int32_t *__restrict__ order, int32_t *__restrict__ first) {
  const int64_t tot = nelem * arity;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < tot;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t pos = q / arity;
    const int k = (int)(q - pos * arity);
    const int64_t e = order ? order[pos] : pos;
    atomicMin(&first[map[e * arity + k]], (int32_t)q);
  }
}

__global__ void fu_flag_kernel(const int32_t *__restrict__ map, int arity, int64_t nelem,
                               const int32_t *__restrict__ order, const int32_t *__restrict__ first,
                               int32_t *__restrict__ flag) {
  const int64_t tot = nelem * arity;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < tot;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t pos = q / arity;
    const int k = (int)(q - pos * arity);
    const int64_t e = order ? order[pos] : pos;
    flag[q] = first[map[e * arity + k]] == (int32_t)q;
  }
}

__global__ void fu_scatter_kernel(const int32_t *__restrict__ map, int arity, int64_t nelem,
                                  const int32_t *__restrict__ order,
                                  const int32_t *__restrict__ first,
                                  const int32_t *__restrict__ rank, int32_t *__restrict__ out) {
  const int64_t tot = nelem * arity;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < tot;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t pos = q / arity;
    const int k = (int)(q - pos * arity);
    const int64_t e = order ? order[pos] : pos;
    const int32_t t = map[e * arity + k];
    if (first[t] == (int32_t)q) out[rank[q]] = t;
  }
}

__global__ void fu_unused_flag_kernel(const int32_t *__restrict__ first, int32_t ntargets,
                                      int32_t *__restrict__ flag) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ntargets;
       t += (int64_t)gridDim.x * blockDim.x)
    flag[t] = first[t] == INT_MAX;
}

__global__ void fu_unused_scatter_kernel(const int32_t *__restrict__ first, int32_t ntargets,
                                         const int32_t *__restrict__ rank,
                                         const int32_t *__restrict__ nused,
                                         int32_t *__restrict__ out) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ntargets;
       t += (int64_t)gridDim.x * blockDim.x)
    if (first[t] == INT_MAX) out[*nused + rank[t]] = (int32_t)t;
}

__global__ void fu_fill_kernel(int32_t *__restrict__ a, int64_t n, int32_t v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    a[i] = v;
}

// ---- row gather and Map renumbering (READ replicas in first-use order)
__global__ void rows_gather_kernel(uint32_t *__restrict__ dst, const uint32_t *__restrict__ src,
                                   const int32_t *__restrict__ index, int64_t n, int words) {
  const int64_t tot = n * words;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < tot;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = q / words;
    const int w = (int)(q - i * words);
    dst[q] = src[(int64_t)index[i] * words + w];
  }
}

__global__ void inverse_kernel(const int32_t *__restrict__ order, int32_t n,
                               int32_t *__restrict__ inv) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    inv[order[i]] = (int32_t)i;
}

__global__ void renumber_kernel(int32_t *__restrict__ dst, const int32_t *__restrict__ map,
                                int64_t n, const int32_t *__restrict__ inv) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x)
    dst[q] = inv[map[q]];
}

}  // namespace op2b

using namespace op2b;

static void incidence_release(Incidence *I, cudaStream_t s) {
  if (!I) return;
  dev_free(I->ptr, s);
  dev_free(I->list, s);
  delete I;
}

extern "C" {

int op2b_incidence_build(uint64_t map, int32_t nelem, int32_t arity, int32_t ntargets,
                         uint64_t stream, uint64_t *out) {
  OP2B_REQUIRE_INIT();
  if (nelem < 0 || arity <= 0 || ntargets < 0)
    return set_error(OP2B_ERR_ARG, "incidence: nelem %d arity %d targets %d", nelem, arity, ntargets);
  const int64_t tot = (int64_t)nelem * arity;
  if (tot > INT_MAX) return set_error(OP2B_ERR_ARG, "incidence: %lld map entries", (long long)tot);
  cudaStream_t s = stream_of(stream);
  Incidence *I = new Incidence();
  I->ntargets = ntargets;
  I->nentries = tot;
  int32_t *cursor = nullptr, *scal = nullptr;
  int rc = dev_alloc((void **)&I->ptr, sizeof(int32_t) * ((size_t)ntargets + 1), s);
  if (!rc) rc = dev_alloc((void **)&I->list, sizeof(int32_t) * std::max<int64_t>(tot, 1), s);
  if (!rc) rc = dev_alloc((void **)&cursor, sizeof(int32_t) * ((size_t)ntargets + 1), s);
  if (!rc) rc = dev_alloc((void **)&scal, sizeof(int32_t) * 4, s);
  auto fail = [&](int code) {
    dev_free(cursor, s);
    dev_free(scal, s);
    incidence_release(I, s);
    return code;
  };
  if (rc) return fail(rc);
  cudaMemsetAsync(I->ptr, 0, sizeof(int32_t) * ((size_t)ntargets + 1), s);
  cudaMemsetAsync(cursor, 0, sizeof(int32_t) * ((size_t)ntargets + 1), s);
  cudaMemsetAsync(scal, 0, sizeof(int32_t) * 4, s);
  const int grid = std::max(1, std::min<int>((int)((tot + 255) / 256), sm_count() * 8));
  const int32_t *m = reinterpret_cast<const int32_t *>(map);
  inc_count_kernel<<<grid, 256, 0, s>>>(m, tot, ntargets, I->ptr, scal + 1);
  rc = device_excl_scan(I->ptr, I->ptr, (int64_t)ntargets + 1, scal, s);
  if (rc) return fail(rc);
  inc_fill_kernel<<<grid, 256, 0, s>>>(m, tot, ntargets, I->ptr, cursor, I->list);
  const int sgrid = std::max(1, std::min(op2b_div_up(ntargets, kIncWarps), sm_count() * 16));
  if (ntargets > 0) inc_sort_kernel<<<sgrid, kIncWarps * 32, 0, s>>>(I->ptr, I->list, ntargets, scal + 2);
  int32_t h[4];
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, scal, sizeof h, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(check_cuda(e, "op2b_incidence_build"));
  if (h[1]) return fail(set_error(OP2B_ERR_MAP, "incidence: a map value lies outside [0, %d)", ntargets));
  I->max_degree = h[2];
  dev_free(cursor, s);
  dev_free(scal, s);
  *out = reinterpret_cast<uint64_t>(I);
  return OP2B_OK;
}

int op2b_incidence_arrays(uint64_t inc, uint64_t *ptr, uint64_t *list, int32_t *max_degree) {
  Incidence *I = reinterpret_cast<Incidence *>(inc);
  if (!I) return set_error(OP2B_ERR_ARG, "null incidence");
  if (ptr) *ptr = reinterpret_cast<uint64_t>(I->ptr);
  if (list) *list = reinterpret_cast<uint64_t>(I->list);
  if (max_degree) *max_degree = I->max_degree;
  return OP2B_OK;
}

int op2b_first_use_order(uint64_t map, int32_t arity, int64_t nelem, uint64_t elem_order,
                         int32_t ntargets, uint64_t target_order, uint64_t stream) {
  OP2B_REQUIRE_INIT();
  if (arity <= 0 || nelem < 0 || ntargets < 0 || (ntargets > 0 && !target_order) ||
      (nelem > 0 && !map))
    return set_error(OP2B_ERR_ARG, "first_use_order: arity %d nelem %lld targets %d", arity,
                     (long long)nelem, ntargets);
  const int64_t tot = nelem * arity;
  if (tot >= INT_MAX) return set_error(OP2B_ERR_ARG, "first_use_order: %lld map entries", (long long)tot);
  if (ntargets == 0) return OP2B_OK;
  cudaStream_t s = stream_of(stream);
  int32_t *first = nullptr, *flag = nullptr, *tflag = nullptr, *scal = nullptr;
  const int32_t *m = reinterpret_cast<const int32_t *>(map);
  const int32_t *ord = reinterpret_cast<const int32_t *>(elem_order);
  int32_t *out = reinterpret_cast<int32_t *>(target_order);
  int rc = dev_alloc((void **)&first, sizeof(int32_t) * (size_t)ntargets, s);
  if (!rc) rc = dev_alloc((void **)&flag, sizeof(int32_t) * (size_t)std::max<int64_t>(tot, 1), s);
  if (!rc) rc = dev_alloc((void **)&tflag, sizeof(int32_t) * (size_t)ntargets, s);
  if (!rc) rc = dev_alloc((void **)&scal, sizeof(int32_t) * 2, s);
  auto done = [&](int code) {
    dev_free(first, s);
    dev_free(flag, s);
    dev_free(tflag, s);
    dev_free(scal, s);
    return code;
  };
  if (rc) return done(rc);
  const int g1 = std::max(1, std::min<int>((int)((tot + 255) / 256), sm_count() * 8));
  const int g2 = std::max(1, std::min<int>((int)((ntargets + 255) / 256), sm_count() * 8));
  fu_fill_kernel<<<g2, 256, 0, s>>>(first, ntargets, INT_MAX);
  if (tot > 0) {
    fu_first_kernel<<<g1, 256, 0, s>>>(m, arity, nelem, ord, first);
    fu_flag_kernel<<<g1, 256, 0, s>>>(m, arity, nelem, ord, first, flag);
  }
  rc = device_excl_scan(flag, flag, tot, scal, s);
  if (rc) return done(rc);
  if (tot > 0) fu_scatter_kernel<<<g1, 256, 0, s>>>(m, arity, nelem, ord, first, flag, out);
  fu_unused_flag_kernel<<<g2, 256, 0, s>>>(first, ntargets, tflag);
  rc = device_excl_scan(tflag, tflag, ntargets, scal + 1, s);
  if (rc) return done(rc);
  fu_unused_scatter_kernel<<<g2, 256, 0, s>>>(first, ntargets, tflag, scal, out);
  return done(check_cuda(cudaGetLastError(), "op2b_first_use_order"));
}

int op2b_rows_gather(uint64_t dst, uint64_t src, uint64_t index, int64_t n, int32_t row_bytes,
                     uint64_t stream) {
  OP2B_REQUIRE_INIT();
  if (n < 0 || row_bytes <= 0 || row_bytes % 4 || (n > 0 && (!dst || !src || !index)))
    return set_error(OP2B_ERR_ARG, "rows_gather: n %lld row_bytes %d", (long long)n, row_bytes);
  if (n == 0) return OP2B_OK;
  const int words = row_bytes / 4;
  const int64_t tot = n * words;
  const int grid = std::max(1, std::min<int>((int)std::min<int64_t>((tot + 255) / 256, INT_MAX),
                                             sm_count() * 8));
  rows_gather_kernel<<<grid, 256, 0, stream_of(stream)>>>(
      reinterpret_cast<uint32_t *>(dst), reinterpret_cast<const uint32_t *>(src),
      reinterpret_cast<const int32_t *>(index), n, words);
  return check_cuda(cudaGetLastError(), "rows_gather_kernel");
}

int op2b_map_renumber(uint64_t dst_map, uint64_t map, int64_t n_entries, uint64_t order,
                      int32_t ntargets, uint64_t stream) {
  OP2B_REQUIRE_INIT();
  if (n_entries < 0 || ntargets < 0 || (n_entries > 0 && (!dst_map || !map || !order)))
    return set_error(OP2B_ERR_ARG, "map_renumber: %lld entries, %d targets", (long long)n_entries,
                     ntargets);
  if (n_entries == 0 || ntargets == 0) return OP2B_OK;
  cudaStream_t s = stream_of(stream);
  int32_t *inv = nullptr;
  int rc = dev_alloc((void **)&inv, sizeof(int32_t) * (size_t)ntargets, s);
  if (rc) return rc;
  const int g1 = std::max(1, std::min<int>((int)((ntargets + 255) / 256), sm_count() * 8));
  const int g2 = std::max(1, std::min<int>((int)std::min<int64_t>((n_entries + 255) / 256, INT_MAX),
                                           sm_count() * 8));
  inverse_kernel<<<g1, 256, 0, s>>>(reinterpret_cast<const int32_t *>(order), ntargets, inv);
  renumber_kernel<<<g2, 256, 0, s>>>(reinterpret_cast<int32_t *>(dst_map),
                                     reinterpret_cast<const int32_t *>(map), n_entries, inv);
  rc = check_cuda(cudaGetLastError(), "renumber_kernel");
  dev_free(inv, s);
  return rc;
}

int op2b_incidence_free(uint64_t inc) {
  OP2B_REQUIRE_INIT();
  incidence_release(reinterpret_cast<Incidence *>(inc), stream_of(0));
  return OP2B_OK;
}

}  // extern "C"
