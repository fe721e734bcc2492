// GPU Sparsity (CSR pattern) construction.
//
// Produces what build_sparsity_pattern_seq (pyop2/sparsity_utils.cxx:5-51)
// produces: for every map pair and element e, every row rmult*rmap[e][i]+r
// receives the columns cmult*cmap[e][d]+c; per-row column sets are sorted and
// duplicate-free; rowptr is their prefix sum and nnz their sizes.
//
// Instead of one std::set per row filled element by element, the rows are
// built in parallel: a counting sort buckets (pair, element) incidences by row
// node, then one warp per row node gathers the column nodes of its incident
// elements and removes duplicates by ranking (small rows, in shared memory) or
// by repeated warp-min selection (rows with many incidences).  Two passes share
// that gather: the first counts, the second writes colidx after the scan.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <vector>

#include "op2b_internal.h"
#include "op2b_scan.cuh"

namespace op2b {

struct Sparsity {
  int32_t rmult = 1, cmult = 1, nrows = 0, ncols = 0, lsize = 0;
  int64_t nz = 0;
  int32_t *rowptr = nullptr, *colidx = nullptr, *nnz = nullptr;
};

struct SpMap {
  const int32_t *rmap, *cmap;
  int32_t rarity, carity, n;
};

constexpr int kSpWarps = 8;
constexpr int kSpBuf = 256;  // keys kept in shared memory per warp

__global__ void sp_count_rows(const SpMap *__restrict__ maps, int nmaps, int nrows,
                              int32_t *__restrict__ count, int32_t *__restrict__ err) {
  for (int m = 0; m < nmaps; ++m) {
    const SpMap M = maps[m];
    const int64_t tot = (int64_t)M.n * M.rarity;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot;
         i += (int64_t)gridDim.x * blockDim.x) {
      int r = M.rmap[i];
      if (r < 0 || r >= nrows) {
        atomicExch(err, 1);
        continue;
      }
      atomicAdd(&count[r], 1);
    }
  }
}

__global__ void sp_fill_rows(const SpMap *__restrict__ maps, int nmaps, int nrows,
                             const int32_t *__restrict__ ptr, int32_t *__restrict__ cursor,
                             int32_t *__restrict__ inc_e, int32_t *__restrict__ inc_m) {
  for (int m = 0; m < nmaps; ++m) {
    const SpMap M = maps[m];
    const int64_t tot = (int64_t)M.n * M.rarity;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot;
         i += (int64_t)gridDim.x * blockDim.x) {
      int r = M.rmap[i];
      if (r < 0 || r >= nrows) continue;
      int pos = ptr[r] + atomicAdd(&cursor[r], 1);
      inc_e[pos] = (int32_t)(i / M.rarity);
      inc_m[pos] = m;
    }
  }
}

// Column node k of row node r's gathered list (incidence-major order).
__device__ __forceinline__ int sp_key(const SpMap *maps, const int32_t *inc_e, const int32_t *inc_m,
                                     int p0, int nmaps, int k, int carity0) {
  if (nmaps == 1) {
    int q = k / carity0, d = k - q * carity0;
    return maps[0].cmap[(int64_t)inc_e[p0 + q] * carity0 + d];
  }
  // General case: walk incidences (their column arities may differ).
  int q = p0;
  for (;;) {
    const SpMap &M = maps[inc_m[q]];
    if (k < M.carity) return M.cmap[(int64_t)inc_e[q] * M.carity + k];
    k -= M.carity;
    ++q;
  }
}

// One warp per row node.  pass 0: nnz of the node's rows; pass 1: colidx.
__global__ void __launch_bounds__(kSpWarps * 32)
sp_rows_kernel(const SpMap *__restrict__ maps, int nmaps, int nrows, int rmult, int cmult,
               const int32_t *__restrict__ ptr, const int32_t *__restrict__ inc_e,
               const int32_t *__restrict__ inc_m, int pass, int32_t *__restrict__ nnz,
               const int32_t *__restrict__ rowptr, int32_t *__restrict__ colidx) {
  __shared__ int buf[kSpWarps][kSpBuf];
  __shared__ unsigned char first[kSpWarps][kSpBuf];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int carity0 = maps[0].carity;
  for (int64_t r = (int64_t)blockIdx.x * kSpWarps + w; r < nrows; r += (int64_t)gridDim.x * kSpWarps) {
    const int p0 = ptr[r], p1 = ptr[r + 1];
    int k = 0;
    if (nmaps == 1) {
      k = (p1 - p0) * carity0;
    } else {
      for (int q = p0 + lane; q < p1; q += 32) k += maps[inc_m[q]].carity;
      for (int o = 16; o > 0; o >>= 1) k += __shfl_xor_sync(0xffffffffu, k, o);
    }
    int u = 0;
    if (k <= kSpBuf) {
      for (int i = lane; i < k; i += 32) buf[w][i] = sp_key(maps, inc_e, inc_m, p0, nmaps, i, carity0);
      __syncwarp();
      for (int i = lane; i < k; i += 32) {
        const int v = buf[w][i];
        bool f = true;
        for (int j = 0; j < i; ++j)
          if (buf[w][j] == v) {
            f = false;
            break;
          }
        first[w][i] = f;
      }
      __syncwarp();
      int cnt = 0;
      for (int i = lane; i < k; i += 32) cnt += first[w][i];
      for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
      u = cnt;
      if (pass == 1) {
        for (int i = lane; i < k; i += 32) {
          if (!first[w][i]) continue;
          const int v = buf[w][i];
          int rank = 0;
          for (int j = 0; j < k; ++j) rank += (first[w][j] && buf[w][j] < v);
          for (int rr = 0; rr < rmult; ++rr) {
            int64_t base = rowptr[r * rmult + rr] + (int64_t)rank * cmult;
            for (int c = 0; c < cmult; ++c) colidx[base + c] = v * cmult + c;
          }
        }
      }
      __syncwarp();
    } else {
      // Many incidences: emit the distinct keys in increasing order by
      // repeated warp-wide minimum above the previous key.
      int prev = -1;
      for (;;) {
        int mn = INT_MAX;
        for (int i = lane; i < k; i += 32) {
          int v = sp_key(maps, inc_e, inc_m, p0, nmaps, i, carity0);
          if (v > prev && v < mn) mn = v;
        }
        for (int o = 16; o > 0; o >>= 1) mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        if (mn == INT_MAX) break;
        if (pass == 1 && lane == 0) {
          for (int rr = 0; rr < rmult; ++rr) {
            int64_t base = rowptr[r * rmult + rr] + (int64_t)u * cmult;
            for (int c = 0; c < cmult; ++c) colidx[base + c] = mn * cmult + c;
          }
        }
        ++u;
        prev = mn;
      }
    }
    if (pass == 0 && lane < rmult) {
      for (int rr = lane; rr < rmult; rr += 32) nnz[r * rmult + rr] = u * cmult;
    }
  }
}

}  // namespace op2b

using namespace op2b;

static void sparsity_release(Sparsity *sp, cudaStream_t s) {
  if (!sp) return;
  dev_free(sp->rowptr, s);
  dev_free(sp->colidx, s);
  dev_free(sp->nnz, s);
  delete sp;
}

extern "C" {

int op2b_sparsity_build(int32_t rmult, int32_t cmult, int32_t nrows, int32_t ncols, int32_t nmaps,
                        const uint64_t *rmaps, const int32_t *rarity, const uint64_t *cmaps,
                        const int32_t *carity, const int32_t *iterset_size, uint64_t stream,
                        uint64_t *out) {
  OP2B_REQUIRE_INIT();
  if (rmult <= 0 || cmult <= 0 || nrows < 0 || nmaps <= 0)
    return set_error(OP2B_ERR_ARG, "sparsity: rmult %d cmult %d nrows %d nmaps %d", rmult, cmult,
                     nrows, nmaps);
  if ((int64_t)nrows * rmult > INT_MAX - 1)
    return set_error(OP2B_ERR_ARG, "sparsity: %lld rows exceed int32", (long long)nrows * rmult);
  cudaStream_t s = stream_of(stream);
  std::vector<SpMap> h(nmaps);
  for (int m = 0; m < nmaps; ++m) {
    h[m].rmap = reinterpret_cast<const int32_t *>(rmaps[m]);
    h[m].cmap = reinterpret_cast<const int32_t *>(cmaps[m]);
    h[m].rarity = rarity[m];
    h[m].carity = carity[m];
    h[m].n = iterset_size[m];
    if (h[m].rarity <= 0 || h[m].carity <= 0 || h[m].n < 0)
      return set_error(OP2B_ERR_ARG, "sparsity: map pair %d has arity %d/%d size %d", m,
                       h[m].rarity, h[m].carity, h[m].n);
  }
  Sparsity *sp = new Sparsity();
  sp->rmult = rmult;
  sp->cmult = cmult;
  sp->nrows = nrows;
  sp->ncols = ncols;
  sp->lsize = nrows * rmult;
  std::vector<void *> temps;
  auto fail = [&](int rc) {
    for (void *t : temps) dev_free(t, s);
    sparsity_release(sp, s);
    return rc;
  };
#define SP_TRY(call)            \
  do {                          \
    int _rc = (call);           \
    if (_rc) return fail(_rc);  \
  } while (0)
#define SP_CUDA(call) SP_TRY(check_cuda((call), #call))

  int64_t ninc = 0;
  for (auto &M : h) ninc += (int64_t)M.n * M.rarity;
  if (ninc > INT_MAX) return fail(set_error(OP2B_ERR_ARG, "sparsity: %lld incidences", (long long)ninc));
  SpMap *d_maps = nullptr;
  int32_t *ptr = nullptr, *cursor = nullptr, *inc_e = nullptr, *inc_m = nullptr, *d_scal = nullptr;
  SP_TRY(dev_alloc((void **)&d_maps, sizeof(SpMap) * nmaps, s));
  temps.push_back(d_maps);
  SP_TRY(dev_alloc((void **)&ptr, sizeof(int32_t) * ((size_t)nrows + 1), s));
  temps.push_back(ptr);
  SP_TRY(dev_alloc((void **)&cursor, sizeof(int32_t) * ((size_t)nrows + 1), s));
  temps.push_back(cursor);
  SP_TRY(dev_alloc((void **)&inc_e, sizeof(int32_t) * std::max<int64_t>(ninc, 1), s));
  temps.push_back(inc_e);
  SP_TRY(dev_alloc((void **)&inc_m, sizeof(int32_t) * std::max<int64_t>(ninc, 1), s));
  temps.push_back(inc_m);
  SP_TRY(dev_alloc((void **)&d_scal, sizeof(int32_t) * 4, s));
  temps.push_back(d_scal);
  SP_CUDA(cudaMemcpyAsync(d_maps, h.data(), sizeof(SpMap) * nmaps, cudaMemcpyHostToDevice, s));
  SP_CUDA(cudaMemsetAsync(ptr, 0, sizeof(int32_t) * ((size_t)nrows + 1), s));
  SP_CUDA(cudaMemsetAsync(cursor, 0, sizeof(int32_t) * ((size_t)nrows + 1), s));
  SP_CUDA(cudaMemsetAsync(d_scal, 0, sizeof(int32_t) * 4, s));
  const int grid = std::max(1, std::min<int>((int)((ninc + 255) / 256), sm_count() * 8));
  sp_count_rows<<<grid, 256, 0, s>>>(d_maps, nmaps, nrows, ptr, d_scal + 2);
  SP_TRY(device_excl_scan(ptr, ptr, (int64_t)nrows + 1, d_scal, s));
  sp_fill_rows<<<grid, 256, 0, s>>>(d_maps, nmaps, nrows, ptr, cursor, inc_e, inc_m);
  SP_CUDA(cudaGetLastError());

  const int lsize = sp->lsize;
  SP_TRY(dev_alloc((void **)&sp->nnz, sizeof(int32_t) * std::max(lsize, 1), s));
  SP_TRY(dev_alloc((void **)&sp->rowptr, sizeof(int32_t) * ((size_t)lsize + 1), s));
  SP_CUDA(cudaMemsetAsync(sp->nnz, 0, sizeof(int32_t) * std::max(lsize, 1), s));
  const int rgrid = std::max(1, std::min<int>(op2b_div_up(nrows, kSpWarps), sm_count() * 16));
  if (nrows > 0)
    sp_rows_kernel<<<rgrid, kSpWarps * 32, 0, s>>>(d_maps, nmaps, nrows, rmult, cmult, ptr, inc_e,
                                                  inc_m, 0, sp->nnz, nullptr, nullptr);
  SP_CUDA(cudaGetLastError());
  SP_CUDA(cudaMemcpyAsync(sp->rowptr, sp->nnz, sizeof(int32_t) * lsize, cudaMemcpyDeviceToDevice, s));
  SP_CUDA(cudaMemsetAsync(sp->rowptr + lsize, 0, sizeof(int32_t), s));
  SP_TRY(device_excl_scan(sp->rowptr, sp->rowptr, (int64_t)lsize + 1, d_scal + 1, s));
  int32_t h_scal[4] = {0, 0, 0, 0};
  SP_CUDA(cudaMemcpyAsync(h_scal, d_scal, sizeof(h_scal), cudaMemcpyDeviceToHost, s));
  SP_CUDA(cudaStreamSynchronize(s));
  if (h_scal[2]) return fail(set_error(OP2B_ERR_MAP, "sparsity: a row map value lies outside [0, %d)", nrows));
  sp->nz = h_scal[1];
  SP_TRY(dev_alloc((void **)&sp->colidx, sizeof(int32_t) * std::max<int64_t>(sp->nz, 1), s));
  if (nrows > 0)
    sp_rows_kernel<<<rgrid, kSpWarps * 32, 0, s>>>(d_maps, nmaps, nrows, rmult, cmult, ptr, inc_e,
                                                  inc_m, 1, sp->nnz, sp->rowptr, sp->colidx);
  SP_CUDA(cudaGetLastError());
  SP_CUDA(cudaStreamSynchronize(s));
  for (void *t : temps) dev_free(t, s);
  *out = reinterpret_cast<uint64_t>(sp);
  return OP2B_OK;
#undef SP_TRY
#undef SP_CUDA
}

int op2b_sparsity_info(uint64_t sparsity, int32_t *lsize, int64_t *nz) {
  Sparsity *sp = reinterpret_cast<Sparsity *>(sparsity);
  if (!sp) return set_error(OP2B_ERR_ARG, "null sparsity");
  if (lsize) *lsize = sp->lsize;
  if (nz) *nz = sp->nz;
  return OP2B_OK;
}

int op2b_sparsity_arrays(uint64_t sparsity, uint64_t *rowptr, uint64_t *colidx, uint64_t *nnz) {
  Sparsity *sp = reinterpret_cast<Sparsity *>(sparsity);
  if (!sp) return set_error(OP2B_ERR_ARG, "null sparsity");
  if (rowptr) *rowptr = reinterpret_cast<uint64_t>(sp->rowptr);
  if (colidx) *colidx = reinterpret_cast<uint64_t>(sp->colidx);
  if (nnz) *nnz = reinterpret_cast<uint64_t>(sp->nnz);
  return OP2B_OK;
}

int op2b_sparsity_free(uint64_t sparsity) {
  OP2B_REQUIRE_INIT();
  sparsity_release(reinterpret_cast<Sparsity *>(sparsity), stream_of(0));
  return OP2B_OK;
}

}  // extern "C"
