// GPU plan construction: block partition, staging maps and conflict colouring.
//
// Restates the outputs of pyop2/plan.pyx (Plan.__cinit__ :93-105):
//  * partition (:107-110): contiguous blocks of part_size elements;
//  * staging (:112-212): per block and unique (Dat, Map) pair the sorted unique
//    map values (ind_map, what numpy.unique returns) and, per element and map
//    index, the position of its value in that list (loc_map, int16), with
//    ind_sizes / ind_offs / nindirect / nshared in the reference layout;
//  * thread colouring (:282-324): per block, the reference's greedy algorithm
//    in element order with 32-colour bit masks, run by one thread per block on
//    block-local target ids, so thrcol/nthrcol equal the reference's;
//  * block colouring (:326-376): a Jones-Plassmann colouring with hashed
//    priorities over the node->block incidence (valid, parallel; the colours
//    differ from the reference's sequential greedy order).
// The layouts of the arrays follow plan.pyx so the oracle can compare them.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <vector>

#include "op2b_internal.h"
#include "op2b_block_sort.cuh"
#include "op2b_scan.cuh"

namespace op2b {

struct Plan {
  int32_t set_size = 0, part_size = 0, nblocks = 0, ncolors = 0, nshared = 0, ninds = 0;
  int32_t max_nthrcol = 0, loc_rows = 0;
  int64_t ind_map_len = 0;
  int32_t *nelems = nullptr, *offset = nullptr, *ind_map = nullptr, *ind_sizes = nullptr;
  int32_t *ind_offs = nullptr, *nindirect = nullptr, *thrcol = nullptr, *nthrcol = nullptr;
  int32_t *blkmap = nullptr, *ncolblk = nullptr, *blkcol = nullptr;
  int16_t *loc_map = nullptr;
  std::vector<int32_t> h_ncolblk;
  int64_t counts[12] = {0};
};

constexpr int kPlanThreads = 256;
constexpr int kMaxBlockKeys = 16384;   // part_size * map indices per pair/group
constexpr int kMaxBlockColors = 2048;  // Jones-Plassmann colour mask capacity

static int next_pow2(int v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}

struct StageArgs {
  const int32_t *map;
  int32_t arity, nidx, idx_off, loc_row;
  int64_t cap;     // temp capacity per block = part_size * nidx
  int32_t *tmp;    // [nblocks][cap] uniques
};

// grid (nblocks, nstage): sort-unique of the block's map values for one pair.
__global__ void plan_stage_kernel(const StageArgs *__restrict__ pairs, const int32_t *__restrict__ idx_all,
                                  int nstage, int set_size, int part_size, int npow2,
                                  int32_t *__restrict__ ind_sizes, int16_t *__restrict__ loc_map) {
  extern __shared__ int smem_i[];
  const int blk = blockIdx.x, s = blockIdx.y;
  const StageArgs p = pairs[s];
  const int start = blk * part_size;
  const int nelem = min(part_size, set_size - start);
  const int nkeys = nelem * p.nidx;
  int *a = smem_i;
  int *u = smem_i + npow2;
  const int *idx = idx_all + p.idx_off;
  const int n = next_pow2_dev(nkeys);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    int v = INT_MAX;
    if (i < nkeys) {
      int e = i / p.nidx, j = i - e * p.nidx;
      v = p.map[(int64_t)(start + e) * p.arity + idx[j]];
    }
    a[i] = v;
  }
  __syncthreads();
  block_bitonic_sort(a, n);
  int nu = block_unique(a, nkeys, n, u);
  for (int i = threadIdx.x; i < nu; i += blockDim.x) p.tmp[(int64_t)blk * p.cap + i] = u[i];
  for (int i = threadIdx.x; i < nkeys; i += blockDim.x) {
    int e = i / p.nidx, j = i - e * p.nidx;
    int v = p.map[(int64_t)(start + e) * p.arity + idx[j]];
    loc_map[(int64_t)(p.loc_row + j) * set_size + start + e] = (int16_t)lower_bound(u, nu, v);
  }
  if (threadIdx.x == 0) ind_sizes[blk * nstage + s] = nu;
}

__global__ void plan_stage_compact_kernel(const StageArgs *__restrict__ pairs, int nstage,
                                          const int64_t *__restrict__ ind_base,
                                          const int32_t *__restrict__ ind_sizes,
                                          const int32_t *__restrict__ ind_offs,
                                          int32_t *__restrict__ ind_map) {
  const int blk = blockIdx.x, s = blockIdx.y;
  const StageArgs p = pairs[s];
  const int nu = ind_sizes[blk * nstage + s];
  const int64_t dst = ind_base[s] + ind_offs[blk * nstage + s];
  for (int i = threadIdx.x; i < nu; i += blockDim.x)
    ind_map[dst + i] = p.tmp[(int64_t)blk * p.cap + i];
}

struct RaceEntry {
  const int32_t *map;
  int32_t arity, idx;
};

struct RaceGroup {
  int32_t first, nent, size;
  int64_t cap;      // part_size * nent
  int32_t *tmp;     // [nblocks][cap] unique targets
  int32_t *node_ptr, *node_blk;  // node -> incident blocks (filled later)
};

// One CTA per block: unique targets per race group (for block colouring) and,
// if requested, the reference's greedy thread colouring in element order.
__global__ void plan_race_kernel(const RaceGroup *__restrict__ groups, const RaceEntry *__restrict__ ents,
                                 int nrace, int nent_total, int set_size, int part_size, int npow2,
                                 int thread_coloring, int32_t *__restrict__ race_cnt,
                                 int32_t *__restrict__ thrcol, int32_t *__restrict__ nthrcol) {
  extern __shared__ int smem_i[];
  const int blk = blockIdx.x;
  const int start = blk * part_size;
  const int nelem = min(part_size, set_size - start);
  int *a = smem_i;                                  // npow2
  int *u = a + npow2;                               // npow2
  uint32_t *masks = (uint32_t *)(u + npow2);        // part_size * nent_total
  int16_t *lid = (int16_t *)(masks + (int64_t)part_size * nent_total);  // nelem * nent_total
  int *col = (int *)(lid + (((int64_t)part_size * nent_total + 1) & ~1LL));  // part_size
  __shared__ int s_remaining;

  int mbase = 0;
  for (int g = 0; g < nrace; ++g) {
    const RaceGroup G = groups[g];
    const int nkeys = nelem * G.nent;
    const int n = next_pow2_dev(nkeys);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      int v = INT_MAX;
      if (i < nkeys) {
        int e = i / G.nent, k = i - e * G.nent;
        const RaceEntry E = ents[G.first + k];
        v = E.map[(int64_t)(start + e) * E.arity + E.idx];
      }
      a[i] = v;
    }
    __syncthreads();
    block_bitonic_sort(a, n);
    int nu = block_unique(a, nkeys, n, u);
    for (int i = threadIdx.x; i < nu; i += blockDim.x) G.tmp[(int64_t)blk * G.cap + i] = u[i];
    for (int i = threadIdx.x; i < nkeys; i += blockDim.x) {
      int e = i / G.nent, k = i - e * G.nent;
      const RaceEntry E = ents[G.first + k];
      int v = E.map[(int64_t)(start + e) * E.arity + E.idx];
      lid[e * nent_total + G.first + k] = (int16_t)(mbase + lower_bound(u, nu, v));
    }
    if (threadIdx.x == 0) race_cnt[blk * nrace + g] = nu;
    mbase += nu;
    __syncthreads();
  }
  if (!thread_coloring) return;

  for (int e = threadIdx.x; e < nelem; e += blockDim.x) col[e] = -1;
  if (threadIdx.x == 0) s_remaining = nelem;
  __syncthreads();
  int base = 0;
  while (s_remaining > 0) {
    for (int i = threadIdx.x; i < mbase; i += blockDim.x) masks[i] = 0u;
    __syncthreads();
    if (threadIdx.x == 0) {
      int rem = 0;
      for (int e = 0; e < nelem; ++e) {
        if (col[e] != -1) continue;
        uint32_t m = 0u;
        for (int k = 0; k < nent_total; ++k) m |= masks[lid[e * nent_total + k]];
        if (m == 0xffffffffu) {
          ++rem;
          continue;
        }
        int c = __ffs(~m) - 1;
        col[e] = base + c;
        uint32_t bit = 1u << c;
        for (int k = 0; k < nent_total; ++k) masks[lid[e * nent_total + k]] |= bit;
      }
      s_remaining = rem;
    }
    base += 32;
    __syncthreads();
  }
  int mx = -1;
  for (int e = threadIdx.x; e < nelem; e += blockDim.x) {
    thrcol[start + e] = col[e];
    mx = max(mx, col[e]);
  }
  // block max of mx
  for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  __shared__ int wmax[32];
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    int m = -1;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = max(m, wmax[w]);
    nthrcol[blk] = m + 1;
  }
}

// node_count[t] += 1 for every (block, unique target t) of a group.
__global__ void incidence_count_kernel(RaceGroup G, int g, int nrace, const int32_t *race_cnt,
                                       int32_t *node_count) {
  const int blk = blockIdx.x;
  const int nu = race_cnt[blk * nrace + g];
  for (int i = threadIdx.x; i < nu; i += blockDim.x)
    atomicAdd(&node_count[G.tmp[(int64_t)blk * G.cap + i]], 1);
}

__global__ void incidence_fill_kernel(RaceGroup G, int g, int nrace, const int32_t *race_cnt,
                                      int32_t *cursor) {
  const int blk = blockIdx.x;
  const int nu = race_cnt[blk * nrace + g];
  for (int i = threadIdx.x; i < nu; i += blockDim.x) {
    int t = G.tmp[(int64_t)blk * G.cap + i];
    int pos = G.node_ptr[t] + atomicAdd(&cursor[t], 1);
    G.node_blk[pos] = blk;
  }
}

__device__ __forceinline__ uint32_t block_priority(uint32_t b) {
  // 32-bit integer hash (xorshift-multiply); ties broken by block index.
  b ^= b >> 16;
  b *= 0x7feb352dU;
  b ^= b >> 15;
  b *= 0x846ca68bU;
  b ^= b >> 16;
  return b;
}

__device__ __forceinline__ bool beats(uint32_t b1, uint32_t b2) {
  uint32_t p1 = block_priority(b1), p2 = block_priority(b2);
  return p1 > p2 || (p1 == p2 && b1 < b2);
}

// One Jones-Plassmann round: an uncoloured block whose priority beats every
// uncoloured neighbour takes the smallest colour no neighbour holds.
__global__ void jp_round_kernel(const RaceGroup *__restrict__ groups, int nrace,
                                const int32_t *__restrict__ race_cnt, int32_t *blkcol,
                                int32_t *remaining, int32_t *overflow) {
  __shared__ uint32_t used[kMaxBlockColors / 32];
  __shared__ int s_wait;
  const int b = blockIdx.x;
  if (blkcol[b] >= 0) return;
  for (int i = threadIdx.x; i < kMaxBlockColors / 32; i += blockDim.x) used[i] = 0u;
  if (threadIdx.x == 0) s_wait = 0;
  __syncthreads();
  for (int g = 0; g < nrace; ++g) {
    const RaceGroup G = groups[g];
    const int nu = race_cnt[b * nrace + g];
    for (int i = threadIdx.x; i < nu; i += blockDim.x) {
      int t = G.tmp[(int64_t)b * G.cap + i];
      for (int q = G.node_ptr[t]; q < G.node_ptr[t + 1]; ++q) {
        int nb = G.node_blk[q];
        if (nb == b) continue;
        int c = *((volatile int32_t *)&blkcol[nb]);
        if (c < 0) {
          if (beats((uint32_t)nb, (uint32_t)b)) s_wait = 1;
        } else if (c < kMaxBlockColors) {
          atomicOr(&used[c >> 5], 1u << (c & 31));
        }
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (s_wait) {
      atomicAdd(remaining, 1);
    } else {
      int c = -1;
      for (int w = 0; w < kMaxBlockColors / 32; ++w) {
        if (used[w] != 0xffffffffu) {
          c = w * 32 + __ffs(~used[w]) - 1;
          break;
        }
      }
      if (c < 0) {
        atomicExch(overflow, 1);
        c = kMaxBlockColors;  // reported as an error by the host
      }
      blkcol[b] = c;
    }
  }
}

}  // namespace op2b

using namespace op2b;

static void plan_release(Plan *p, cudaStream_t s) {
  if (!p) return;
  int32_t *arrs[] = {p->nelems, p->offset, p->ind_map, p->ind_sizes, p->ind_offs, p->nindirect,
                     p->thrcol, p->nthrcol, p->blkmap, p->ncolblk, p->blkcol};
  for (int32_t *a : arrs) dev_free(a, s);
  dev_free(p->loc_map, s);
  delete p;
}

#define PLAN_TRY(call)               \
  do {                               \
    int _rc = (call);                \
    if (_rc) {                       \
      for (void *t : temps) dev_free(t, s); \
      plan_release(P, s);            \
      return _rc;                    \
    }                                \
  } while (0)

#define PLAN_CUDA(call) PLAN_TRY(check_cuda((call), #call))

extern "C" {

int op2b_plan_build(int32_t set_size, int32_t part_size, int32_t nstage, const uint64_t *stage_map,
                    const int32_t *stage_arity, const int32_t *stage_nidx,
                    const int32_t *stage_idx_off, const int32_t *stage_idx,
                    const int32_t *stage_bytes, int32_t nrace, const int32_t *race_nent,
                    const int32_t *race_size, const uint64_t *race_map, const int32_t *race_arity,
                    const int32_t *race_idx, int32_t flags, uint64_t stream, uint64_t *plan_out) {
  OP2B_REQUIRE_INIT();
  if (set_size < 0 || part_size <= 0)
    return set_error(OP2B_ERR_ARG, "plan: set_size %d part_size %d", set_size, part_size);
  if (nrace > 64) return set_error(OP2B_ERR_ARG, "plan: more than 64 race groups");
  cudaStream_t s = stream_of(stream);
  std::vector<void *> temps;
  Plan *P = new Plan();
  P->set_size = set_size;
  P->part_size = part_size;
  const int nblocks = set_size ? op2b_div_up(set_size, part_size) : 0;
  P->nblocks = nblocks;
  const bool staging = flags & OP2B_PLAN_STAGING;
  const bool tc = flags & OP2B_PLAN_THREAD_COLORING;

  // ---- partition (plan.pyx:107-110) and offsets (:199-204)
  std::vector<int32_t> h_nelems(nblocks), h_offset(nblocks);
  for (int b = 0; b < nblocks; ++b) {
    h_nelems[b] = std::min(part_size, set_size - b * part_size);
    h_offset[b] = b * part_size;
  }
  auto alloc32 = [&](int32_t **p, int64_t n) { return dev_alloc((void **)p, sizeof(int32_t) * std::max<int64_t>(n, 1), s); };
  PLAN_TRY(alloc32(&P->nelems, nblocks));
  PLAN_TRY(alloc32(&P->offset, nblocks));
  PLAN_CUDA(cudaMemcpyAsync(P->nelems, h_nelems.data(), sizeof(int32_t) * nblocks, cudaMemcpyHostToDevice, s));
  PLAN_CUDA(cudaMemcpyAsync(P->offset, h_offset.data(), sizeof(int32_t) * nblocks, cudaMemcpyHostToDevice, s));
  P->counts[0] = nblocks;
  P->counts[1] = nblocks;

  // ---- staging (plan.pyx:112-212)
  P->ninds = staging ? nstage : 0;
  int loc_rows = 0;
  std::vector<int64_t> h_ind_base(std::max(nstage, 1), 0);
  if (staging && nstage > 0 && nblocks > 0) {
    std::vector<StageArgs> h_pairs(nstage);
    int64_t ind_len = 0;
    int max_keys = 0;
    for (int q = 0; q < nstage; ++q) {
      StageArgs &p = h_pairs[q];
      p.map = reinterpret_cast<const int32_t *>(stage_map[q]);
      p.arity = stage_arity[q];
      p.nidx = stage_nidx[q];
      p.idx_off = stage_idx_off[q];
      p.loc_row = loc_rows;
      p.cap = (int64_t)part_size * p.nidx;
      for (int j = 0; j < p.nidx; ++j) {
        int ix = stage_idx[p.idx_off + j];
        if (ix < 0 || ix >= p.arity) {
          plan_release(P, s);
          return set_error(OP2B_ERR_ARG, "plan: map index %d outside arity %d", ix, p.arity);
        }
      }
      loc_rows += p.nidx;
      h_ind_base[q] = ind_len;
      ind_len += (int64_t)p.nidx * set_size;
      max_keys = std::max<int>(max_keys, part_size * p.nidx);
      PLAN_TRY(alloc32(&p.tmp, (int64_t)nblocks * p.cap));
      temps.push_back(p.tmp);
    }
    if (max_keys > kMaxBlockKeys || max_keys > 32767) {
      for (void *t : temps) dev_free(t, s);
      plan_release(P, s);
      return set_error(OP2B_ERR_ARG,
                       "plan: part_size %d x map indices gives %d staged keys per block "
                       "(limit %d, int16 loc_map)", part_size, max_keys, std::min(kMaxBlockKeys, 32767));
    }
    P->ind_map_len = ind_len;
    P->loc_rows = loc_rows;
    PLAN_TRY(alloc32(&P->ind_map, ind_len));
    PLAN_CUDA(cudaMemsetAsync(P->ind_map, 0xff, sizeof(int32_t) * std::max<int64_t>(ind_len, 1), s));
    PLAN_TRY(dev_alloc((void **)&P->loc_map, sizeof(int16_t) * std::max<int64_t>((int64_t)loc_rows * set_size, 1), s));
    PLAN_TRY(alloc32(&P->ind_sizes, (int64_t)nblocks * nstage));
    PLAN_TRY(alloc32(&P->ind_offs, (int64_t)nblocks * nstage));
    PLAN_TRY(alloc32(&P->nindirect, nstage));
    StageArgs *d_pairs = nullptr;
    int32_t *d_idx = nullptr;
    int64_t *d_base = nullptr;
    int nidx_total = stage_idx_off[nstage - 1] + stage_nidx[nstage - 1];
    PLAN_TRY(dev_alloc((void **)&d_pairs, sizeof(StageArgs) * nstage, s));
    temps.push_back(d_pairs);
    PLAN_TRY(dev_alloc((void **)&d_idx, sizeof(int32_t) * std::max(nidx_total, 1), s));
    temps.push_back(d_idx);
    PLAN_TRY(dev_alloc((void **)&d_base, sizeof(int64_t) * nstage, s));
    temps.push_back(d_base);
    PLAN_CUDA(cudaMemcpyAsync(d_pairs, h_pairs.data(), sizeof(StageArgs) * nstage, cudaMemcpyHostToDevice, s));
    PLAN_CUDA(cudaMemcpyAsync(d_idx, stage_idx, sizeof(int32_t) * nidx_total, cudaMemcpyHostToDevice, s));
    PLAN_CUDA(cudaMemcpyAsync(d_base, h_ind_base.data(), sizeof(int64_t) * nstage, cudaMemcpyHostToDevice, s));
    const int npow2 = next_pow2(max_keys);
    const int smem = 2 * npow2 * (int)sizeof(int);
    PLAN_CUDA(cudaFuncSetAttribute(plan_stage_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    plan_stage_kernel<<<dim3(nblocks, nstage), kPlanThreads, smem, s>>>(
        d_pairs, d_idx, nstage, set_size, part_size, npow2, P->ind_sizes, P->loc_map);
    PLAN_CUDA(cudaGetLastError());
    // ind_offs / nindirect / nshared from the per-block sizes (small, host).
    std::vector<int32_t> h_sizes((size_t)nblocks * nstage), h_offs((size_t)nblocks * nstage);
    PLAN_CUDA(cudaMemcpyAsync(h_sizes.data(), P->ind_sizes, sizeof(int32_t) * h_sizes.size(), cudaMemcpyDeviceToHost, s));
    PLAN_CUDA(cudaStreamSynchronize(s));
    std::vector<int32_t> h_nind(nstage, 0);
    int nshared = 0;
    for (int b = 0; b < nblocks; ++b) {
      int sh = 0;
      for (int q = 0; q < nstage; ++q) {
        int sz = h_sizes[(size_t)b * nstage + q];
        h_offs[(size_t)b * nstage + q] = h_nind[q];
        h_nind[q] += sz;
        sh += ((sz * stage_bytes[q]) + 15) / 16 * 16;
      }
      nshared = std::max(nshared, sh);
    }
    P->nshared = nshared;
    PLAN_CUDA(cudaMemcpyAsync(P->ind_offs, h_offs.data(), sizeof(int32_t) * h_offs.size(), cudaMemcpyHostToDevice, s));
    PLAN_CUDA(cudaMemcpyAsync(P->nindirect, h_nind.data(), sizeof(int32_t) * nstage, cudaMemcpyHostToDevice, s));
    plan_stage_compact_kernel<<<dim3(nblocks, nstage), kPlanThreads, 0, s>>>(
        d_pairs, nstage, d_base, P->ind_sizes, P->ind_offs, P->ind_map);
    PLAN_CUDA(cudaGetLastError());
    P->counts[2] = ind_len;
    P->counts[3] = (int64_t)loc_rows * set_size;
    P->counts[4] = (int64_t)nblocks * nstage;
    P->counts[5] = (int64_t)nblocks * nstage;
    P->counts[6] = nstage;
  }

  // ---- colouring (plan.pyx:214-376)
  PLAN_TRY(alloc32(&P->thrcol, set_size));
  PLAN_TRY(alloc32(&P->nthrcol, nblocks));
  PLAN_TRY(alloc32(&P->blkcol, nblocks));
  PLAN_CUDA(cudaMemsetAsync(P->thrcol, 0xff, sizeof(int32_t) * std::max(set_size, 1), s));
  PLAN_CUDA(cudaMemsetAsync(P->nthrcol, 0, sizeof(int32_t) * std::max(nblocks, 1), s));
  P->counts[7] = set_size;
  P->counts[8] = nblocks;
  P->counts[11] = nblocks;
  std::vector<int32_t> h_blkcol(nblocks, 0);
  int32_t max_nthrcol = tc ? 1 : 0;
  if (nblocks > 0 && nrace > 0) {
    int nent_total = 0;
    for (int g = 0; g < nrace; ++g) nent_total += race_nent[g];
    if ((int64_t)part_size * nent_total > 32767) {
      for (void *t : temps) dev_free(t, s);
      plan_release(P, s);
      return set_error(OP2B_ERR_ARG, "plan: part_size %d x %d race entries exceeds 32767",
                       part_size, nent_total);
    }
    std::vector<RaceEntry> h_ents(nent_total);
    std::vector<RaceGroup> h_groups(nrace);
    int max_keys = 0;
    for (int g = 0, k = 0; g < nrace; ++g) {
      RaceGroup &G = h_groups[g];
      G.first = k;
      G.nent = race_nent[g];
      G.size = race_size[g];
      G.cap = (int64_t)part_size * G.nent;
      max_keys = std::max<int>(max_keys, part_size * G.nent);
      for (int j = 0; j < G.nent; ++j, ++k) {
        h_ents[k].map = reinterpret_cast<const int32_t *>(race_map[k]);
        h_ents[k].arity = race_arity[k];
        h_ents[k].idx = race_idx[k];
        if (race_idx[k] < 0 || race_idx[k] >= race_arity[k]) {
          for (void *t : temps) dev_free(t, s);
          plan_release(P, s);
          return set_error(OP2B_ERR_ARG, "plan: race map index %d outside arity %d", race_idx[k], race_arity[k]);
        }
      }
      PLAN_TRY(alloc32(&G.tmp, (int64_t)nblocks * G.cap));
      temps.push_back(G.tmp);
    }
    int32_t *race_cnt = nullptr;
    PLAN_TRY(alloc32(&race_cnt, (int64_t)nblocks * nrace));
    temps.push_back(race_cnt);
    RaceGroup *d_groups = nullptr;
    RaceEntry *d_ents = nullptr;
    PLAN_TRY(dev_alloc((void **)&d_ents, sizeof(RaceEntry) * nent_total, s));
    temps.push_back(d_ents);
    PLAN_CUDA(cudaMemcpyAsync(d_ents, h_ents.data(), sizeof(RaceEntry) * nent_total, cudaMemcpyHostToDevice, s));
    // node -> block incidence per group
    for (int g = 0; g < nrace; ++g) {
      RaceGroup &G = h_groups[g];
      PLAN_TRY(alloc32(&G.node_ptr, (int64_t)G.size + 1));
      temps.push_back(G.node_ptr);
    }
    PLAN_TRY(dev_alloc((void **)&d_groups, sizeof(RaceGroup) * nrace, s));
    temps.push_back(d_groups);
    PLAN_CUDA(cudaMemcpyAsync(d_groups, h_groups.data(), sizeof(RaceGroup) * nrace, cudaMemcpyHostToDevice, s));
    const int npow2 = next_pow2(max_keys);
    int64_t smem64 = 2LL * npow2 * 4 + (int64_t)part_size * nent_total * 4 +
                     (((int64_t)part_size * nent_total + 1) & ~1LL) * 2 + (int64_t)part_size * 4;
    if (smem64 > smem_optin()) {
      for (void *t : temps) dev_free(t, s);
      plan_release(P, s);
      return set_error(OP2B_ERR_ARG, "plan: colouring needs %lld bytes of shared memory per block; "
                       "reduce the partition size", (long long)smem64);
    }
    const int smem = (int)smem64;
    PLAN_CUDA(cudaFuncSetAttribute(plan_race_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    plan_race_kernel<<<nblocks, kPlanThreads, smem, s>>>(d_groups, d_ents, nrace, nent_total, set_size,
                                                       part_size, npow2, tc ? 1 : 0, race_cnt,
                                                       P->thrcol, P->nthrcol);
    PLAN_CUDA(cudaGetLastError());
    int32_t *d_scalar = nullptr;
    PLAN_TRY(alloc32(&d_scalar, 4));
    temps.push_back(d_scalar);
    for (int g = 0; g < nrace; ++g) {
      RaceGroup &G = h_groups[g];
      int32_t *cursor = nullptr;
      PLAN_TRY(alloc32(&cursor, (int64_t)G.size + 1));
      temps.push_back(cursor);
      PLAN_CUDA(cudaMemsetAsync(G.node_ptr, 0, sizeof(int32_t) * ((size_t)G.size + 1), s));
      incidence_count_kernel<<<nblocks, kPlanThreads, 0, s>>>(G, g, nrace, race_cnt, G.node_ptr);
      PLAN_TRY(device_excl_scan(G.node_ptr, G.node_ptr, (int64_t)G.size + 1, d_scalar, s));
      int32_t total = 0;
      PLAN_CUDA(cudaMemcpyAsync(&total, G.node_ptr + G.size, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
      PLAN_CUDA(cudaStreamSynchronize(s));
      PLAN_TRY(alloc32(&G.node_blk, total));
      temps.push_back(G.node_blk);
      PLAN_CUDA(cudaMemsetAsync(cursor, 0, sizeof(int32_t) * ((size_t)G.size + 1), s));
      incidence_fill_kernel<<<nblocks, kPlanThreads, 0, s>>>(G, g, nrace, race_cnt, cursor);
      PLAN_CUDA(cudaGetLastError());
    }
    PLAN_CUDA(cudaMemcpyAsync(d_groups, h_groups.data(), sizeof(RaceGroup) * nrace, cudaMemcpyHostToDevice, s));
    PLAN_CUDA(cudaMemsetAsync(P->blkcol, 0xff, sizeof(int32_t) * nblocks, s));
    for (int round = 0; round < nblocks + 1; ++round) {
      PLAN_CUDA(cudaMemsetAsync(d_scalar, 0, 2 * sizeof(int32_t), s));
      jp_round_kernel<<<nblocks, 128, 0, s>>>(d_groups, nrace, race_cnt, P->blkcol, d_scalar, d_scalar + 1);
      int32_t h[2] = {0, 0};
      PLAN_CUDA(cudaMemcpyAsync(h, d_scalar, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
      PLAN_CUDA(cudaStreamSynchronize(s));
      if (h[1]) {
        for (void *t : temps) dev_free(t, s);
        plan_release(P, s);
        return set_error(OP2B_ERR_ARG, "plan: more than %d block colours", kMaxBlockColors);
      }
      if (h[0] == 0) break;
    }
    PLAN_CUDA(cudaMemcpyAsync(h_blkcol.data(), P->blkcol, sizeof(int32_t) * nblocks, cudaMemcpyDeviceToHost, s));
    if (tc) {
      std::vector<int32_t> h_nthr(nblocks);
      PLAN_CUDA(cudaMemcpyAsync(h_nthr.data(), P->nthrcol, sizeof(int32_t) * nblocks, cudaMemcpyDeviceToHost, s));
      PLAN_CUDA(cudaStreamSynchronize(s));
      for (int v : h_nthr) max_nthrcol = std::max(max_nthrcol, v);
    }
    PLAN_CUDA(cudaStreamSynchronize(s));
  } else if (nblocks > 0) {
    // No race arguments: every element colour 0, one block colour
    // (plan.pyx:296-311 with an empty mask).
    if (tc) {
      PLAN_CUDA(cudaMemsetAsync(P->thrcol, 0, sizeof(int32_t) * set_size, s));
      std::vector<int32_t> ones(nblocks, 1);
      PLAN_CUDA(cudaMemcpyAsync(P->nthrcol, ones.data(), sizeof(int32_t) * nblocks, cudaMemcpyHostToDevice, s));
      PLAN_CUDA(cudaStreamSynchronize(s));
    }
    PLAN_CUDA(cudaMemsetAsync(P->blkcol, 0, sizeof(int32_t) * nblocks, s));
  }
  P->max_nthrcol = max_nthrcol;

  // ncolblk = bincount(colours), blkmap = stable argsort (plan.pyx:374-376)
  int ncolors = 0;
  for (int c : h_blkcol) ncolors = std::max(ncolors, c + 1);
  if (nblocks == 0) ncolors = 0;
  std::vector<int32_t> h_ncolblk(ncolors, 0), h_blkmap(nblocks);
  for (int c : h_blkcol) h_ncolblk[c]++;
  std::vector<int32_t> start(ncolors, 0);
  for (int c = 1; c < ncolors; ++c) start[c] = start[c - 1] + h_ncolblk[c - 1];
  for (int b = 0; b < nblocks; ++b) h_blkmap[start[h_blkcol[b]]++] = b;
  P->ncolors = ncolors;
  P->h_ncolblk = h_ncolblk;
  PLAN_TRY(alloc32(&P->blkmap, nblocks));
  PLAN_TRY(alloc32(&P->ncolblk, ncolors));
  PLAN_CUDA(cudaMemcpyAsync(P->blkmap, h_blkmap.data(), sizeof(int32_t) * nblocks, cudaMemcpyHostToDevice, s));
  PLAN_CUDA(cudaMemcpyAsync(P->ncolblk, h_ncolblk.data(), sizeof(int32_t) * ncolors, cudaMemcpyHostToDevice, s));
  P->counts[9] = nblocks;
  P->counts[10] = ncolors;
  PLAN_CUDA(cudaStreamSynchronize(s));
  for (void *t : temps) dev_free(t, s);
  *plan_out = reinterpret_cast<uint64_t>(P);
  return OP2B_OK;
}

int op2b_plan_info(uint64_t plan, int32_t *nblocks, int32_t *ncolors, int32_t *nshared,
                   int32_t *ninds, int32_t *max_nthrcol, int64_t *ind_map_len, int32_t *loc_rows) {
  Plan *P = reinterpret_cast<Plan *>(plan);
  if (!P) return set_error(OP2B_ERR_ARG, "null plan");
  if (nblocks) *nblocks = P->nblocks;
  if (ncolors) *ncolors = P->ncolors;
  if (nshared) *nshared = P->nshared;
  if (ninds) *ninds = P->ninds;
  if (max_nthrcol) *max_nthrcol = P->max_nthrcol;
  if (ind_map_len) *ind_map_len = P->ind_map_len;
  if (loc_rows) *loc_rows = P->loc_rows;
  return OP2B_OK;
}

int op2b_plan_array(uint64_t plan, int32_t which, uint64_t *dptr, int64_t *count) {
  Plan *P = reinterpret_cast<Plan *>(plan);
  if (!P) return set_error(OP2B_ERR_ARG, "null plan");
  void *arr[12] = {P->nelems, P->offset, P->ind_map, P->loc_map, P->ind_sizes, P->ind_offs,
                   P->nindirect, P->thrcol, P->nthrcol, P->blkmap, P->ncolblk, P->blkcol};
  if (which < 0 || which >= 12) return set_error(OP2B_ERR_ARG, "plan array %d", which);
  *dptr = reinterpret_cast<uint64_t>(arr[which]);
  if (count) *count = P->counts[which];
  return OP2B_OK;
}

int op2b_plan_ncolblk_host(uint64_t plan, int32_t *out, int32_t n) {
  Plan *P = reinterpret_cast<Plan *>(plan);
  if (!P) return set_error(OP2B_ERR_ARG, "null plan");
  for (int i = 0; i < n && i < P->ncolors; ++i) out[i] = P->h_ncolblk[i];
  return OP2B_OK;
}

int op2b_plan_free(uint64_t plan) {
  OP2B_REQUIRE_INIT();
  plan_release(reinterpret_cast<Plan *>(plan), stream_of(0));
  return OP2B_OK;
}

}  // extern "C"
