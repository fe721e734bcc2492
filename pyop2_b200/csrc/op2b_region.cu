// Locality partition of an iteration set for staged indirect loops.
//
// The reference partitions an iteration set into blocks of consecutive
// elements (pyop2/plan.pyx:107-110) and stages each block's indirectly
// accessed rows in shared memory (:112-212).  Consecutive elements share
// targets only if the mesh numbering is local; on a permuted numbering a
// block of 1024 edges touches ~1300 distinct cells and staging saves nothing.
// This builder reorders the set instead:
//  * regions: seeds are picked by hashing element ids (about one per
//    region_size elements); a multi-source breadth-first search over the
//    element graph (two elements adjacent when they share a target of the
//    growth Map) gives every element the key (level, region) of the nearest
//    seed, ties to the smaller region id, so the result does not depend on
//    scheduling;
//  * order: elements sorted by (region, level, element id);
//  * blocks: each region cut into nearly equal runs of at most part_size
//    elements;
//  * staging: per block and staged Map the distinct targets over all Map
//    rows in order of first use (tlist / toff / tcnt) and, per position of
//    the reordered set and Map row, the target's index in that list (loc,
//    int16);
//  * thread colouring: per block, the reference's greedy colouring
//    (pyop2/plan.pyx:282-324: elements in order, 32-colour masks per round)
//    over the targets of the staged Maps marked as INC targets, so elements
//    of one colour never add to the same staged row (thrcol per position,
//    nthrcol per block); then the block's positions are sorted by colour
//    (stable), so a run of consecutive positions spans few colours.
// A staged stub (see codegen) walks block b over positions
// boff[b] .. boff[b+1], element order[pos], and finds row r of staged Map s
// at tlist[toff[b][s] + loc[row_base(s) + r][pos]].
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <vector>

#include "op2b_block_sort.cuh"
#include "op2b_internal.h"
#include "op2b_scan.cuh"

extern "C" int op2b_incidence_build(uint64_t map, int32_t nelem, int32_t arity, int32_t ntargets,
                                    uint64_t stream, uint64_t *incidence);
extern "C" int op2b_incidence_arrays(uint64_t incidence, uint64_t *ptr, uint64_t *list,
                                     int32_t *max_degree);
extern "C" int op2b_incidence_free(uint64_t incidence);

namespace op2b {

struct RegionPlan {
  int32_t set_size = 0, part_size = 0, nblocks = 0, nstage = 0, nregions = 0, levels = 0;
  int32_t loc_rows = 0;
  int64_t tlist_len = 0;
  int32_t *order = nullptr, *boff = nullptr, *tlist = nullptr, *toff = nullptr, *tcnt = nullptr;
  int32_t *thrcol = nullptr, *nthrcol = nullptr;
  int16_t *loc = nullptr;
  int32_t max_nthrcol = 0;
  std::vector<int32_t> max_count;   // per staged Map: largest tcnt over blocks
  std::vector<int32_t> arity;       // per staged Map: rows per element (loc rows from row_base)
  bool bank_slots = false;          // op2b_region_plan_bank_slots applied
};

constexpr int kRgThreads = 256;
constexpr int kRgStageThreads = 128;     // staging: more CTAs per SM than 256-thread ones
constexpr int kRgMaxKeys = 16384;          // part_size * arity per staged Map
constexpr uint64_t kUnset = ~0ull;
constexpr int kRgLevelChunk = 8;           // BFS levels between two looks at progress
constexpr int kRgMaxLevels = 1 << 16;

__device__ __forceinline__ uint32_t rg_hash(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352dU;
  x ^= x >> 15;
  x *= 0x846ca68bU;
  x ^= x >> 16;
  return x;
}

__global__ void rg_seed_kernel(int n, int region_size, int32_t *__restrict__ flag) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x)
    flag[e] = (e == 0 || rg_hash((uint32_t)e) % (uint32_t)region_size == 0) ? 1 : 0;
}

// key = level << 32 | region; seeds start at level 0 with their rank as region.
__global__ void rg_init_kernel(int n, const int32_t *__restrict__ flag, const int32_t *__restrict__ rank,
                               uint64_t *__restrict__ ekey) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x)
    ekey[e] = flag[e] ? (uint64_t)(uint32_t)rank[e] : kUnset;
}

// Elements of level L hand their key to their targets (the smallest wins).
__global__ void rg_push_kernel(int n, const int32_t *__restrict__ map, int arity, int ntargets,
                               uint32_t level,
                               const uint64_t *__restrict__ ekey,
                               unsigned long long *__restrict__ tkey) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const uint64_t k = ekey[e];
    if (k == kUnset || (uint32_t)(k >> 32) != level) continue;
    for (int r = 0; r < arity; ++r) {
      const int t = map[(int64_t)e * arity + r];
      if (t >= 0 && t < ntargets) atomicMin(&tkey[t], (unsigned long long)k);
    }
  }
}

// One level of the search in one pass: unlabelled elements take the
// smallest key of level <= `level` among their targets, one level further,
// and hand the new key to their own targets at once.  Keys of level
// `level` + 1 written during the pass are ignored by the pass's readers (a
// level-`level` target would have labelled them earlier otherwise; the key's
// level sits in its high word, so atomicMin never lets a level-`level`+1 key
// replace an older one), so every pass reads what a separate push after the
// whole previous pass would have left: the labels do not depend on
// scheduling.  Every labelled target of an unlabelled element carries level
// `level` (an earlier one would have labelled the element earlier).
__global__ void rg_level_kernel(int n, const int32_t *__restrict__ map, int arity, int ntargets,
                                uint32_t level, uint64_t *__restrict__ ekey,
                                unsigned long long *__restrict__ tkey, int32_t *__restrict__ changed) {
  int any = 0;
  const uint64_t limit = ((uint64_t)level + 1) << 32;   // keys below it: level <= `level`
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    if (ekey[e] != kUnset) continue;
    uint64_t best = kUnset;
    for (int r = 0; r < arity; ++r) {
      const int t = map[(int64_t)e * arity + r];
      if (t >= 0 && t < ntargets) {
        const uint64_t k = (uint64_t)((volatile unsigned long long *)tkey)[t];
        if (k < limit) best = min(best, k);
      }
    }
    if (best != kUnset) {
      const uint64_t k = ((best >> 32) + 1) << 32 | (best & 0xffffffffull);
      ekey[e] = k;
      any = 1;
      for (int r = 0; r < arity; ++r) {
        const int t = map[(int64_t)e * arity + r];
        if (t >= 0 && t < ntargets) atomicMin(&tkey[t], (unsigned long long)k);
      }
    }
  }
  if (__syncthreads_or(any) && threadIdx.x == 0) *changed = 1;
}

// Bucket of each element: region * nlevels + level; elements the search did
// not reach (components without a seed) form regions of consecutive ids.
__global__ void rg_bucket_kernel(int n, const uint64_t *__restrict__ ekey, int nseeds, int part_size,
                                 int nlevels, int32_t *__restrict__ bucket) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const uint64_t k = ekey[e];
    int64_t region, level;
    if (k == kUnset) {
      region = nseeds + e / part_size;
      level = 0;
    } else {
      region = (int64_t)(k & 0xffffffffull);
      level = (int64_t)(k >> 32);
    }
    bucket[e] = (int32_t)(region * nlevels + (nlevels > 1 ? level : 0));
  }
}

// First position of every region in the sorted order.
__global__ void rg_region_start_kernel(const int32_t *__restrict__ bptr, int nregions, int nlevels,
                                       int32_t *__restrict__ rstart) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r <= nregions; r += gridDim.x * blockDim.x)
    rstart[r] = bptr[(int64_t)r * nlevels];
}

struct RgStage {
  const int32_t *map;
  int32_t arity, loc_row;
  int64_t cap;       // part_size * arity
  int32_t *tmp;      // [nblocks][cap] distinct targets
};

// grid (nblocks, nstage): the distinct targets of the block's elements over
// all rows of one staged Map, numbered in order of first use (keys taken
// position by position, rows in order), and each (position, row)'s number.
// Neighbouring elements of a block (one ring of the breadth-first search)
// touch neighbouring targets, so first-use numbers put the rows a warp reads
// close together in shared memory.
// The distinct targets are found with an open-addressing hash table in
// shared memory (npow2 >= keys slots, so probing always ends); each slot
// records the first key index that holds its target, and a scan over the key
// indices of the flags "first use here" numbers the targets.  Which slot a
// target lands in depends on the order of the inserts, the numbers do not.
constexpr int kRgEmpty = INT_MIN;

__global__ void rg_stage_kernel(const RgStage *__restrict__ stages, int nstage, int set_size,
                                const int32_t *__restrict__ order, const int32_t *__restrict__ boff,
                                int npow2, int keep_keys, int32_t *__restrict__ tcnt,
                                int16_t *__restrict__ loc) {
  extern __shared__ int rg_smem[];
  const int blk = blockIdx.x, s = blockIdx.y;
  const RgStage st = stages[s];
  const int start = boff[blk], nelem = boff[blk + 1] - start;
  const int nkeys = nelem * st.arity;
  const int H = npow2;
  int *tab = rg_smem;           // [H] target of each slot
  int *first = tab + H;         // [H] first key index of the slot's target, then -1 - its number
  int *slot = first + H;        // [npow2] each key's slot
  int *key = slot + npow2;      // [npow2] keys in position order (when keep_keys)
  auto key_at = [&](int i) {
    if (keep_keys) return key[i];
    const int q = i / st.arity, r = i - q * st.arity;
    return st.map[(int64_t)order[start + q] * st.arity + r];
  };
  for (int h = threadIdx.x; h < H; h += blockDim.x) {
    tab[h] = kRgEmpty;
    first[h] = INT_MAX;
  }
  if (keep_keys)
    for (int i = threadIdx.x; i < nkeys; i += blockDim.x) {
      const int q = i / st.arity, r = i - q * st.arity;
      key[i] = st.map[(int64_t)order[start + q] * st.arity + r];
    }
  __syncthreads();
  for (int i = threadIdx.x; i < nkeys; i += blockDim.x) {
    const int v = key_at(i);
    int h = (int)(rg_hash((uint32_t)v) & (uint32_t)(H - 1));
    for (int probe = 0; probe < H; ++probe) {
      const int cur = atomicCAS(&tab[h], kRgEmpty, v);
      if (cur == kRgEmpty || cur == v) break;
      h = (h + 1) & (H - 1);
    }
    slot[i] = h;
    atomicMin(&first[h], i);
  }
  __syncthreads();
  // number the distinct targets by first use: a scan, in key order, of the
  // flags "this key is its target's first use"; a numbered slot's entry
  // becomes negative, which no later key index equals
  int carry = 0;
  for (int base = 0; base < nkeys; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const int h = i < nkeys ? slot[i] : 0;
    const int flag = (i < nkeys && first[h] == i) ? 1 : 0;
    int tot;
    const int pos = block_excl_scan(flag, &tot);
    if (flag) {
      first[h] = -1 - (carry + pos);
      st.tmp[(int64_t)blk * st.cap + carry + pos] = tab[h];
    }
    carry += tot;
    __syncthreads();
  }
  for (int i = threadIdx.x; i < nkeys; i += blockDim.x) {
    const int q = i / st.arity, r = i - q * st.arity;
    loc[(int64_t)(st.loc_row + r) * set_size + start + q] = (int16_t)(-1 - first[slot[i]]);
  }
  if (threadIdx.x == 0) tcnt[blk * nstage + s] = carry;
}

// Lane 0's part of the thread colouring: one round (colours base ..
// base + 31) of the greedy rule over the block's positions in order, R
// targets per position (R = 0: `rows` read at run time).  With R known the
// position's targets sit in registers and both mask loads issue together.
template <int R>
__device__ __forceinline__ int rg_greedy_round(const int *__restrict__ tgt, int rows, int nelem,
                                               int base, uint32_t *__restrict__ masks,
                                               int *__restrict__ col, int &ncol) {
  int remaining = 0;
  for (int i = 0; i < nelem; ++i) {
    if (base > 0 && col[i] >= 0) continue;
    uint32_t m = 0u;
    if (R > 0) {
      int t[R > 0 ? R : 1];
#pragma unroll
      for (int k = 0; k < R; ++k) t[k] = tgt[i * R + k];
#pragma unroll
      for (int k = 0; k < R; ++k) m |= masks[t[k]];
      if (m == 0xffffffffu) {
        ++remaining;
        continue;
      }
      const int c = __ffs(~m) - 1;
      col[i] = base + c;
      ncol = max(ncol, base + c + 1);
#pragma unroll
      for (int k = 0; k < R; ++k) masks[t[k]] |= 1u << c;
    } else {
      for (int k = 0; k < rows; ++k) m |= masks[tgt[i * rows + k]];
      if (m == 0xffffffffu) {
        ++remaining;
        continue;
      }
      const int c = __ffs(~m) - 1;
      col[i] = base + c;
      ncol = max(ncol, base + c + 1);
      for (int k = 0; k < rows; ++k) masks[tgt[i * rows + k]] |= 1u << c;
    }
  }
  return remaining;
}

// One warp per block: greedy thread colouring in position order over the
// block-local targets of the INC staged Maps (masks of 32 colours per round,
// as pyop2/plan.pyx:282-324).  The warp gathers every element's INC targets
// (block-local numbers, offset per staged Map) into shared memory, lane 0
// colours from there (the rule is sequential), and the warp then sorts the
// positions by colour, stably: per chunk of 32 positions, a lane's rank is
// the count of its colour so far plus the earlier lanes of the chunk with
// the same colour.  One-warp CTAs let many blocks colour at once per SM.
__global__ void rg_color_kernel(const RgStage *__restrict__ stages, const int32_t *__restrict__ inc,
                                int nstage, int set_size, int inc_rows, int part_size,
                                const int32_t *__restrict__ boff, const int32_t *__restrict__ tcnt,
                                const int16_t *__restrict__ loc, int32_t *__restrict__ thrcol,
                                int32_t *__restrict__ nthrcol, int32_t *__restrict__ newpos) {
  extern __shared__ uint32_t rg_masks[];  // [mask words][part_size*inc_rows targets][part_size
                                          //  colours][part_size+1 counts]
  const int blk = blockIdx.x, lane = threadIdx.x;
  const int start = boff[blk], nelem = boff[blk + 1] - start;
  // local target numbering: the INC staged Maps' lists one after the other
  __shared__ int s_base[64];
  __shared__ int s_total;
  if (lane == 0) {
    int b = 0;
    for (int q = 0; q < nstage; ++q) {
      s_base[q] = b;
      if (inc[q]) b += tcnt[blk * nstage + q];
    }
    s_total = b;
  }
  __syncwarp();
  const int total = s_total;
  int *tgt = reinterpret_cast<int *>(rg_masks + total);   // [nelem][inc_rows]
  int row = 0;
  for (int q = 0; q < nstage; ++q) {
    if (!inc[q]) continue;
    for (int r = 0; r < stages[q].arity; ++r, ++row)
      for (int i = lane; i < nelem; i += 32)
        tgt[i * inc_rows + row] = s_base[q] + loc[(int64_t)(stages[q].loc_row + r) * set_size + start + i];
  }
  int *col = tgt + part_size * inc_rows;                   // [nelem]
  int *cnt = col + part_size;                              // [ncol + 1]
  for (int i = lane; i < nelem; i += 32) col[i] = -1;
  int ncol = 0;
  for (int base = 0, more = nelem > 0; more; base += 32) {
    for (int i = lane; i < total; i += 32) rg_masks[i] = 0u;
    __syncwarp();
    int remaining = 0;
    if (lane == 0) {
      switch (inc_rows) {
        case 1: remaining = rg_greedy_round<1>(tgt, 1, nelem, base, rg_masks, col, ncol); break;
        case 2: remaining = rg_greedy_round<2>(tgt, 2, nelem, base, rg_masks, col, ncol); break;
        case 3: remaining = rg_greedy_round<3>(tgt, 3, nelem, base, rg_masks, col, ncol); break;
        case 4: remaining = rg_greedy_round<4>(tgt, 4, nelem, base, rg_masks, col, ncol); break;
        default: remaining = rg_greedy_round<0>(tgt, inc_rows, nelem, base, rg_masks, col, ncol);
      }
    }
    more = __shfl_sync(0xffffffffu, remaining, 0) > 0;
    __syncwarp();
  }
  ncol = __shfl_sync(0xffffffffu, ncol, 0);
  if (lane == 0) nthrcol[blk] = ncol;
  // stable counting sort of the positions by colour
  for (int c = lane; c <= ncol; c += 32) cnt[c] = 0;
  __syncwarp();
  for (int i = lane; i < nelem; i += 32) atomicAdd(&cnt[col[i] + 1], 1);
  __syncwarp();
  if (lane == 0)
    for (int c = 0; c < ncol; ++c) cnt[c + 1] += cnt[c];   // cnt[c]: first rank of colour c
  __syncwarp();
  const unsigned below = (1u << lane) - 1u;
  for (int i0 = 0; i0 < nelem; i0 += 32) {
    const int i = i0 + lane;
    const int c = i < nelem ? col[i] : -1 - lane;          // idle lanes match nobody
    const unsigned peers = __match_any_sync(0xffffffffu, c);
    const int rank = i < nelem ? cnt[c] + __popc(peers & below) : 0;
    __syncwarp();
    if (i < nelem) {
      if (lane == 31 - __clz(peers)) cnt[c] += __popc(peers);
      thrcol[start + rank] = c;
      newpos[start + i] = start + rank;
    }
    __syncwarp();
  }
}

// Move every position's element id and loc rows to its colour-sorted place.
__global__ void rg_permute_kernel(int n, int loc_rows, const int32_t *__restrict__ newpos,
                                  const int32_t *__restrict__ order, const int16_t *__restrict__ loc,
                                  int32_t *__restrict__ order2, int16_t *__restrict__ loc2) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const int q = newpos[p];
    order2[q] = order[p];
    for (int r = 0; r < loc_rows; ++r) loc2[(int64_t)r * n + q] = loc[(int64_t)r * n + p];
  }
}

__global__ void rg_compact_kernel(const RgStage *__restrict__ stages, int nstage,
                                  const int32_t *__restrict__ tcnt, const int32_t *__restrict__ toff,
                                  int32_t *__restrict__ tlist) {
  const int blk = blockIdx.x, s = blockIdx.y;
  const RgStage st = stages[s];
  const int nu = tcnt[blk * nstage + s];
  const int64_t dst = toff[blk * nstage + s];
  for (int i = threadIdx.x; i < nu; i += blockDim.x) tlist[dst + i] = st.tmp[(int64_t)blk * st.cap + i];
}

// Bank-aware slot numbering (op2b_region_plan_bank_slots).  A staged stub's
// lanes 8k..8k+7 of a warp (positions start+8g .. start+8g+7 of a block,
// whatever the CTA size) read one staged row each with one 16-byte shared
// access per chunk; the access is conflict-free when their rows lie in
// distinct 16-byte bank groups, which with the rows' chunk permutation
// (op2b_srow_layout) means distinct slot numbers mod 8.  Thread 0 of a
// (block, staged Map) CTA walks the groups of 8 positions, row by row, and
// gives every target not yet placed the residue mod 8 unused in its group
// with the fewest targets so far (any residue when all 8 are taken); slots
// are then residue + 8 * (rank in its residue class, in first-use order), so
// a block's slot count becomes 8 x its largest class (unused slots are
// padding, tlist -1).  perm[b][s][old slot] = new slot, ncnt[b][s] = count.
__global__ void rg_slot_kernel(int nstage, int set_size, const int32_t *__restrict__ boff,
                               const int32_t *__restrict__ tcnt, const int16_t *__restrict__ loc,
                               const int32_t *__restrict__ arity, const int32_t *__restrict__ row0,
                               int maxc, int16_t *__restrict__ perm, int32_t *__restrict__ ncnt) {
  extern __shared__ int8_t rg_res[];      // [maxc] residue per old slot
  const int blk = blockIdx.x, s = blockIdx.y;
  const int start = boff[blk], nelem = boff[blk + 1] - start;
  const int nu = tcnt[blk * nstage + s];
  const int A = arity[s], rb = row0[s];
  int16_t *pm = perm + ((int64_t)blk * nstage + s) * maxc;
  for (int k = threadIdx.x; k < nu; k += blockDim.x) rg_res[k] = -1;
  __syncthreads();
  if (threadIdx.x != 0) return;
  int cls[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int g = 0; g < nelem; g += 8) {
    const int m = min(8, nelem - g);
    for (int r = 0; r < A; ++r) {
      const int16_t *row = loc + (int64_t)(rb + r) * set_size + start + g;
      unsigned used = 0u;
      for (int i = 0; i < m; ++i) {
        const int t = row[i];
        if (rg_res[t] >= 0) used |= 1u << rg_res[t];
      }
      for (int i = 0; i < m; ++i) {
        const int t = row[i];
        if (rg_res[t] >= 0) continue;
        const unsigned freec = used == 0xffu ? 0xffu : (~used & 0xffu);
        int best = -1;
        for (int c = 0; c < 8; ++c)
          if (((freec >> c) & 1u) && (best < 0 || cls[c] < cls[best])) best = c;
        rg_res[t] = (int8_t)best;
        ++cls[best];
        used |= 1u << best;
      }
    }
  }
  int next[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int top = 0;
  for (int k = 0; k < nu; ++k) {
    const int c = rg_res[k] < 0 ? 0 : rg_res[k];   // every slot is used, so c >= 0
    const int v = c + 8 * next[c]++;
    top = max(top, v + 1);
    pm[k] = (int16_t)(v <= 32767 ? v : -1);          // loc rows are int16
  }
  ncnt[blk * nstage + s] = top <= 32768 ? top : -1;
}

// New target lists (padding -1) and loc rows in the new numbering; bad[0] is
// set if any renumbered slot falls outside its block's new count.
__global__ void rg_slot_apply_kernel(int nstage, int set_size, const int32_t *__restrict__ boff,
                                     const int32_t *__restrict__ tcnt, const int32_t *__restrict__ toff,
                                     const int32_t *__restrict__ tlist, const int32_t *__restrict__ ncnt,
                                     const int32_t *__restrict__ ntoff, int32_t *__restrict__ ntlist,
                                     const int16_t *__restrict__ loc, int16_t *__restrict__ nloc,
                                     const int32_t *__restrict__ arity, const int32_t *__restrict__ row0,
                                     int maxc, const int16_t *__restrict__ perm, int32_t *bad) {
  const int blk = blockIdx.x, s = blockIdx.y;
  const int start = boff[blk], nelem = boff[blk + 1] - start;
  const int bs = blk * nstage + s;
  const int nu = tcnt[bs], nn = ncnt[bs];
  const int16_t *pm = perm + (int64_t)bs * maxc;
  for (int k = threadIdx.x; k < nu; k += blockDim.x) {
    const int v = pm[k];
    if (v < 0 || v >= nn) {
      atomicExch(bad, 1);
      continue;
    }
    ntlist[ntoff[bs] + v] = tlist[toff[bs] + k];
  }
  const int A = arity[s], rb = row0[s];
  for (int q = threadIdx.x; q < nelem * A; q += blockDim.x) {
    const int i = q / A, r = q - i * A;
    const int64_t at = (int64_t)(rb + r) * set_size + start + i;
    const int o = loc[at];
    if (o < 0 || o >= nu) {
      atomicExch(bad, 1);
      continue;
    }
    nloc[at] = pm[o];
  }
}

static int rg_grid(int64_t n) {
  return std::max(1, std::min(op2b_div_up(std::max<int64_t>(n, 1), kRgThreads), sm_count() * 8));
}

}  // namespace op2b

using namespace op2b;

static void region_release(RegionPlan *p, cudaStream_t s) {
  if (!p) return;
  int32_t *arrs[] = {p->order, p->boff, p->tlist, p->toff, p->tcnt, p->thrcol, p->nthrcol};
  for (int32_t *a : arrs) dev_free(a, s);
  dev_free(p->loc, s);
  delete p;
}

extern "C" {

int op2b_region_plan_build(int32_t set_size, int32_t part_size, int32_t region_size,
                           uint64_t grow_map, int32_t grow_arity, int32_t grow_ntargets,
                           int32_t nstage, const uint64_t *stage_map, const int32_t *stage_arity,
                           const int32_t *stage_inc, uint64_t stream, uint64_t *plan_out) {
  OP2B_REQUIRE_INIT();
  if (set_size < 0 || part_size <= 0 || region_size <= 0 || grow_arity <= 0 || grow_ntargets < 0 ||
      nstage < 0 || nstage > 64 || !plan_out ||
      (nstage > 0 && (!stage_map || !stage_arity || !stage_inc)))
    return set_error(OP2B_ERR_ARG, "region plan: set_size %d part_size %d region_size %d",
                     set_size, part_size, region_size);
  int max_arity = 1, loc_rows = 0;
  for (int q = 0; q < nstage; ++q) {
    if (stage_arity[q] <= 0) return set_error(OP2B_ERR_ARG, "region plan: arity %d", stage_arity[q]);
    max_arity = std::max(max_arity, (int)stage_arity[q]);
    loc_rows += stage_arity[q];
  }
  if ((int64_t)part_size * max_arity > kRgMaxKeys)
    return set_error(OP2B_ERR_ARG,
                     "region plan: part_size %d x arity %d exceeds %d staged keys per block",
                     part_size, max_arity, kRgMaxKeys);
  cudaStream_t s = stream_of(stream);
  RegionPlan *P = new RegionPlan();
  P->set_size = set_size;
  P->part_size = part_size;
  P->nstage = nstage;
  P->loc_rows = loc_rows;
  P->max_count.assign(nstage, 0);
  P->arity.assign(stage_arity, stage_arity + nstage);
  std::vector<void *> temps;
  uint64_t inc = 0;
  auto fail = [&](int rc) {
    for (void *t : temps) dev_free(t, s);
    if (inc) op2b_incidence_free(inc);
    region_release(P, s);
    return rc;
  };
#define RG_TRY(call)              \
  do {                            \
    int _rc = (call);             \
    if (_rc) return fail(_rc);    \
  } while (0)
#define RG_CUDA(call) RG_TRY(check_cuda((call), #call))
  auto alloc = [&](void **p, size_t bytes, bool temp) {
    int rc = dev_alloc(p, std::max<size_t>(bytes, 16), s);
    if (!rc && temp) temps.push_back(*p);
    return rc;
  };
  const int n = set_size;
  const int grid = rg_grid(n);
  const int32_t *gmap = reinterpret_cast<const int32_t *>(grow_map);

  // ---- regions: seeds, then a multi-source breadth-first search
  int32_t *flag = nullptr, *rank = nullptr, *scal = nullptr;
  uint64_t *ekey = nullptr;
  unsigned long long *tkey = nullptr;
  RG_TRY(alloc((void **)&flag, sizeof(int32_t) * n, true));
  RG_TRY(alloc((void **)&rank, sizeof(int32_t) * n, true));
  RG_TRY(alloc((void **)&scal, sizeof(int32_t) * (kRgLevelChunk + 2), true));
  RG_TRY(alloc((void **)&ekey, sizeof(uint64_t) * n, true));
  RG_TRY(alloc((void **)&tkey, sizeof(uint64_t) * (size_t)grow_ntargets, true));
  int nseeds = 0, levels = 0;
  if (n > 0) {
    rg_seed_kernel<<<grid, kRgThreads, 0, s>>>(n, region_size, flag);
    RG_TRY(device_excl_scan(flag, rank, n, scal, s));
    RG_CUDA(cudaMemcpyAsync(&nseeds, scal, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    rg_init_kernel<<<grid, kRgThreads, 0, s>>>(n, flag, rank, ekey);
    RG_CUDA(cudaMemsetAsync(tkey, 0xff, sizeof(uint64_t) * (size_t)grow_ntargets, s));
    // the seeds hand their keys to their targets; each level's pass then
    // hands on the keys of the elements it labels
    rg_push_kernel<<<grid, kRgThreads, 0, s>>>(n, gmap, grow_arity, grow_ntargets, 0u, ekey, tkey);
    // levels in chunks; changed[j] records whether level base+j labelled anything
    for (int base = 0; base < kRgMaxLevels; base += kRgLevelChunk) {
      RG_CUDA(cudaMemsetAsync(scal, 0, sizeof(int32_t) * kRgLevelChunk, s));
      for (int j = 0; j < kRgLevelChunk; ++j)
        rg_level_kernel<<<grid, kRgThreads, 0, s>>>(n, gmap, grow_arity, grow_ntargets,
                                                    (uint32_t)(base + j), ekey, tkey, scal + j);
      int32_t changed[kRgLevelChunk];
      RG_CUDA(cudaGetLastError());
      RG_CUDA(cudaMemcpyAsync(changed, scal, sizeof changed, cudaMemcpyDeviceToHost, s));
      RG_CUDA(cudaStreamSynchronize(s));
      int last = -1;
      for (int j = 0; j < kRgLevelChunk; ++j)
        if (changed[j]) last = j;
      if (last >= 0) levels = base + last + 1;
      if (last < kRgLevelChunk - 1) break;
    }
  }
  const int nlevels_all = levels + 1;   // levels 0 .. levels
  const int nregions = nseeds + op2b_div_up(std::max(n, 1), part_size);
  // sort key: (region, level) when the bucket count stays moderate, else region
  int nlevels = nlevels_all;
  if ((int64_t)nregions * nlevels > std::max<int64_t>(4LL * n, 1 << 20) ||
      (int64_t)nregions * nlevels >= INT_MAX)
    nlevels = 1;
  P->nregions = nregions;
  P->levels = nlevels_all;

  // ---- order: counting sort by bucket, element ids ascending inside one
  int32_t *bucket = rank;   // reuse
  std::vector<int32_t> h_rstart(nregions + 1, 0);
  RG_TRY(alloc((void **)&P->order, sizeof(int32_t) * n, false));
  if (n > 0) {
    rg_bucket_kernel<<<grid, kRgThreads, 0, s>>>(n, ekey, nseeds, part_size, nlevels, bucket);
    RG_CUDA(cudaGetLastError());
    const int nbuckets = nregions * nlevels;
    RG_TRY(op2b_incidence_build(reinterpret_cast<uint64_t>(bucket), n, 1, nbuckets, stream, &inc));
    uint64_t bptr = 0, blist = 0;
    int32_t maxdeg = 0;
    RG_TRY(op2b_incidence_arrays(inc, &bptr, &blist, &maxdeg));
    RG_CUDA(cudaMemcpyAsync(P->order, reinterpret_cast<void *>(blist), sizeof(int32_t) * n,
                            cudaMemcpyDeviceToDevice, s));
    int32_t *rstart = nullptr;
    RG_TRY(alloc((void **)&rstart, sizeof(int32_t) * (nregions + 1), true));
    rg_region_start_kernel<<<rg_grid(nregions + 1), kRgThreads, 0, s>>>(
        reinterpret_cast<const int32_t *>(bptr), nregions, nlevels, rstart);
    RG_CUDA(cudaGetLastError());
    RG_CUDA(cudaMemcpyAsync(h_rstart.data(), rstart, sizeof(int32_t) * (nregions + 1),
                            cudaMemcpyDeviceToHost, s));
    RG_CUDA(cudaStreamSynchronize(s));
    RG_TRY(op2b_incidence_free(inc));
    inc = 0;
  }

  // ---- blocks: every region cut into nearly equal runs of <= part_size
  std::vector<int32_t> h_boff;
  h_boff.push_back(0);
  for (int r = 0; r < nregions; ++r) {
    const int a = h_rstart[r], cnt = h_rstart[r + 1] - a;
    if (cnt <= 0) continue;
    const int pieces = op2b_div_up(cnt, part_size);
    for (int q = 1; q <= pieces; ++q) h_boff.push_back(a + (int)((int64_t)cnt * q / pieces));
  }
  const int nblocks = (int)h_boff.size() - 1;
  P->nblocks = nblocks;
  RG_TRY(alloc((void **)&P->boff, sizeof(int32_t) * (nblocks + 1), false));
  RG_CUDA(cudaMemcpyAsync(P->boff, h_boff.data(), sizeof(int32_t) * (nblocks + 1),
                          cudaMemcpyHostToDevice, s));

  // ---- staging lists of every staged Map
  RG_TRY(alloc((void **)&P->tcnt, sizeof(int32_t) * (size_t)nblocks * nstage, false));
  RG_TRY(alloc((void **)&P->toff, sizeof(int32_t) * ((size_t)nblocks * nstage + 1), false));
  RG_TRY(alloc((void **)&P->loc, sizeof(int16_t) * (size_t)loc_rows * n, false));
  RG_TRY(alloc((void **)&P->thrcol, sizeof(int32_t) * n, false));
  RG_TRY(alloc((void **)&P->nthrcol, sizeof(int32_t) * nblocks, false));
  if (nblocks > 0 && nstage > 0) {
    std::vector<RgStage> h_st(nstage);
    int row = 0;
    for (int q = 0; q < nstage; ++q) {
      h_st[q].map = reinterpret_cast<const int32_t *>(stage_map[q]);
      h_st[q].arity = stage_arity[q];
      h_st[q].loc_row = row;
      h_st[q].cap = (int64_t)part_size * stage_arity[q];
      row += stage_arity[q];
      RG_TRY(alloc((void **)&h_st[q].tmp, sizeof(int32_t) * (size_t)nblocks * h_st[q].cap, true));
    }
    RgStage *d_st = nullptr;
    RG_TRY(alloc((void **)&d_st, sizeof(RgStage) * nstage, true));
    RG_CUDA(cudaMemcpyAsync(d_st, h_st.data(), sizeof(RgStage) * nstage, cudaMemcpyHostToDevice, s));
    int npow2 = 1;
    while (npow2 < part_size * max_arity) npow2 <<= 1;
    // the block's keys stay in shared memory when they fit beside the three
    // working arrays, else they are read again from the Map
    const int keep_keys = 4LL * npow2 * (int64_t)sizeof(int) <= smem_optin() ? 1 : 0;
    const int smem = (3 + keep_keys) * npow2 * (int)sizeof(int);
    RG_CUDA(cudaFuncSetAttribute(rg_stage_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    rg_stage_kernel<<<dim3(nblocks, nstage), kRgStageThreads, smem, s>>>(
        d_st, nstage, n, P->order, P->boff, npow2, keep_keys, P->tcnt, P->loc);
    RG_CUDA(cudaGetLastError());
    std::vector<int32_t> h_cnt((size_t)nblocks * nstage);
    RG_CUDA(cudaMemcpyAsync(h_cnt.data(), P->tcnt, sizeof(int32_t) * h_cnt.size(),
                            cudaMemcpyDeviceToHost, s));
    RG_CUDA(cudaStreamSynchronize(s));
    std::vector<int32_t> h_off(h_cnt.size() + 1);
    int64_t tot = 0;
    for (size_t i = 0; i < h_cnt.size(); ++i) {
      h_off[i] = (int32_t)tot;
      tot += h_cnt[i];
      int q = (int)(i % nstage);
      P->max_count[q] = std::max(P->max_count[q], h_cnt[i]);
    }
    if (tot > INT_MAX) return fail(set_error(OP2B_ERR_ARG, "region plan: %lld staged targets", (long long)tot));
    h_off[h_cnt.size()] = (int32_t)tot;
    P->tlist_len = tot;
    RG_CUDA(cudaMemcpyAsync(P->toff, h_off.data(), sizeof(int32_t) * h_off.size(),
                            cudaMemcpyHostToDevice, s));
    RG_TRY(alloc((void **)&P->tlist, sizeof(int32_t) * (size_t)tot, false));
    rg_compact_kernel<<<dim3(nblocks, nstage), kRgThreads, 0, s>>>(d_st, nstage, P->tcnt, P->toff,
                                                                   P->tlist);
    RG_CUDA(cudaGetLastError());
    // thread colours over the INC staged Maps' block-local targets
    int32_t *d_inc = nullptr;
    RG_TRY(alloc((void **)&d_inc, sizeof(int32_t) * nstage, true));
    RG_CUDA(cudaMemcpyAsync(d_inc, stage_inc, sizeof(int32_t) * nstage, cudaMemcpyHostToDevice, s));
    int64_t mask_words = 0;
    int inc_rows = 0;
    for (int q = 0; q < nstage; ++q)
      if (stage_inc[q]) {
        mask_words += P->max_count[q];
        inc_rows += stage_arity[q];
      }
    const int64_t cwords = mask_words + (int64_t)part_size * inc_rows + 2LL * part_size + 1;
    if (cwords * 4 > smem_optin())
      return fail(set_error(OP2B_ERR_ARG, "region plan: colouring needs %lld bytes of shared memory",
                            (long long)(cwords * 4)));
    const int csmem = (int)sizeof(uint32_t) * (int)std::max<int64_t>(cwords, 1);
    RG_CUDA(cudaFuncSetAttribute(rg_color_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, csmem));
    int32_t *newpos = nullptr, *order2 = nullptr;
    int16_t *loc2 = nullptr;
    RG_TRY(alloc((void **)&newpos, sizeof(int32_t) * n, true));
    RG_TRY(alloc((void **)&order2, sizeof(int32_t) * n, true));
    RG_TRY(alloc((void **)&loc2, sizeof(int16_t) * (size_t)loc_rows * n, true));
    rg_color_kernel<<<nblocks, 32, csmem, s>>>(d_st, d_inc, nstage, n, inc_rows, part_size, P->boff,
                                                P->tcnt, P->loc, P->thrcol, P->nthrcol, newpos);
    RG_CUDA(cudaGetLastError());
    rg_permute_kernel<<<grid, kRgThreads, 0, s>>>(n, loc_rows, newpos, P->order, P->loc, order2, loc2);
    RG_CUDA(cudaGetLastError());
    // the permuted arrays replace the originals, which become temporaries
    temps.erase(std::remove(temps.begin(), temps.end(), (void *)order2), temps.end());
    temps.erase(std::remove(temps.begin(), temps.end(), (void *)loc2), temps.end());
    temps.push_back(P->order);
    temps.push_back(P->loc);
    P->order = order2;
    P->loc = loc2;
    std::vector<int32_t> h_nc(nblocks);
    RG_CUDA(cudaMemcpyAsync(h_nc.data(), P->nthrcol, sizeof(int32_t) * nblocks, cudaMemcpyDeviceToHost, s));
    RG_CUDA(cudaStreamSynchronize(s));
    for (int b = 0; b < nblocks; ++b) P->max_nthrcol = std::max(P->max_nthrcol, h_nc[b]);
  } else {
    RG_TRY(alloc((void **)&P->tlist, 16, false));
    RG_CUDA(cudaMemsetAsync(P->toff, 0, sizeof(int32_t) * ((size_t)nblocks * nstage + 1), s));
    RG_CUDA(cudaMemsetAsync(P->thrcol, 0, sizeof(int32_t) * std::max(n, 1), s));
    RG_CUDA(cudaMemsetAsync(P->nthrcol, 0, sizeof(int32_t) * std::max(nblocks, 1), s));
    if (nblocks > 0) P->max_nthrcol = 1;
  }
  RG_CUDA(cudaStreamSynchronize(s));
  for (void *t : temps) dev_free(t, s);
  temps.clear();
#undef RG_TRY
#undef RG_CUDA
  *plan_out = reinterpret_cast<uint64_t>(P);
  return OP2B_OK;
}

int op2b_region_plan_info(uint64_t plan, int32_t *nblocks, int32_t *nregions, int32_t *levels,
                          int32_t *max_count, int64_t *tlist_len, int32_t *max_nthrcol) {
  RegionPlan *P = reinterpret_cast<RegionPlan *>(plan);
  if (!P) return set_error(OP2B_ERR_ARG, "null region plan");
  if (max_nthrcol) *max_nthrcol = P->max_nthrcol;
  if (nblocks) *nblocks = P->nblocks;
  if (nregions) *nregions = P->nregions;
  if (levels) *levels = P->levels;
  if (max_count)
    for (int q = 0; q < P->nstage; ++q) max_count[q] = P->max_count[q];
  if (tlist_len) *tlist_len = P->tlist_len;
  return OP2B_OK;
}

int op2b_region_plan_array(uint64_t plan, int32_t which, uint64_t *dptr, int64_t *count) {
  RegionPlan *P = reinterpret_cast<RegionPlan *>(plan);
  if (!P || !dptr) return set_error(OP2B_ERR_ARG, "null region plan");
  const int64_t nbs = (int64_t)P->nblocks * P->nstage;
  void *ptrs[] = {P->order, P->boff, P->tlist, P->toff, P->tcnt, P->loc, P->thrcol, P->nthrcol};
  const int64_t counts[] = {P->set_size, P->nblocks + 1, P->tlist_len, nbs + 1, nbs,
                            (int64_t)P->loc_rows * P->set_size, P->set_size, P->nblocks};
  if (which < 0 || which > 7) return set_error(OP2B_ERR_ARG, "region plan array %d", which);
  *dptr = reinterpret_cast<uint64_t>(ptrs[which]);
  if (count) *count = counts[which];
  return OP2B_OK;
}

int op2b_region_plan_bank_slots(uint64_t plan, uint64_t stream) {
  OP2B_REQUIRE_INIT();
  RegionPlan *P = reinterpret_cast<RegionPlan *>(plan);
  if (!P) return set_error(OP2B_ERR_ARG, "null region plan");
  if (P->bank_slots || P->nblocks == 0 || P->nstage == 0) {
    P->bank_slots = true;
    return OP2B_OK;
  }
  cudaStream_t s = stream_of(stream);
  const int nb = P->nblocks, ns = P->nstage, n = P->set_size;
  const int64_t nbs = (int64_t)nb * ns;
  int maxc = 1;
  for (int q = 0; q < ns; ++q) maxc = std::max(maxc, P->max_count[q]);
  std::vector<int32_t> h_row0(ns);
  for (int q = 0, r = 0; q < ns; ++q) {
    h_row0[q] = r;
    r += P->arity[q];
  }
  std::vector<void *> temps;
  auto alloc = [&](void **ptr, size_t bytes, bool temp) -> int {
    int rc = dev_alloc(ptr, bytes, s);
    if (rc == OP2B_OK && temp) temps.push_back(*ptr);
    return rc;
  };
  auto done = [&](int rc) {
    for (void *t : temps) dev_free(t, s);
    return rc;
  };
#define BS_TRY(x) do { int _rc = (x); if (_rc) return done(_rc); } while (0)
#define BS_CUDA(x) BS_TRY(check_cuda((x), #x))
  int32_t *d_ar = nullptr, *d_row0 = nullptr, *ncnt = nullptr, *ntoff = nullptr, *ntlist = nullptr,
          *bad = nullptr;
  int16_t *perm = nullptr, *nloc = nullptr;
  BS_TRY(alloc((void **)&d_ar, sizeof(int32_t) * ns, true));
  BS_TRY(alloc((void **)&d_row0, sizeof(int32_t) * ns, true));
  BS_CUDA(cudaMemcpyAsync(d_ar, P->arity.data(), sizeof(int32_t) * ns, cudaMemcpyHostToDevice, s));
  BS_CUDA(cudaMemcpyAsync(d_row0, h_row0.data(), sizeof(int32_t) * ns, cudaMemcpyHostToDevice, s));
  BS_TRY(alloc((void **)&perm, sizeof(int16_t) * (size_t)nbs * maxc, true));
  BS_TRY(alloc((void **)&ncnt, sizeof(int32_t) * (size_t)nbs, false));
  BS_CUDA(cudaFuncSetAttribute(rg_slot_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, maxc));
  rg_slot_kernel<<<dim3(nb, ns), 32, maxc, s>>>(ns, n, P->boff, P->tcnt, P->loc, d_ar, d_row0, maxc,
                                                perm, ncnt);
  BS_CUDA(cudaGetLastError());
  std::vector<int32_t> h_cnt((size_t)nbs);
  BS_CUDA(cudaMemcpyAsync(h_cnt.data(), ncnt, sizeof(int32_t) * h_cnt.size(), cudaMemcpyDeviceToHost, s));
  BS_CUDA(cudaStreamSynchronize(s));
  std::vector<int32_t> h_off(h_cnt.size() + 1);
  std::vector<int32_t> mc(ns, 0);
  int64_t tot = 0;
  for (size_t i = 0; i < h_cnt.size(); ++i) {
    h_off[i] = (int32_t)tot;
    tot += h_cnt[i];
    mc[i % ns] = std::max(mc[i % ns], h_cnt[i]);
  }
  if (tot > INT_MAX) {
    dev_free(ncnt, s);
    return done(set_error(OP2B_ERR_ARG, "region plan: %lld staged slots", (long long)tot));
  }
  for (size_t i = 0; i < h_cnt.size(); ++i)
    if (h_cnt[i] < 0) {
      dev_free(ncnt, s);
      return done(set_error(OP2B_ERR_ARG, "region plan: block %zu needs more than 32768 slots",
                            i / ns));
    }
  h_off[h_cnt.size()] = (int32_t)tot;
  BS_TRY(alloc((void **)&ntoff, sizeof(int32_t) * h_off.size(), false));
  BS_CUDA(cudaMemcpyAsync(ntoff, h_off.data(), sizeof(int32_t) * h_off.size(), cudaMemcpyHostToDevice, s));
  BS_TRY(alloc((void **)&ntlist, sizeof(int32_t) * (size_t)std::max<int64_t>(tot, 1), false));
  BS_CUDA(cudaMemsetAsync(ntlist, 0xff, sizeof(int32_t) * (size_t)std::max<int64_t>(tot, 1), s));
  BS_TRY(alloc((void **)&nloc, sizeof(int16_t) * (size_t)P->loc_rows * std::max(n, 1), false));
  BS_TRY(alloc((void **)&bad, sizeof(int32_t), true));
  BS_CUDA(cudaMemsetAsync(bad, 0, sizeof(int32_t), s));
  rg_slot_apply_kernel<<<dim3(nb, ns), kRgThreads, 0, s>>>(ns, n, P->boff, P->tcnt, P->toff, P->tlist,
                                                          ncnt, ntoff, ntlist, P->loc, nloc, d_ar,
                                                          d_row0, maxc, perm, bad);
  BS_CUDA(cudaGetLastError());
  int32_t h_bad = 0;
  BS_CUDA(cudaMemcpyAsync(&h_bad, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  BS_CUDA(cudaStreamSynchronize(s));
  if (h_bad) {
    dev_free(ncnt, s);
    dev_free(ntoff, s);
    dev_free(ntlist, s);
    dev_free(nloc, s);
    return done(set_error(OP2B_ERR_STATE, "region plan: slot renumbering out of range"));
  }
  temps.push_back(P->tcnt);
  temps.push_back(P->toff);
  temps.push_back(P->tlist);
  temps.push_back(P->loc);
  P->tcnt = ncnt;
  P->toff = ntoff;
  P->tlist = ntlist;
  P->loc = nloc;
  P->tlist_len = tot;
  P->max_count = mc;
  P->bank_slots = true;
#undef BS_TRY
#undef BS_CUDA
  return done(OP2B_OK);
}

int op2b_region_plan_free(uint64_t plan) {
  OP2B_REQUIRE_INIT();
  region_release(reinterpret_cast<RegionPlan *>(plan), stream_of(0));
  return OP2B_OK;
}

}  // extern "C"
