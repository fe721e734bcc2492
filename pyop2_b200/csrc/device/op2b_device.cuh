// Device helpers prepended to every JIT-compiled par_loop stub (NVRTC, sm_100a).
//
//  * op2b_load / op2b_store: move one Dat row of N elements of T between
//    global memory and a register array with the widest aligned vector access
//    (16-byte when the row size is a multiple of 16, then 8, then 4 bytes).
//    The register arrays are declared __align__(16) by the generated stubs.
//    Dat rows start at base + i * N * sizeof(T) with a 256-byte aligned base,
//    so a row whose size is a multiple of 16 (8) bytes is 16 (8) byte aligned.
//  * op2b_csr_find: position of (row, col) in a CSR pattern (binary search in
//    the sorted colidx of the row), -1 if the pattern does not store it.
//  * op2b_reduce: deterministic Global reduction (INC / MIN / MAX) of one
//    register value per thread: warp shuffles, one partial per CTA, and the
//    last CTA to finish folds the partials in CTA order into the Global.
#pragma once

typedef signed char op2b_i8;
typedef unsigned char op2b_u8;
typedef long long op2b_i64;
typedef unsigned long long op2b_u64;

#define OP2B_FULL_MASK 0xffffffffu

// First statement of every generated stub: wait until the kernel before it
// on the stream has completed and its writes are visible (a no-op when the
// stub was launched without programmatic serialisation), then allow the
// kernel after it to be scheduled.
__device__ __forceinline__ void op2b_stub_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Asynchronous copy (cp.async) of one row of B bytes, B a multiple of 4,
// from global to shared memory in 16-, 8- or 4-byte pieces as the size
// allows; both addresses must be aligned to the piece size.
// op2b_cp_async_wait() waits for every copy the thread has issued.
template <int B>
__device__ __forceinline__ void op2b_cp_async_row(void *dst, const void *src) {
  unsigned long long s;
  asm("cvta.to.shared.u64 %0, %1;" : "=l"(s) : "l"(dst));
  const unsigned sa = (unsigned)s;
  const char *g = reinterpret_cast<const char *>(src);
  if constexpr (B % 16 == 0) {
#pragma unroll
    for (int i = 0; i < B / 16; ++i)
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa + 16 * i), "l"(g + 16 * i)
                   : "memory");
  } else if constexpr (B % 8 == 0) {
#pragma unroll
    for (int i = 0; i < B / 8; ++i)
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa + 8 * i), "l"(g + 8 * i)
                   : "memory");
  } else {
    static_assert(B % 4 == 0, "cp.async rows are multiples of 4 bytes");
#pragma unroll
    for (int i = 0; i < B / 4; ++i)
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(sa + 4 * i), "l"(g + 4 * i)
                   : "memory");
  }
}

__device__ __forceinline__ void op2b_cp_async_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

template <typename T, int N, bool RO>
__device__ __forceinline__ void op2b_load(T (&dst)[N], const T *__restrict__ src) {
  constexpr int B = N * (int)sizeof(T);
  if constexpr (B % 16 == 0) {
#pragma unroll
    for (int i = 0; i < B / 16; ++i) {
      uint4 v = RO ? __ldg(reinterpret_cast<const uint4 *>(src) + i)
                   : reinterpret_cast<const uint4 *>(src)[i];
      reinterpret_cast<uint4 *>(dst)[i] = v;
    }
  } else if constexpr (B % 8 == 0) {
#pragma unroll
    for (int i = 0; i < B / 8; ++i) {
      uint2 v = RO ? __ldg(reinterpret_cast<const uint2 *>(src) + i)
                   : reinterpret_cast<const uint2 *>(src)[i];
      reinterpret_cast<uint2 *>(dst)[i] = v;
    }
  } else if constexpr (B % 4 == 0 && sizeof(T) >= 4) {
#pragma unroll
    for (int i = 0; i < B / 4; ++i) {
      unsigned v = RO ? __ldg(reinterpret_cast<const unsigned *>(src) + i)
                      : reinterpret_cast<const unsigned *>(src)[i];
      reinterpret_cast<unsigned *>(dst)[i] = v;
    }
  } else {
#pragma unroll
    for (int i = 0; i < N; ++i) dst[i] = src[i];
  }
}

template <typename T, int N>
__device__ __forceinline__ void op2b_store(T *__restrict__ dst, const T (&src)[N]) {
  constexpr int B = N * (int)sizeof(T);
  if constexpr (B % 16 == 0) {
#pragma unroll
    for (int i = 0; i < B / 16; ++i) {
      reinterpret_cast<uint4 *>(dst)[i] = reinterpret_cast<const uint4 *>(src)[i];
    }
  } else if constexpr (B % 8 == 0) {
#pragma unroll
    for (int i = 0; i < B / 8; ++i) {
      reinterpret_cast<uint2 *>(dst)[i] = reinterpret_cast<const uint2 *>(src)[i];
    }
  } else {
#pragma unroll
    for (int i = 0; i < N; ++i) dst[i] = src[i];
  }
}

// Staged rows in shared memory (the staged form's READ rows and INC
// accumulators).  Row r of B bytes starts at base + r * B.  When B is 32, 64
// or 128 (m = B / 16 chunks of 16 bytes), chunk j of row r is kept at chunk
// j ^ ((r / (8 / m)) mod m) of the row: otherwise chunk j of every row falls
// in the same m-th of the 32 banks (rows of 32 bytes: only the even or only
// the odd 16-byte bank groups), and eight threads reading chunk j of eight
// rows conflict at least two ways.  Other sizes keep the plain layout.
template <int B>
struct op2b_srow_layout {
  static constexpr int M = B / 16;
  static constexpr bool swizzled = B % 16 == 0 && (M == 2 || M == 4 || M == 8);
  static constexpr int L = swizzled ? 8 / M : 1;
  static __device__ __forceinline__ int chunk(int r, int j) {
    if constexpr (swizzled) return j ^ ((r / L) & (M - 1));
    else return j;
  }
};

// Row r of a staged array into registers.
template <typename T, int N>
__device__ __forceinline__ void op2b_srow_load(T (&dst)[N], const T *base, int r) {
  using Lay = op2b_srow_layout<N * (int)sizeof(T)>;
  if constexpr (Lay::swizzled) {
    const uint4 *row = reinterpret_cast<const uint4 *>(base + (op2b_i64)r * N);
#pragma unroll
    for (int j = 0; j < Lay::M; ++j) reinterpret_cast<uint4 *>(dst)[j] = row[Lay::chunk(r, j)];
  } else {
    op2b_load<T, N, false>(dst, base + (op2b_i64)r * N);
  }
}

// Registers into row r of a staged array.
template <typename T, int N>
__device__ __forceinline__ void op2b_srow_store(T *base, int r, const T (&src)[N]) {
  using Lay = op2b_srow_layout<N * (int)sizeof(T)>;
  if constexpr (Lay::swizzled) {
    uint4 *row = reinterpret_cast<uint4 *>(base + (op2b_i64)r * N);
#pragma unroll
    for (int j = 0; j < Lay::M; ++j) row[Lay::chunk(r, j)] = reinterpret_cast<const uint4 *>(src)[j];
  } else {
    op2b_store(base + (op2b_i64)r * N, src);
  }
}

// Index in a staged array of element k of row r.
template <typename T, int N>
__device__ __forceinline__ int op2b_srow_index(int r, int k) {
  using Lay = op2b_srow_layout<N * (int)sizeof(T)>;
  if constexpr (Lay::swizzled) {
    constexpr int E = 16 / (int)sizeof(T);
    return r * N + Lay::chunk(r, k / E) * E + k % E;
  } else {
    return r * N + k;
  }
}

// cp.async of one row (B bytes at src) into row r of a staged array.
template <int B>
__device__ __forceinline__ void op2b_cp_async_srow(void *base, int r, const void *src) {
  using Lay = op2b_srow_layout<B>;
  char *row = reinterpret_cast<char *>(base) + (op2b_i64)r * B;
  if constexpr (Lay::swizzled) {
    const char *g = reinterpret_cast<const char *>(src);
#pragma unroll
    for (int j = 0; j < Lay::M; ++j) op2b_cp_async_row<16>(row + 16 * Lay::chunk(r, j), g + 16 * j);
  } else {
    op2b_cp_async_row<B>(row, src);
  }
}

// SoA row: component k of element e lives at base[k * stride + e].
template <typename T, int N>
__device__ __forceinline__ void op2b_load_soa(T (&dst)[N], const T *__restrict__ base, op2b_i64 e,
                                              op2b_i64 stride) {
#pragma unroll
  for (int k = 0; k < N; ++k) dst[k] = base[k * stride + e];
}

template <typename T, int N>
__device__ __forceinline__ void op2b_store_soa(T *__restrict__ base, op2b_i64 e, op2b_i64 stride,
                                               const T (&src)[N]) {
#pragma unroll
  for (int k = 0; k < N; ++k) base[k * stride + e] = src[k];
}

template <typename T, int N>
__device__ __forceinline__ void op2b_zero(T (&a)[N]) {
#pragma unroll
  for (int k = 0; k < N; ++k) a[k] = T(0);
}

// Row of the contribution of element e at position k (of K) in a two-phase
// contribution array: tiles of 32 elements, position-major inside a tile.
__device__ __forceinline__ op2b_i64 op2b_lma_index(op2b_i64 e, int k, int K) {
  return (((e >> 5) * K + k) << 5) + (e & 31);
}

__device__ __forceinline__ int op2b_csr_find(const int *__restrict__ rowptr,
                                             const int *__restrict__ colidx, int row, int col) {
  int lo = rowptr[row], hi = rowptr[row + 1];
  const int end = hi;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (colidx[mid] < col)
      lo = mid + 1;
    else
      hi = mid;
  }
  return (lo < end && colidx[lo] == col) ? lo : -1;
}

// Atomic increment for the atomic INC mode (no plan, no colouring).  The
// result is unused, so the compiler emits a reduction (RED) to L2.
__device__ __forceinline__ void op2b_atomic_add(double *a, double v) { atomicAdd(a, v); }
__device__ __forceinline__ void op2b_atomic_add(float *a, float v) { atomicAdd(a, v); }
__device__ __forceinline__ void op2b_atomic_add(int *a, int v) { atomicAdd(a, v); }
__device__ __forceinline__ void op2b_atomic_add(unsigned *a, unsigned v) { atomicAdd(a, v); }
__device__ __forceinline__ void op2b_atomic_add(unsigned long long *a, unsigned long long v) {
  atomicAdd(a, v);
}
__device__ __forceinline__ void op2b_atomic_add(long long *a, long long v) {
  atomicAdd(reinterpret_cast<unsigned long long *>(a), (unsigned long long)v);
}

template <typename T, int N>
__device__ __forceinline__ void op2b_atomic_row(T *dst, const T (&v)[N]) {
#pragma unroll
  for (int k = 0; k < N; ++k) op2b_atomic_add(dst + k, v[k]);
}

// Record the first Mat insertion outside the Sparsity (PETSc raises
// NEW_NONZERO_ALLOCATION_ERR there); err[1..2] = offending (row, col).
__device__ __forceinline__ void op2b_flag_missing(int *err, int row, int col) {
  if (atomicCAS(err, 0, 1) == 0) {
    err[1] = row;
    err[2] = col;
  }
}

// ------------------------------------------------------------- reductions
template <int OP, typename T>
__device__ __forceinline__ T op2b_combine(T a, T b) {
  if constexpr (OP == 0) return a + b;
  else if constexpr (OP == 1) return b < a ? b : a;
  else return b > a ? b : a;
}

template <int OP, typename T>
__device__ __forceinline__ T op2b_warp_reduce(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = op2b_combine<OP>(v, __shfl_xor_sync(OP2B_FULL_MASK, v, o));
  return v;
}

// Reduce v over the CTA; the result is valid in thread 0.  scratch holds 32 T.
template <int OP, typename T>
__device__ __forceinline__ T op2b_block_reduce(T v, T *scratch) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = op2b_warp_reduce<OP>(v);
  __syncthreads();
  if (lane == 0) scratch[wid] = v;
  __syncthreads();
  if (wid == 0) {
    // lanes past the last warp repeat warp 0's value: harmless for MIN/MAX,
    // replaced by zero for sums.
    T t = scratch[lane < nw ? lane : 0];
    if (OP == 0 && lane >= nw) t = T(0);
    v = op2b_warp_reduce<OP>(t);
  }
  return v;
}

// OP: 0 = INC (sum), 1 = MIN, 2 = MAX.  gbl: the Global's device value;
// partials: >= gridDim.x * N values; counter: zero before the launch, reset to
// zero by the last CTA.  from_init: the last CTA combines with init[] (the
// value before the loop, carried in the launch parameters, so a Global the
// host has just set needs no upload) instead of reading gbl.
template <int OP, typename T, int N>
__device__ __forceinline__ void op2b_reduce(const T (&v)[N], T *gbl, T *partials, unsigned *counter,
                                            bool from_init = false, const T *init = nullptr) {
  __shared__ T red_scratch[32];
  __shared__ bool red_last;
#pragma unroll
  for (int k = 0; k < N; ++k) {
    T r = op2b_block_reduce<OP>(v[k], red_scratch);
    if (threadIdx.x == 0) partials[blockIdx.x * N + k] = r;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) red_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!red_last) return;
  __threadfence();
#pragma unroll
  for (int k = 0; k < N; ++k) {
    T acc = OP == 0 ? T(0) : __ldcg(&partials[k]);
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
      acc = op2b_combine<OP>(acc, __ldcg(&partials[b * N + k]));
    acc = op2b_block_reduce<OP>(acc, red_scratch);
    if (threadIdx.x == 0) gbl[k] = op2b_combine<OP>(from_init ? init[k] : gbl[k], acc);
  }
  if (threadIdx.x == 0) *counter = 0u;
}
