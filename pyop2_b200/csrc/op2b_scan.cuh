// Device-wide exclusive prefix sum of int32 counts, used by the plan and the
// Sparsity builders.  Three phases: per-CTA scan of a 4096-item chunk, one CTA
// scanning the chunk totals, then a uniform add.  In-place (out == in) is
// allowed: every CTA reads its chunk before it writes it.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "op2b_internal.h"

namespace op2b {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;  // per thread -> 4096 items per CTA
constexpr int kScanChunk = kScanThreads * kScanItems;

__device__ __forceinline__ int warp_incl_scan(int v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// Exclusive scan of one value per thread across the CTA; returns the CTA total
// in *total.  blockDim.x must be a multiple of 32 and at most 1024.
__device__ __forceinline__ int block_excl_scan(int v, int *total) {
  __shared__ int warp_tot[33];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  int incl = warp_incl_scan(v);
  if (lane == 31) warp_tot[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    int w = lane < nw ? warp_tot[lane] : 0;
    int wi = warp_incl_scan(w);
    if (lane < nw) warp_tot[lane] = wi - w;
    if (lane == nw - 1) warp_tot[32] = wi;
  }
  __syncthreads();
  int res = incl - v + warp_tot[wid];
  int tot = warp_tot[32];
  __syncthreads();
  *total = tot;
  return res;
}

static __global__ void scan_chunk_kernel(const int *in, int *out, int *chunk_sums, int64_t n) {
  const int64_t base = (int64_t)blockIdx.x * kScanChunk + (int64_t)threadIdx.x * kScanItems;
  int v[kScanItems];
  int s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t i = base + k;
    v[k] = i < n ? in[i] : 0;
    s += v[k];
  }
  int total;
  int pre = block_excl_scan(s, &total);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t i = base + k;
    if (i < n) out[i] = pre;
    pre += v[k];
  }
  if (threadIdx.x == 0) chunk_sums[blockIdx.x] = total;
}

// One CTA: exclusive scan of the chunk totals in place; grand total to *total.
static __global__ void scan_sums_kernel(int *sums, int nchunks, int *total) {
  int carry = 0;
  for (int start = 0; start < nchunks; start += blockDim.x) {
    int i = start + threadIdx.x;
    int v = i < nchunks ? sums[i] : 0;
    int t;
    int pre = block_excl_scan(v, &t);
    if (i < nchunks) sums[i] = pre + carry;
    carry += t;
  }
  if (threadIdx.x == 0) *total = carry;
}

static __global__ void scan_add_kernel(int *out, const int *chunk_sums, int64_t n) {
  const int add = chunk_sums[blockIdx.x];
  const int64_t base = (int64_t)blockIdx.x * kScanChunk;
  for (int k = threadIdx.x; k < kScanChunk; k += blockDim.x) {
    int64_t i = base + k;
    if (i < n) out[i] += add;
  }
}

// out[i] = sum(in[0..i)); *d_total (device int) receives the grand total.
// Needs scratch of (n/4096 + 1) ints, allocated here stream-ordered.
inline int device_excl_scan(const int *in, int *out, int64_t n, int *d_total, cudaStream_t s) {
  if (n <= 0) {
    OP2B_CUDA(cudaMemsetAsync(d_total, 0, sizeof(int), s));
    return OP2B_OK;
  }
  const int nchunks = (int)((n + kScanChunk - 1) / kScanChunk);
  int *sums = nullptr;
  int rc = dev_alloc((void **)&sums, sizeof(int) * (size_t)nchunks, s);
  if (rc) return rc;
  scan_chunk_kernel<<<nchunks, kScanThreads, 0, s>>>(in, out, sums, n);
  scan_sums_kernel<<<1, 1024, 0, s>>>(sums, nchunks, d_total);
  scan_add_kernel<<<nchunks, kScanThreads, 0, s>>>(out, sums, n);
  dev_free(sums, s);
  OP2B_CUDA(cudaGetLastError());
  return OP2B_OK;
}

}  // namespace op2b
