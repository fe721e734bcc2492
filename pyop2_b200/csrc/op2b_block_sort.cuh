// Block-wide sort and unique in shared memory, shared by the plan builders
// (op2b_plan.cu, op2b_region.cu).
#pragma once

#include <climits>

#include "op2b_scan.cuh"

namespace op2b {

__device__ __forceinline__ int next_pow2_dev(int v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}

// In-place ascending bitonic sort of a[0..n), n a power of two.
__device__ __forceinline__ void block_bitonic_sort(int *a, int n) {
  for (int k = 2; k <= n; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        int ixj = i ^ j;
        if (ixj > i) {
          int x = a[i], y = a[ixj];
          bool up = (i & k) == 0;
          if ((x > y) == up) {
            a[i] = y;
            a[ixj] = x;
          }
        }
      }
      __syncthreads();
    }
  }
}

// Sorted a[0..n) (first nkeys valid) -> unique values in u[0..return).
__device__ __forceinline__ int block_unique(const int *a, int nkeys, int n, int *u) {
  int carry = 0;
  for (int start = 0; start < n; start += blockDim.x) {
    int i = start + threadIdx.x;
    int flag = (i < nkeys && (i == 0 || a[i] != a[i - 1])) ? 1 : 0;
    int tot;
    int pos = block_excl_scan(flag, &tot);
    if (flag) u[carry + pos] = a[i];
    carry += tot;
  }
  __syncthreads();
  return carry;
}

__device__ __forceinline__ int lower_bound(const int *u, int n, int key) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (u[mid] < key)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

}  // namespace op2b
