// Linear algebra on the device CSR Mats and Dat vectors: sparse
// matrix-vector product, vector operations, reductions, and a
// Jacobi-preconditioned conjugate-gradient solve.
//
// Replaces the reference's PETSc KSP solve (pyop2/petsc_base.py:160-220,
// defaults linear_solver 'cg', preconditioner 'jacobi', pyop2/base.py:1591-
// 1601) and the Cusp CG of the CUDA backend (pyop2/cuda.py:445-600); the Dat
// arithmetic of pyop2/base.py:749-797 and Dat.norm (:836-839).
//
// Reductions are deterministic: each CTA reduces its share in a fixed order,
// and the partials are combined in CTA order by one CTA (or, inside the CG
// iteration, identically by every CTA that needs the total), so a result
// depends only on the data and the launch shape, never on scheduling.
//
// The CG iteration runs three kernels per step with every scalar (alpha,
// beta, residual norms) kept on the device; the convergence test runs on the
// device too and sets a stop flag that turns the remaining launched steps
// into no-ops, so the host launches steps in chunks and synchronises once per
// chunk while the solve still stops at the exact iteration.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "op2b_internal.h"

namespace op2b {

constexpr int kLinBlock = 256;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum over the CTA in a fixed order; valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double *scratch) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) scratch[wid] = v;
  __syncthreads();
  double t = 0.0;
  if (wid == 0) {
    t = lane < nw ? scratch[lane] : 0.0;
    t = warp_sum(t);
  }
  return t;
}

// Sum of n partials in a fixed order by the whole CTA; every thread gets it.
__device__ __forceinline__ double reduce_partials(const double *__restrict__ part, int n,
                                                  double *scratch) {
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += part[i];
  s = block_sum(s, scratch);
  __shared__ double total;
  if (threadIdx.x == 0) total = s;
  __syncthreads();
  return total;
}

// ------------------------------------------------------------------ SpMV
// One group of G lanes per row: strided partial products, then a shuffle
// tree inside the group (fixed order).
// Every lane of the warp must call it (the shuffles use the full mask): a
// lane past the last row passes live = false and contributes nothing.
template <int G>
__device__ __forceinline__ double row_dot(const int32_t *__restrict__ rowptr,
                                          const int32_t *__restrict__ colidx,
                                          const double *__restrict__ vals,
                                          const double *__restrict__ x, int row, int lane,
                                          bool live) {
  double s = 0.0;
  const int k0 = live ? rowptr[row] : 0, k1 = live ? rowptr[row + 1] : 0;
  for (int k = k0 + lane; k < k1; k += G) s += vals[k] * __ldg(x + colidx[k]);
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, G);
  return s;
}

// y = alpha * A x + beta * y (beta == 0: y is not read)
template <int G>
__global__ void __launch_bounds__(kLinBlock)
    spmv_kernel(const int32_t *__restrict__ rowptr, const int32_t *__restrict__ colidx,
                const double *__restrict__ vals, int nrows, const double *__restrict__ x,
                double *__restrict__ y, double alpha, double beta) {
  const int lane = threadIdx.x % G;
  const int groups = (gridDim.x * blockDim.x) / G;
  // every lane of a group walks the same rows (the row count padded to a
  // multiple of the groups), so the group shuffles stay converged
  const int rows_padded = ((nrows + groups - 1) / groups) * groups;
  for (int row = (blockIdx.x * blockDim.x + threadIdx.x) / G; row < rows_padded; row += groups) {
    const bool live = row < nrows;
    const double s = row_dot<G>(rowptr, colidx, vals, x, row, lane, live);
    if (live && lane == 0) y[row] = beta == 0.0 ? alpha * s : alpha * s + beta * y[row];
  }
}

__global__ void diag_inv_kernel(const int32_t *__restrict__ rowptr,
                                const int32_t *__restrict__ colidx,
                                const double *__restrict__ vals, int nrows,
                                double *__restrict__ dinv) {
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < nrows; row += gridDim.x * blockDim.x) {
    double d = 0.0;
    for (int k = rowptr[row]; k < rowptr[row + 1]; ++k)
      if (colidx[k] == row) d = vals[k];
    // a missing or zero diagonal leaves that row unpreconditioned
    dinv[row] = d != 0.0 ? 1.0 / d : 1.0;
  }
}

// --------------------------------------------------------- vector kernels
template <typename T>
__global__ void binop_kernel(T *__restrict__ out, const T *__restrict__ x,
                             const T *__restrict__ y, T ys, int64_t n, int op) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const T a = x[i], b = y ? y[i] : ys;
    T r;
    switch (op) {
      case 0: r = a + b; break;
      case 1: r = a - b; break;
      case 2: r = a * b; break;
      default: r = a / b; break;
    }
    out[i] = r;
  }
}

__global__ void dot_partial_kernel(const double *__restrict__ x, const double *__restrict__ y,
                                   int64_t n, double *__restrict__ part) {
  __shared__ double scratch[32];
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    s += x[i] * y[i];
  s = block_sum(s, scratch);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void sum_partials_kernel(const double *__restrict__ part, int n,
                                    double *__restrict__ out) {
  __shared__ double scratch[32];
  const double s = reduce_partials(part, n, scratch);
  if (threadIdx.x == 0) *out = s;
}

// ------------------------------------------------------------------ CG
// Device state of one solve.
struct CgState {
  double *x, *r, *z, *p, *q, *dinv;
  const double *b;
  double *part_pq, *part_rz, *part_zz;   // [grid] each
  double *rz;                             // [max_it + 2]: r.z of each iteration
  double *hist;                           // [max_it + 1]: ||z|| of each iteration
  double *ttol;                           // convergence threshold, divergence threshold
  int *stop;                              // [0] reason (0 running, 1 converged, 2 diverged,
                                          //  3 breakdown), [1] iterations
  int n, grid;
};

// x = 0, r = b, z = D^-1 b, p = z; partial r.z and z.z
__global__ void __launch_bounds__(kLinBlock) cg_init_kernel(CgState s) {
  __shared__ double scratch[32];
  double rz = 0.0, zz = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < s.n; i += gridDim.x * blockDim.x) {
    const double bi = s.b[i], zi = s.dinv[i] * bi;
    s.x[i] = 0.0;
    s.r[i] = bi;
    s.z[i] = zi;
    s.p[i] = zi;
    rz += bi * zi;
    zz += zi * zi;
  }
  rz = block_sum(rz, scratch);
  zz = block_sum(zz, scratch);
  if (threadIdx.x == 0) {
    s.part_rz[blockIdx.x] = rz;
    s.part_zz[blockIdx.x] = zz;
  }
}

__global__ void cg_init_finish_kernel(CgState s, double rtol, double atol, double dtol) {
  __shared__ double scratch[32];
  const double rz = reduce_partials(s.part_rz, s.grid, scratch);
  const double zz = reduce_partials(s.part_zz, s.grid, scratch);
  if (threadIdx.x == 0) {
    const double rnorm0 = sqrt(zz);
    s.rz[0] = rz;
    s.hist[0] = rnorm0;
    s.ttol[0] = fmax(rtol * rnorm0, atol);
    s.ttol[1] = dtol * rnorm0;
    s.stop[1] = 0;
    s.stop[0] = (rnorm0 <= s.ttol[0]) ? 1 : (isfinite(rnorm0) ? 0 : 3);
  }
}

// q = A p; partial p.q
template <int G>
__global__ void __launch_bounds__(kLinBlock)
    cg_spmv_kernel(CgState s, const int32_t *__restrict__ rowptr,
                   const int32_t *__restrict__ colidx, const double *__restrict__ vals) {
  __shared__ double scratch[32];
  if (*(volatile int *)s.stop) return;
  const int lane = threadIdx.x % G;
  const int groups = (gridDim.x * blockDim.x) / G;
  const int rows_padded = ((s.n + groups - 1) / groups) * groups;
  double pq = 0.0;
  for (int row = (blockIdx.x * blockDim.x + threadIdx.x) / G; row < rows_padded; row += groups) {
    const bool live = row < s.n;
    const double v = row_dot<G>(rowptr, colidx, vals, s.p, row, lane, live);
    if (live && lane == 0) {
      s.q[row] = v;
      pq += s.p[row] * v;
    }
  }
  pq = block_sum(pq, scratch);
  if (threadIdx.x == 0) s.part_pq[blockIdx.x] = pq;
}

// alpha = r.z / p.q; x += alpha p; r -= alpha q; z = D^-1 r; partial r.z, z.z
__global__ void __launch_bounds__(kLinBlock) cg_update_kernel(CgState s, int k) {
  __shared__ double scratch[32];
  if (*(volatile int *)s.stop) return;
  const double pq = reduce_partials(s.part_pq, s.grid, scratch);
  const double rzk = s.rz[k];
  const double alpha = (pq != 0.0 && isfinite(pq)) ? rzk / pq : 0.0;
  double rz = 0.0, zz = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < s.n; i += gridDim.x * blockDim.x) {
    s.x[i] += alpha * s.p[i];
    const double ri = s.r[i] - alpha * s.q[i];
    const double zi = s.dinv[i] * ri;
    s.r[i] = ri;
    s.z[i] = zi;
    rz += ri * zi;
    zz += zi * zi;
  }
  rz = block_sum(rz, scratch);
  zz = block_sum(zz, scratch);
  if (threadIdx.x == 0) {
    s.part_rz[blockIdx.x] = rz;
    s.part_zz[blockIdx.x] = zz;
  }
}

// beta = r.z(k+1) / r.z(k); p = z + beta p; convergence test
__global__ void __launch_bounds__(kLinBlock) cg_direction_kernel(CgState s, int k, int max_it) {
  __shared__ double scratch[32];
  if (*(volatile int *)s.stop) return;
  const double rz = reduce_partials(s.part_rz, s.grid, scratch);
  const double rzk = s.rz[k];
  const double beta = (rzk != 0.0 && isfinite(rzk)) ? rz / rzk : 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < s.n; i += gridDim.x * blockDim.x)
    s.p[i] = s.z[i] + beta * s.p[i];
  if (blockIdx.x == 0) {
    const double zz = reduce_partials(s.part_zz, s.grid, scratch);
    if (threadIdx.x == 0) {
      const double rnorm = sqrt(zz);
      s.rz[k + 1] = rz;
      s.hist[k + 1] = rnorm;
      int reason = 0;
      if (!isfinite(rnorm)) reason = 3;
      else if (rnorm <= s.ttol[0]) reason = 1;
      else if (rnorm >= s.ttol[1]) reason = 2;
      else if (k + 1 >= max_it) reason = 4;    // iteration limit
      if (reason) {
        s.stop[1] = k + 1;
        __threadfence();
        s.stop[0] = reason;
      }
    }
  }
}

// Lanes per row from the mean row length: on the P2 mass matrix (11.5
// entries per row) 4 lanes measured 0.150 ms per product, 2 lanes 0.152, 8
// lanes 0.221, 16 lanes 0.373 -- fewer lanes keep more rows in flight.
static int group_for(int64_t nnz, int nrows) {
  const double avg = nrows > 0 ? (double)nnz / nrows : 0.0;
  return avg <= 16 ? 4 : avg <= 48 ? 8 : avg <= 96 ? 16 : 32;
}

static int lin_grid(int64_t work) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((work + kLinBlock - 1) / kLinBlock,
                                                     (int64_t)sm_count() * 8));
}

}  // namespace op2b

using namespace op2b;

extern "C" {

int op2b_csr_spmv(uint64_t rowptr, uint64_t colidx, uint64_t vals, int32_t nrows, int64_t nnz,
                  uint64_t x, uint64_t y, double alpha, double beta, int32_t group,
                  uint64_t stream) {
  OP2B_REQUIRE_INIT();
  if (nrows < 0 || nnz < 0) return set_error(OP2B_ERR_ARG, "op2b_csr_spmv: bad sizes");
  if (group != 0 && group != 1 && group != 2 && group != 4 && group != 8 && group != 16 &&
      group != 32)
    return set_error(OP2B_ERR_ARG, "op2b_csr_spmv: group %d (0 or a power of two up to 32)",
                     group);
  if (nrows == 0) return OP2B_OK;
  const int G = group ? group : group_for(nnz, nrows);
  const int grid = lin_grid((int64_t)nrows * G);
  cudaStream_t s = stream_of(stream);
  auto rp = (const int32_t *)rowptr;
  auto ci = (const int32_t *)colidx;
  auto v = (const double *)vals;
  switch (G) {
    case 1: spmv_kernel<1><<<grid, kLinBlock, 0, s>>>(rp, ci, v, nrows, (const double *)x, (double *)y, alpha, beta); break;
    case 2: spmv_kernel<2><<<grid, kLinBlock, 0, s>>>(rp, ci, v, nrows, (const double *)x, (double *)y, alpha, beta); break;
    case 4: spmv_kernel<4><<<grid, kLinBlock, 0, s>>>(rp, ci, v, nrows, (const double *)x, (double *)y, alpha, beta); break;
    case 8: spmv_kernel<8><<<grid, kLinBlock, 0, s>>>(rp, ci, v, nrows, (const double *)x, (double *)y, alpha, beta); break;
    case 16: spmv_kernel<16><<<grid, kLinBlock, 0, s>>>(rp, ci, v, nrows, (const double *)x, (double *)y, alpha, beta); break;
    default: spmv_kernel<32><<<grid, kLinBlock, 0, s>>>(rp, ci, v, nrows, (const double *)x, (double *)y, alpha, beta); break;
  }
  return check_cuda(cudaGetLastError(), "spmv_kernel");
}

int op2b_vec_binop(uint64_t out, uint64_t x, uint64_t y, double yscalar, int64_t n, int32_t op,
                   int32_t dtype, uint64_t stream) {
  OP2B_REQUIRE_INIT();
  if (n < 0 || op < 0 || op > 3) return set_error(OP2B_ERR_ARG, "op2b_vec_binop: bad arguments");
  if (n == 0) return OP2B_OK;
  cudaStream_t s = stream_of(stream);
  const int grid = lin_grid(n);
  switch (dtype) {
    case 0:
      binop_kernel<double><<<grid, kLinBlock, 0, s>>>((double *)out, (const double *)x,
                                                      (const double *)y, yscalar, n, op);
      break;
    case 1:
      binop_kernel<float><<<grid, kLinBlock, 0, s>>>((float *)out, (const float *)x,
                                                     (const float *)y, (float)yscalar, n, op);
      break;
    case 2:
      binop_kernel<int32_t><<<grid, kLinBlock, 0, s>>>((int32_t *)out, (const int32_t *)x,
                                                       (const int32_t *)y, (int32_t)yscalar, n, op);
      break;
    default:
      return set_error(OP2B_ERR_ARG, "op2b_vec_binop: dtype %d", dtype);
  }
  return check_cuda(cudaGetLastError(), "binop_kernel");
}

int op2b_vec_dot(uint64_t x, uint64_t y, int64_t n, double *result, uint64_t stream) {
  OP2B_REQUIRE_INIT();
  if (n < 0 || !result) return set_error(OP2B_ERR_ARG, "op2b_vec_dot: bad arguments");
  cudaStream_t s = stream_of(stream);
  const int grid = lin_grid(n);
  double *part = nullptr;
  int rc = dev_alloc((void **)&part, sizeof(double) * (grid + 1), s);
  if (rc) return rc;
  dot_partial_kernel<<<grid, kLinBlock, 0, s>>>((const double *)x, (const double *)y, n, part);
  sum_partials_kernel<<<1, kLinBlock, 0, s>>>(part, grid, part + grid);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(result, part + grid, sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  dev_free(part, s);
  return check_cuda(e, "op2b_vec_dot");
}

int op2b_cg_solve(uint64_t rowptr, uint64_t colidx, uint64_t vals, int32_t nrows, int64_t nnz,
                  uint64_t x, uint64_t b, int32_t jacobi, double rtol, double atol, double dtol,
                  int32_t max_it, int32_t *iterations, int32_t *reason, double *history,
                  uint64_t stream) {
  OP2B_REQUIRE_INIT();
  if (nrows < 0 || nnz < 0 || max_it < 0 || !iterations || !reason)
    return set_error(OP2B_ERR_ARG, "op2b_cg_solve: bad arguments");
  *iterations = 0;
  *reason = 1;
  if (nrows == 0) return OP2B_OK;
  cudaStream_t st = stream_of(stream);
  CgState s{};
  s.n = nrows;
  s.grid = lin_grid(nrows);
  s.x = (double *)x;
  s.b = (const double *)b;
  const int G = group_for(nnz, nrows);
  const int sgrid = lin_grid((int64_t)nrows * G);      // CTAs of the SpMV step
  const size_t pmax = (size_t)std::max(s.grid, sgrid);  // partials per array
  const size_t nv = (size_t)nrows;
  double *work = nullptr;
  int *flags = nullptr;
  const size_t nwork = 5 * nv + 3 * pmax + (size_t)(max_it + 2) + (size_t)(max_it + 1) + 2;
  int rc = dev_alloc((void **)&work, sizeof(double) * nwork, st);
  if (!rc) rc = dev_alloc((void **)&flags, sizeof(int) * 2, st);
  if (rc) {
    dev_free(work, st);
    return rc;
  }
  double *w = work;
  s.r = w; w += nv;
  s.z = w; w += nv;
  s.p = w; w += nv;
  s.q = w; w += nv;
  s.dinv = w; w += nv;
  s.part_pq = w; w += pmax;
  s.part_rz = w; w += pmax;
  s.part_zz = w; w += pmax;
  s.rz = w; w += max_it + 2;
  s.hist = w; w += max_it + 1;
  s.ttol = w;
  s.stop = flags;
  auto rp = (const int32_t *)rowptr;
  auto ci = (const int32_t *)colidx;
  auto v = (const double *)vals;
  if (jacobi) {
    diag_inv_kernel<<<lin_grid(nrows), kLinBlock, 0, st>>>(rp, ci, v, nrows, s.dinv);
  } else {
    // no preconditioner: dinv = 0 + 1
    cudaMemsetAsync(s.dinv, 0, sizeof(double) * nv, st);
    binop_kernel<double><<<lin_grid(nrows), kLinBlock, 0, st>>>(s.dinv, s.dinv, nullptr, 1.0,
                                                                nrows, 0);
  }
  cg_init_kernel<<<s.grid, kLinBlock, 0, st>>>(s);
  cg_init_finish_kernel<<<1, kLinBlock, 0, st>>>(s, rtol, atol, dtol);
  // the update step combines the SpMV's sgrid partials of p.q; the direction
  // step combines the update's s.grid partials of r.z and z.z
  CgState sq = s;
  sq.grid = sgrid;
  int host_stop[2] = {0, 0};
  const int chunk = 16;   // steps launched between two looks at the stop flag
  cudaError_t e = cudaGetLastError();
  int k = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(host_stop, flags, sizeof host_stop, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  while (e == cudaSuccess && host_stop[0] == 0 && k < max_it) {
    const int kend = std::min(max_it, k + chunk);
    for (; k < kend; ++k) {
      switch (G) {
        case 4: cg_spmv_kernel<4><<<sgrid, kLinBlock, 0, st>>>(sq, rp, ci, v); break;
        case 8: cg_spmv_kernel<8><<<sgrid, kLinBlock, 0, st>>>(sq, rp, ci, v); break;
        case 16: cg_spmv_kernel<16><<<sgrid, kLinBlock, 0, st>>>(sq, rp, ci, v); break;
        default: cg_spmv_kernel<32><<<sgrid, kLinBlock, 0, st>>>(sq, rp, ci, v); break;
      }
      cg_update_kernel<<<s.grid, kLinBlock, 0, st>>>(sq, k);
      cg_direction_kernel<<<s.grid, kLinBlock, 0, st>>>(s, k, max_it);
    }
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(host_stop, flags, sizeof host_stop, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  if (e == cudaSuccess) {
    *reason = host_stop[0] == 0 ? 4 : host_stop[0];
    *iterations = host_stop[0] == 0 ? k : host_stop[1];
    if (history) {
      const int nh = *iterations + 1;
      e = cudaMemcpyAsync(history, s.hist, sizeof(double) * nh, cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
  }
  dev_free(work, st);
  dev_free(flags, st);
  return check_cuda(e, "op2b_cg_solve");
}

}  // extern "C"
