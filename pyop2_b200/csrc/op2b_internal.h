// Host-side internals shared by the translation units of libop2b200.so.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

#include "op2b200.h"

namespace op2b {

// Records msg as the calling thread's last error and returns code.
int set_error(int code, const char *fmt, ...);
int check_cuda(cudaError_t err, const char *what);
bool initialised();
cudaStream_t stream_of(uint64_t s);   // 0 -> the library's default stream
int sm_count();
int smem_optin();

// Stream-ordered device allocation helpers for library-internal scratch.
int dev_alloc(void **p, size_t bytes, cudaStream_t s);
void dev_free(void *p, cudaStream_t s);

}  // namespace op2b

#define OP2B_CUDA(call)                                              \
  do {                                                               \
    cudaError_t _e = (call);                                         \
    if (_e != cudaSuccess) return op2b::check_cuda(_e, #call);       \
  } while (0)

#define OP2B_REQUIRE_INIT()                                          \
  do {                                                               \
    if (!op2b::initialised())                                        \
      return op2b::set_error(OP2B_ERR_STATE, "op2b_init not called"); \
  } while (0)

static inline int op2b_div_up(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }
