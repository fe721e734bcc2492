// libop2b200 runtime: context, device memory, streams/events/graphs, NVRTC
// JIT modules and launches.  See include/op2b200.h for the contract.
#include <cuda_runtime.h>
#include <nvrtc.h>

#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "op2b_internal.h"

namespace op2b {

static thread_local std::string g_last_error;
static bool g_init = false;
static int g_device = -1;
static cudaStream_t g_stream = nullptr;
static int g_sm_count = 0;
static int g_smem_optin = 0;
// Generated stubs launched through op2b_launch / op2b_launch_colored may
// start while the previous kernel on the stream drains (programmatic
// dependent launch); every stub waits for its predecessor's completion
// (griddepcontrol.wait) before it touches memory.
static bool g_programmatic = false;
static std::mutex g_init_mutex;

int set_error(int code, const char *fmt, ...) {
  char buf[2048];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int check_cuda(cudaError_t err, const char *what) {
  if (err == cudaSuccess) return OP2B_OK;
  int code = (err == cudaErrorMemoryAllocation) ? OP2B_ERR_NOMEM : OP2B_ERR_CUDA;
  return set_error(code, "%s failed: %s (%s)", what, cudaGetErrorString(err),
                   cudaGetErrorName(err));
}

bool initialised() { return g_init; }
cudaStream_t stream_of(uint64_t s) { return s ? reinterpret_cast<cudaStream_t>(s) : g_stream; }
int sm_count() { return g_sm_count; }
int smem_optin() { return g_smem_optin; }

int dev_alloc(void **p, size_t bytes, cudaStream_t s) {
  *p = nullptr;
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMallocAsync(p, bytes, s);
  if (e != cudaSuccess) return check_cuda(e, "cudaMallocAsync");
  return OP2B_OK;
}

void dev_free(void *p, cudaStream_t s) {
  if (p) cudaFreeAsync(p, s);
}

// [n][dim] <-> [dim][n]; one thread per element row, elements of E bytes.
template <typename T>
__global__ void transpose_kernel(T *__restrict__ dst, const T *__restrict__ src, int64_t n,
                                 int dim, int to_soa) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    for (int k = 0; k < dim; ++k) {
      if (to_soa)
        dst[k * n + i] = src[i * dim + k];
      else
        dst[i * dim + k] = src[k * n + i];
    }
  }
}

// Host bytes carried by value in the launch parameters: a small upload that
// needs no staging buffer and never waits for the stream.
struct SmallBytes {
  unsigned char b[256];
};

__global__ void small_copy_kernel(unsigned char *__restrict__ dst, SmallBytes v, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = v.b[i];
}

// Writes the smallest offending position (or INT64_MAX) to *bad.
__global__ void map_validate_kernel(const int32_t *__restrict__ map, int64_t n, int32_t to_size,
                                    unsigned long long *bad) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int32_t v = map[i];
    if (v < 0 || v >= to_size) atomicMin(bad, (unsigned long long)i);
  }
}

// The graph's nodes in chain order; fails unless every node has at most one
// dependency and one dependent and there is one root.
int graph_chain(cudaGraph_t g, std::vector<cudaGraphNode_t> &chain) {
  size_t n = 0;
  OP2B_CUDA(cudaGraphGetNodes(g, nullptr, &n));
  chain.clear();
  if (!n) return OP2B_OK;
  size_t nr = 0;
  OP2B_CUDA(cudaGraphGetRootNodes(g, nullptr, &nr));
  if (nr != 1) return set_error(OP2B_ERR_STATE, "graph: %zu roots, not a chain", nr);
  cudaGraphNode_t cur = nullptr;
  OP2B_CUDA(cudaGraphGetRootNodes(g, &cur, &nr));
  chain.reserve(n);
  while (cur) {
    chain.push_back(cur);
    if (chain.size() > n) return set_error(OP2B_ERR_STATE, "graph: cycle");
    size_t nd = 0;
    OP2B_CUDA(cudaGraphNodeGetDependentNodes(cur, nullptr, &nd));
    if (nd > 1) return set_error(OP2B_ERR_STATE, "graph: node with %zu dependents", nd);
    cudaGraphNode_t next = nullptr;
    if (nd) OP2B_CUDA(cudaGraphNodeGetDependentNodes(cur, &next, &nd));
    cur = nd ? next : nullptr;
  }
  if (chain.size() != n) return set_error(OP2B_ERR_STATE, "graph: %zu of %zu nodes on the chain",
                                          chain.size(), n);
  return OP2B_OK;
}

}  // namespace op2b

using namespace op2b;

extern "C" {

int op2b_version(void) { return 1; }

int op2b_last_error(char *buf, size_t len) {
  if (!buf || len == 0) return OP2B_ERR_ARG;
  std::snprintf(buf, len, "%s", g_last_error.c_str());
  return OP2B_OK;
}

int op2b_init(int device) {
  std::lock_guard<std::mutex> lock(g_init_mutex);
  if (g_init) {
    if (device != g_device)
      return set_error(OP2B_ERR_STATE, "already initialised on device %d", g_device);
    return OP2B_OK;
  }
  int n = 0;
  OP2B_CUDA(cudaGetDeviceCount(&n));
  if (device < 0 || device >= n)
    return set_error(OP2B_ERR_ARG, "device %d out of range (%d devices)", device, n);
  OP2B_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  OP2B_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10)
    return set_error(OP2B_ERR_STATE,
                     "device %d is sm_%d%d; this library is built for sm_100a (B200)",
                     device, prop.major, prop.minor);
  g_sm_count = prop.multiProcessorCount;
  g_smem_optin = (int)prop.sharedMemPerBlockOptin;
  OP2B_CUDA(cudaStreamCreateWithFlags(&g_stream, cudaStreamNonBlocking));
  // Keep freed stream-ordered memory in the pool instead of returning it to
  // the driver at every synchronisation: Globals and scratch are recycled.
  cudaMemPool_t pool;
  OP2B_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
  uint64_t threshold = UINT64_MAX;
  OP2B_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
  g_device = device;
  g_init = true;
  return OP2B_OK;
}

int op2b_shutdown(void) {
  std::lock_guard<std::mutex> lock(g_init_mutex);
  if (!g_init) return OP2B_OK;
  cudaStreamSynchronize(g_stream);
  cudaStreamDestroy(g_stream);
  g_stream = nullptr;
  g_init = false;
  return OP2B_OK;
}

int op2b_device_info(int32_t *sm, int32_t *smem, int32_t *major, int32_t *minor,
                     uint64_t *total_mem, uint64_t *l2_bytes) {
  OP2B_REQUIRE_INIT();
  cudaDeviceProp prop;
  OP2B_CUDA(cudaGetDeviceProperties(&prop, g_device));
  if (sm) *sm = prop.multiProcessorCount;
  if (smem) *smem = (int32_t)prop.sharedMemPerBlockOptin;
  if (major) *major = prop.major;
  if (minor) *minor = prop.minor;
  if (total_mem) *total_mem = prop.totalGlobalMem;
  if (l2_bytes) *l2_bytes = prop.l2CacheSize;
  return OP2B_OK;
}

int op2b_set_l2_fetch_granularity(int32_t bytes) {
  OP2B_REQUIRE_INIT();
  if (bytes != 32 && bytes != 64 && bytes != 128)
    return set_error(OP2B_ERR_ARG, "L2 fetch granularity %d (32, 64 or 128)", bytes);
  OP2B_CUDA(cudaDeviceSetLimit(cudaLimitMaxL2FetchGranularity, (size_t)bytes));
  return OP2B_OK;
}

// ---------------------------------------------------------------- memory
int op2b_malloc(uint64_t *dptr, uint64_t bytes) {
  OP2B_REQUIRE_INIT();
  if (!dptr) return set_error(OP2B_ERR_ARG, "op2b_malloc: null out pointer");
  void *p = nullptr;
  int rc = dev_alloc(&p, bytes, g_stream);
  if (rc) return rc;
  *dptr = reinterpret_cast<uint64_t>(p);
  return OP2B_OK;
}

int op2b_free(uint64_t dptr) {
  OP2B_REQUIRE_INIT();
  if (dptr) OP2B_CUDA(cudaFreeAsync(reinterpret_cast<void *>(dptr), g_stream));
  return OP2B_OK;
}

int op2b_host_alloc(uint64_t *hptr, uint64_t bytes) {
  OP2B_REQUIRE_INIT();
  void *p = nullptr;
  OP2B_CUDA(cudaMallocHost(&p, bytes ? bytes : 16));
  *hptr = reinterpret_cast<uint64_t>(p);
  return OP2B_OK;
}

int op2b_host_free(uint64_t hptr) {
  OP2B_REQUIRE_INIT();
  if (hptr) OP2B_CUDA(cudaFreeHost(reinterpret_cast<void *>(hptr)));
  return OP2B_OK;
}

int op2b_memcpy_h2d(uint64_t dst, const void *src, uint64_t bytes, uint64_t stream) {
  OP2B_REQUIRE_INIT();
  if (!bytes) return OP2B_OK;
  OP2B_CUDA(cudaMemcpyAsync(reinterpret_cast<void *>(dst), src, bytes,
                            cudaMemcpyHostToDevice, stream_of(stream)));
  return OP2B_OK;
}

int op2b_memcpy_d2h(void *dst, uint64_t src, uint64_t bytes, uint64_t stream) {
  OP2B_REQUIRE_INIT();
  if (!bytes) return OP2B_OK;
  cudaStream_t s = stream_of(stream);
  OP2B_CUDA(cudaMemcpyAsync(dst, reinterpret_cast<const void *>(src), bytes,
                            cudaMemcpyDeviceToHost, s));
  OP2B_CUDA(cudaStreamSynchronize(s));
  return OP2B_OK;
}

int op2b_memcpy_h2d_small(uint64_t dst, const void *src, uint64_t bytes, uint64_t stream) {
  OP2B_REQUIRE_INIT();
  if (bytes > sizeof(SmallBytes::b))
    return set_error(OP2B_ERR_ARG, "op2b_memcpy_h2d_small: %llu bytes (at most %zu)",
                     (unsigned long long)bytes, sizeof(SmallBytes::b));
  if (!bytes) return OP2B_OK;
  SmallBytes v;
  std::memcpy(v.b, src, bytes);
  small_copy_kernel<<<1, 64, 0, stream_of(stream)>>>(reinterpret_cast<unsigned char *>(dst), v,
                                                    static_cast<int>(bytes));
  return check_cuda(cudaGetLastError(), "small_copy_kernel");
}

int op2b_memcpy_d2h_async(void *dst, uint64_t src, uint64_t bytes, uint64_t stream) {
  OP2B_REQUIRE_INIT();
  if (!bytes) return OP2B_OK;
  OP2B_CUDA(cudaMemcpyAsync(dst, reinterpret_cast<const void *>(src), bytes,
                            cudaMemcpyDeviceToHost, stream_of(stream)));
  return OP2B_OK;
}

int op2b_memcpy_d2d(uint64_t dst, uint64_t src, uint64_t bytes, uint64_t stream) {
  OP2B_REQUIRE_INIT();
  if (!bytes) return OP2B_OK;
  OP2B_CUDA(cudaMemcpyAsync(reinterpret_cast<void *>(dst), reinterpret_cast<const void *>(src),
                            bytes, cudaMemcpyDeviceToDevice, stream_of(stream)));
  return OP2B_OK;
}

int op2b_memset(uint64_t dst, int value, uint64_t bytes, uint64_t stream) {
  OP2B_REQUIRE_INIT();
  if (!bytes) return OP2B_OK;
  OP2B_CUDA(cudaMemsetAsync(reinterpret_cast<void *>(dst), value, bytes, stream_of(stream)));
  return OP2B_OK;
}

int op2b_transpose(uint64_t dst, uint64_t src, int64_t n, int32_t dim, int32_t elem_bytes,
                   int32_t to_soa, uint64_t stream) {
  OP2B_REQUIRE_INIT();
  if (n <= 0) return OP2B_OK;
  cudaStream_t s = stream_of(stream);
  int grid = (int)std::min<int64_t>((n + 255) / 256, (int64_t)g_sm_count * 8);
  switch (elem_bytes) {
    case 1: transpose_kernel<uint8_t><<<grid, 256, 0, s>>>((uint8_t *)dst, (const uint8_t *)src, n, dim, to_soa); break;
    case 2: transpose_kernel<uint16_t><<<grid, 256, 0, s>>>((uint16_t *)dst, (const uint16_t *)src, n, dim, to_soa); break;
    case 4: transpose_kernel<uint32_t><<<grid, 256, 0, s>>>((uint32_t *)dst, (const uint32_t *)src, n, dim, to_soa); break;
    case 8: transpose_kernel<uint64_t><<<grid, 256, 0, s>>>((uint64_t *)dst, (const uint64_t *)src, n, dim, to_soa); break;
    default: return set_error(OP2B_ERR_ARG, "op2b_transpose: elem_bytes %d", elem_bytes);
  }
  OP2B_CUDA(cudaGetLastError());
  return OP2B_OK;
}

int op2b_map_validate(uint64_t map, int64_t n_values, int32_t to_size, int64_t *bad_index,
                      uint64_t stream) {
  OP2B_REQUIRE_INIT();
  if (bad_index) *bad_index = -1;
  if (n_values <= 0) return OP2B_OK;
  cudaStream_t s = stream_of(stream);
  unsigned long long *d_bad = nullptr;
  int rc = dev_alloc((void **)&d_bad, sizeof(unsigned long long), s);
  if (rc) return rc;
  OP2B_CUDA(cudaMemsetAsync(d_bad, 0xff, sizeof(unsigned long long), s));
  int grid = (int)std::min<int64_t>((n_values + 255) / 256, (int64_t)g_sm_count * 8);
  map_validate_kernel<<<grid, 256, 0, s>>>((const int32_t *)map, n_values, to_size, d_bad);
  unsigned long long h_bad = 0;
  cudaError_t e = cudaMemcpyAsync(&h_bad, d_bad, sizeof h_bad, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  dev_free(d_bad, s);
  if (e != cudaSuccess) return check_cuda(e, "op2b_map_validate");
  if (h_bad != ~0ull) {
    if (bad_index) *bad_index = (int64_t)h_bad;
    return set_error(OP2B_ERR_MAP, "map value at flat position %lld outside [0, %d)",
                     (long long)h_bad, to_size);
  }
  return OP2B_OK;
}

// ------------------------------------------------------ streams and events
int op2b_default_stream(uint64_t *stream) {
  OP2B_REQUIRE_INIT();
  *stream = reinterpret_cast<uint64_t>(g_stream);
  return OP2B_OK;
}

int op2b_stream_create(uint64_t *stream) {
  OP2B_REQUIRE_INIT();
  cudaStream_t s;
  OP2B_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  *stream = reinterpret_cast<uint64_t>(s);
  return OP2B_OK;
}

int op2b_stream_destroy(uint64_t stream) {
  OP2B_REQUIRE_INIT();
  if (stream) OP2B_CUDA(cudaStreamDestroy(reinterpret_cast<cudaStream_t>(stream)));
  return OP2B_OK;
}

int op2b_stream_sync(uint64_t stream) {
  OP2B_REQUIRE_INIT();
  OP2B_CUDA(cudaStreamSynchronize(stream_of(stream)));
  return OP2B_OK;
}

int op2b_device_sync(void) {
  OP2B_REQUIRE_INIT();
  OP2B_CUDA(cudaDeviceSynchronize());
  return OP2B_OK;
}

int op2b_event_create(uint64_t *event) {
  OP2B_REQUIRE_INIT();
  cudaEvent_t e;
  OP2B_CUDA(cudaEventCreate(&e));
  *event = reinterpret_cast<uint64_t>(e);
  return OP2B_OK;
}

int op2b_event_destroy(uint64_t event) {
  OP2B_REQUIRE_INIT();
  if (event) OP2B_CUDA(cudaEventDestroy(reinterpret_cast<cudaEvent_t>(event)));
  return OP2B_OK;
}

int op2b_event_record(uint64_t event, uint64_t stream) {
  OP2B_REQUIRE_INIT();
  OP2B_CUDA(cudaEventRecord(reinterpret_cast<cudaEvent_t>(event), stream_of(stream)));
  return OP2B_OK;
}

int op2b_event_record_node(uint64_t event, uint64_t stream) {
  OP2B_REQUIRE_INIT();
  OP2B_CUDA(cudaEventRecordWithFlags(reinterpret_cast<cudaEvent_t>(event), stream_of(stream),
                                     cudaEventRecordExternal));
  return OP2B_OK;
}

int op2b_event_sync(uint64_t event) {
  OP2B_REQUIRE_INIT();
  OP2B_CUDA(cudaEventSynchronize(reinterpret_cast<cudaEvent_t>(event)));
  return OP2B_OK;
}

int op2b_event_query(uint64_t event, int32_t *done) {
  OP2B_REQUIRE_INIT();
  if (!done) return set_error(OP2B_ERR_ARG, "op2b_event_query: null out pointer");
  cudaError_t e = cudaEventQuery(reinterpret_cast<cudaEvent_t>(event));
  if (e == cudaErrorNotReady) {
    *done = 0;
    return OP2B_OK;
  }
  OP2B_CUDA(e);
  *done = 1;
  return OP2B_OK;
}

int op2b_event_elapsed_ms(uint64_t start, uint64_t stop, float *ms) {
  OP2B_REQUIRE_INIT();
  OP2B_CUDA(cudaEventElapsedTime(ms, reinterpret_cast<cudaEvent_t>(start),
                                 reinterpret_cast<cudaEvent_t>(stop)));
  return OP2B_OK;
}

int op2b_stream_wait_event(uint64_t stream, uint64_t event) {
  OP2B_REQUIRE_INIT();
  OP2B_CUDA(cudaStreamWaitEvent(stream_of(stream), reinterpret_cast<cudaEvent_t>(event), 0));
  return OP2B_OK;
}

int op2b_graph_begin(uint64_t stream) {
  OP2B_REQUIRE_INIT();
  OP2B_CUDA(cudaStreamBeginCapture(stream_of(stream), cudaStreamCaptureModeRelaxed));
  return OP2B_OK;
}

int op2b_graph_end(uint64_t stream, uint64_t *graph_exec) {
  OP2B_REQUIRE_INIT();
  cudaGraph_t g = nullptr;
  OP2B_CUDA(cudaStreamEndCapture(stream_of(stream), &g));
  cudaGraphExec_t ge = nullptr;
  cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return check_cuda(e, "cudaGraphInstantiate");
  *graph_exec = reinterpret_cast<uint64_t>(ge);
  return OP2B_OK;
}

// ---- overlapped capture: a capture on one stream records a linear chain of
// nodes; the host marks the chain's tail around each par_loop, computes which
// loops must follow which from their accesses, and the chain edges between
// independent loops are replaced by those dependencies before instantiation.
int op2b_graph_capture_tail(uint64_t stream, uint64_t *node) {
  OP2B_REQUIRE_INIT();
  if (!node) return set_error(OP2B_ERR_ARG, "op2b_graph_capture_tail: null");
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  const cudaGraphNode_t *deps = nullptr;
  size_t nd = 0;
  OP2B_CUDA(cudaStreamGetCaptureInfo(stream_of(stream), &st, nullptr, nullptr, &deps, &nd));
  if (st != cudaStreamCaptureStatusActive)
    return set_error(OP2B_ERR_STATE, "op2b_graph_capture_tail: the stream is not capturing");
  if (nd > 1)
    return set_error(OP2B_ERR_STATE, "op2b_graph_capture_tail: the capture has %zu tails", nd);
  *node = nd ? reinterpret_cast<uint64_t>(deps[0]) : 0;
  return OP2B_OK;
}

int op2b_graph_end_capture(uint64_t stream, uint64_t *graph) {
  OP2B_REQUIRE_INIT();
  if (!graph) return set_error(OP2B_ERR_ARG, "op2b_graph_end_capture: null");
  cudaGraph_t g = nullptr;
  OP2B_CUDA(cudaStreamEndCapture(stream_of(stream), &g));
  *graph = reinterpret_cast<uint64_t>(g);
  return OP2B_OK;
}


int op2b_graph_chain_positions(uint64_t graph, const uint64_t *marks, int32_t nmarks,
                               int64_t *pos, int64_t *nnodes) {
  OP2B_REQUIRE_INIT();
  if (!graph || nmarks < 0 || (nmarks && (!marks || !pos)) || !nnodes)
    return set_error(OP2B_ERR_ARG, "op2b_graph_chain_positions: bad arguments");
  std::vector<cudaGraphNode_t> chain;
  int rc = graph_chain(reinterpret_cast<cudaGraph_t>(graph), chain);
  if (rc) return rc;
  *nnodes = (int64_t)chain.size();
  std::unordered_map<uint64_t, int64_t> at;
  for (size_t k = 0; k < chain.size(); ++k) at[reinterpret_cast<uint64_t>(chain[k])] = (int64_t)k;
  for (int32_t m = 0; m < nmarks; ++m) {
    if (!marks[m]) {
      pos[m] = -1;
      continue;
    }
    auto it = at.find(marks[m]);
    if (it == at.end()) return set_error(OP2B_ERR_STATE, "graph: mark %d is not a node", m);
    pos[m] = it->second;
  }
  return OP2B_OK;
}

int op2b_graph_relax(uint64_t graph, const int64_t *seg_first, const int64_t *seg_last,
                     int32_t nseg, const int32_t *dep_ptr, const int32_t *dep_idx,
                     uint64_t *graph_exec) {
  OP2B_REQUIRE_INIT();
  if (!graph || !graph_exec || nseg < 0 || (nseg && (!seg_first || !seg_last || !dep_ptr)))
    return set_error(OP2B_ERR_ARG, "op2b_graph_relax: bad arguments");
  cudaGraph_t g = reinterpret_cast<cudaGraph_t>(graph);
  if (nseg) {
    std::vector<cudaGraphNode_t> chain;
    int rc = graph_chain(g, chain);
    if (rc) return rc;
    const int64_t n = (int64_t)chain.size();
    // the segments tile the chain in order
    int64_t expect = 0;
    for (int32_t s = 0; s < nseg; ++s) {
      if (seg_first[s] != expect || seg_last[s] < seg_first[s] || seg_last[s] >= n)
        return set_error(OP2B_ERR_ARG, "op2b_graph_relax: segment %d [%lld, %lld] does not tile "
                         "the chain of %lld nodes", s, (long long)seg_first[s],
                         (long long)seg_last[s], (long long)n);
      expect = seg_last[s] + 1;
      for (int32_t k = dep_ptr[s]; k < dep_ptr[s + 1]; ++k)
        if (dep_idx[k] < 0 || dep_idx[k] >= s)
          return set_error(OP2B_ERR_ARG, "op2b_graph_relax: segment %d depends on %d", s,
                           dep_idx[k]);
    }
    if (expect != n)
      return set_error(OP2B_ERR_ARG, "op2b_graph_relax: segments cover %lld of %lld nodes",
                       (long long)expect, (long long)n);
    std::vector<cudaGraphNode_t> from, to;
    for (int32_t s = 1; s < nseg; ++s) {
      cudaGraphNode_t first = chain[seg_first[s]], prev = chain[seg_first[s] - 1];
      OP2B_CUDA(cudaGraphRemoveDependencies(g, &prev, &first, 1));
      for (int32_t k = dep_ptr[s]; k < dep_ptr[s + 1]; ++k) {
        from.push_back(chain[seg_last[dep_idx[k]]]);
        to.push_back(first);
      }
    }
    if (!from.empty()) OP2B_CUDA(cudaGraphAddDependencies(g, from.data(), to.data(), from.size()));
  }
  cudaGraphExec_t ge = nullptr;
  cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
  if (e != cudaSuccess) return check_cuda(e, "cudaGraphInstantiate");
  *graph_exec = reinterpret_cast<uint64_t>(ge);
  return OP2B_OK;
}

int op2b_graph_free(uint64_t graph) {
  OP2B_REQUIRE_INIT();
  if (graph) OP2B_CUDA(cudaGraphDestroy(reinterpret_cast<cudaGraph_t>(graph)));
  return OP2B_OK;
}

int op2b_graph_launch(uint64_t graph_exec, uint64_t stream) {
  OP2B_REQUIRE_INIT();
  OP2B_CUDA(cudaGraphLaunch(reinterpret_cast<cudaGraphExec_t>(graph_exec), stream_of(stream)));
  return OP2B_OK;
}

int op2b_graph_destroy(uint64_t graph_exec) {
  OP2B_REQUIRE_INIT();
  if (graph_exec) OP2B_CUDA(cudaGraphExecDestroy(reinterpret_cast<cudaGraphExec_t>(graph_exec)));
  return OP2B_OK;
}

// -------------------------------------------------------- NVRTC / modules
int op2b_nvrtc_compile(const char *src, const char *name, const char *const *opts, int32_t nopts,
                       void **cubin, uint64_t *cubin_bytes, char *log, uint64_t log_len) {
  if (!src || !cubin || !cubin_bytes) return set_error(OP2B_ERR_ARG, "op2b_nvrtc_compile: null");
  *cubin = nullptr;
  *cubin_bytes = 0;
  if (log && log_len) log[0] = 0;
  nvrtcProgram prog;
  nvrtcResult r = nvrtcCreateProgram(&prog, src, name ? name : "op2b_stub.cu", 0, nullptr, nullptr);
  if (r != NVRTC_SUCCESS)
    return set_error(OP2B_ERR_NVRTC, "nvrtcCreateProgram: %s", nvrtcGetErrorString(r));
  r = nvrtcCompileProgram(prog, nopts, opts);
  size_t lsz = 0;
  nvrtcGetProgramLogSize(prog, &lsz);
  std::string plog(lsz, '\0');
  if (lsz) nvrtcGetProgramLog(prog, &plog[0]);
  if (log && log_len) std::snprintf(log, log_len, "%s", plog.c_str());
  if (r != NVRTC_SUCCESS) {
    nvrtcDestroyProgram(&prog);
    return set_error(OP2B_ERR_NVRTC, "nvrtcCompileProgram: %s\n%s", nvrtcGetErrorString(r),
                     plog.c_str());
  }
  size_t csz = 0;
  r = nvrtcGetCUBINSize(prog, &csz);
  if (r != NVRTC_SUCCESS || csz == 0) {
    nvrtcDestroyProgram(&prog);
    return set_error(OP2B_ERR_NVRTC, "nvrtcGetCUBINSize: %s (compile for a real sm_ arch)",
                     nvrtcGetErrorString(r));
  }
  void *buf = std::malloc(csz);
  if (!buf) {
    nvrtcDestroyProgram(&prog);
    return set_error(OP2B_ERR_NOMEM, "cubin buffer");
  }
  nvrtcGetCUBIN(prog, (char *)buf);
  nvrtcDestroyProgram(&prog);
  *cubin = buf;
  *cubin_bytes = csz;
  return OP2B_OK;
}

int op2b_cubin_free(void *cubin) {
  std::free(cubin);
  return OP2B_OK;
}

int op2b_module_load(const void *cubin, uint64_t *module) {
  OP2B_REQUIRE_INIT();
  cudaLibrary_t lib;
  OP2B_CUDA(cudaLibraryLoadData(&lib, cubin, nullptr, nullptr, 0, nullptr, nullptr, 0));
  *module = reinterpret_cast<uint64_t>(lib);
  return OP2B_OK;
}

int op2b_module_unload(uint64_t module) {
  OP2B_REQUIRE_INIT();
  if (module) OP2B_CUDA(cudaLibraryUnload(reinterpret_cast<cudaLibrary_t>(module)));
  return OP2B_OK;
}

int op2b_module_function(uint64_t module, const char *name, uint64_t *fn) {
  OP2B_REQUIRE_INIT();
  cudaKernel_t k;
  OP2B_CUDA(cudaLibraryGetKernel(&k, reinterpret_cast<cudaLibrary_t>(module), name));
  *fn = reinterpret_cast<uint64_t>(k);
  return OP2B_OK;
}

int op2b_module_global(uint64_t module, const char *name, uint64_t *dptr, uint64_t *bytes) {
  OP2B_REQUIRE_INIT();
  void *p = nullptr;
  size_t sz = 0;
  OP2B_CUDA(cudaLibraryGetGlobal(&p, &sz, reinterpret_cast<cudaLibrary_t>(module), name));
  *dptr = reinterpret_cast<uint64_t>(p);
  if (bytes) *bytes = sz;
  return OP2B_OK;
}

int op2b_function_set_smem(uint64_t fn, int32_t bytes) {
  OP2B_REQUIRE_INIT();
  if (bytes > g_smem_optin)
    return set_error(OP2B_ERR_ARG, "dynamic shared memory %d exceeds the device limit %d", bytes,
                     g_smem_optin);
  OP2B_CUDA(cudaFuncSetAttribute(reinterpret_cast<const void *>(fn),
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  return OP2B_OK;
}

int op2b_function_occupancy(uint64_t fn, uint32_t block, uint32_t smem, int32_t *blocks_per_sm) {
  OP2B_REQUIRE_INIT();
  if (!blocks_per_sm || block == 0) return set_error(OP2B_ERR_ARG, "bad occupancy query");
  int n = 0;
  OP2B_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, reinterpret_cast<const void *>(fn),
                                                          static_cast<int>(block), smem));
  *blocks_per_sm = n;
  return OP2B_OK;
}

// One launch of a generated stub, with the programmatic-serialisation
// attribute when that is on.
static cudaError_t launch_stub(uint64_t fn, uint32_t grid, uint32_t block, uint32_t smem,
                               cudaStream_t s, void **args) {
  if (!g_programmatic)
    return cudaLaunchKernel(reinterpret_cast<const void *>(fn), dim3(grid), dim3(block), args,
                            smem, s);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelExC(&cfg, reinterpret_cast<const void *>(fn), args);
}

int op2b_set_programmatic_launch(int32_t on) {
  OP2B_REQUIRE_INIT();
  g_programmatic = on != 0;
  return OP2B_OK;
}

int op2b_launch(uint64_t fn, uint32_t grid, uint32_t block, uint32_t smem, uint64_t stream,
                const void *params, uint64_t nbytes) {
  OP2B_REQUIRE_INIT();
  (void)nbytes;
  if (grid == 0) return OP2B_OK;
  void *args[1] = {const_cast<void *>(params)};
  OP2B_CUDA(launch_stub(fn, grid, block, smem, stream_of(stream), args));
  return OP2B_OK;
}

int op2b_launch_colored(uint64_t fn, int32_t ncolors, const int32_t *ncolblk, uint32_t block,
                        uint32_t smem, uint64_t stream, void *params, uint64_t nbytes,
                        uint64_t col_field_offset) {
  OP2B_REQUIRE_INIT();
  if (col_field_offset + 2 * sizeof(int32_t) > nbytes)
    return set_error(OP2B_ERR_ARG, "colour field offset outside the parameter block");
  int32_t *fields = reinterpret_cast<int32_t *>(static_cast<char *>(params) + col_field_offset);
  int32_t first = 0;
  void *args[1] = {params};
  for (int c = 0; c < ncolors; ++c) {
    int32_t nb = ncolblk[c];
    if (nb > 0) {
      fields[0] = first;
      fields[1] = nb;
      // The parameter block is copied at launch, so it may be patched for the
      // next colour straight away.
      OP2B_CUDA(launch_stub(fn, nb, block, smem, stream_of(stream), args));
    }
    first += nb;
  }
  return OP2B_OK;
}

}  // extern "C"
