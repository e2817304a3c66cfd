// Test infrastructure only: a stand-in CUDA runtime for exercising libbcgpu's
// HOST logic on a machine without a GPU. The library's own objects (built by
// build.py) are linked against this file instead of cudart: "device" memory
// is host memory (filled with a byte pattern when allocated, as cudaMalloc's
// memory is undefined), copies and memsets are memcpy/memset, kernel launches do
// nothing but are counted, stream capture records the stream's copies and
// memsets (and counts its launches) into a replayable list. Eight identical
// fake sm_100 devices with 148 SMs (one per rank under torchrun); memory is
// not per device. Nothing here computes BC: tests built on it check plan
// construction, routing, unit bookkeeping, graph record/replay, argument
// validation and error paths -- never numbers, which the GPU tests pin.
#include <cuda_runtime_api.h>

#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <vector>

namespace {

// Containers are function-local statics: the registration calls below run from
// other objects' static initialisers, possibly before this file's globals exist.
std::mutex g_mu;  // constant-initialised
std::atomic<long long> g_launches{0};
std::atomic<long long> g_live{0};        // device allocations not yet freed
std::atomic<long long> g_mallocs{0};     // device allocation calls so far
std::atomic<long long> g_h2d{0}, g_d2h{0};  // bytes copied host->device, device->host (when executed)
std::atomic<long long> g_fail_after{-1};  // allocations left before one fails (-1: none fails)
std::map<const void *, size_t> &var_size() {  // registered __device__ variables: host shadow -> size
  static std::map<const void *, size_t> m;
  return m;
}
std::map<const void *, void *> &var_storage() {  // their stand-in device storage
  static std::map<const void *, void *> m;
  return m;
}

struct Capture {
  std::vector<std::function<void()>> ops;
  long long launches = 0;
};
std::map<cudaStream_t, Capture *> &capturing() {
  static std::map<cudaStream_t, Capture *> m;
  return m;
}

struct Graph {
  std::vector<std::function<void()>> ops;
  long long launches = 0;
};

// Runs op now, or records it when the stream is being captured.
cudaError_t on_stream(cudaStream_t s, std::function<void()> op) {
  std::lock_guard<std::mutex> lock(g_mu);
  auto it = capturing().find(s);
  if (it != capturing().end()) it->second->ops.push_back(std::move(op));
  else op();
  return cudaSuccess;
}

cudaError_t launch(cudaStream_t s) {
  std::lock_guard<std::mutex> lock(g_mu);
  auto it = capturing().find(s);
  if (it != capturing().end()) ++it->second->launches;
  else ++g_launches;
  return cudaSuccess;
}

thread_local dim3 t_grid, t_block;
thread_local size_t t_smem;
thread_local cudaStream_t t_stream;

}  // namespace

extern "C" {

// ---- test hooks
long long stub_cudart_launches() { return g_launches.load(); }
long long stub_cudart_live_allocs() { return g_live.load(); }
long long stub_cudart_mallocs() { return g_mallocs.load(); }
long long stub_cudart_h2d() { return g_h2d.load(); }
long long stub_cudart_d2h() { return g_d2h.load(); }
// The (n+1)-th device allocation from now on fails (n < 0: none fails).
void stub_cudart_fail_malloc_after(long long n) { g_fail_after = n; }

// ---- module registration (called by nvcc-generated static initialisers)
void **__cudaRegisterFatBinary(void *) {
  static void *handle = nullptr;
  return &handle;
}
void __cudaRegisterFatBinaryEnd(void **) {}
void __cudaUnregisterFatBinary(void **) {}
void __cudaRegisterFunction(void **, const char *, char *, const char *, int, uint3 *, uint3 *, dim3 *, dim3 *, int *) {}
void __cudaRegisterVar(void **, char *hostVar, char *, const char *, int, size_t size, int, int) {
  std::lock_guard<std::mutex> lock(g_mu);
  var_size()[hostVar] = size;
}
unsigned __cudaPushCallConfiguration(dim3 grid, dim3 block, size_t smem, struct CUstream_st *stream) {
  t_grid = grid; t_block = block; t_smem = smem; t_stream = stream;
  return 0;
}
cudaError_t __cudaPopCallConfiguration(dim3 *grid, dim3 *block, size_t *smem, void *stream) {
  *grid = t_grid; *block = t_block; *smem = t_smem; *(cudaStream_t *)stream = t_stream;
  return cudaSuccess;
}

}  // extern "C"

// ---- device and errors
constexpr int kDevices = 8;
thread_local int t_device = 0;
cudaError_t cudaGetDeviceCount(int *count) { *count = kDevices; return cudaSuccess; }
cudaError_t cudaSetDevice(int device) {
  if (device < 0 || device >= kDevices) return cudaErrorInvalidDevice;
  t_device = device;
  return cudaSuccess;
}
cudaError_t cudaGetDevice(int *device) { *device = t_device; return cudaSuccess; }
cudaError_t cudaGetDeviceProperties_v2(cudaDeviceProp *prop, int device) {
  if (device < 0 || device >= kDevices) return cudaErrorInvalidDevice;
  std::memset(prop, 0, sizeof(*prop));
  std::strcpy(prop->name, "stub sm_100 (no GPU)");
  prop->major = 10;
  prop->minor = 0;
  prop->multiProcessorCount = 148;
  prop->cooperativeLaunch = 1;
  return cudaSuccess;
}
cudaError_t cudaDeviceGetAttribute(int *value, cudaDeviceAttr attr, int) {
  *value = attr == cudaDevAttrMultiProcessorCount        ? 148
           : attr == cudaDevAttrCooperativeLaunch        ? 1
           : attr == cudaDevAttrMaxSharedMemoryPerBlockOptin ? 232448  // B200: 227 KB per CTA
                                                         : 0;
  return cudaSuccess;
}
cudaError_t cudaFuncSetAttribute(const void *, cudaFuncAttribute, int) { return cudaSuccess; }
cudaError_t cudaOccupancyMaxActiveBlocksPerMultiprocessorWithFlags(int *n, const void *, int, size_t, unsigned) {
  *n = 4;
  return cudaSuccess;
}
cudaError_t cudaOccupancyMaxActiveBlocksPerMultiprocessor(int *n, const void *, int, size_t) {
  *n = 4;
  return cudaSuccess;
}
cudaError_t cudaGetLastError() { return cudaSuccess; }
const char *cudaGetErrorName(cudaError_t e) { return e == cudaSuccess ? "cudaSuccess" : "cudaErrorStub"; }
const char *cudaGetErrorString(cudaError_t e) { return e == cudaSuccess ? "no error" : "stub runtime error"; }
cudaError_t cudaMemGetInfo(size_t *free_b, size_t *total_b) {
  *free_b = (size_t)8 << 30;  // keeps plans small: device memory is host memory here
  *total_b = (size_t)16 << 30;
  return cudaSuccess;
}

// ---- memory
cudaError_t cudaMalloc(void **p, size_t bytes) {
  ++g_mallocs;
  *p = nullptr;
  if (g_fail_after.load() == 0) {
    g_fail_after = -1;
    return cudaErrorMemoryAllocation;
  }
  if (g_fail_after.load() > 0) --g_fail_after;
  *p = std::malloc(bytes ? bytes : 1);
  if (!*p) return cudaErrorMemoryAllocation;
  std::memset(*p, 0xA5, bytes ? bytes : 1);  // device memory starts undefined: never zero here either
  ++g_live;
  return cudaSuccess;
}
cudaError_t cudaFree(void *p) {
  if (p) --g_live;
  std::free(p);
  return cudaSuccess;
}
cudaError_t cudaMallocAsync(void **p, size_t bytes, cudaStream_t) { return cudaMalloc(p, bytes); }
// pinned host memory: ordinary host memory here
cudaError_t cudaMallocHost(void **p, size_t bytes) {
  *p = std::malloc(bytes ? bytes : 1);
  return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
cudaError_t cudaFreeHost(void *p) {
  std::free(p);
  return cudaSuccess;
}
cudaError_t cudaFreeAsync(void *p, cudaStream_t) { return cudaFree(p); }
// Memory pools: a pool is a tag; its allocations are ordinary stand-in
// allocations. An injected failure of a pool allocation also fails the
// allocation that follows it (the library retries once after trimming the
// pool), so that every allocation can still be made to fail.
struct StubPool { int id; };
static bool g_pool_refail = false;
cudaError_t cudaMemPoolCreate(cudaMemPool_t *pool, const cudaMemPoolProps *) {
  *pool = reinterpret_cast<cudaMemPool_t>(new StubPool{0});
  return cudaSuccess;
}
cudaError_t cudaMemPoolDestroy(cudaMemPool_t pool) {
  delete reinterpret_cast<StubPool *>(pool);
  return cudaSuccess;
}
cudaError_t cudaMemPoolSetAttribute(cudaMemPool_t, cudaMemPoolAttr, void *) { return cudaSuccess; }
cudaError_t cudaMemPoolGetAttribute(cudaMemPool_t, cudaMemPoolAttr, void *value) {
  *static_cast<uint64_t *>(value) = 0;  // nothing held in reserve
  return cudaSuccess;
}
cudaError_t cudaMemPoolTrimTo(cudaMemPool_t, size_t) { return cudaSuccess; }
cudaError_t cudaMallocFromPoolAsync(void **p, size_t bytes, cudaMemPool_t, cudaStream_t) {
  if (g_pool_refail) {
    g_pool_refail = false;
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  const cudaError_t e = cudaMalloc(p, bytes);
  g_pool_refail = e == cudaErrorMemoryAllocation;
  return e;
}
cudaError_t cudaMemcpyAsync(void *dst, const void *src, size_t bytes, cudaMemcpyKind kind, cudaStream_t s) {
  return on_stream(s, [=] {
    std::memcpy(dst, src, bytes);
    if (kind == cudaMemcpyHostToDevice) g_h2d += (long long)bytes;
    if (kind == cudaMemcpyDeviceToHost) g_d2h += (long long)bytes;
  });
}
cudaError_t cudaMemsetAsync(void *dst, int value, size_t bytes, cudaStream_t s) {
  return on_stream(s, [=] { std::memset(dst, value, bytes); });
}
cudaError_t cudaGetSymbolAddress(void **p, const void *symbol) {
  std::lock_guard<std::mutex> lock(g_mu);
  auto it = var_size().find(symbol);
  if (it == var_size().end()) return cudaErrorInvalidSymbol;
  void *&storage = var_storage()[symbol];
  if (!storage) storage = std::calloc(1, it->second);
  *p = storage;
  return storage ? cudaSuccess : cudaErrorMemoryAllocation;
}

// ---- launches: counted, nothing runs
cudaError_t cudaLaunchKernel(const void *, dim3, dim3, void **, size_t, cudaStream_t s) { return launch(s); }
cudaError_t cudaLaunchCooperativeKernel(const void *, dim3, dim3, void **, size_t, cudaStream_t s) { return launch(s); }
cudaError_t cudaLaunchKernelExC(const cudaLaunchConfig_t *cfg, const void *, void **) { return launch(cfg->stream); }

// ---- streams and events
cudaError_t cudaStreamCreateWithFlags(cudaStream_t *s, unsigned) {
  *s = reinterpret_cast<cudaStream_t>(new char);
  return cudaSuccess;
}
cudaError_t cudaStreamDestroy(cudaStream_t s) { delete reinterpret_cast<char *>(s); return cudaSuccess; }
cudaError_t cudaStreamSynchronize(cudaStream_t) { return cudaSuccess; }
cudaError_t cudaEventCreate(cudaEvent_t *e) { *e = reinterpret_cast<cudaEvent_t>(new char); return cudaSuccess; }
cudaError_t cudaEventCreateWithFlags(cudaEvent_t *e, unsigned) { return cudaEventCreate(e); }
cudaError_t cudaEventDestroy(cudaEvent_t e) { delete reinterpret_cast<char *>(e); return cudaSuccess; }
cudaError_t cudaEventRecord(cudaEvent_t, cudaStream_t) { return cudaSuccess; }
cudaError_t cudaEventSynchronize(cudaEvent_t) { return cudaSuccess; }
cudaError_t cudaEventElapsedTime(float *ms, cudaEvent_t, cudaEvent_t) { *ms = 1.0f; return cudaSuccess; }

// ---- stream capture and graphs
cudaError_t cudaStreamBeginCapture(cudaStream_t s, cudaStreamCaptureMode) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (capturing().count(s)) return cudaErrorIllegalState;
  capturing()[s] = new Capture;
  return cudaSuccess;
}
cudaError_t cudaStreamEndCapture(cudaStream_t s, cudaGraph_t *graph) {
  std::lock_guard<std::mutex> lock(g_mu);
  auto it = capturing().find(s);
  if (it == capturing().end()) return cudaErrorIllegalState;
  auto *g = new Graph{std::move(it->second->ops), it->second->launches};
  delete it->second;
  capturing().erase(it);
  *graph = reinterpret_cast<cudaGraph_t>(g);
  return cudaSuccess;
}
cudaError_t cudaStreamIsCapturing(cudaStream_t s, cudaStreamCaptureStatus *status) {
  std::lock_guard<std::mutex> lock(g_mu);
  *status = capturing().count(s) ? cudaStreamCaptureStatusActive : cudaStreamCaptureStatusNone;
  return cudaSuccess;
}
cudaError_t cudaGraphInstantiate(cudaGraphExec_t *exec, cudaGraph_t graph, unsigned long long) {
  *exec = reinterpret_cast<cudaGraphExec_t>(new Graph(*reinterpret_cast<Graph *>(graph)));
  return cudaSuccess;
}
cudaError_t cudaGraphDestroy(cudaGraph_t graph) { delete reinterpret_cast<Graph *>(graph); return cudaSuccess; }
cudaError_t cudaGraphExecDestroy(cudaGraphExec_t exec) { delete reinterpret_cast<Graph *>(exec); return cudaSuccess; }
cudaError_t cudaGraphLaunch(cudaGraphExec_t exec, cudaStream_t s) {
  Graph *g = reinterpret_cast<Graph *>(exec);
  for (auto &op : g->ops) on_stream(s, op);
  for (long long k = 0; k < g->launches; ++k) launch(s);
  return cudaSuccess;
}
