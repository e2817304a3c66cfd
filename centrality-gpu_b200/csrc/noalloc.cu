// bc_begin_free_noalloc: the free-source BC call for callers that cannot
// allocate device memory (no cudaMalloc, cudaFree or allocating library call
// on this path). Everything the PLAIN kernel needs beyond the caller's own
// device buffers lives in one file-scope __device__ array of fixed size, which
// every GPU that loads this library holds until the process exits.
#include "bcgpu.h"
#include "common.cuh"
#include "internal.h"
#include "plain.h"

#include <algorithm>
#include <cstdio>
#include <mutex>
#include <string>

namespace bcg {
namespace {

// Limits of one call: a BCC of at most kMaxVertices vertices and at most
// kMaxVertices sources, run on kSlots CTAs (one source each at a time).
constexpr int64_t kMaxVertices = 16384;
constexpr int64_t kSlots = 16;
constexpr int64_t kRowCap = kMaxVertices + 2;  // per-slot row capacity the kernel checks

constexpr int64_t align256(int64_t x) { return (x + 255) / 256 * 256; }
constexpr int64_t kOffWsI = 0;
constexpr int64_t kBytesWsI = align256(kSlots * kWsIntRows * kRowCap * 4);
constexpr int64_t kOffWsF = kOffWsI + kBytesWsI;
constexpr int64_t kBytesWsF = align256(kSlots * kWsDblRows * kRowCap * 8);
constexpr int64_t kOffRow = kOffWsF + kBytesWsF;
constexpr int64_t kBytesRow = align256((kMaxVertices + 1) * 8);
constexpr int64_t kOffItems = kOffRow + kBytesRow;
constexpr int64_t kBytesItems = align256(kMaxVertices * (int64_t)sizeof(PlainItem));
constexpr int64_t kOffAcc = kOffItems + kBytesItems;  // fixed-point BC counters, kAccDigits per vertex
constexpr int64_t kBytesAcc = align256(kMaxVertices * kAccDigits * 8);
constexpr int64_t kOffCtl = kOffAcc + kBytesAcc;  // vtx_off[2], counter, epochs[2*kSlots], err
constexpr int64_t kBytesCtl = align256(16 + 8 + 8 * kSlots + 4);
constexpr int64_t kScratchBytes = kOffCtl + kBytesCtl;  // 20,909,056 bytes (about 20 MiB)
static_assert(kScratchBytes == 20909056, "the size the header documents");
static_assert(kMaxVertices <= kAccMaxAdds, "one call's sources must fit the fixed-point counters' headroom");

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

struct Layout {
  int32_t *ws_i;
  double *ws_f;
  int64_t *row;
  PlainItem *items;
  unsigned long long *acc;
  int64_t *vtx_off;
  unsigned long long *counter;
  int32_t *epochs;
  int *err;
};

Layout layout(unsigned char *base) {
  Layout L;
  L.ws_i = reinterpret_cast<int32_t *>(base + kOffWsI);
  L.ws_f = reinterpret_cast<double *>(base + kOffWsF);
  L.row = reinterpret_cast<int64_t *>(base + kOffRow);
  L.items = reinterpret_cast<PlainItem *>(base + kOffItems);
  L.acc = reinterpret_cast<unsigned long long *>(base + kOffAcc);
  L.vtx_off = reinterpret_cast<int64_t *>(base + kOffCtl);
  L.counter = reinterpret_cast<unsigned long long *>(base + kOffCtl + 16);
  L.epochs = reinterpret_cast<int32_t *>(base + kOffCtl + 24);
  L.err = reinterpret_cast<int *>(base + kOffCtl + 24 + 8 * kSlots);
  return L;
}

// Builds the work items of one call: row offsets widened to int64, one item
// per source. Malformed input (offsets, neighbour ids, sources) sets the error
// flag, and the BC kernel then takes no work. On the first call on a device
// (first != 0) it also sets the level-stamp epochs to 1; the workspace rows
// and the fixed-point counters were cleared just before. Later calls keep the
// epochs and stamps the previous call left (every stamp is below its row's
// epoch, and the kernel wraps a row back to zero before an epoch could
// overflow) and find the counters cleared by the previous call's fold.
__global__ void setup_kernel(Layout L, const int32_t *R, const int32_t *C, int32_t n, int32_t m, const int32_t *src,
                             int32_t nsrc, int first) {
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = tid; i <= n; i += stride) {
    const int32_t r = R[i];
    if (r < 0 || r > m || (i == 0 && r != 0) || (i == n && r != m) || (i < n && R[i + 1] < r))
      set_err(L.err, kDevBadItem);
    L.row[i] = r;
  }
  for (int64_t e = tid; e < m; e += stride)
    if (C[e] < 0 || C[e] >= n) set_err(L.err, kDevBadItem);
  for (int64_t i = tid; i < nsrc; i += stride) {
    int32_t s = src[i];
    if (s < 0 || s >= n) {
      set_err(L.err, kDevBadItem);
      s = 0;
    }
    L.items[i] = PlainItem{0, s, 0, 0, 1};
  }
  if (first && tid < 2 * kSlots) L.epochs[tid] = 1;
  if (tid == 0) {
    L.vtx_off[0] = 0;
    L.vtx_off[1] = n;
    *L.counter = 0;
  }
}

// Device address of g_scratch per device, looked up once with that device
// current; g_ready: the array's rows, epochs and counters are in the state a
// finished call leaves (false before the first call and after a failed one,
// which then clears them again).
std::mutex g_mu;
unsigned char *g_addr[64] = {nullptr};
bool g_ready[64] = {false};

}  // namespace
}  // namespace bcg

extern "C" int bc_begin_free_noalloc(bc_ctx *ctx, const int32_t *R, const int32_t *C, int32_t n, int32_t m,
                                     const int32_t *req_nodes, int32_t n_req, const int32_t *reach, double *bc,
                                     double *time_s) {
  using namespace bcg;
  if (!ctx || !R || !C || !reach || !bc || (n_req > 0 && !req_nodes)) return BCGPU_EINVAL;
  if (n < 3 || m < 0 || n_req < 0) return BCGPU_EINVAL;
  if (n > kMaxVertices || n_req > kMaxVertices) {
    char msg[160];
    std::snprintf(msg, sizeof msg,
                  "bc_begin_free_noalloc: %d vertices / %d sources exceed the fixed scratch limit of %lld each", n,
                  n_req, (long long)kMaxVertices);
    ctx_set_error(ctx, msg);
    return BCGPU_EOVERFLOW;
  }
  int dev = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;  // the context's own events: nothing is created here
  ctx_device_stream(ctx, &dev, &stream, &e0, &e1);
  if (dev < 0 || dev >= 64 || cudaSetDevice(dev) != cudaSuccess) return BCGPU_ECUDA;
  unsigned char *base = nullptr;
  bool first = false;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
      void *p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);  // first call on this device
      if (e != cudaSuccess) {
        ctx_set_error(ctx, cudaGetErrorString(e));
        return BCGPU_ECUDA;
      }
      g_addr[dev] = static_cast<unsigned char *>(p);
    }
    base = g_addr[dev];
    first = !g_ready[dev];
    g_ready[dev] = false;  // set again once this call has finished cleanly
  }
  const Layout L = layout(base);
  const bool timing = time_s != nullptr;
  if (timing) cudaEventRecord(e0, stream);
  // the previous call's error flag is still in the array: clear it (and, on a
  // device's first call or after a failed one, the rows and the counters)
  cudaError_t e = cudaMemsetAsync(L.err, 0, sizeof(int), stream);
  if (e == cudaSuccess && first) e = cudaMemsetAsync(L.ws_f, 0, (size_t)kBytesWsF, stream);  // row records: unvisited
  if (e == cudaSuccess && first) e = cudaMemsetAsync(L.acc, 0, (size_t)kBytesAcc, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(bc, 0, sizeof(double) * (size_t)n, stream);
  if (e == cudaSuccess) {
    setup_kernel<<<64, 256, 0, stream>>>(L, R, C, n, m, req_nodes, n_req, first ? 1 : 0);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && n_req > 0) {
    PlainArgs a{};
    a.row = L.row;
    a.col = C;
    a.reach = reach;
    a.vtx_off = L.vtx_off;
    a.items = L.items;
    a.item_begin = 0;
    a.item_end = n_req;
    a.next_item = L.counter;
    a.acc = L.acc;
    a.ws_i = L.ws_i;
    a.ws_f = L.ws_f;
    a.ws_n = kRowCap;
    a.epochs = L.epochs;
    a.rows_slot = -1;  // no row export on this path (launch_rows is never called with these arguments)
    a.rescale_exp = 900;
    a.err = L.err;
    e = launch_plain(a, 256, (int)std::min<int64_t>(kSlots, n_req), stream);
    if (e == cudaSuccess) e = launch_fold(L.acc, bc, 0, n, stream);  // counters -> bc, counters cleared
  }
  int h_err = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_err, L.err, sizeof(int), cudaMemcpyDeviceToHost, stream);
  if (timing) cudaEventRecord(e1, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (timing) {
    float ms = 0.f;
    if (e == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) *time_s += ms * 1e-3;
  }
  if (e != cudaSuccess) {
    ctx_set_error(ctx, cudaGetErrorString(e));
    return BCGPU_ECUDA;
  }
  if (h_err != kDevOk) {
    const std::string msg = std::string("bc_begin_free_noalloc: ") +
                            (h_err == kDevBadItem ? "malformed CSR or source list (offsets, neighbour or source ids)"
                                                  : dev_err_text(h_err));
    ctx_set_error(ctx, msg.c_str());
    return dev_err_status(h_err);
  }
  std::lock_guard<std::mutex> lock(g_mu);
  g_ready[dev] = true;
  return BCGPU_OK;
}
