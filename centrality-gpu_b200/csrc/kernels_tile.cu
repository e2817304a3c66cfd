// Small-BCC schedule: one CTA per range of sources of one BCC, one warp per
// source, the BCC's CSR slice in shared memory.
//
// The reference runs every BCC through the same per-source kernel, one
// source per CTA (Codes/kernels_free.cu:154-473, launch shape
// Codes/begin_gpupgm.cu:52-65), whatever its size; on a batch of thousands of
// small graphs most of a CTA then waits at its per-level barriers. Here a
// BCC that fits shared memory is run warp-synchronously:
//  * the slice (local row offsets, neighbours, reach; tile.h TileSlice) is
//    brought into shared memory by one cp.async.bulk (a plain bulk copy from
//    this GPU's global memory into this CTA's shared memory, completion on an
//    mbarrier whose wait is bounded) and serves every source of the range;
//  * each warp runs one source at a time: a level-synchronous BFS whose levels
//    live in shared memory (one int32 row per warp), each frontier vertex
//    pulling sigma from its predecessors and claiming its successors in one
//    scan of its row (lane per vertex; a vertex of more than 32 arcs is
//    scanned by the whole warp), then the successor-form dependency sweep
//    q(w) = (reach(w)+1+delta(w))/sigma(w), delta(v) = sigma(v) * sum q
//    (Codes/kernels_free.cu:391,409), q overwriting sigma in place;
//  * chain (degree-2) vertices are ordinary vertices and sources here: their
//    BFS costs no more than the endpoint merge of the per-source schedule on
//    a BCC this small;
//  * BC: each contribution delta * (reach(s)+1) (Codes/kernels_free.cu:425) is
//    added to the CTA's fixed-point counters in shared memory (integer
//    atomics: the result does not depend on the order of the warps), which
//    are added to the global counters once per work item.
// Path counts are FP64 without per-level scaling: the plan routes a BCC here
// only when no path count can pass 2^1000 ((2 ecc + 1) levels of at most
// maxdeg predecessors each); a non-finite value still flags kDevOverflow.
#include "accum.cuh"
#include "common.cuh"
#include "tile.h"

namespace bcg {

namespace {

constexpr int kThreads = kTileWarps * 32;
constexpr int kWarpScan = 32;  // rows longer than this are scanned by the whole warp

// Shared memory: control words, then the counters, the per-warp level rows
// and the staged slice, each on a 16-byte boundary.
struct Ctl {
  unsigned long long bar;  // mbarrier of the slice copy
  int item, next, bcc, pad;
  int tail[kTileWarps];
};

__host__ __device__ constexpr int64_t align16(int64_t x) { return (x + 15) / 16 * 16; }

struct Smem {
  Ctl *ctl;
  unsigned long long *cnt;  // [nmax][kAccDigits]
  int32_t *lev;             // [kTileWarps][nmax]
  unsigned char *slice;
};

__device__ __forceinline__ Smem smem_of(unsigned char *base, int nmax) {
  Smem s;
  s.ctl = reinterpret_cast<Ctl *>(base);
  int64_t off = align16(sizeof(Ctl));
  s.cnt = reinterpret_cast<unsigned long long *>(base + off);
  off += align16((int64_t)nmax * kAccDigits * 8);
  s.lev = reinterpret_cast<int32_t *>(base + off);
  off += align16((int64_t)kTileWarps * nmax * 4);
  s.slice = base + off;
  return s;
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// mbarrier and bulk-copy primitives (PTX ISA: mbarrier, cp.async.bulk).
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// Global -> this CTA's shared memory, bytes a multiple of 16, both ends 16-byte aligned.
__device__ __forceinline__ void bulk_copy(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // earlier reads of dst before the copy's writes
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

// Waits for phase `parity` of the barrier, at most limit_ns; false on timeout.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity, unsigned long long limit_ns) {
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (global_ns() - t0 > limit_ns) return false;
  }
  return true;
}

// One BCC as the kernel reads it: local row offsets, neighbours, reach.
struct View {
  const int32_t *R, *C, *rch;
};

// Forward BFS of one warp from s: levels in d (-1 = unvisited), path counts in
// sq, visit order in S, level offsets lv[0..nlev]. Returns nlev.
__device__ int warp_bfs(const View &g, int32_t nb, int32_t s, int32_t *d, double *sq, int32_t *S, int32_t *lv,
                        int *tail, int lane, int *err) {
  for (int v = lane; v < nb; v += 32) d[v] = -1;
  __syncwarp();
  if (lane == 0) {
    d[s] = 0;
    S[0] = s;
    sq[s] = 1.0;
    lv[0] = 0;
    lv[1] = 1;
    *tail = 1;
  }
  __syncwarp();
  int lev = 0, f0 = 0, f1 = 1;
  while (true) {
    const int dprev = lev == 0 ? INT_MIN : lev - 1, dnext = lev + 1;
    for (int c0 = f0; c0 < f1; c0 += 32) {
      const int i = c0 + lane;
      int32_t w = -1, e0 = 0, e1 = 0;
      if (i < f1) {
        w = S[i];
        e0 = g.R[w];
        e1 = g.R[w + 1];
      }
      const bool big = e1 - e0 > kWarpScan;
      if (w >= 0 && !big) {
        double acc = 0.0;
        for (int e = e0; e < e1; e += 4) {  // four arcs' loads in flight; sums in arc order
          int32_t x[4], dx[4];
          double sv[4];
#pragma unroll
          for (int j = 0; j < 4; ++j) x[j] = e + j < e1 ? g.C[e + j] : -1;
#pragma unroll
          for (int j = 0; j < 4; ++j) dx[j] = x[j] >= 0 ? d[x[j]] : INT_MAX;
#pragma unroll
          for (int j = 0; j < 4; ++j) sv[j] = dx[j] == dprev ? __ldcg(sq + x[j]) : 0.0;
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            if (dx[j] == dprev) {
              acc += sv[j];
            } else if (dx[j] == -1 && atomicCAS(d + x[j], -1, dnext) == -1) {
              S[atomicAdd(tail, 1)] = x[j];
            }
          }
        }
        if (lev > 0) sq[w] = acc;
      }
      uint32_t bigs = __ballot_sync(0xffffffffu, w >= 0 && big);
      while (bigs) {  // rows longer than kWarpScan: the whole warp, lanes over arcs
        const int j = __ffs(bigs) - 1;
        bigs &= bigs - 1;
        const int32_t wj = __shfl_sync(0xffffffffu, w, j);
        const int32_t a0 = __shfl_sync(0xffffffffu, e0, j), a1 = __shfl_sync(0xffffffffu, e1, j);
        double acc = 0.0;
        for (int e = a0 + lane; e < a1; e += 32) {
          const int32_t x = g.C[e];
          const int dx = d[x];
          if (dx == dprev) acc += __ldcg(sq + x);
          else if (dx == -1 && atomicCAS(d + x, -1, dnext) == -1) S[atomicAdd(tail, 1)] = x;
        }
        acc = warp_sum(acc);
        if (lane == 0 && lev > 0) sq[wj] = acc;
      }
    }
    __syncwarp();
    const int t = *(volatile int *)tail;
    if (t == f1) break;
    if (lane == 0) lv[lev + 2] = t;
    f0 = f1;
    f1 = t;
    ++lev;
    __syncwarp();
  }
  (void)err;
  return lev + 1;
}

// Dependency sweep of one warp, deepest level first; q overwrites sigma in
// sq; contributions delta * wsrc go to the shared-memory counters.
__device__ void warp_sweep(const View &g, int32_t nlev, const int32_t *d, double *sq, const int32_t *S,
                           const int32_t *lv, double wsrc, unsigned long long *cnt, int lane, int *err) {
  for (int lev = nlev - 1; lev >= 1; --lev) {
    const int dsucc = lev + 1, a0 = lv[lev], a1 = lv[lev + 1];
    for (int c0 = a0; c0 < a1; c0 += 32) {
      const int i = c0 + lane;
      int32_t w = -1, e0 = 0, e1 = 0;
      if (i < a1) {
        w = S[i];
        e0 = g.R[w];
        e1 = g.R[w + 1];
      }
      const bool big = e1 - e0 > kWarpScan;
      double acc = 0.0;
      if (w >= 0 && !big) {
        for (int e = e0; e < e1; e += 4) {
          int32_t x[4];
          bool hit[4];
          double qv[4];
#pragma unroll
          for (int j = 0; j < 4; ++j) x[j] = e + j < e1 ? g.C[e + j] : -1;
#pragma unroll
          for (int j = 0; j < 4; ++j) hit[j] = x[j] >= 0 && d[x[j]] == dsucc;
#pragma unroll
          for (int j = 0; j < 4; ++j) qv[j] = hit[j] ? __ldcg(sq + x[j]) : 0.0;
#pragma unroll
          for (int j = 0; j < 4; ++j)
            if (hit[j]) acc += qv[j];
        }
      }
      uint32_t bigs = __ballot_sync(0xffffffffu, w >= 0 && big);
      while (bigs) {
        const int j = __ffs(bigs) - 1;
        bigs &= bigs - 1;
        const int32_t a0j = __shfl_sync(0xffffffffu, e0, j), a1j = __shfl_sync(0xffffffffu, e1, j);
        double part = 0.0;
        for (int e = a0j + lane; e < a1j; e += 32) {
          const int32_t x = g.C[e];
          if (d[x] == dsucc) part += __ldcg(sq + x);
        }
        part = warp_sum(part);
        if (lane == j) acc = part;
      }
      if (w >= 0) {
        const double sw = __ldcg(sq + w);
        const double delta = sw * acc;
        const double qw = ((double)g.rch[w] + 1.0 + delta) / sw;
        if (exp_bits(qw) == 0x7ff || exp_bits(delta) == 0x7ff || exp_bits(sw) == 0) set_err(err, kDevOverflow);
        sq[w] = qw;  // this level's q: read only by the level above (after the warp barrier)
        if (delta != 0.0) acc_add(cnt + (int64_t)kAccDigits * w, delta * wsrc, err);
      }
    }
    __syncwarp();
  }
}

__global__ void __launch_bounds__(kThreads, 1) tile_kernel(TileArgs a) {
  extern __shared__ __align__(16) unsigned char s_raw[];
  const Smem sm = smem_of(s_raw, a.nmax);
  Ctl &ctl = *sm.ctl;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t slot = (int64_t)blockIdx.x * kTileWarps + warp;
  int32_t *S = a.ws_S + slot * a.cap, *lv = a.ws_lv + slot * a.cap;
  double *sq = a.ws_sq + slot * a.cap;
  int32_t *dl = sm.lev + (int64_t)warp * a.nmax;
  if (tid == 0) {
    mbar_init(&ctl.bar, 1);
    ctl.bcc = -1;
  }
  __syncthreads();
  unsigned phase = 0;
  while (true) {
    if (tid == 0) {
      const int64_t k = (int64_t)atomicAdd(a.next_item, 1ull);
      ctl.item = (*(volatile int *)a.err != kDevOk || a.item_begin + k >= a.item_end) ? -1 : (int)k;
      ctl.next = 0;
    }
    __syncthreads();  // also: every warp is done with the previous item's slice and counters
    if (ctl.item < 0) break;
    const TileItem it = a.items[a.item_begin + ctl.item];
    const int64_t vo = a.vtx_off[it.bcc];
    const int32_t nb = (int32_t)(a.vtx_off[it.bcc + 1] - vo);
    const int64_t soff = a.slice_off[it.bcc];
    if (nb > a.nmax || soff < 0) {  // uniform over the CTA
      set_err(a.err, kDevBadItem);
      continue;
    }
    if (ctl.bcc != it.bcc) {  // stage the BCC's slice (uniform: ctl.bcc was last written before a barrier)
      if (tid == 0) {
        const unsigned bytes = (unsigned)a.slice_bytes[it.bcc];
        mbar_expect_tx(&ctl.bar, bytes);
        bulk_copy(sm.slice, a.slices + soff, bytes, &ctl.bar);
      }
      const bool ok = mbar_wait(&ctl.bar, phase, a.wait_ns);
      if (!ok) {
        // the copy did not complete in time: record it, wait (again bounded)
        // for the copy in flight to land in this CTA's shared memory, stop
        set_err(a.err, kDevTimeout);
        mbar_wait(&ctl.bar, phase, a.wait_ns);
        break;
      }
      phase ^= 1u;
    }
    for (int64_t k = tid; k < (int64_t)kAccDigits * nb; k += kThreads) sm.cnt[k] = 0ull;
    __syncthreads();
    if (tid == 0) ctl.bcc = it.bcc;  // read again only after the next top-of-loop barrier
    const int32_t *sl = reinterpret_cast<const int32_t *>(sm.slice);
    const View g{sl, sl + TileSlice::col_at(nb) / 4,
                 reinterpret_cast<const int32_t *>(sm.slice + TileSlice::reach_at(nb, sl[nb]))};
    while (true) {  // warps take the item's sources one at a time
      int k = 0;
      if (lane == 0) k = atomicAdd(&ctl.next, 1);
      k = __shfl_sync(0xffffffffu, k, 0);
      const int32_t s = it.s0 + k;
      if (s >= it.s1) break;
      if (s < 0 || s >= nb) {
        set_err(a.err, kDevBadItem);
        break;
      }
      const int nlev = warp_bfs(g, nb, s, dl, sq, S, lv, &ctl.tail[warp], lane, a.err);
      warp_sweep(g, nlev, dl, sq, S, lv, (double)g.rch[s] + 1.0, sm.cnt, lane, a.err);
    }
    __syncthreads();
    // the item's contributions into the global counters (integer adds: any order)
    unsigned long long *acc = a.acc + (int64_t)kAccDigits * vo;
    for (int64_t k = tid; k < (int64_t)kAccDigits * nb; k += kThreads) {
      const unsigned long long c = sm.cnt[k];
      if (c) atomicAdd(acc + k, c);
    }
  }
}

}  // namespace

size_t tile_smem_bytes(int64_t nmax, int64_t slice_max) {
  return (size_t)(align16(sizeof(Ctl)) + align16(nmax * kAccDigits * 8) + align16((int64_t)kTileWarps * nmax * 4) +
                  align16(slice_max));
}

size_t tile_smem_limit(int device) {
  int v = 0;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess) return 0;
  return (size_t)v;
}

int tile_ctas_per_sm(size_t smem) {
  int n = 0;
  if (cudaFuncSetAttribute(tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, tile_kernel, kThreads, smem) != cudaSuccess) return 0;
  return n;
}

cudaError_t launch_tile(const TileArgs &a, int grid, size_t smem, cudaStream_t stream) {
  cudaError_t e = cudaFuncSetAttribute(tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  tile_kernel<<<grid, kThreads, smem, stream>>>(a);
  return cudaGetLastError();
}

}  // namespace bcg
