// Breadth-first batched join: every query descends the tree level by level,
// all queries at once.  A frontier item is (query, node); a group of G lanes
// (G = fanout rounded up to a power of two) tests the node's entries against
// the query box, a warp ballot compacts the hits, and one atomicAdd per warp
// reserves their slots in the next frontier (or, at the leaf level, in the
// pair output).  Frontier counts stay on the device and every launch
// grid-strides over the current count, so a whole join is a fixed sequence of
// launches with no host round trip until the final count is read.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <vector>

#include "prt_internal.cuh"

namespace prt {
namespace {

constexpr int kJoinBlock = 256;

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

struct JoinLevel {
  const void *mbr;          // entries of node level l (Box<T>)
  int64_t n_entries;        // entries at level l
  const uint2 *in;          // frontier (query, node); nullptr = (q, 0) for all queries
  const unsigned long long *in_count;
  int64_t in_cap;
  uint2 *out;               // next frontier, or pairs at the leaf level
  unsigned long long *out_count;
  int64_t out_cap;
  int leaf;                 // 1: emit (entry, query) pairs
  int64_t nq;
  long long *counts;        // optional per-query reference counters
  int td_slots;
};

// One block iteration takes kJoinRounds rounds of kGroups items per warp: the
// frontier items of all rounds are loaded first, then their node entries, so
// each warp has that many independent loads in flight; the hits of the whole
// iteration are reserved with one atomicAdd per block.  Measured on the
// 1M-window join of the 10M-box tree (F = 16) with the grid sized to one
// resident wave: 3, 4, 6 rounds take 3.00, 3.29, 3.07 ms.
constexpr int kJoinRounds = 3;

template <typename T, int G>
__global__ void __launch_bounds__(kJoinBlock) expand_kernel(JoinLevel J, const Box<T> *__restrict__ queries,
                                                            int fanout) {
  const Box<T> *mbr = reinterpret_cast<const Box<T> *>(J.mbr);
  const int lane = threadIdx.x & 31;
  const int sub = lane / G;           // group within the warp
  const int e = lane % G;             // entry within the node
  constexpr int kGroups = 32 / G;
  constexpr int kWarps = kJoinBlock / 32;
  const uint32_t gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (sub * G));
  const uint32_t lt = lanemask_lt();
  int64_t count = J.in ? (int64_t)min((unsigned long long)J.in_cap, *J.in_count) : J.nq;
  __shared__ uint32_t s_wcount[2][kWarps];
  __shared__ unsigned long long s_base[2];
  const int warp = threadIdx.x >> 5;
  const int64_t per_warp = (int64_t)kJoinRounds * kGroups;
  const int64_t per_block = (int64_t)kWarps * per_warp;
  int par = 0;
  for (int64_t bb = blockIdx.x * per_block; bb < count; bb += (int64_t)gridDim.x * per_block, par ^= 1) {
    const int64_t wb = bb + warp * per_warp;
    uint32_t q[kJoinRounds], node[kJoinRounds];
#pragma unroll
    for (int r = 0; r < kJoinRounds; r++) {
      const int64_t item = wb + r * kGroups + sub;
      q[r] = 0;
      node[r] = 0;
      if (item < count) {
        if (J.in) {
          const uint2 it = J.in[item];
          q[r] = it.x;
          node[r] = it.y;
        } else {
          q[r] = (uint32_t)item;
        }
      }
    }
    uint32_t ballots[kJoinRounds];
    uint32_t wtot = 0;
#pragma unroll
    for (int r = 0; r < kJoinRounds; r++) {
      const int64_t item = wb + r * kGroups + sub;
      const bool live = item < count;
      bool hit = false;
      if (live && e < fanout) {
        const Box<T> qb = load_box(queries, q[r]);
        const Box<T> eb = load_box(mbr, (int64_t)node[r] * fanout + e);  // padded slots intersect nothing
        hit = overlaps(eb, qb);
      }
      ballots[r] = __ballot_sync(0xffffffffu, hit);
      wtot += __popc(ballots[r]);
      if (J.counts && live && e == 0) {
        const int k = __popc(ballots[r] & gmask);
        const int64_t fill = J.td_slots ? fanout : min((int64_t)fanout, J.n_entries - (int64_t)node[r] * fanout);
        atomicAdd(reinterpret_cast<unsigned long long *>(&J.counts[3 * (int64_t)q[r]]), (unsigned long long)fill);
        if (k > 1)
          atomicAdd(reinterpret_cast<unsigned long long *>(&J.counts[3 * (int64_t)q[r] + 1]),
                    (unsigned long long)(k - 1));
        if (J.leaf && k)
          atomicAdd(reinterpret_cast<unsigned long long *>(&J.counts[3 * (int64_t)q[r] + 2]), (unsigned long long)k);
      }
    }
    // one reservation per block iteration (warp counts double-buffered by
    // iteration parity, so one barrier separates the writes and the reads)
    if (lane == 0) s_wcount[par][warp] = wtot;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t tot = 0;
#pragma unroll
      for (int w = 0; w < kWarps; w++) tot += s_wcount[par][w];
      s_base[par] = tot ? atomicAdd(J.out_count, (unsigned long long)tot) : 0ull;
    }
    __syncthreads();
    if (wtot) {
      unsigned long long slot = s_base[par];
#pragma unroll
      for (int w = 0; w < kWarps; w++) slot += w < warp ? s_wcount[par][w] : 0u;
#pragma unroll
      for (int r = 0; r < kJoinRounds; r++) {
        if (ballots[r] >> lane & 1u) {
          const unsigned long long at = slot + __popc(ballots[r] & lt);
          const uint32_t entry = node[r] * (uint32_t)fanout + (uint32_t)e;
          if ((int64_t)at < J.out_cap) J.out[at] = J.leaf ? make_uint2(entry, q[r]) : make_uint2(q[r], entry);
        }
        slot += __popc(ballots[r]);
      }
    }
  }
}

// Resident blocks per SM of expand_kernel<T, G> (once per instantiation): the
// grid is exactly one wave, since a block beyond it would process its share
// of every grid-stride loop after the others.
template <typename T, int G>
int expand_blocks() {
  static std::atomic<int> per_sm{0};
  int b = per_sm.load(std::memory_order_relaxed);
  if (b == 0) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, expand_kernel<T, G>, kJoinBlock, 0) != cudaSuccess || b < 1) {
      cudaGetLastError();
      b = 4;
    }
    per_sm.store(b, std::memory_order_relaxed);
  }
  return kSMs * b;
}

template <typename T>
int launch_expand(const JoinLevel &J, const void *queries, int fanout, cudaStream_t s) {
  const Box<T> *q = reinterpret_cast<const Box<T> *>(queries);
  if (fanout <= 2) {
    PRT_PROF("expand", s);
    expand_kernel<T, 2><<<expand_blocks<T, 2>(), kJoinBlock, 0, s>>>(J, q, fanout);
  }
  else if (fanout <= 4) {
    PRT_PROF("expand", s);
    expand_kernel<T, 4><<<expand_blocks<T, 4>(), kJoinBlock, 0, s>>>(J, q, fanout);
  }
  else if (fanout <= 8) {
    PRT_PROF("expand", s);
    expand_kernel<T, 8><<<expand_blocks<T, 8>(), kJoinBlock, 0, s>>>(J, q, fanout);
  }
  else if (fanout <= 16) {
    PRT_PROF("expand", s);
    expand_kernel<T, 16><<<expand_blocks<T, 16>(), kJoinBlock, 0, s>>>(J, q, fanout);
  }
  else {
    PRT_PROF("expand", s);
    expand_kernel<T, 32><<<expand_blocks<T, 32>(), kJoinBlock, 0, s>>>(J, q, fanout);
  }
  return PRT_OK;
}

// Overlapping pairs of sibling entries (the reference's RtreeSearch1,
// BotomUp-rtree.cu:574-590, TopDown-rtree.cu:78-93): for every node of every
// level, the entry pairs j < i < fill whose boxes intersect.  One warp per
// node, lane i holds entry i and counts its overlaps with the entries before
// it, which it receives by shuffles; one atomic per warp.
template <typename T>
__global__ void __launch_bounds__(256) sibling_kernel(const Box<T> *__restrict__ lv, int64_t n_entries, int fanout,
                                                      unsigned long long *__restrict__ total) {
  const int lane = threadIdx.x & 31;
  const int64_t nodes = (n_entries + fanout - 1) / fanout;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long acc = 0;
  for (int64_t node = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; node < nodes; node += nw) {
    const int64_t first = node * fanout;
    const int fill = (int)min((int64_t)fanout, n_entries - first);
    Box<T> b = empty_box<T>();
    if (lane < fill) b = load_box(lv, first + lane);
    unsigned c = 0;
    for (int j = 0; j < fill - 1; j++) {
      Box<T> o;
      o.x1 = __shfl_sync(0xffffffffu, b.x1, j);
      o.y1 = __shfl_sync(0xffffffffu, b.y1, j);
      o.x2 = __shfl_sync(0xffffffffu, b.x2, j);
      o.y2 = __shfl_sync(0xffffffffu, b.y2, j);
      c += (j < lane && lane < fill && overlaps(b, o)) ? 1u : 0u;
    }
    acc += c;
  }
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0 && acc) atomicAdd(total, acc);
}

// Frontier capacity that worked last time (grows across calls; shared by the
// process's threads, so it is atomic).
std::atomic<int64_t> g_frontier_hint{1 << 20};

// Runs the traversal.  pairs may be nullptr with cap 0 (count only).
int run_join(const prt_tree *t, const void *d_queries, int coord, int64_t nq, uint2 *d_pairs, int64_t cap,
             int64_t *h_count, long long *d_counts, int td_slots, cudaStream_t s) {
  PRT_CHECK(t != nullptr, PRT_ERR_INVALID, "tree is NULL");
  PRT_CHECK(coord == t->coord, PRT_ERR_INVALID, "query coordinate type %d differs from the tree's %d", coord,
            t->coord);
  PRT_CHECK(nq >= 0 && nq < (1ll << 31), PRT_ERR_INVALID, "nq=%lld", (long long)nq);
  PRT_CHECK(cap >= 0, PRT_ERR_INVALID, "cap < 0");
  PRT_CHECK((reinterpret_cast<uintptr_t>(d_queries) & 15) == 0 && (reinterpret_cast<uintptr_t>(d_pairs) & 7) == 0,
            PRT_ERR_INVALID, "d_queries must be 16-byte and d_pairs 8-byte aligned");
  if (h_count) *h_count = 0;
  if (nq == 0) return PRT_OK;
  const TreeLevels &L = t->lv;
  const size_t bs = 4 * coord_size(t->coord);
  int64_t fcap = std::max<int64_t>(g_frontier_hint.load(std::memory_order_relaxed), 4 * nq);
  for (int attempt = 0; attempt < 8; attempt++) {
    unsigned long long *cnt = nullptr;
    uint2 *fr[2] = {nullptr, nullptr};
    int rc = dalloc(&cnt, PRT_MAX_LEVELS + 2, s);
    if (!rc && L.levels > 1) rc = dalloc(&fr[0], fcap, s);
    if (!rc && L.levels > 2) rc = dalloc(&fr[1], fcap, s);
    if (!rc) {
      cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * (PRT_MAX_LEVELS + 2), s);
      if (e != cudaSuccess) rc = cuda_status(e, "memset");
    }
    if (!rc && d_counts) {
      cudaError_t e = cudaMemsetAsync(d_counts, 0, sizeof(long long) * 3 * nq, s);
      if (e != cudaSuccess) rc = cuda_status(e, "memset");
    }
    // level L-1 (root node) down to 0
    int cur = -1;
    for (int l = L.levels - 1; l >= 0 && !rc; l--) {
      JoinLevel J;
      J.mbr = reinterpret_cast<const char *>(t->d_mbr) + L.offset[l] * bs;
      J.n_entries = L.count[l];
      J.in = cur < 0 ? nullptr : fr[cur];
      J.in_count = cur < 0 ? nullptr : &cnt[l + 1];
      J.in_cap = fcap;
      J.leaf = l == 0;
      int nxt = cur < 0 ? 0 : 1 - cur;
      J.out = J.leaf ? d_pairs : fr[nxt];
      J.out_count = J.leaf ? &cnt[PRT_MAX_LEVELS] : &cnt[l];
      J.out_cap = J.leaf ? cap : fcap;
      J.nq = nq;
      J.counts = d_counts;
      J.td_slots = td_slots;
      rc = dispatch_coord(t->coord, [&](auto tag) {
        using T = decltype(tag);
        return launch_expand<T>(J, d_queries, t->fanout, s);
      });
      cur = nxt;
    }
    if (!rc) {
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) rc = cuda_status(e, "join launch");
    }
    std::vector<unsigned long long> h(PRT_MAX_LEVELS + 2, 0);
    if (!rc) {
      cudaError_t e = cudaMemcpyAsync(h.data(), cnt, sizeof(unsigned long long) * (PRT_MAX_LEVELS + 2),
                                      cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) rc = cuda_status(e, "join");
    }
    dfree(cnt, s);
    dfree(fr[0], s);
    dfree(fr[1], s);
    if (rc) return rc;
    unsigned long long worst = 0;
    for (int l = 1; l < L.levels; l++) worst = std::max(worst, h[l]);
    if ((int64_t)worst > fcap) {
      fcap = (int64_t)(worst + worst / 4 + 1024);
      int64_t seen = g_frontier_hint.load(std::memory_order_relaxed);
      while (seen < fcap && !g_frontier_hint.compare_exchange_weak(seen, fcap, std::memory_order_relaxed)) {
      }
      continue;
    }
    int64_t np = (int64_t)h[PRT_MAX_LEVELS];
    if (h_count) *h_count = np;
    if (np > cap && d_pairs) {
      set_error("join: %lld pairs exceed capacity %lld", (long long)np, (long long)cap);
      return PRT_ERR_CAPACITY;
    }
    return PRT_OK;
  }
  set_error("join: frontier kept overflowing");
  return PRT_ERR_CAPACITY;
}

__global__ void pair_key_kernel(const uint2 *__restrict__ p, int64_t n, uint64_t *__restrict__ k,
                                uint32_t *__restrict__ v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint2 x = p[i];
    k[i] = ((uint64_t)x.y << 32) | x.x;
    v[i] = x.x;
  }
}

__global__ void pair_unkey_kernel(const uint64_t *k0, const uint64_t *k1, const int *sel, int64_t n,
                                  uint2 *__restrict__ p) {
  const uint64_t *k = *sel ? k1 : k0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t x = k[i];
    p[i] = make_uint2((uint32_t)x, (uint32_t)(x >> 32));
  }
}

}  // namespace
}  // namespace prt

using namespace prt;

extern "C" {

int prt_join(const prt_tree *t, const void *d_queries, int coord_type, int64_t nq, prt_pair *d_pairs, int64_t cap,
             int64_t *h_count, void *stream) {
  return run_join(t, d_queries, coord_type, nq, reinterpret_cast<uint2 *>(d_pairs), d_pairs ? cap : 0, h_count,
                  nullptr, 0, reinterpret_cast<cudaStream_t>(stream));
}

int prt_join_sorted(const prt_tree *t, const void *d_queries, int coord_type, int64_t nq, prt_pair *d_pairs,
                    int64_t cap, int64_t *h_count, void *stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int64_t np = 0;
  int rc = run_join(t, d_queries, coord_type, nq, reinterpret_cast<uint2 *>(d_pairs), d_pairs ? cap : 0, &np,
                    nullptr, 0, s);
  if (h_count) *h_count = np;
  if (rc || np == 0) return rc;
  PRT_CHECK(np < (1ll << 30), PRT_ERR_INVALID, "join_sorted: %lld pairs (sort limit 2^30)", (long long)np);
  unsigned char *scr = nullptr;
  rc = dmalloc(reinterpret_cast<void **>(&scr), 64 + np * (8 + 8 + 4 + 4), s);
  if (rc) return rc;
  unsigned *err = reinterpret_cast<unsigned *>(scr);
  int *sel = reinterpret_cast<int *>(scr + 8);
  uint64_t *k0 = reinterpret_cast<uint64_t *>(scr + 64), *k1 = k0 + np;
  uint32_t *v0 = reinterpret_cast<uint32_t *>(k1 + np), *v1 = v0 + np;
  cudaMemsetAsync(err, 0, 8, s);
  int g = grid_for(np, 256, 16);
  {
    PRT_PROF("pair_key", s);
    pair_key_kernel<<<g, 256, 0, s>>>(reinterpret_cast<const uint2 *>(d_pairs), np, k0, v0);
  }
  rc = radix_sort_pairs<uint64_t>(k0, v0, k1, v1, np, 64, sel, err, s);
  if (!rc) {
    PRT_PROF("pair_unkey", s);
    pair_unkey_kernel<<<g, 256, 0, s>>>(k0, k1, sel, np, reinterpret_cast<uint2 *>(d_pairs));
  }
  unsigned herr = 0;
  if (!rc) {
    cudaError_t e = cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = cuda_status(e, "join_sorted");
  }
  dfree(scr, s);
  if (!rc && (herr & kErrTimeout)) {
    set_error("join_sorted: sort look-back timed out");
    rc = PRT_ERR_TIMEOUT;
  }
  return rc;
}

int prt_query_counts(const prt_tree *t, const void *d_queries, int coord_type, int64_t nq, int td_slots,
                     int64_t *d_counts, void *stream) {
  PRT_CHECK(d_counts != nullptr, PRT_ERR_INVALID, "d_counts is NULL");
  int64_t np = 0;
  return run_join(t, d_queries, coord_type, nq, nullptr, 0, &np, reinterpret_cast<long long *>(d_counts), td_slots,
                  reinterpret_cast<cudaStream_t>(stream));
}

int prt_tree_sibling_overlaps(const prt_tree *t, int64_t *h_count, void *stream) {
  PRT_CHECK(t && h_count, PRT_ERR_INVALID, "NULL argument");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  *h_count = 0;
  unsigned long long *d = nullptr;
  int rc = dalloc(&d, 1, s);
  if (rc) return rc;
  cudaError_t e = cudaMemsetAsync(d, 0, 8, s);
  const size_t bs = 4 * coord_size(t->coord);
  for (int l = 0; l < t->lv.levels && e == cudaSuccess; l++) {
    const int64_t nodes = (t->lv.count[l] + t->fanout - 1) / t->fanout;
    const void *lv = reinterpret_cast<const char *>(t->d_mbr) + t->lv.offset[l] * bs;
    rc = dispatch_coord(t->coord, [&](auto tag) {
      using T = decltype(tag);
      PRT_PROF("sibling", s);
      sibling_kernel<T><<<grid_for(nodes * 32, 256, 8), 256, 0, s>>>(reinterpret_cast<const Box<T> *>(lv),
                                                                     t->lv.count[l], t->fanout, d);
      return PRT_OK;
    });
    e = cudaGetLastError();
  }
  unsigned long long h = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d, 8, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  dfree(d, s);
  if (e != cudaSuccess) return cuda_status(e, "sibling overlaps");
  *h_count = (int64_t)h;
  return rc;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free join.
//
// prt_join takes its frontier buffers and level counters from the
// stream-ordered allocator.  Some callers may not allocate device memory at
// the moment they join: a host process that hands the whole device budget to
// its own pool and treats any other allocation as a failure, or an embedding
// that forbids the library from calling cudaMalloc / cudaMallocAsync at all.
// prt_join_noalloc runs the same breadth-first traversal with its scratch in
// the file-scope array below instead: the caller passes the queries and the
// pair buffer, and the library allocates nothing.  The call still waits for
// its stream once, at the end, to read the level and pair counts.
//
// The array is reserved on every GPU that loads the library, for the life of
// the process.  Its device address is looked up once per device
// (cudaGetSymbolAddress, with that device current) on the first call made
// there and kept for the process, so make that first call before any stream
// capture, and do not call again on a device after cudaDeviceReset (the kept
// address would be stale).  All calls on a device share the one array and its
// contents stay from one call to the next (every call clears the counters):
// calls that can overlap on the GPU (different streams, or host threads) race
// on it and must be serialised by the caller.
#include <mutex>

namespace prt {
namespace {

// Frontier items per buffer: two (query, node) buffers of 4 Mi items each
// (64 MiB) plus the level counters.
constexpr int64_t kNoAllocFrontier = 1ll << 22;
constexpr size_t kNoAllocCounterBytes = 512;  // 64 x uint64, room for PRT_MAX_LEVELS + 2
constexpr size_t kNoAllocBytes = kNoAllocCounterBytes + 2 * sizeof(uint2) * (size_t)kNoAllocFrontier;

static __device__ __align__(256) unsigned char g_join_scratch[kNoAllocBytes];

std::mutex g_noalloc_mu;
unsigned char *g_noalloc_addr[256] = {nullptr};  // per device, set on first use

int noalloc_scratch(unsigned char **out) {
  int dev = 0;
  PRT_CUDA(cudaGetDevice(&dev));
  PRT_CHECK(dev >= 0 && dev < 256, PRT_ERR_INVALID, "device %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_join_scratch);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(join scratch)");
    g_noalloc_addr[dev] = reinterpret_cast<unsigned char *>(p);
  }
  *out = g_noalloc_addr[dev];
  return PRT_OK;
}

}  // namespace
}  // namespace prt

extern "C" {

int prt_join_noalloc(const prt_tree *t, const void *d_queries, int coord_type, int64_t nq, prt_pair *d_pairs,
                     int64_t cap, int64_t *h_count, void *stream) {
  using namespace prt;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  PRT_CHECK(t != nullptr, PRT_ERR_INVALID, "tree is NULL");
  PRT_CHECK(coord_type == t->coord, PRT_ERR_INVALID, "query coordinate type %d differs from the tree's %d",
            coord_type, t->coord);
  PRT_CHECK(nq >= 0 && nq < (1ll << 31), PRT_ERR_INVALID, "nq=%lld", (long long)nq);
  PRT_CHECK(cap >= 0 && (cap == 0 || d_pairs != nullptr), PRT_ERR_INVALID, "pair buffer");
  PRT_CHECK((reinterpret_cast<uintptr_t>(d_queries) & 15) == 0 && (reinterpret_cast<uintptr_t>(d_pairs) & 7) == 0,
            PRT_ERR_INVALID, "d_queries must be 16-byte and d_pairs 8-byte aligned");
  PRT_CHECK(t->lv.levels + 2 <= (int)(kNoAllocCounterBytes / 8), PRT_ERR_INVALID, "tree too deep");
  if (h_count) *h_count = 0;
  if (nq == 0) return PRT_OK;
  unsigned char *scr = nullptr;
  int rc = noalloc_scratch(&scr);
  if (rc) return rc;
  unsigned long long *cnt = reinterpret_cast<unsigned long long *>(scr);
  uint2 *fr[2] = {reinterpret_cast<uint2 *>(scr + kNoAllocCounterBytes),
                  reinterpret_cast<uint2 *>(scr + kNoAllocCounterBytes) + kNoAllocFrontier};
  // the counters must start at zero; the frontier buffers are written before read
  PRT_CUDA(cudaMemsetAsync(cnt, 0, kNoAllocCounterBytes, s));
  const TreeLevels &L = t->lv;
  const size_t bs = 4 * coord_size(t->coord);
  const int leaf_slot = PRT_MAX_LEVELS;  // counter of emitted pairs
  int cur = -1;
  for (int l = L.levels - 1; l >= 0 && !rc; l--) {
    JoinLevel J;
    J.mbr = reinterpret_cast<const char *>(t->d_mbr) + L.offset[l] * bs;
    J.n_entries = L.count[l];
    J.in = cur < 0 ? nullptr : fr[cur];
    J.in_count = cur < 0 ? nullptr : &cnt[l + 1];
    J.in_cap = kNoAllocFrontier;
    J.leaf = l == 0;
    int nxt = cur < 0 ? 0 : 1 - cur;
    J.out = J.leaf ? reinterpret_cast<uint2 *>(d_pairs) : fr[nxt];
    J.out_count = J.leaf ? &cnt[leaf_slot] : &cnt[l];
    J.out_cap = J.leaf ? cap : kNoAllocFrontier;
    J.nq = nq;
    J.counts = nullptr;
    J.td_slots = 0;
    rc = dispatch_coord(t->coord, [&](auto tag) {
      using T = decltype(tag);
      return launch_expand<T>(J, d_queries, t->fanout, s);
    });
    cur = nxt;
  }
  if (rc) return rc;
  PRT_CUDA(cudaGetLastError());
  unsigned long long h[PRT_MAX_LEVELS + 2];
  PRT_CUDA(cudaMemcpyAsync(h, cnt, sizeof h, cudaMemcpyDeviceToHost, s));
  PRT_CUDA(cudaStreamSynchronize(s));
  for (int l = 1; l < L.levels; l++) {
    if ((int64_t)h[l] > kNoAllocFrontier) {
      set_error("prt_join_noalloc: a frontier of %llu (query, node) items exceeds the fixed scratch of %lld items; "
                "use prt_join or fewer queries per call",
                h[l], (long long)kNoAllocFrontier);
      return PRT_ERR_CAPACITY;
    }
  }
  const int64_t np = (int64_t)h[leaf_slot];
  if (h_count) *h_count = np;
  if (np > cap) {
    set_error("prt_join_noalloc: %lld pairs exceed capacity %lld", (long long)np, (long long)cap);
    return PRT_ERR_CAPACITY;
  }
  return PRT_OK;
}

}  // extern "C"

namespace prt {

// Breadth-first join into caller-owned buffers, nothing synchronised: the
// capture-safe form used by the graph pipeline (prt_pipeline_*).
int join_enqueue(const prt_tree *t, const void *d_queries, int64_t nq, uint2 *d_pairs, int64_t cap, uint2 *fr0,
                 uint2 *fr1, int64_t fcap, unsigned long long *cnt, cudaStream_t s) {
  PRT_CHECK(t != nullptr && nq >= 0, PRT_ERR_INVALID, "join_enqueue arguments");
  if (nq == 0) return PRT_OK;
  const TreeLevels &L = t->lv;
  const size_t bs = 4 * coord_size(t->coord);
  uint2 *fr[2] = {fr0, fr1};
  int cur = -1;
  int rc = PRT_OK;
  for (int l = L.levels - 1; l >= 0 && !rc; l--) {
    JoinLevel J;
    J.mbr = reinterpret_cast<const char *>(t->d_mbr) + L.offset[l] * bs;
    J.n_entries = L.count[l];
    J.in = cur < 0 ? nullptr : fr[cur];
    J.in_count = cur < 0 ? nullptr : &cnt[l + 1];
    J.in_cap = fcap;
    J.leaf = l == 0;
    int nxt = cur < 0 ? 0 : 1 - cur;
    J.out = J.leaf ? d_pairs : fr[nxt];
    J.out_count = J.leaf ? &cnt[PRT_MAX_LEVELS] : &cnt[l];
    J.out_cap = J.leaf ? cap : fcap;
    J.nq = nq;
    J.counts = nullptr;
    J.td_slots = 0;
    rc = dispatch_coord(t->coord, [&](auto tag) {
      using T = decltype(tag);
      return launch_expand<T>(J, d_queries, t->fanout, s);
    });
    cur = nxt;
  }
  if (rc) return rc;
  PRT_CUDA(cudaGetLastError());
  return PRT_OK;
}

}  // namespace prt
