// Overlay: clip every candidate pair with GPC semantics.
//
// Two schedules over the same device clipper (prt_gpc.cuh):
//   PLAIN    one thread per pair in the order given (the reference's Execute,
//            vector_map_overlay_gpc_kernel.cu:81-113), each with an arena
//            slice sized for its own vertex count; launched in chunks that fit
//            the memory budget.
//   BATCHED  pairs sorted by vertex count (radix sort, descending) and cut
//            into size bins; each bin is ONE persistent launch whose workers
//            own a fixed arena slice and take the next 32 pairs per warp from
//            an atomic ticket, so a warp's lanes clip pairs of similar cost.
// Results go to shared pools through atomic bump reservations (contours and
// vertices), the device analogue of the reference's per-pair device malloc
// (GPC:703-718).  Pairs whose slice or pool reservation was too small are
// retried with larger slices / grown pools.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include <mutex>

#include "prt_gpc.cuh"
#include "prt_internal.cuh"
#include "prt_overlay.cuh"
#include "prt_wgpc.cuh"

namespace prt {

// per-pair status: ok, arena slice too small (retried), pair ids out of range,
// result pool full (retried), malformed internal list (reported as an error)
enum : int { kPairOk = 0, kPairArena = 1, kPairInvalid = 2, kPairPool = 3, kPairCorrupt = 4 };

struct ClipOut {
  int32_t *status;
  int64_t *pair_cstart;
  int32_t *pair_ncont;
  int64_t *cont_vstart;
  int32_t *cont_nverts;
  int32_t *cont_hole;
  double *xy;
  unsigned long long *pool;  // [0] contours reserved, [1] vertices reserved
  int64_t cap_c, cap_v;
  double *area;  // area-only mode when non-null
};

__device__ inline bool resolve(const PairSrc &S, int64_t i, gpc::PolyView &a, gpc::PolyView &b, int64_t &nv) {
  int64_t pa, pb;
  if (S.pairs) {
    uint2 p = S.pairs[i];
    int64_t leaf = (int64_t)(int32_t)p.x - S.offset;
    pa = S.leaf_to_poly ? (leaf >= 0 ? (int64_t)S.leaf_to_poly[leaf] : -1) : leaf;
    pb = (int64_t)(int32_t)p.y;
  } else {
    pa = S.pa[i];
    pb = S.pb[i];
  }
  if (pa < 0 || pa >= S.base.n_poly || pb < 0 || pb >= S.over.n_poly) return false;
  a.ring_vert = S.base.ring_vert;
  a.xy = S.base.xy;
  a.r0 = S.base.poly_ring[pa];
  a.r1 = S.base.poly_ring[pa + 1];
  b.ring_vert = S.over.ring_vert;
  b.xy = S.over.xy;
  b.r0 = S.over.poly_ring[pb];
  b.r1 = S.over.poly_ring[pb + 1];
  nv = (a.ring_vert[a.r1] - a.ring_vert[a.r0]) + (b.ring_vert[b.r1] - b.ring_vert[b.r0]);
  return true;
}

// Records the clip result of pair i (arena A, output list head): per-pair
// area, or contours and vertices reserved from the result pools.
__device__ __noinline__ void finish_pair(const ClipOut &O, int64_t i, gpc::Arena &A, int head) {
  int nc = 0;
  int64_t nvt = 0;
  if (!A.status) gpc::count_result(A, head, &nc, &nvt);
  if (A.status) {
    O.status[i] = A.status == gpc::kClipCapacity ? kPairArena : kPairCorrupt;
    if (O.pair_ncont) O.pair_ncont[i] = 0;
    return;
  }
  if (O.area) {
    O.area[i] = nc ? gpc::result_area(A, head) : 0.0;
    O.status[i] = kPairOk;
    return;
  }
  int64_t cbase = 0, vbase = 0;
  if (nc) {
    cbase = (int64_t)atomicAdd(&O.pool[0], (unsigned long long)nc);
    vbase = (int64_t)atomicAdd(&O.pool[1], (unsigned long long)nvt);
    if (cbase + nc > O.cap_c || vbase + nvt > O.cap_v) {
      // record what the pair needs so the host grows the pools enough
      O.pair_ncont[i] = nc;
      O.pair_cstart[i] = nvt;
      O.status[i] = kPairPool;
      return;
    }
    gpc::write_result(A, head, O.cont_nverts, O.cont_hole, O.cont_vstart, O.xy, cbase, vbase);
  }
  O.pair_cstart[i] = cbase;
  O.pair_ncont[i] = nc;
  O.status[i] = kPairOk;
}

__device__ inline void invalid_pair(const ClipOut &O, int64_t i) {
  O.status[i] = kPairInvalid;
  if (O.pair_ncont) O.pair_ncont[i] = 0;
  if (O.area) O.area[i] = 0.0;
}

// One pair on the calling thread.
__device__ __noinline__ void process_pair(const PairSrc &S, const ClipOut &O, int64_t i, unsigned char *slice, int scale) {
  gpc::PolyView a, b;
  int64_t nv = 0;
  if (!resolve(S, i, a, b, nv)) {
    invalid_pair(O, i);
    return;
  }
  gpc::Arena A;
  gpc::arena_init(A, slice, gpc::caps_for(nv, scale));
  int head = gpc::clip_pair(A, S.op, a, b);
  finish_pair(O, i, A, head);
}

// One pair on the calling warp (all lanes): the warp clipper, or the thread
// clipper on lane 0 when the pair outgrows the warp's active-edge slots.
__device__ __noinline__ void process_pair_warp(const PairSrc &S, const ClipOut &O, int64_t i, unsigned char *slice, int scale,
                                  gpc::WAet &W, unsigned long long *fallbacks) {
  const int lane = threadIdx.x & 31;
  gpc::PolyView a, b;
  int64_t nv = 0;
  if (!resolve(S, i, a, b, nv)) {
    if (lane == 0) invalid_pair(O, i);
    __syncwarp();
    return;
  }
  gpc::Arena A;
  const gpc::Caps caps = gpc::caps_for(nv, scale);
  gpc::arena_init(A, slice, caps);
  int mode = gpc::kWarpOk;
  int head = gpc::wclip_pair(A, S.op, a, b, W, &mode);
  __syncwarp();
  if (lane == 0) {
    if (mode == gpc::kWarpFallback) {
      if (fallbacks) atomicAdd(fallbacks, 1ull);
      gpc::arena_init(A, slice, caps);
      head = gpc::clip_pair(A, S.op, a, b);
    }
    finish_pair(O, i, A, head);
  }
  __syncwarp();
}

namespace {

__global__ void nv_kernel(PairSrc S, int64_t n, const int64_t *__restrict__ idx, int scale, int64_t *__restrict__ nv,
                          int64_t *__restrict__ demand) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t i = idx ? idx[t] : t;
    gpc::PolyView a, b;
    int64_t v = 0;
    if (!resolve(S, i, a, b, v)) v = 0;
    if (nv) nv[t] = v;
    if (demand) demand[t] = (int64_t)gpc::arena_bytes(gpc::caps_for(v, scale));
  }
}

__global__ void __launch_bounds__(128) clip_plain_kernel(PairSrc S, ClipOut O, const int64_t *__restrict__ idx,
                                                         int64_t begin, int64_t count, unsigned char *arena,
                                                         const int64_t *__restrict__ arena_off, int64_t off_base,
                                                         int scale) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= count) return;
  int64_t k = begin + t;
  int64_t i = idx ? idx[k] : k;
  process_pair(S, O, i, arena + (arena_off[k] - off_base), scale);
}

// One persistent launch over all bins (longest pairs first): each warp drains
// its own bin from the bin's atomic ticket (one pair per ticket in warp mode,
// 32 in thread mode), then steals from the smaller bins after it.  One warp
// per block spreads the big-pair warps over every SM; the block's dynamic
// shared memory holds the warp clipper's active-edge slots.
// The body of the persistent launch; kWarp = false compiles the warp clipper
// out (every bin in thread mode).
template <bool kWarp>
__device__ __forceinline__ void lpt_body(const PairSrc &S, const ClipOut &O, const uint32_t *__restrict__ order,
                                         const BinPlan &plan, unsigned long long *tickets, unsigned char *arena,
                                         int scale, const int64_t *__restrict__ dyn_ranges) {
  __shared__ int64_t s_begin[PRT_MAX_BINS], s_end[PRT_MAX_BINS];
  __shared__ int32_t s_mode[PRT_MAX_BINS];
  const int lane = threadIdx.x & 31;
  const int64_t w = blockIdx.x;
  const int nbins = plan.nbins;
  if (lane < nbins) {
    // bin ranges from the plan, or computed on the device (graph mode)
    s_begin[lane] = dyn_ranges ? dyn_ranges[2 * lane] : plan.begin[lane];
    s_end[lane] = dyn_ranges ? dyn_ranges[2 * lane + 1] : plan.end[lane];
    s_mode[lane] = plan.warp_mode[lane];
  }
  __syncwarp();
  gpc::WAet W = gpc::waet_carve(plan.wcap);
  int g = 0;
  while (g + 1 < nbins && w >= plan.warp0[g + 1]) g++;
  unsigned char *region = arena + plan.arena_off[g] + (w - plan.warp0[g]) * plan.region[g];
  unsigned char *slice = region + (int64_t)lane * ((plan.region[g] / 32) & ~(int64_t)15);
  unsigned long long *fallbacks = tickets + PRT_MAX_BINS;
  for (int b = g; b < nbins; b++) {
    const int64_t begin = s_begin[b], end = s_end[b];
    if (kWarp && s_mode[b]) {
      for (;;) {
        unsigned long long t = 0;
        if (lane == 0) t = atomicAdd(&tickets[b], 1ull);
        t = __shfl_sync(0xffffffffu, t, 0);
        const int64_t k = begin + (int64_t)t;
        if (k >= end) break;
        const int64_t i = (int64_t)order[k];
        if (i < plan.n_pairs) process_pair_warp(S, O, i, region, scale, W, fallbacks);
      }
    } else {
      for (;;) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(&tickets[b], 32ull);
        base = __shfl_sync(0xffffffffu, base, 0);
        const int64_t k0 = begin + (int64_t)base;
        if (k0 >= end) break;
        const int64_t k = k0 + lane;
        if (k < end && (int64_t)order[k] < plan.n_pairs) process_pair(S, O, (int64_t)order[k], slice, scale);
        __syncwarp();
      }
    }
  }
}

// Compiled for kLptWarpsPerSM resident warps per SM (at most 168 registers a
// thread): with fewer, the warp clipper's shuffle and FP64 latencies go
// unhidden; with more, its register loop spills.
__global__ void __launch_bounds__(32, kLptWarpsPerSM)
    clip_lpt_kernel(PairSrc S, ClipOut O, const uint32_t *__restrict__ order, BinPlan plan,
                    unsigned long long *tickets, unsigned char *arena, int scale,
                    const int64_t *__restrict__ dyn_ranges) {
  lpt_body<true>(S, O, order, plan, tickets, arena, scale, dyn_ranges);
}

// The same launch when no bin with pairs is in warp mode: without the warp
// clipper the thread clipper fits kLptThreadWarpsPerSM resident warps per SM,
// which hide more of its list-walking latency.
__global__ void __launch_bounds__(32, kLptThreadWarpsPerSM)
    clip_lpt_thread_kernel(PairSrc S, ClipOut O, const uint32_t *__restrict__ order, BinPlan plan,
                           unsigned long long *tickets, unsigned char *arena, int scale) {
  lpt_body<false>(S, O, order, plan, tickets, arena, scale, nullptr);
}

// Sort keys: larger vertex counts first.
__global__ void size_key_kernel(const int64_t *__restrict__ nv, int64_t n, uint32_t *__restrict__ key,
                                uint32_t *__restrict__ val) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t v = nv[i];
    key[i] = 0xFFFFFFFFu - (uint32_t)(v > 0xFFFFFFFFll ? 0xFFFFFFFFll : v);
    val[i] = (uint32_t)i;
  }
}

// bounds[b] = first sorted position whose vertex count is <= thr[b]
// (counts descend along the sorted order); maxnv[b] = count at that position.
__global__ void bin_bounds_kernel(const uint32_t *__restrict__ k0, const uint32_t *__restrict__ k1,
                                  const int *__restrict__ sel, int64_t n, const int64_t *__restrict__ thr, int nbins,
                                  int64_t *__restrict__ bounds, int64_t *__restrict__ maxnv) {
  const uint32_t *k = *sel ? k1 : k0;
  int b = threadIdx.x;
  if (b >= nbins) return;
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t mid = (lo + hi) / 2;
    int64_t v = (int64_t)(0xFFFFFFFFu - k[mid]);
    if (v > thr[b]) lo = mid + 1;
    else hi = mid;
  }
  bounds[b] = lo;
  maxnv[b] = lo < n ? (int64_t)(0xFFFFFFFFu - k[lo]) : 0;
}

// dst[i] = the sorted value i (from a or b per *sel), mapped through idx when given.
__global__ void select_u32_kernel(const uint32_t *a, const uint32_t *b, const int *sel, int64_t n, uint32_t *dst,
                                  const int64_t *__restrict__ idx = nullptr) {
  const uint32_t *src = *sel ? b : a;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t k = src[i];
    // a timed-out sort can leave any value here: out-of-range positions are
    // marked, skipped by the clip, and the caller reports the timeout
    dst[i] = (int64_t)k >= n ? 0xFFFFFFFFu : idx ? (uint32_t)idx[k] : k;
  }
}

__global__ void area_from_results_kernel(const int64_t *__restrict__ pair_cstart, const int32_t *__restrict__ pair_ncont,
                                         const int64_t *__restrict__ cont_vstart, const int32_t *__restrict__ cont_nverts,
                                         const int32_t *__restrict__ cont_hole, const double *__restrict__ xy, int64_t n,
                                         double *__restrict__ area) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double total = 0.0;
    for (int c = 0; c < pair_ncont[i]; c++) {
      int64_t cc = pair_cstart[i] + c;
      const double *v = xy + 2 * cont_vstart[cc];
      int m = cont_nverts[cc];
      double a = 0.0;
      // relative to the first vertex, in output order (as the oracle sums)
      const double x0 = v[0], y0 = v[1];
      for (int j = 0; j < m; j++) {
        int k = (j + 1) % m;
        a += (v[2 * j] - x0) * (v[2 * k + 1] - y0) - (v[2 * k] - x0) * (v[2 * j + 1] - y0);
      }
      a = 0.5 * fabs(a);
      total += cont_hole[cc] ? -a : a;
    }
    area[i] = total;
  }
}

// contours, vertices and non-empty pairs over the live results
__global__ void result_totals_kernel(const int64_t *__restrict__ pair_cstart, const int32_t *__restrict__ pair_ncont,
                                     const int32_t *__restrict__ cont_nverts, int64_t n,
                                     unsigned long long *__restrict__ tot) {
  unsigned long long c = 0, v = 0, ne = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int k = pair_ncont[i];
    c += k;
    ne += k > 0;
    for (int j = 0; j < k; j++) v += cont_nverts[pair_cstart[i] + j];
  }
  for (int o = 16; o; o >>= 1) {
    c += __shfl_xor_sync(0xffffffffu, c, o);
    v += __shfl_xor_sync(0xffffffffu, v, o);
    ne += __shfl_xor_sync(0xffffffffu, ne, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&tot[0], c);
    atomicAdd(&tot[1], v);
    atomicAdd(&tot[2], ne);
  }
}

size_t arena_budget() {
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
    cudaGetLastError();
    return (size_t)1 << 30;
  }
  size_t b = fr / 3;
  const size_t cap = (size_t)48 << 30;
  return std::max<size_t>(std::min(b, cap), (size_t)64 << 20);
}

}  // namespace

// ---- batched schedule ----------------------------------------------------------
// Default: pairs above 128 vertices are clipped one per warp, smaller ones one
// per thread (32 pairs of up to 256 vertices in one warp's ticket made the
// ticket long enough to leave a tail; below 128, one pair per thread is the
// faster mode); kLptWarpsPerSM warps per SM, what an SM holds at the clip
// kernel's register count; 64 shared-memory slots per warp (the warp
// clipper keeps active edge tables of up to 32 edges in registers).
static prt_schedule default_schedule() {
  prt_schedule d;
  memset(&d, 0, sizeof d);
  d.nbins = 6;
  d.aet_slots = 64;
  d.warps_per_sm = kLptWarpsPerSM;
  const int64_t thr[6] = {1ll << 40, 4096, 1024, 256, 128, 64};
  const int32_t wm[6] = {1, 1, 1, 1, 0, 0};
  for (int b = 0; b < 6; b++) {
    d.bin_thresholds[b] = thr[b];
    d.bin_warp_mode[b] = wm[b];
  }
  return d;
}

static std::mutex g_sched_mu;
static prt_schedule g_sched = default_schedule();

prt_schedule current_schedule() {
  std::lock_guard<std::mutex> lk(g_sched_mu);
  return g_sched;
}

int schedule_valid(const prt_schedule &s) {
  PRT_CHECK(s.nbins >= 1 && s.nbins <= PRT_MAX_BINS, PRT_ERR_INVALID, "schedule: nbins %d", s.nbins);
  PRT_CHECK(s.aet_slots >= 32 && s.aet_slots <= 2048 && s.aet_slots % 32 == 0, PRT_ERR_INVALID,
            "schedule: aet_slots %d (a multiple of 32 in [32, 2048])", s.aet_slots);
  for (int b = 0; b < s.nbins; b++) {
    PRT_CHECK(s.bin_thresholds[b] > 0, PRT_ERR_INVALID, "schedule: threshold %d", b);
    PRT_CHECK(b == 0 || s.bin_thresholds[b] < s.bin_thresholds[b - 1], PRT_ERR_INVALID,
              "schedule: thresholds must descend");
    PRT_CHECK(s.bin_warp_mode[b] == 0 || s.bin_warp_mode[b] == 1, PRT_ERR_INVALID, "schedule: warp mode of bin %d",
              b);
  }
  PRT_CHECK(s.bin_thresholds[0] >= (1ll << 31), PRT_ERR_INVALID, "schedule: bin 0 must hold every pair size");
  PRT_CHECK(s.warps_per_sm >= 1 && s.warps_per_sm <= 64, PRT_ERR_INVALID, "schedule: warps_per_sm %d",
            s.warps_per_sm);
  return PRT_OK;
}

size_t plan_bins(const prt_schedule &sc, const int64_t *counts, const int64_t *maxnv, size_t budget, BinPlan &plan,
                 size_t *smem, int scale, bool thread_kernel) {
  memset(&plan, 0, sizeof plan);
  plan.nbins = sc.nbins;
  plan.wcap = sc.aet_slots;
  int64_t need[PRT_MAX_BINS];
  bool any_warp = false;
  for (int b = 0; b < sc.nbins; b++) {
    const gpc::Caps caps = gpc::caps_for(maxnv[b] > 0 ? maxnv[b] : 4, scale);
    plan.warp_mode[b] = sc.bin_warp_mode[b];
    const int64_t sl = (int64_t)gpc::align16(sc.bin_warp_mode[b] ? gpc::warp_arena_bytes(caps) : gpc::arena_bytes(caps));
    need[b] = counts[b] > 0 ? (sc.bin_warp_mode[b] ? sl : 32 * sl) : 0;
    any_warp |= sc.bin_warp_mode[b] && counts[b] > 0;
  }
  // one group: every warp starts on the largest bin and moves down as bins
  // drain, so its arena region holds the largest need of any bin
  int64_t region = 512, work = 0;
  for (int b = 0; b < sc.nbins; b++) {
    region = std::max(region, need[b]);
    work += sc.bin_warp_mode[b] ? counts[b] : (counts[b] + 31) / 32;
  }
  region = (region + 511) & ~(int64_t)511;
  // no more warps than can be resident: the persistent launch must not queue
  // (a launch without warp-mode pairs uses the thread-only kernel, whose
  // resident limit is higher; the schedule's warps_per_sm is for the other)
  plan.thread_only = thread_kernel && !any_warp ? 1 : 0;
  const int per_sm = plan.thread_only ? kLptThreadWarpsPerSM : std::min(sc.warps_per_sm, kLptWarpsPerSM);
  int64_t warps = std::min<int64_t>(work, (int64_t)kSMs * per_sm);
  warps = std::min<int64_t>(warps, (int64_t)(budget / (size_t)region));
  if (work > 0) warps = std::max<int64_t>(warps, 1);
  for (int b = 0; b <= sc.nbins; b++) plan.warp0[b] = b == 0 ? 0 : warps;
  plan.arena_off[0] = 0;
  plan.region[0] = region;
  const size_t bytes = (size_t)warps * (size_t)region;
  plan.warp0[sc.nbins] = warps;
  *smem = any_warp ? gpc::waet_bytes(sc.aet_slots) : 0;
  return bytes;
}

struct OverlayState {
  PairSrc S;
  ClipOut O;
  int64_t n;
  int sched = PRT_SCHED_PLAIN;
  int64_t retried = 0;
};

static int grow_pools(OverlayState &st, cudaStream_t s, int64_t need_c, int64_t need_v) {
  unsigned long long used[2];
  PRT_CUDA(cudaMemcpyAsync(used, st.O.pool, sizeof used, cudaMemcpyDeviceToHost, s));
  PRT_CUDA(cudaStreamSynchronize(s));
  int64_t nc = std::max<int64_t>(2 * st.O.cap_c, (int64_t)used[0] + need_c + 1024);
  int64_t nvv = std::max<int64_t>(2 * st.O.cap_v, (int64_t)used[1] + need_v + 1024);
  int64_t *cvs = nullptr;
  int32_t *cnv = nullptr, *ch = nullptr;
  double *xy = nullptr;
  int rc = dalloc(&cvs, nc, s);
  if (!rc) rc = dalloc(&cnv, nc, s);
  if (!rc) rc = dalloc(&ch, nc, s);
  if (!rc) rc = dalloc(&xy, 2 * nvv, s);
  if (rc) {
    dfree(cvs, s);
    dfree(cnv, s);
    dfree(ch, s);
    return rc;
  }
  int64_t kc = std::min<int64_t>((int64_t)used[0], st.O.cap_c), kv = std::min<int64_t>((int64_t)used[1], st.O.cap_v);
  if (kc) {
    cudaMemcpyAsync(cvs, st.O.cont_vstart, 8 * kc, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(cnv, st.O.cont_nverts, 4 * kc, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(ch, st.O.cont_hole, 4 * kc, cudaMemcpyDeviceToDevice, s);
  }
  if (kv) cudaMemcpyAsync(xy, st.O.xy, 16 * kv, cudaMemcpyDeviceToDevice, s);
  dfree(st.O.cont_vstart, s);
  dfree(st.O.cont_nverts, s);
  dfree(st.O.cont_hole, s);
  dfree(st.O.xy, s);
  st.O.cont_vstart = cvs;
  st.O.cont_nverts = cnv;
  st.O.cont_hole = ch;
  st.O.xy = xy;
  st.O.cap_c = nc;
  st.O.cap_v = nvv;
  PRT_CUDA(cudaGetLastError());
  return PRT_OK;
}

// Plain launches over items [0, count) of idx (or all pairs when idx is
// NULL), chunked by the arena budget.
static int run_plain(OverlayState &st, const int64_t *d_idx, int64_t count, int scale, cudaStream_t s) {
  if (count == 0) return PRT_OK;
  int64_t *demand = nullptr, *off = nullptr;
  int rc = dalloc(&demand, count, s);
  if (!rc) rc = dalloc(&off, count + 1, s);
  if (rc) {
    dfree(demand, s);
    return rc;
  }
  {
    PRT_PROF("nv", s);
    nv_kernel<<<grid_for(count, 256, 16), 256, 0, s>>>(st.S, count, d_idx, scale, nullptr, demand);
  }
  rc = exclusive_scan<int64_t>(demand, count, off, off + count, s);
  std::vector<int64_t> h_off(count + 1);
  if (!rc) {
    cudaError_t e = cudaMemcpyAsync(h_off.data(), off, 8 * (count + 1), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = cuda_status(e, "overlay plain");
  }
  const int64_t budget = (int64_t)arena_budget();
  unsigned char *arena = nullptr;
  int64_t arena_cap = 0;
  int64_t b = 0;
  while (!rc && b < count) {
    int64_t e = b + 1;
    // largest chunk [b, e) that fits the budget (at least one pair)
    int64_t lo = b + 1, hi = count;
    while (lo < hi) {
      int64_t mid = (lo + hi + 1) / 2;
      if (h_off[mid] - h_off[b] <= budget) lo = mid;
      else hi = mid - 1;
    }
    e = lo;
    int64_t bytes = h_off[e] - h_off[b];
    if (bytes > arena_cap) {
      dfree(arena, s);
      arena = nullptr;
      rc = dmalloc(reinterpret_cast<void **>(&arena), bytes, s);
      if (rc) break;
      arena_cap = bytes;
    }
    int64_t cnt = e - b;
    {
      PRT_PROF("clip_plain", s);
      clip_plain_kernel<<<(unsigned)((cnt + 127) / 128), 128, 0, s>>>(st.S, st.O, d_idx, b, cnt, arena, off, h_off[b],
                                                                    scale);
    }
    b = e;
  }
  if (!rc) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) rc = cuda_status(e, "clip_plain_kernel");
  }
  dfree(arena, s);
  dfree(demand, s);
  dfree(off, s);
  return rc;
}

// Lets the persistent clip kernel take `smem` bytes of dynamic shared memory
// (the warp clipper's slots); called before any launch or capture.
int prepare_lpt_launch(size_t smem) {
  if (smem > 48 * 1024)
    PRT_CUDA(cudaFuncSetAttribute(clip_lpt_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  return PRT_OK;
}

// Batched launch over items [0, count) of idx (or all pairs when idx is NULL)
// with arena slices of `scale` times the first size.
static int run_batched(OverlayState &st, const int64_t *d_idx, int64_t count, int scale, cudaStream_t s) {
  if (count == 0) return PRT_OK;
  const int64_t n = count;
  const prt_schedule sc = current_schedule();
  const int nb = sc.nbins;
  int64_t *nv = nullptr;
  unsigned char *scr = nullptr;
  int rc = dalloc(&nv, n, s);
  if (!rc) rc = dmalloc(reinterpret_cast<void **>(&scr), 512 + 16 * n + 4 * n, s);
  if (rc) {
    dfree(nv, s);
    return rc;
  }
  unsigned *err = reinterpret_cast<unsigned *>(scr);
  int *sel = reinterpret_cast<int *>(scr + 8);
  int64_t *thr = reinterpret_cast<int64_t *>(scr + 16);                            // PRT_MAX_BINS
  int64_t *bnd = thr + PRT_MAX_BINS;                                               // PRT_MAX_BINS
  int64_t *mx = bnd + PRT_MAX_BINS;                                                // PRT_MAX_BINS
  unsigned long long *tickets = reinterpret_cast<unsigned long long *>(mx + PRT_MAX_BINS);  // bins + fallbacks
  uint32_t *k0 = reinterpret_cast<uint32_t *>(scr + 512);
  uint32_t *k1 = k0 + n, *v0 = k1 + n, *v1 = v0 + n, *order = v1 + n;
  cudaMemsetAsync(scr, 0, 512, s);
  cudaMemcpyAsync(thr, sc.bin_thresholds, sizeof(int64_t) * nb, cudaMemcpyHostToDevice, s);
  const int g = grid_for(n, 256, 16);
  {
    PRT_PROF("nv", s);
    nv_kernel<<<g, 256, 0, s>>>(st.S, n, d_idx, 1, nv, nullptr);
  }
  {
    PRT_PROF("size_key", s);
    size_key_kernel<<<g, 256, 0, s>>>(nv, n, k0, v0);
  }
  rc = radix_sort_pairs<uint32_t>(k0, v0, k1, v1, n, 32, sel, err, s);
  int64_t hb[PRT_MAX_BINS + 1] = {0}, hm[PRT_MAX_BINS] = {0};
  if (!rc) {
    {
      PRT_PROF("select_u32", s);
      select_u32_kernel<<<g, 256, 0, s>>>(v0, v1, sel, n, order, d_idx);
    }
    {
      PRT_PROF("bin_bounds", s);
      bin_bounds_kernel<<<1, 32, 0, s>>>(k0, k1, sel, n, thr, nb, bnd, mx);
    }
    unsigned herr = 0;
    cudaMemcpyAsync(hb, bnd, sizeof(int64_t) * nb, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(hm, mx, sizeof(int64_t) * nb, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&herr, err, sizeof herr, cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = cuda_status(e, "overlay batched");
    if (!rc && (herr & kErrTimeout)) {
      set_error("overlay batched: size sort look-back wait timed out");
      rc = PRT_ERR_TIMEOUT;
    }
  }
  // bin b covers sorted positions [bnd[b], bnd[b+1]) (bnd[nbins] = n)
  hb[nb] = n;
  BinPlan plan;
  int64_t counts[PRT_MAX_BINS];
  for (int b = 0; b < nb; b++) counts[b] = hb[b + 1] - hb[b];
  // Too few pairs to keep the GPU busy one per thread (under half a wave of
  // the thread-only launch, e.g. the 2 x 10,000-star overlay's ~21k pairs in
  // ~650 warps): clip every pair with a whole warp instead, so there are as
  // many warps as pairs.  Both clippers give the same output.
  prt_schedule run_sc = sc;
  {
    int64_t thread_warps = 0;
    for (int b = 0; b < nb; b++)
      if (!sc.bin_warp_mode[b]) thread_warps += (counts[b] + 31) / 32;
    if (thread_warps > 0 && thread_warps < (int64_t)kSMs * kLptThreadWarpsPerSM / 2)
      for (int b = 0; b < nb; b++) run_sc.bin_warp_mode[b] = 1;
  }
  size_t smem = 0;
  const size_t bytes = plan_bins(run_sc, counts, hm, arena_budget(), plan, &smem, scale, true);
  plan.n_pairs = st.n;
  for (int b = 0; b < nb; b++) {
    plan.begin[b] = hb[b];
    plan.end[b] = hb[b + 1];
  }
  const int64_t warps = plan.warp0[nb];
  unsigned char *arena = nullptr;
  if (!rc) rc = prepare_lpt_launch(smem);
  if (!rc && warps > 0) rc = dmalloc(reinterpret_cast<void **>(&arena), bytes, s);
  if (!rc && warps > 0) {
    PRT_PROF("clip_batched", s);
    if (plan.thread_only)
      clip_lpt_thread_kernel<<<(unsigned)warps, 32, 0, s>>>(st.S, st.O, order, plan, tickets, arena, scale);
    else
      clip_lpt_kernel<<<(unsigned)warps, 32, smem, s>>>(st.S, st.O, order, plan, tickets, arena, scale, nullptr);
  }
  if (!rc) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) rc = cuda_status(e, "clip_batched_kernel");
  }
  dfree(arena, s);
  dfree(nv, s);
  dfree(scr, s);
  return rc;
}

// Retries pairs whose arena slice or pool reservation was too small.
static int retry_failed(OverlayState &st, cudaStream_t s) {
  const int64_t n = st.n;
  std::vector<int32_t> hs(n);
  std::vector<int32_t> scale(n, 1);  // arena scale per pair: x4 after each arena overflow
  for (int round = 0; round < 8; round++) {
    PRT_CUDA(cudaMemcpyAsync(hs.data(), st.O.status, 4 * n, cudaMemcpyDeviceToHost, s));
    PRT_CUDA(cudaStreamSynchronize(s));
    std::vector<int64_t> pool_fail;
    bool any = false;
    for (int64_t i = 0; i < n; i++) {
      if (hs[i] == kPairArena) {
        if (scale[i] >= (1 << 12)) {
          set_error("overlay: pair %lld exceeds the largest arena slice", (long long)i);
          return PRT_ERR_CAPACITY;
        }
        scale[i] *= 4;
        any = true;
      } else if (hs[i] == kPairPool) {
        pool_fail.push_back(i);
        any = true;
      } else if (hs[i] == kPairInvalid) {
        set_error("overlay: pair %lld names a polygon outside its layer", (long long)i);
        return PRT_ERR_INVALID;
      } else if (hs[i] == kPairCorrupt) {
        set_error("overlay: pair %lld: clipper list walk exceeded its bound", (long long)i);
        return PRT_ERR_INVALID;
      }
    }
    if (!any) return PRT_OK;
    if (!pool_fail.empty()) {
      // the failing pairs recorded their needs in pair_ncont / pair_cstart
      std::vector<int32_t> nc(n);
      std::vector<int64_t> nvt(n);
      PRT_CUDA(cudaMemcpyAsync(nc.data(), st.O.pair_ncont, 4 * n, cudaMemcpyDeviceToHost, s));
      PRT_CUDA(cudaMemcpyAsync(nvt.data(), st.O.pair_cstart, 8 * n, cudaMemcpyDeviceToHost, s));
      PRT_CUDA(cudaStreamSynchronize(s));
      int64_t need_c = 0, need_v = 0;
      for (int64_t i : pool_fail) {
        need_c += nc[i];
        need_v += nvt[i];
      }
      int rc = grow_pools(st, s, need_c, need_v);
      if (rc) return rc;
    }
    // rerun every failed pair, grouped by arena scale
    std::vector<int32_t> scales;
    for (int64_t i = 0; i < n; i++)
      if (hs[i] == kPairArena || hs[i] == kPairPool) scales.push_back(scale[i]);
    std::sort(scales.begin(), scales.end());
    scales.erase(std::unique(scales.begin(), scales.end()), scales.end());
    for (int32_t sc : scales) {
      std::vector<int64_t> idx;
      for (int64_t i = 0; i < n; i++)
        if ((hs[i] == kPairArena || hs[i] == kPairPool) && scale[i] == sc) idx.push_back(i);
      st.retried += (int64_t)idx.size();
      int64_t *d_idx = nullptr;
      int rc = dalloc(&d_idx, idx.size(), s);
      if (rc) return rc;
      cudaMemcpyAsync(d_idx, idx.data(), 8 * idx.size(), cudaMemcpyHostToDevice, s);
      rc = st.sched == PRT_SCHED_PLAIN ? run_plain(st, d_idx, (int64_t)idx.size(), sc, s)
                                       : run_batched(st, d_idx, (int64_t)idx.size(), sc, s);
      dfree(d_idx, s);
      if (rc) return rc;
    }
  }
  set_error("overlay: pairs still failing after retries");
  return PRT_ERR_CAPACITY;
}

// ---- capture-safe overlay (graph pipeline) ----------------------------------

// Size keys of the first *d_count pairs (larger first); the padding slots up to
// cap sort last.
__global__ void graph_size_key_kernel(PairSrc S, const unsigned long long *__restrict__ d_count, int64_t cap,
                                      uint32_t *__restrict__ key, uint32_t *__restrict__ val) {
  const int64_t count = (int64_t)min((unsigned long long)cap, *d_count);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < cap; i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t k = 0xFFFFFFFFu;
    if (i < count) {
      gpc::PolyView a, b;
      int64_t v = 0;
      if (!resolve(S, i, a, b, v)) v = 0;
      if (v > 0xFFFFFFFEll) v = 0xFFFFFFFEll;
      k = 0xFFFFFFFEu - (uint32_t)v;
    }
    key[i] = k;
    val[i] = (uint32_t)i;
  }
}

// ranges[2b], ranges[2b+1]: sorted positions of bin b among the first count
__global__ void graph_bins_kernel(const uint32_t *__restrict__ k0, const uint32_t *__restrict__ k1,
                                  const int *__restrict__ sel, const unsigned long long *__restrict__ d_count,
                                  int64_t cap, const int64_t *__restrict__ thr, int nbins, int64_t *__restrict__ ranges) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const uint32_t *k = *sel ? k1 : k0;
  const int64_t count = (int64_t)min((unsigned long long)cap, *d_count);
  for (int b = 0; b < nbins; b++) {
    int64_t lo = 0, hi = count;
    while (lo < hi) {
      int64_t mid = (lo + hi) / 2;
      int64_t v = (int64_t)(0xFFFFFFFEu - k[mid]);
      if (v > thr[b]) lo = mid + 1;
      else hi = mid;
    }
    if (b > 0) ranges[2 * (b - 1) + 1] = lo;
    ranges[2 * b] = lo;
  }
  ranges[2 * (nbins - 1) + 1] = count;
}

__global__ void graph_totals_kernel(const int64_t *__restrict__ pair_cstart, const int32_t *__restrict__ pair_ncont,
                                    const int32_t *__restrict__ cont_nverts, const int32_t *__restrict__ status,
                                    const unsigned long long *__restrict__ d_count, int64_t cap,
                                    unsigned long long *__restrict__ tot) {
  const int64_t n = (int64_t)min((unsigned long long)cap, *d_count);
  unsigned long long c = 0, v = 0, ne = 0, bad = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (status[i] != kPairOk) {
      bad++;
      continue;
    }
    int k = pair_ncont[i];
    c += k;
    ne += k > 0;
    for (int j = 0; j < k; j++) v += cont_nverts[pair_cstart[i] + j];
  }
  for (int o = 16; o; o >>= 1) {
    c += __shfl_xor_sync(0xffffffffu, c, o);
    v += __shfl_xor_sync(0xffffffffu, v, o);
    ne += __shfl_xor_sync(0xffffffffu, ne, o);
    bad += __shfl_xor_sync(0xffffffffu, bad, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&tot[0], c);
    atomicAdd(&tot[1], v);
    atomicAdd(&tot[2], ne);
    atomicAdd(&tot[3], bad);
  }
}

int overlay_graph_enqueue(const PairSrc &S, const unsigned long long *d_npairs, GraphOverlay &G, cudaStream_t s) {
  const int64_t cap = G.cap_pairs;
  PRT_CUDA(cudaMemsetAsync(G.status, 0, 4 * cap, s));
  PRT_CUDA(cudaMemsetAsync(G.pair_ncont, 0, 4 * cap, s));
  PRT_CUDA(cudaMemsetAsync(G.tickets, 0, 8 * (PRT_MAX_BINS + 1), s));
  PRT_CUDA(cudaMemsetAsync(G.pool, 0, 16, s));
  PRT_CUDA(cudaMemsetAsync(G.totals, 0, 32, s));
  PRT_CUDA(cudaMemsetAsync(G.err, 0, 4, s));
  const int g = grid_for(cap, 256, 16);
  {
    PRT_PROF("size_key", s);
    graph_size_key_kernel<<<g, 256, 0, s>>>(S, d_npairs, cap, G.k0, G.v0);
  }
  int rc = radix_sort_pairs<uint32_t>(G.k0, G.v0, G.k1, G.v1, cap, 32, G.sel, G.err, s);
  if (rc) return rc;
  {
    PRT_PROF("select_u32", s);
    select_u32_kernel<<<g, 256, 0, s>>>(G.v0, G.v1, G.sel, cap, G.order);
  }
  {
    PRT_PROF("bin_bounds", s);
    graph_bins_kernel<<<1, 32, 0, s>>>(G.k0, G.k1, G.sel, d_npairs, cap, G.thresholds, G.plan.nbins, G.ranges);
  }
  ClipOut O;
  memset(&O, 0, sizeof O);
  O.status = G.status;
  O.pair_cstart = G.pair_cstart;
  O.pair_ncont = G.pair_ncont;
  O.cont_vstart = G.cont_vstart;
  O.cont_nverts = G.cont_nverts;
  O.cont_hole = G.cont_hole;
  O.xy = G.xy;
  O.pool = G.pool;
  O.cap_c = G.cap_c;
  O.cap_v = G.cap_v;
  const int64_t warps = G.plan.warp0[G.plan.nbins];
  if (warps > 0) {
    PRT_PROF("clip_batched", s);
    clip_lpt_kernel<<<(unsigned)warps, 32, G.smem, s>>>(S, O, G.order, G.plan, G.tickets, G.arena, 1, G.ranges);
  }
  {
    PRT_PROF("result_totals", s);
    graph_totals_kernel<<<grid_for(cap, 256, 8), 256, 0, s>>>(G.pair_cstart, G.pair_ncont, G.cont_nverts, G.status,
                                                             d_npairs, cap, G.totals);
  }
  PRT_CUDA(cudaGetLastError());
  return PRT_OK;
}

}  // namespace prt

namespace prt {

static void free_state(OverlayState &st, cudaStream_t s) {
  dfree(st.O.status, s);
  dfree(st.O.pair_cstart, s);
  dfree(st.O.pair_ncont, s);
  dfree(st.O.cont_vstart, s);
  dfree(st.O.cont_nverts, s);
  dfree(st.O.cont_hole, s);
  dfree(st.O.xy, s);
  dfree(st.O.pool, s);
}

// area != nullptr: area-only mode (no contour output, no results object).
int overlay_impl(const PairSrc &S, int64_t n, int sched, double *d_area, cudaStream_t s, prt_results **out) {
  PRT_CHECK(n >= 0 && n < (1ll << 31), PRT_ERR_INVALID, "n_pairs=%lld", (long long)n);
  PRT_CHECK(S.op >= 0 && S.op <= 3, PRT_ERR_INVALID, "op %d", S.op);
  PRT_CHECK(sched == PRT_SCHED_PLAIN || sched == PRT_SCHED_BATCHED, PRT_ERR_INVALID, "sched %d", sched);
  OverlayState st;
  st.S = S;
  st.n = n;
  st.sched = sched;
  memset(&st.O, 0, sizeof st.O);
  st.O.area = d_area;
  int rc = dalloc(&st.O.status, std::max<int64_t>(n, 1), s);
  if (!rc) rc = dalloc(&st.O.pool, 2, s);
  if (!rc && !d_area) rc = dalloc(&st.O.pair_cstart, std::max<int64_t>(n, 1), s);
  if (!rc && !d_area) rc = dalloc(&st.O.pair_ncont, std::max<int64_t>(n, 1), s);
  int64_t total_nv = 0;
  if (!rc && !d_area && n > 0) {
    int64_t *nv = nullptr, *tmp = nullptr;
    rc = dalloc(&nv, n, s);
    if (!rc) rc = dalloc(&tmp, n + 1, s);
    if (!rc) {
      {
        PRT_PROF("nv", s);
        nv_kernel<<<grid_for(n, 256, 16), 256, 0, s>>>(S, n, nullptr, 1, nv, nullptr);
      }
      rc = exclusive_scan<int64_t>(nv, n, tmp, tmp + n, s);
    }
    if (!rc) {
      cudaError_t e = cudaMemcpyAsync(&total_nv, tmp + n, 8, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) rc = cuda_status(e, "overlay sizes");
    }
    dfree(nv, s);
    dfree(tmp, s);
  }
  if (!rc && !d_area) {
    // first guess at the result size (grown on demand): half of the input
    // vertices, one contour per 64 of them
    st.O.cap_c = total_nv / 64 + 1024;
    st.O.cap_v = total_nv / 2 + 4096;
    rc = dalloc(&st.O.cont_vstart, st.O.cap_c, s);
    if (!rc) rc = dalloc(&st.O.cont_nverts, st.O.cap_c, s);
    if (!rc) rc = dalloc(&st.O.cont_hole, st.O.cap_c, s);
    if (!rc) rc = dalloc(&st.O.xy, 2 * st.O.cap_v, s);
  }
  if (!rc) {
    cudaError_t e = cudaMemsetAsync(st.O.pool, 0, 16, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(st.O.status, 0, 4 * std::max<int64_t>(n, 1), s);
    if (e != cudaSuccess) rc = cuda_status(e, "memset");
  }
  if (!rc && n > 0) rc = sched == PRT_SCHED_PLAIN ? run_plain(st, nullptr, n, 1, s) : run_batched(st, nullptr, n, 1, s);
  if (!rc && n > 0) rc = retry_failed(st, s);
  if (rc || d_area) {
    if (!rc) {
      cudaError_t e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) rc = cuda_status(e, "overlay");
    }
    free_state(st, s);
    return rc;
  }
  prt_results *r = new prt_results();
  r->n_pairs = n;
  r->retried = st.retried;
  r->pair_cstart = st.O.pair_cstart;
  r->pair_ncont = st.O.pair_ncont;
  r->status = st.O.status;
  r->cont_vstart = st.O.cont_vstart;
  r->cont_nverts = st.O.cont_nverts;
  r->cont_hole = st.O.cont_hole;
  r->xy = st.O.xy;
  r->pool = st.O.pool;
  // exact totals of the live results (pools may hold abandoned reservations)
  {
    unsigned long long *tot = nullptr;
    int rc2 = dalloc(&tot, 3, s);
    unsigned long long h[3] = {0, 0, 0};
    cudaError_t e = rc2 ? cudaErrorMemoryAllocation : cudaMemsetAsync(tot, 0, 24, s);
    if (e == cudaSuccess && n > 0) {
      PRT_PROF("result_totals", s);
      result_totals_kernel<<<grid_for(n, 256, 8), 256, 0, s>>>(r->pair_cstart, r->pair_ncont, r->cont_nverts, n, tot);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, tot, sizeof h, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    dfree(tot, s);
    if (e != cudaSuccess) {
      prt_results_free(r);
      return cuda_status(e, "overlay results");
    }
    r->n_cont = (int64_t)h[0];
    r->n_vert = (int64_t)h[1];
    r->nonempty = (int64_t)h[2];
  }
  *out = r;
  return PRT_OK;
}

__global__ void ident_rings_kernel(int64_t n, int64_t *poly_ring) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= n; i += (int64_t)gridDim.x * blockDim.x)
    poly_ring[i] = i;
}

__global__ void ring_vert_from_ref_kernel(const int32_t *num, const int64_t *prefix, int64_t n, int64_t *ring_vert) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    ring_vert[i] = prefix[i];
    if (i == n - 1) ring_vert[n] = prefix[i] + num[i];
  }
}

}  // namespace prt

using namespace prt;

extern "C" {

int prt_schedule_set(const prt_schedule *sched) {
  prt_schedule s = sched ? *sched : prt::default_schedule();
  int rc = prt::schedule_valid(s);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(prt::g_sched_mu);
  prt::g_sched = s;
  return PRT_OK;
}

int prt_schedule_get(prt_schedule *sched) {
  PRT_CHECK(sched != nullptr, PRT_ERR_INVALID, "NULL argument");
  *sched = prt::current_schedule();
  return PRT_OK;
}


int prt_overlay_run(const prt_pair *d_pairs, int64_t n_pairs, int32_t offset, const int32_t *d_leaf_to_poly,
                    const prt_layer *base, const prt_layer *overlay, int op, int sched, void *stream,
                    prt_results **out) {
  PRT_CHECK(out && base && overlay, PRT_ERR_INVALID, "NULL argument");
  PRT_CHECK(d_pairs || n_pairs == 0, PRT_ERR_INVALID, "d_pairs is NULL");
  *out = nullptr;
  PairSrc S;
  memset(&S, 0, sizeof S);
  S.pairs = reinterpret_cast<const uint2 *>(d_pairs);
  S.offset = offset;
  S.leaf_to_poly = d_leaf_to_poly;
  S.base = layer_dev(base);
  S.over = layer_dev(overlay);
  S.op = op;
  return overlay_impl(S, n_pairs, sched, nullptr, reinterpret_cast<cudaStream_t>(stream), out);
}

// The reference's per-polygon CSR (readData packs polygon i's vertices at
// [prefix[i], prefix[i] + num[i]) with prefix[i+1] = prefix[i] + num[i]) is a
// ring CSR with one ring per polygon: poly_ring = 0..n, ring_vert = prefix
// followed by the total.  The packing is checked before use.
static int ref_layer(const int32_t *num, const int64_t *prefix, int64_t n, int64_t **pr, int64_t **rv,
                     cudaStream_t s) {
  std::vector<int32_t> hn(n);
  std::vector<int64_t> hp(n);
  PRT_CUDA(cudaMemcpyAsync(hn.data(), num, 4 * n, cudaMemcpyDeviceToHost, s));
  PRT_CUDA(cudaMemcpyAsync(hp.data(), prefix, 8 * n, cudaMemcpyDeviceToHost, s));
  PRT_CUDA(cudaStreamSynchronize(s));
  for (int64_t i = 0; i + 1 < n; i++)
    PRT_CHECK(hp[i + 1] == hp[i] + hn[i], PRT_ERR_INVALID, "prefix[%lld] is not prefix[%lld] + num[%lld]",
              (long long)(i + 1), (long long)i, (long long)i);
  int rc = dalloc(pr, n + 1, s);
  if (!rc) rc = dalloc(rv, n + 1, s);
  if (rc) return rc;
  {
    PRT_PROF("ident_rings", s);
    ident_rings_kernel<<<grid_for(n + 1, 256, 4), 256, 0, s>>>(n, *pr);
  }
  {
    PRT_PROF("ring_vert_from_ref", s);
    ring_vert_from_ref_kernel<<<grid_for(n, 256, 4), 256, 0, s>>>(num, prefix, n, *rv);
  }
  PRT_CUDA(cudaGetLastError());
  return PRT_OK;
}

int prt_overlay_run_ref(const prt_pair *d_pairs, int64_t n_pairs, int32_t offset, const int32_t *d_leaf_to_poly,
                        const int32_t *d_num_base, const int64_t *d_prefix_base, const double *d_vertex_base,
                        const int32_t *d_hole_base, int64_t n_base, const int32_t *d_num_overlay,
                        const int64_t *d_prefix_overlay, const double *d_vertex_overlay,
                        const int32_t *d_hole_overlay, int64_t n_overlay, int op, int sched, void *stream,
                        prt_results **out) {
  PRT_CHECK(out, PRT_ERR_INVALID, "out is NULL");
  PRT_CHECK(n_base > 0 && n_overlay > 0, PRT_ERR_INVALID, "empty layer");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  // the hole flags are carried by the reference but not read by its clip
  (void)d_hole_base;
  (void)d_hole_overlay;
  int64_t *pr_b = nullptr, *rv_b = nullptr, *pr_o = nullptr, *rv_o = nullptr;
  int rc = ref_layer(d_num_base, d_prefix_base, n_base, &pr_b, &rv_b, s);
  if (!rc) rc = ref_layer(d_num_overlay, d_prefix_overlay, n_overlay, &pr_o, &rv_o, s);
  if (!rc) {
    PairSrc S;
    memset(&S, 0, sizeof S);
    S.pairs = reinterpret_cast<const uint2 *>(d_pairs);
    S.offset = offset;
    S.leaf_to_poly = d_leaf_to_poly;
    S.op = op;
    S.base.poly_ring = pr_b;
    S.base.ring_vert = rv_b;
    S.base.xy = d_vertex_base;
    S.base.n_poly = n_base;
    S.over.poly_ring = pr_o;
    S.over.ring_vert = rv_o;
    S.over.xy = d_vertex_overlay;
    S.over.n_poly = n_overlay;
    rc = overlay_impl(S, n_pairs, sched, nullptr, s, out);
  }
  cudaStreamSynchronize(s);
  dfree(pr_b, s);
  dfree(rv_b, s);
  dfree(pr_o, s);
  dfree(rv_o, s);
  return rc;
}

int prt_results_sizes(const prt_results *r, int64_t *sizes) {
  PRT_CHECK(r && sizes, PRT_ERR_INVALID, "NULL argument");
  sizes[0] = r->n_pairs;
  sizes[1] = r->n_cont;
  sizes[2] = r->n_vert;
  sizes[3] = r->nonempty;
  sizes[4] = r->retried;
  return PRT_OK;
}

int prt_results_device(const prt_results *r, const int64_t **pair_cont_start, const int32_t **pair_ncont,
                       const int64_t **cont_vert_start, const int32_t **cont_nverts, const int32_t **cont_hole,
                       const double **xy) {
  PRT_CHECK(r, PRT_ERR_INVALID, "NULL argument");
  if (pair_cont_start) *pair_cont_start = r->pair_cstart;
  if (pair_ncont) *pair_ncont = r->pair_ncont;
  if (cont_vert_start) *cont_vert_start = r->cont_vstart;
  if (cont_nverts) *cont_nverts = r->cont_nverts;
  if (cont_hole) *cont_hole = r->cont_hole;
  if (xy) *xy = r->xy;
  return PRT_OK;
}

int prt_results_copy(const prt_results *r, int64_t *h_pair_cont_off, int32_t *h_cont_nverts, int32_t *h_cont_hole,
                     double *h_xy) {
  PRT_CHECK(r && h_pair_cont_off && h_cont_nverts && h_cont_hole && h_xy, PRT_ERR_INVALID, "NULL argument");
  const int64_t n = r->n_pairs;
  unsigned long long used[2];
  PRT_CUDA(cudaDeviceSynchronize());
  PRT_CUDA(cudaMemcpy(used, r->pool, sizeof used, cudaMemcpyDeviceToHost));
  std::vector<int64_t> cs(n), cvs(used[0]);
  std::vector<int32_t> nc(n), cnv(used[0]), ch(used[0]);
  std::vector<double> xy(2 * used[1]);
  PRT_CUDA(cudaMemcpy(cs.data(), r->pair_cstart, 8 * n, cudaMemcpyDeviceToHost));
  PRT_CUDA(cudaMemcpy(nc.data(), r->pair_ncont, 4 * n, cudaMemcpyDeviceToHost));
  if (used[0]) {
    PRT_CUDA(cudaMemcpy(cvs.data(), r->cont_vstart, 8 * used[0], cudaMemcpyDeviceToHost));
    PRT_CUDA(cudaMemcpy(cnv.data(), r->cont_nverts, 4 * used[0], cudaMemcpyDeviceToHost));
    PRT_CUDA(cudaMemcpy(ch.data(), r->cont_hole, 4 * used[0], cudaMemcpyDeviceToHost));
  }
  if (used[1]) PRT_CUDA(cudaMemcpy(xy.data(), r->xy, 16 * used[1], cudaMemcpyDeviceToHost));
  int64_t c = 0, v = 0;
  h_pair_cont_off[0] = 0;
  for (int64_t i = 0; i < n; i++) {
    for (int k = 0; k < nc[i]; k++) {
      int64_t cc = cs[i] + k;
      h_cont_nverts[c] = cnv[cc];
      h_cont_hole[c] = ch[cc];
      memcpy(h_xy + 2 * v, xy.data() + 2 * cvs[cc], 16 * (size_t)cnv[cc]);
      v += cnv[cc];
      c++;
    }
    h_pair_cont_off[i + 1] = c;
  }
  return PRT_OK;
}

int prt_results_copy_pairs(const prt_results *r, const int64_t *h_pairs, int64_t k, int64_t *h_pair_cont_off,
                           int32_t *h_cont_nverts, int32_t *h_cont_hole, double *h_xy, int64_t cont_cap,
                           int64_t vert_cap, int64_t *h_need) {
  PRT_CHECK(r && (k == 0 || h_pairs) && h_pair_cont_off && h_need, PRT_ERR_INVALID, "NULL argument");
  PRT_CHECK(k >= 0, PRT_ERR_INVALID, "k < 0");
  for (int64_t j = 0; j < k; j++)
    PRT_CHECK(h_pairs[j] >= 0 && h_pairs[j] < r->n_pairs, PRT_ERR_INVALID, "pair %lld out of range",
              (long long)h_pairs[j]);
  PRT_CUDA(cudaDeviceSynchronize());
  std::vector<int64_t> cs(k);
  std::vector<int32_t> nc(k);
  for (int64_t j = 0; j < k; j++) {
    PRT_CUDA(cudaMemcpy(&cs[j], r->pair_cstart + h_pairs[j], 8, cudaMemcpyDeviceToHost));
    PRT_CUDA(cudaMemcpy(&nc[j], r->pair_ncont + h_pairs[j], 4, cudaMemcpyDeviceToHost));
  }
  // contour headers of the listed pairs, then their vertices
  std::vector<int64_t> cvs;
  std::vector<int32_t> cnv, ch;
  h_pair_cont_off[0] = 0;
  for (int64_t j = 0; j < k; j++) {
    const size_t o = cvs.size();
    cvs.resize(o + nc[j]);
    cnv.resize(o + nc[j]);
    ch.resize(o + nc[j]);
    if (nc[j]) {
      PRT_CUDA(cudaMemcpy(cvs.data() + o, r->cont_vstart + cs[j], 8 * (size_t)nc[j], cudaMemcpyDeviceToHost));
      PRT_CUDA(cudaMemcpy(cnv.data() + o, r->cont_nverts + cs[j], 4 * (size_t)nc[j], cudaMemcpyDeviceToHost));
      PRT_CUDA(cudaMemcpy(ch.data() + o, r->cont_hole + cs[j], 4 * (size_t)nc[j], cudaMemcpyDeviceToHost));
    }
    h_pair_cont_off[j + 1] = (int64_t)cvs.size();
  }
  int64_t nv = 0;
  for (int32_t v : cnv) nv += v;
  h_need[0] = (int64_t)cvs.size();
  h_need[1] = nv;
  if (h_need[0] > cont_cap || nv > vert_cap) {
    set_error("results_copy_pairs: %lld contours / %lld vertices exceed the buffers", (long long)h_need[0],
              (long long)nv);
    return PRT_ERR_CAPACITY;
  }
  PRT_CHECK(cvs.empty() || (h_cont_nverts && h_cont_hole && h_xy), PRT_ERR_INVALID, "NULL argument");
  int64_t v = 0;
  for (size_t c = 0; c < cvs.size(); c++) {
    h_cont_nverts[c] = cnv[c];
    h_cont_hole[c] = ch[c];
    if (cnv[c]) PRT_CUDA(cudaMemcpy(h_xy + 2 * v, r->xy + 2 * cvs[c], 16 * (size_t)cnv[c], cudaMemcpyDeviceToHost));
    v += cnv[c];
  }
  return PRT_OK;
}

int prt_results_area(const prt_results *r, double *d_area, void *stream) {
  PRT_CHECK(r && d_area, PRT_ERR_INVALID, "NULL argument");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (r->n_pairs == 0) return PRT_OK;
  {
    PRT_PROF("area_from_results", s);
    area_from_results_kernel<<<grid_for(r->n_pairs, 256, 16), 256, 0, s>>>(
      r->pair_cstart, r->pair_ncont, r->cont_vstart, r->cont_nverts, r->cont_hole, r->xy, r->n_pairs, d_area);
  }
  PRT_CUDA(cudaGetLastError());
  return PRT_OK;
}

int prt_results_free(prt_results *r) {
  if (!r) return PRT_OK;
  // stream-ordered release on the legacy default stream: no device-wide sync
  void *ptrs[] = {r->pair_cstart, r->pair_ncont, r->status, r->cont_vstart,
                  r->cont_nverts, r->cont_hole, r->xy, r->pool};
  for (void *p : ptrs)
    if (p) cudaFreeAsync(p, 0);
  cudaGetLastError();
  delete r;
  return PRT_OK;
}

int prt_clip_pair_host(int op, int s_ncont, const int32_t *s_nverts, const double *s_xy, int c_ncont,
                       const int32_t *c_nverts, const double *c_xy, int32_t *out_ncont, int32_t cont_cap,
                       int32_t *out_nverts, int32_t *out_hole, int64_t *out_nv, int64_t vert_cap, double *out_xy) {
  PRT_CHECK(out_ncont && out_nv && (s_ncont == 0 || (s_nverts && s_xy)) && (c_ncont == 0 || (c_nverts && c_xy)),
            PRT_ERR_INVALID, "NULL argument");
  PRT_CHECK(s_ncont >= 0 && c_ncont >= 0, PRT_ERR_INVALID, "negative contour count");
  // layers with one polygon each (zero-ring polygons allowed)
  std::vector<int64_t> pr_s = {0, s_ncont}, pr_c = {0, c_ncont};
  std::vector<int64_t> rv_s(s_ncont + 1, 0), rv_c(c_ncont + 1, 0);
  for (int i = 0; i < s_ncont; i++) rv_s[i + 1] = rv_s[i] + s_nverts[i];
  for (int i = 0; i < c_ncont; i++) rv_c[i + 1] = rv_c[i] + c_nverts[i];
  int64_t vs = rv_s[s_ncont], vc = rv_c[c_ncont];
  int64_t *d_i64 = nullptr;
  double *d_xy = nullptr;
  int32_t *d_pair = nullptr;
  size_t ni = 4 + (s_ncont + 1) + (c_ncont + 1);
  PRT_CUDA(cudaMalloc(&d_i64, 8 * ni));
  PRT_CUDA(cudaMalloc(&d_xy, 16 * (vs + vc + 1)));
  PRT_CUDA(cudaMalloc(&d_pair, 8));
  int64_t *d_prs = d_i64, *d_prc = d_i64 + 2, *d_rvs = d_i64 + 4, *d_rvc = d_rvs + s_ncont + 1;
  cudaMemcpy(d_prs, pr_s.data(), 16, cudaMemcpyHostToDevice);
  cudaMemcpy(d_prc, pr_c.data(), 16, cudaMemcpyHostToDevice);
  cudaMemcpy(d_rvs, rv_s.data(), 8 * (s_ncont + 1), cudaMemcpyHostToDevice);
  cudaMemcpy(d_rvc, rv_c.data(), 8 * (c_ncont + 1), cudaMemcpyHostToDevice);
  if (vs) cudaMemcpy(d_xy, s_xy, 16 * vs, cudaMemcpyHostToDevice);
  if (vc) cudaMemcpy(d_xy + 2 * vs, c_xy, 16 * vc, cudaMemcpyHostToDevice);
  int32_t zero[2] = {0, 0};
  cudaMemcpy(d_pair, zero, 8, cudaMemcpyHostToDevice);
  prt_layer Ls = {d_prs, d_rvs, nullptr, d_xy, 1};
  prt_layer Lc = {d_prc, d_rvc, nullptr, d_xy + 2 * vs, 1};
  prt_results *r = nullptr;
  int rc = prt_overlay_run(reinterpret_cast<const prt_pair *>(d_pair), 1, 0, nullptr, &Ls, &Lc, op,
                           PRT_SCHED_PLAIN, nullptr, &r);
  if (!rc) {
    *out_ncont = (int32_t)r->n_cont;
    *out_nv = r->n_vert;
    if (r->n_cont > cont_cap || r->n_vert > vert_cap) {
      set_error("clip_pair_host: result has %lld contours / %lld vertices", (long long)r->n_cont,
                (long long)r->n_vert);
      rc = PRT_ERR_CAPACITY;
    } else if (r->n_cont > 0) {
      std::vector<int64_t> off(2);
      rc = prt_results_copy(r, off.data(), out_nverts, out_hole, out_xy);
    }
  }
  prt_results_free(r);
  cudaFree(d_i64);
  cudaFree(d_xy);
  cudaFree(d_pair);
  return rc;
}

}  // extern "C"
