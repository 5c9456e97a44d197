// Onesweep LSD radix sort of (key, uint32 value) pairs.
//
// One upsweep kernel histograms every 8-bit digit of every key at once; a
// tiny plan kernel scans the histograms and marks passes whose digit is the
// same for all keys (they are skipped without a host round trip, so the whole
// sort can be captured in a CUDA graph).  Each remaining pass is ONE kernel:
// a CTA takes the next tile in launch order (atomic ticket), ranks its keys
// with a warp-level multisplit (lanes with the same digit found by one ballot
// per digit bit), learns its global digit
// offsets by decoupled look-back over the preceding tiles (bounded spin, an
// error flag instead of a hang), stages the tile in shared memory in digit
// order and writes it out in coalesced runs.  Stable: ranks follow the
// original order within a warp, then warp order, then tile order.
#include <cuda_runtime.h>

#include <atomic>

#include "prt_internal.cuh"

namespace prt {
namespace {

constexpr int kRadix = 256;
constexpr int kSortBlock = 256;
constexpr int kSortWarps = kSortBlock / 32;
#ifndef PRT_SORT_ITEMS
#define PRT_SORT_ITEMS 16  // keys per thread of a tile
#endif
#ifndef PRT_SORT_MIN_BLOCKS
// resident blocks per SM the 32-bit-key pass is compiled for: 4 (64
// registers, a 56-byte spill) against 3 (80 registers): 0.0872 ->
// 0.0830-0.0840 ms per 10M-key pass, measured with the look-back batch below.
// The 64-bit-key pass stays at 3: its 58 KB tile fits no more per SM.
#define PRT_SORT_MIN_BLOCKS 4
#endif
constexpr int kItems = PRT_SORT_ITEMS;
constexpr int kTile = kSortBlock * kItems;
static_assert(kTile == kSortRunTile, "the run sort's tile");
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagPrefix = 2u << 30;
constexpr uint32_t kCountMask = (1u << 30) - 1;

struct PassPlan {
  int active, src, dst, pad;
};

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

template <typename KeyT>
__global__ void __launch_bounds__(256) hist_kernel(const KeyT *__restrict__ keys, int64_t n, int passes,
                                                   uint32_t *__restrict__ ghist) {
  extern __shared__ uint32_t sh[];  // passes * 256
  for (int i = threadIdx.x; i < passes * kRadix; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int64_t i0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (sizeof(KeyT) == 4 && (reinterpret_cast<uintptr_t>(keys) & 15) == 0) {
    // four keys per 16-byte load
    const uint4 *k4 = reinterpret_cast<const uint4 *>(keys);
    for (int64_t i = i0; i < n / 4; i += stride) {
      const uint4 q = k4[i];
      const KeyT kk[4] = {(KeyT)q.x, (KeyT)q.y, (KeyT)q.z, (KeyT)q.w};
#pragma unroll
      for (int j = 0; j < 4; j++)
        for (int p = 0; p < passes; p++) atomicAdd(&sh[p * kRadix + (int)((kk[j] >> (8 * p)) & 0xFF)], 1u);
    }
    i0 += (n / 4) * 4;
  }
  for (int64_t i = i0; i < n; i += stride) {
    KeyT k = keys[i];
    for (int p = 0; p < passes; p++) atomicAdd(&sh[p * kRadix + (int)((k >> (8 * p)) & 0xFF)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < passes * kRadix; i += blockDim.x)
    if (sh[i]) atomicAdd(&ghist[i], sh[i]);
}

__global__ void plan_kernel(const uint32_t *__restrict__ ghist, uint32_t *__restrict__ goff, int passes, int64_t n,
                            PassPlan *__restrict__ plan, int *__restrict__ d_sel) {
  __shared__ uint32_t scan[kRadix];
  __shared__ int trivial[PRT_MAX_LEVELS];
  for (int p = 0; p < passes; p++) {
    uint32_t c = ghist[p * kRadix + threadIdx.x];
    scan[threadIdx.x] = c;
    if (threadIdx.x == 0) trivial[p] = 0;
    __syncthreads();
    if ((int64_t)c == n) trivial[p] = 1;
    // inclusive Hillis-Steele scan over 256 bins
    for (int o = 1; o < kRadix; o <<= 1) {
      uint32_t v = threadIdx.x >= o ? scan[threadIdx.x - o] : 0u;
      __syncthreads();
      scan[threadIdx.x] += v;
      __syncthreads();
    }
    goff[p * kRadix + threadIdx.x] = scan[threadIdx.x] - c;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    int cur = 0;
    for (int p = 0; p < passes; p++) {
      PassPlan pp;
      pp.active = !trivial[p];
      pp.src = cur;
      pp.dst = 1 - cur;
      pp.pad = 0;
      if (pp.active) cur = 1 - cur;
      plan[p] = pp;
    }
    *d_sel = cur;
  }
}

template <typename KeyT>
struct PassSmem {
  KeyT keys[kTile];
  uint32_t vals[kTile];
  uint32_t warp_hist[kSortWarps][kRadix];
  uint32_t digit_start[kRadix];  // tile-local exclusive start of each digit
  uint32_t global_start[kRadix];
  uint32_t scan_tmp[kSortWarps];
  int tile;
};

#ifndef PRT_SORT_LOOKBATCH
#define PRT_SORT_LOOKBATCH 4  // 2, 4, 8, 16 measured: 4 best at 4 blocks per SM
#endif
#ifndef PRT_SORT_BACKOFF_NS
#define PRT_SORT_BACKOFF_NS 0  // pause between look-back polls that found nothing new
#endif
constexpr int kLookBatch = PRT_SORT_LOOKBATCH;  // predecessor statuses read per look-back step

template <typename KeyT>
__global__ void __launch_bounds__(kSortBlock, sizeof(KeyT) == 4 ? PRT_SORT_MIN_BLOCKS : 3) onesweep_pass(KeyT *keys0, uint32_t *vals0, KeyT *keys1,
                                                           uint32_t *vals1, int64_t n, int shift,
                                                           const PassPlan *__restrict__ plan,
                                                           const uint32_t *__restrict__ goff,
                                                           uint32_t *status, unsigned *tile_ticket,
                                                           unsigned *err, WaitLimit wl, int64_t tiles_per_run) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  PassSmem<KeyT> &S = *reinterpret_cast<PassSmem<KeyT> *>(smem_raw);
  const PassPlan pp = *plan;
  if (!pp.active) return;
  const KeyT *src_k = pp.src ? keys1 : keys0;
  const uint32_t *src_v = pp.src ? vals1 : vals0;
  KeyT *dst_k = pp.dst ? keys1 : keys0;
  uint32_t *dst_v = pp.dst ? vals1 : vals0;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int d = tid;  // kSortBlock == kRadix: thread d owns digit d
  if (tid == 0) S.tile = (int)atomicAdd(tile_ticket, 1u);
  for (int i = tid; i < kSortWarps * kRadix; i += kSortBlock) (&S.warp_hist[0][0])[i] = 0;
  __syncthreads();
  const int tile = S.tile;
  const int64_t base = (int64_t)tile * kTile;
  const int valid = (int)min((int64_t)kTile, n - base);
  // runs sorted independently (tiles_per_run > 0): the tile's run, its first
  // tile and its digit offsets; otherwise one run
  const int64_t run = tiles_per_run > 0 ? tile / tiles_per_run : 0;
  const int first = (int)(run * tiles_per_run);
  goff += run * kRadix;
  const int wb = warp * 32 * kItems;  // this warp's first item in the tile

  KeyT k[kItems];
  uint32_t v[kItems];
#pragma unroll
  for (int i = 0; i < kItems; i++) {
    const int li = wb + i * 32 + lane;
    k[i] = 0;
    v[i] = 0;
    if (li < valid) {
      k[i] = src_k[base + li];
      v[i] = src_v[base + li];
    }
  }
  // 1. stable ranks and the warps' digit histograms in one sweep: lanes with
  //    the same digit are found by one ballot per digit bit; the lowest of
  //    them reads and bumps the warp's counter, the others get the old count
  //    by shuffle.  Items are ranked in index order (item slot i of lane l is
  //    tile position wb + 32 i + l), which makes the pass stable.
  const uint32_t lt = lanemask_lt();
  uint32_t *wh = S.warp_hist[warp];
  uint32_t dr[kItems];  // rank << 9 | digit (256 + lane: no item)
#pragma unroll
  for (int i = 0; i < kItems; i++) {
    const int li = wb + i * 32 + lane;
    const bool ok = li < valid;
    const uint32_t dg = ok ? (uint32_t)((k[i] >> shift) & 0xFF) : 256u + lane;
    uint32_t peers = __ballot_sync(0xffffffffu, ok);
#pragma unroll
    for (int b = 0; b < 8; b++) {
      const uint32_t m = __ballot_sync(0xffffffffu, (dg >> b) & 1u);
      peers &= ((dg >> b) & 1u) ? m : ~m;
    }
    if (!ok) peers = 1u << lane;
    const int leader = __ffs(peers) - 1;
    uint32_t cnt = 0;
    if (lane == leader && ok) {
      cnt = wh[dg];
      wh[dg] = cnt + __popc(peers);
    }
    cnt = __shfl_sync(0xffffffffu, cnt, leader);
    dr[i] = ((cnt + __popc(peers & lt)) << 9) | dg;
    __syncwarp();  // this item's counter updates before the next item's reads
  }
  __syncthreads();
  // 2. digit d: exclusive prefix over the warps and the tile's count, which
  //    is published at once for the later tiles' look-back
  uint32_t total = 0;
#pragma unroll
  for (int w = 0; w < kSortWarps; w++) {
    const uint32_t c = S.warp_hist[w][d];
    S.warp_hist[w][d] = total;
    total += c;
  }
  uint32_t *st = status + (int64_t)tile * kRadix + d;
  if (tile == first) atomicExch(st, kFlagPrefix | ((goff[d] + total) & kCountMask));
  else atomicExch(st, kFlagAgg | (total & kCountMask));
  // tile-local exclusive scan over digits: shuffle scan per warp of 32
  // digits, then the 8 warp totals
  uint32_t incl = total;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) S.scan_tmp[warp] = incl;
  __syncthreads();
  uint32_t woff = 0;
#pragma unroll
  for (int w = 0; w < kSortWarps; w++) woff += w < warp ? S.scan_tmp[w] : 0u;
  S.digit_start[d] = woff + incl - total;
  __syncthreads();
  // 3. stage the tile in digit order before the look-back: the items leave
  //    the registers, which the look-back's batches then use
#pragma unroll
  for (int i = 0; i < kItems; i++) {
    const uint32_t dg = dr[i] & 511u;
    if (dg < 256u) {
      const uint32_t pos = S.digit_start[dg] + wh[dg] + (dr[i] >> 9);
      S.keys[pos] = k[i];
      S.vals[pos] = v[i];
    }
  }

  // 4. decoupled look-back for digit d, kLookBatch predecessor statuses per
  //    round trip; every wait is bounded
  uint32_t excl = goff[d];
  if (tile > first) {  // the run's first tile publishes a prefix: the look-back stops there
    uint32_t acc = 0;
    int t = tile - 1;
    int spins = 0;
    bool timed_out = false;
    for (;;) {
      uint32_t sv[kLookBatch];
#pragma unroll
      for (int j = 0; j < kLookBatch; j++) {
        uint32_t sj = 2u << 30;  // before tile 0: an empty prefix (never reached)
        if (t - j >= 0) sj = *reinterpret_cast<volatile uint32_t *>(status + (int64_t)(t - j) * kRadix + d);
        sv[j] = wl.blind ? 0u : sj;
      }
      int used = 0;
      bool done = false;
#pragma unroll
      for (int j = 0; j < kLookBatch; j++) {
        if (done || used < j) continue;  // stop at the first prefix or unpublished status
        const uint32_t f = sv[j] & ~kCountMask;
        if (f == 0u) continue;           // not yet published: retry from here
        acc += sv[j] & kCountMask;
        used = j + 1;
        if (f == kFlagPrefix) done = true;
      }
      if (done) break;
      t -= used;
      if (used == 0) {
        if (++spins > wl.polls) {
          timed_out = true;
          break;
        }
        if (PRT_SORT_BACKOFF_NS > 0) __nanosleep(PRT_SORT_BACKOFF_NS);
      }
    }
    if (timed_out) atomicOr(err, kErrTimeout);
    excl = acc;
    atomicExch(st, kFlagPrefix | ((excl + total) & kCountMask));
  }
  // staged position i of digit dd goes to global_start[dd] + i - digit_start[dd]
  S.global_start[d] = excl - S.digit_start[d];
  __syncthreads();

  // 5. write the staged tile out in coalesced runs per digit (a look-back
  //    that timed out leaves the offsets wrong: the bound keeps every write
  //    inside the buffers, and the caller reports the timeout)
  for (int i = tid; i < valid; i += kSortBlock) {
    const KeyT kk = S.keys[i];
    const int dd = (int)((kk >> shift) & 0xFF);
    const uint32_t dst = S.global_start[dd] + (uint32_t)i;
    if ((int64_t)dst < n) {
      dst_k[dst] = kk;
      dst_v[dst] = S.vals[i];
    }
  }
}

// Digit histograms of every pass per run (runs of tiles_per_run tiles): one
// block per tile, block histograms in shared memory, one global add per
// nonzero bin into hist[(run * passes + p) * 256 + digit].
template <typename KeyT>
__global__ void __launch_bounds__(256) run_hist_kernel(const KeyT *__restrict__ keys, int64_t n, int passes,
                                                       int64_t tiles_per_run, uint32_t *__restrict__ hist) {
  extern __shared__ uint32_t sh[];  // passes * 256
  for (int i = threadIdx.x; i < passes * kRadix; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kTile;
  const int64_t end = min(base + (int64_t)kTile, n);
  for (int64_t i = base + threadIdx.x; i < end; i += blockDim.x) {
    const KeyT k = keys[i];
    for (int p = 0; p < passes; p++) atomicAdd(&sh[p * kRadix + (int)((k >> (8 * p)) & 0xFF)], 1u);
  }
  __syncthreads();
  uint32_t *h = hist + (int64_t)(blockIdx.x / tiles_per_run) * passes * kRadix;
  for (int i = threadIdx.x; i < passes * kRadix; i += blockDim.x)
    if (sh[i]) atomicAdd(&h[i], sh[i]);
}

// Per run and pass: goff[(p * runs + run) * 256 + d] = the run's first
// position + the run's exclusive digit scan; trivial[p] is cleared when some
// run has more than one digit in pass p.  One block (256 threads) per run.
__global__ void run_plan_kernel(const uint32_t *__restrict__ hist, int64_t n, int64_t run_len, int64_t runs,
                                int passes, uint32_t *__restrict__ goff, int *__restrict__ trivial) {
  __shared__ uint32_t scan[kRadix];
  const int64_t run = blockIdx.x;
  const int64_t start = run * run_len;
  const int64_t len = min(run_len, n - start);
  const int d = threadIdx.x;
  for (int p = 0; p < passes; p++) {
    const uint32_t c = hist[(run * passes + p) * kRadix + d];
    scan[d] = c;
    __syncthreads();
    if ((int64_t)c != len && c != 0) trivial[p] = 0;
    for (int o = 1; o < kRadix; o <<= 1) {
      const uint32_t v = d >= o ? scan[d - o] : 0u;
      __syncthreads();
      scan[d] += v;
      __syncthreads();
    }
    goff[((int64_t)p * runs + run) * kRadix + d] = (uint32_t)start + scan[d] - c;
    __syncthreads();
  }
}

// Pass plans from the trivial flags (a pass whose digit is constant within
// every run moves nothing and is skipped).
__global__ void run_plan_final_kernel(const int *__restrict__ trivial, int passes, PassPlan *__restrict__ plan,
                                      int *__restrict__ d_sel) {
  int cur = 0;
  for (int p = 0; p < passes; p++) {
    PassPlan pp;
    pp.active = !trivial[p];
    pp.src = cur;
    pp.dst = 1 - cur;
    pp.pad = 0;
    if (pp.active) cur = 1 - cur;
    plan[p] = pp;
  }
  *d_sel = cur;
}

}  // namespace

template <typename KeyT>
int radix_sort_runs(KeyT *keys0, uint32_t *vals0, KeyT *keys1, uint32_t *vals1, int64_t n, int64_t run_len,
                    int *d_sel, unsigned *d_err, cudaStream_t s, const uint32_t *d_hist) {
  PRT_CHECK(n >= 0 && n < (int64_t)kCountMask, PRT_ERR_INVALID, "radix sort: n=%lld out of range",
            (long long)n);
  PRT_CHECK(run_len >= kTile && run_len % kTile == 0, PRT_ERR_INVALID,
            "run sort: run length %lld is not a multiple of the %d-key tile", (long long)run_len, kTile);
  if (n == 0) {
    PRT_CUDA(cudaMemsetAsync(d_sel, 0, sizeof(int), s));
    return PRT_OK;
  }
  const int passes = (int)sizeof(KeyT);
  const int64_t tiles = (n + kTile - 1) / kTile;
  const int64_t tpr = run_len / kTile;
  const int64_t runs = (n + run_len - 1) / run_len;
  // scratch: trivial flags, plan, tickets, per-run histograms, per-run offsets, status
  const size_t triv_b = 64, plan_b = sizeof(PassPlan) * passes, tick_b = 64;
  const size_t hist_b = sizeof(uint32_t) * (size_t)runs * passes * kRadix;
  const size_t stat_b = sizeof(uint32_t) * (size_t)tiles * kRadix * passes;
  unsigned char *scratch = nullptr;
  const size_t head = 256;  // trivial (64) + plan (<= 128) + tickets (64)
  size_t total = head + 2 * hist_b + stat_b;
  int rc = dmalloc(reinterpret_cast<void **>(&scratch), total, s);
  if (rc) return rc;
  int *trivial = reinterpret_cast<int *>(scratch);
  PassPlan *plan = reinterpret_cast<PassPlan *>(scratch + triv_b);
  unsigned *tick = reinterpret_cast<unsigned *>(scratch + triv_b + 128);
  uint32_t *hist = reinterpret_cast<uint32_t *>(scratch + head);
  uint32_t *goff = hist + (size_t)runs * passes * kRadix;
  uint32_t *status = goff + (size_t)runs * passes * kRadix;
  (void)plan_b;
  (void)tick_b;
  cudaError_t e = cudaMemsetAsync(scratch, 0, total, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(trivial, 0xFF, sizeof(int) * passes, s);  // nonzero = trivial
  if (e == cudaSuccess) {
    if (!d_hist) {
      PRT_PROF("run_hist", s);
      run_hist_kernel<KeyT><<<(unsigned)tiles, 256, sizeof(uint32_t) * passes * kRadix, s>>>(keys0, n, passes, tpr,
                                                                                            hist);
    }
    {
      PRT_PROF("plan", s);
      run_plan_kernel<<<(unsigned)runs, kRadix, 0, s>>>(d_hist ? d_hist : hist, n, run_len, runs, passes, goff,
                                                        trivial);
      run_plan_final_kernel<<<1, 1, 0, s>>>(trivial, passes, plan, d_sel);
    }
    size_t smem = sizeof(PassSmem<KeyT>);
    static bool attr_done[256] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 256 || !attr_done[dev]) {
      e = cudaFuncSetAttribute(onesweep_pass<KeyT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e == cudaSuccess && dev >= 0 && dev < 256) attr_done[dev] = true;
    }
    const WaitLimit wl = wait_limit();
    for (int p = 0; p < passes && e == cudaSuccess; p++) {
      PRT_PROF("onesweep_pass", s);
      onesweep_pass<KeyT><<<(unsigned)tiles, kSortBlock, smem, s>>>(
        keys0, vals0, keys1, vals1, n, 8 * p, plan + p, goff + (size_t)p * runs * kRadix,
        status + (size_t)p * tiles * kRadix, tick + p, d_err, wl, tpr);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
  }
  dfree(scratch, s);
  if (e != cudaSuccess) return cuda_status(e, "radix_sort_runs");
  return PRT_OK;
}

template <typename KeyT>
int radix_sort_pairs(KeyT *keys0, uint32_t *vals0, KeyT *keys1, uint32_t *vals1, int64_t n, int key_bits,
                     int *d_sel, unsigned *d_err, cudaStream_t s, const uint32_t *d_hist) {
  PRT_CHECK(n >= 0 && n < (int64_t)kCountMask, PRT_ERR_INVALID, "radix sort: n=%lld out of range",
            (long long)n);
  int passes = (key_bits + 7) / 8;
  if (passes < 1) passes = 1;
  PRT_CHECK(passes <= (int)sizeof(KeyT), PRT_ERR_INVALID, "radix sort: %d key bits", key_bits);
  if (n == 0) {
    PRT_CUDA(cudaMemsetAsync(d_sel, 0, sizeof(int), s));
    return PRT_OK;
  }
  const int64_t tiles = (n + kTile - 1) / kTile;
  // scratch: hist, offsets, plan, tickets, status
  size_t hist_b = sizeof(uint32_t) * passes * kRadix;
  size_t plan_b = sizeof(PassPlan) * passes;
  size_t tick_b = sizeof(unsigned) * passes;
  size_t stat_b = sizeof(uint32_t) * (size_t)tiles * kRadix * passes;
  unsigned char *scratch = nullptr;
  size_t total = 2 * hist_b + plan_b + tick_b + stat_b + 256;
  int rc = dmalloc(reinterpret_cast<void **>(&scratch), total, s);
  if (rc) return rc;
  uint32_t *ghist = reinterpret_cast<uint32_t *>(scratch);
  uint32_t *goff = ghist + passes * kRadix;
  PassPlan *plan = reinterpret_cast<PassPlan *>(goff + passes * kRadix);
  unsigned *tick = reinterpret_cast<unsigned *>(plan + passes);
  uint32_t *status = reinterpret_cast<uint32_t *>(tick + passes);
  cudaError_t e = cudaMemsetAsync(scratch, 0, total, s);
  if (e == cudaSuccess) {
    int g = grid_for(n, 256, 4);
    if (!d_hist) {
      PRT_PROF("hist", s);
      hist_kernel<KeyT><<<g, 256, sizeof(uint32_t) * passes * kRadix, s>>>(keys0, n, passes, ghist);
    }
    {
      PRT_PROF("plan", s);
      plan_kernel<<<1, kRadix, 0, s>>>(d_hist ? d_hist : ghist, goff, passes, n, plan, d_sel);
    }
    size_t smem = sizeof(PassSmem<KeyT>);
    // the shared-memory opt-in is set once per device (not a stream
    // operation, but kept out of graph captures after the first call)
    static bool attr_done[256] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 256 || !attr_done[dev]) {
      e = cudaFuncSetAttribute(onesweep_pass<KeyT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e == cudaSuccess && dev >= 0 && dev < 256) attr_done[dev] = true;
    }
    const WaitLimit wl = wait_limit();
    for (int p = 0; p < passes && e == cudaSuccess; p++) {
      {
        PRT_PROF("onesweep_pass", s);
        onesweep_pass<KeyT><<<(unsigned)tiles, kSortBlock, smem, s>>>(
          keys0, vals0, keys1, vals1, n, 8 * p, plan + p, goff + p * kRadix,
          status + (size_t)p * tiles * kRadix, tick + p, d_err, wl, 0);
      }
    }
    if (e == cudaSuccess) e = cudaGetLastError();
  }
  dfree(scratch, s);
  if (e != cudaSuccess) return cuda_status(e, "radix_sort_pairs");
  return PRT_OK;
}

namespace {
std::atomic<int> g_wait_polls{kSpinLimit};
std::atomic<int> g_wait_blind{0};
}  // namespace

WaitLimit wait_limit() { return WaitLimit{g_wait_polls.load(), g_wait_blind.load()}; }

template int radix_sort_runs<uint32_t>(uint32_t *, uint32_t *, uint32_t *, uint32_t *, int64_t, int64_t, int *,
                                       unsigned *, cudaStream_t, const uint32_t *);
template int radix_sort_runs<uint64_t>(uint64_t *, uint32_t *, uint64_t *, uint32_t *, int64_t, int64_t, int *,
                                       unsigned *, cudaStream_t, const uint32_t *);
template int radix_sort_pairs<uint32_t>(uint32_t *, uint32_t *, uint32_t *, uint32_t *, int64_t, int, int *,
                                        unsigned *, cudaStream_t, const uint32_t *);
template int radix_sort_pairs<uint64_t>(uint64_t *, uint32_t *, uint64_t *, uint32_t *, int64_t, int, int *,
                                        unsigned *, cudaStream_t, const uint32_t *);

}  // namespace prt

extern "C" int prt_debug_wait_limit(int polls, int never_published) {
  using namespace prt;
  g_wait_polls.store(polls > 0 ? polls : kSpinLimit);
  g_wait_blind.store(never_published ? 1 : 0);
  return PRT_OK;
}
