// R-tree bulk loading: key generation, leaf order (bottom-up: one radix sort
// of the keys; top-down: one segmented radix sort per level) and packing of
// the levels.  Device layout of a tree (shared by both builds):
//   level l holds n_l entries, padded to a multiple of the fanout F with boxes
//   that intersect nothing; level 0 = the records in leaf order; entry j of
//   level l+1 = union of entries [jF, jF+F) of level l, so the child of entry
//   j is node j of the level below and no child pointers are stored.
#include <cuda_runtime.h>

#include <limits>
#include <type_traits>

#include <algorithm>
#include <vector>
#include <cstdarg>
#include <cstring>
#include <mutex>

#include "prt_internal.cuh"

namespace prt {

// ------------------------------------------------------------------ errors
static thread_local std::string g_err;

void set_error(const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
}

int cuda_status(cudaError_t e, const char *what) {
  set_error("%s: %s", what, cudaGetErrorString(e));
  cudaGetLastError();
  return e == cudaErrorMemoryAllocation ? PRT_ERR_NOMEM : PRT_ERR_CUDA;
}

// The scratch comes from the device's default stream-ordered pool.  Its release
// threshold is raised once per device so that memory freed by one call stays
// in the pool for the next instead of going back to the driver at every
// synchronisation (a fresh mapping of hundreds of MB per call costs more than
// the kernels that use it).
static void keep_pool_memory() {
  static std::mutex mu;
  static bool done[256] = {false};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) {
    cudaGetLastError();
    return;
  }
  std::lock_guard<std::mutex> lk(mu);
  if (done[dev]) return;
  done[dev] = true;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  cudaGetLastError();
}

int dmalloc(void **p, size_t bytes, cudaStream_t s) {
  if (bytes == 0) bytes = 16;
  keep_pool_memory();
  cudaError_t e = cudaMallocAsync(p, bytes, s);
  if (e != cudaSuccess) {
    *p = nullptr;
    return cuda_status(e, "cudaMallocAsync");
  }
  return PRT_OK;
}

void dfree(void *p, cudaStream_t s) {
  if (p) cudaFreeAsync(p, s);
}

TreeLevels level_layout(int64_t n, int fanout) {
  TreeLevels L;
  memset(&L, 0, sizeof L);
  int64_t c = n;
  int l = 0;
  for (;;) {
    L.count[l] = c;
    L.padded[l] = ((c + fanout - 1) / fanout) * fanout;
    if (L.padded[l] == 0) L.padded[l] = fanout;
    l++;
    if (c <= fanout || l == PRT_MAX_LEVELS) break;
    c = (c + fanout - 1) / fanout;
  }
  L.levels = l;
  int64_t o = 0;
  for (int i = 0; i < l; i++) {
    L.offset[i] = o;
    o += L.padded[i];
  }
  L.total = o;
  return L;
}

namespace {

// ------------------------------------------------------------------ extent

__device__ __forceinline__ unsigned long long ord_f64(double v) {
  unsigned long long u = (unsigned long long)__double_as_longlong(v);
  return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ double unord_f64(unsigned long long u) {
  u = (u & 0x8000000000000000ull) ? (u & 0x7FFFFFFFFFFFFFFFull) : ~u;
  return __longlong_as_double((long long)u);
}

template <typename T>
__device__ __forceinline__ T vmin(T a, T b) {
  if constexpr (std::is_same<T, float>::value) return fminf(a, b);
  else if constexpr (std::is_same<T, double>::value) return fmin(a, b);
  else return b < a ? b : a;
}
template <typename T>
__device__ __forceinline__ T vmax(T a, T b) {
  if constexpr (std::is_same<T, float>::value) return fmaxf(a, b);
  else if constexpr (std::is_same<T, double>::value) return fmax(a, b);
  else return b > a ? b : a;
}

// ext[0..3] = ordered encodings of min x1, min y1, max x2, max y2 (as double).
// The per-thread min / max run in the coordinate type (the conversion to
// double is monotone, so the result is the same as in double).
template <typename T>
__global__ void extent_f64_kernel(const Box<T> *__restrict__ b, int64_t n, unsigned long long *ext) {
  T hi, lo;
  if constexpr (std::is_floating_point<T>::value) {
    hi = (T)__longlong_as_double(0x7FF0000000000000ll);
    lo = -hi;
  } else {
    hi = std::numeric_limits<T>::max();
    lo = std::numeric_limits<T>::lowest();
  }
  T tnx = hi, tny = hi, txx = lo, txy = lo;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    Box<T> x = load_box(b, i);
    tnx = vmin(tnx, x.x1);
    tny = vmin(tny, x.y1);
    txx = vmax(txx, x.x2);
    txy = vmax(txy, x.y2);
  }
  double mnx = (double)tnx, mny = (double)tny, mxx = (double)txx, mxy = (double)txy;
  for (int o = 16; o; o >>= 1) {
    mnx = fmin(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
    mny = fmin(mny, __shfl_xor_sync(0xffffffffu, mny, o));
    mxx = fmax(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
    mxy = fmax(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
  }
  // the block's warps, then one set of atomics per block (the four words
  // are the same for every block, so fewer atomics means less contention)
  __shared__ double red[4][32];
  const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  if ((threadIdx.x & 31) == 0) {
    red[0][w] = mnx;
    red[1][w] = mny;
    red[2][w] = mxx;
    red[3][w] = mxy;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < nw; k++) {
      mnx = fmin(mnx, red[0][k]);
      mny = fmin(mny, red[1][k]);
      mxx = fmax(mxx, red[2][k]);
      mxy = fmax(mxy, red[3][k]);
    }
    atomicMin(&ext[0], ord_f64(mnx));
    atomicMin(&ext[1], ord_f64(mny));
    atomicMax(&ext[2], ord_f64(mxx));
    atomicMax(&ext[3], ord_f64(mxy));
  }
}

__global__ void extent_init_kernel(unsigned long long *ext) {
  ext[0] = ord_f64(__longlong_as_double(0x7FF0000000000000ll));
  ext[1] = ext[0];
  ext[2] = ord_f64(-__longlong_as_double(0x7FF0000000000000ll));
  ext[3] = ext[2];
}

// int64 extent with the reference's start values (BotomUp-rtree.cu:663-666)
__global__ void extent_i64_kernel(const Box<int64_t> *__restrict__ b, int64_t n, long long *ext) {
  long long mnx = 100000000000000000ll, mny = mnx, mxx = 0, mxy = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    Box<int64_t> x = load_box(b, i);
    mnx = min(mnx, (long long)x.x1);
    mny = min(mny, (long long)x.y1);
    mxx = max(mxx, (long long)x.x2);
    mxy = max(mxy, (long long)x.y2);
  }
  for (int o = 16; o; o >>= 1) {
    mnx = min(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
    mny = min(mny, __shfl_xor_sync(0xffffffffu, mny, o));
    mxx = max(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
    mxy = max(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&ext[0], mnx);
    atomicMin(&ext[1], mny);
    atomicMax(&ext[2], mxx);
    atomicMax(&ext[3], mxy);
  }
}

__global__ void extent_i64_init_kernel(long long *ext) {
  ext[0] = 100000000000000000ll;
  ext[1] = 100000000000000000ll;
  ext[2] = 0;
  ext[3] = 0;
}

// ------------------------------------------------------------------ keys

__device__ __forceinline__ uint32_t part1by1_16(uint32_t v) {
  v &= 0xFFFFu;
  v = (v | (v << 8)) & 0x00FF00FFu;
  v = (v | (v << 4)) & 0x0F0F0F0Fu;
  v = (v | (v << 2)) & 0x33333333u;
  v = (v | (v << 1)) & 0x55555555u;
  return v;
}

// MORTON32: centre of each box on a 65536^2 grid over the data extent; the
// expression order matches the oracle exactly (no FMA: built with -fmad=false).
// The four 8-bit digit histograms of the keys are counted on the way (block
// histograms in shared memory, one global add per nonzero bin), so the sort
// need not read the keys again to plan its passes.
template <typename T>
__global__ void __launch_bounds__(256) morton32_kernel(const Box<T> *__restrict__ b, int64_t n,
                                                       const unsigned long long *__restrict__ ext,
                                                       uint32_t *__restrict__ keys, uint32_t *__restrict__ vals,
                                                       uint32_t *__restrict__ ghist) {
  __shared__ uint32_t h[4 * 256];
  for (int i = threadIdx.x; i < 4 * 256; i += blockDim.x) h[i] = 0;
  __syncthreads();
  const double minX = unord_f64(ext[0]), minY = unord_f64(ext[1]);
  const double maxX = unord_f64(ext[2]), maxY = unord_f64(ext[3]);
  const double ex = (maxX - minX) > (maxY - minY) ? (maxX - minX) : (maxY - minY);
  const double inv = ex > 0.0 ? 65535.0 / ex : 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    Box<T> x = load_box(b, i);
    double cx = 0.5 * ((double)x.x1 + (double)x.x2);
    double cy = 0.5 * ((double)x.y1 + (double)x.y2);
    double tx = (cx - minX) * inv;
    double ty = (cy - minY) * inv;
    uint32_t gx = tx >= 65535.0 ? 65535u : (tx > 0.0 ? (uint32_t)tx : 0u);
    uint32_t gy = ty >= 65535.0 ? 65535u : (ty > 0.0 ? (uint32_t)ty : 0u);
    const uint32_t k = part1by1_16(gx) | (part1by1_16(gy) << 1);
    keys[i] = k;
    vals[i] = (uint32_t)i;
#pragma unroll
    for (int p = 0; p < 4; p++) atomicAdd(&h[p * 256 + ((k >> (8 * p)) & 0xFF)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 4 * 256; i += blockDim.x)
    if (h[i]) atomicAdd(&ghist[i], h[i]);
}

// Spreads the low 16 bits of v into 2-bit chunks, one per byte (chunk k ->
// bits 8k..8k+1), by three mask-and-shift rounds; BotomUp-rtree.cu:98-123.
__device__ __forceinline__ uint64_t spread_2bit_chunks(uint64_t v) {
  v = (v | (v << 24)) & 0x000000FF000000FFull;
  v = (v | (v << 12)) & 0x000F000F000F000Full;
  v = (v | (v << 6)) & 0x0303030303030303ull;
  return v;
}

// REF64: shift by (min x1, min y1), power-of-ten scale with extent/scale <=
// 1e4, integer division, 4-D interleave of (x1, y1, x2, y2)
// (BotomUp-rtree.cu:704-716, 81-92).
__global__ void ref64_kernel(const Box<int64_t> *__restrict__ b, int64_t n, const long long *__restrict__ ext,
                             uint64_t *__restrict__ keys, uint32_t *__restrict__ vals) {
  const long long minX = ext[0], minY = ext[1];
  long long e = (ext[2] - minX) > (ext[3] - minY) ? (ext[2] - minX) : (ext[3] - minY);
  long long scale = 1;
  while (e > 10000) {
    scale *= 10;
    e /= 10;
  }
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    Box<int64_t> x = load_box(b, i);
    uint64_t a1 = (uint64_t)((x.x1 - minX) / scale);
    uint64_t a2 = (uint64_t)((x.y1 - minY) / scale);
    uint64_t a3 = (uint64_t)((x.x2 - minX) / scale);
    uint64_t a4 = (uint64_t)((x.y2 - minY) / scale);
    keys[i] = (spread_2bit_chunks(a1) << 6) | (spread_2bit_chunks(a2) << 4) | (spread_2bit_chunks(a3) << 2) |
              spread_2bit_chunks(a4);
    vals[i] = (uint32_t)i;
  }
}

// Order-preserving unsigned image of a coordinate (-0.0 folded onto +0.0).
__device__ __forceinline__ uint32_t ukey(float v) {
  uint32_t u = __float_as_uint(v + 0.0f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ uint32_t ukey(int32_t v) { return (uint32_t)v ^ 0x80000000u; }
__device__ __forceinline__ uint64_t ukey(double v) {
  uint64_t u = (uint64_t)__double_as_longlong(v + 0.0);
  return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ uint64_t ukey(int64_t v) { return (uint64_t)v ^ 0x8000000000000000ull; }

// Top-down level key for 32-bit coordinates: (pos / seg) << 32 | coordinate.
template <typename T>
__global__ void td_key32_kernel(const Box<T> *__restrict__ b, const uint32_t *__restrict__ perm, int64_t n,
                                int64_t seg, int use_y, uint64_t *__restrict__ keys, uint32_t *__restrict__ vals) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t r = perm ? perm[i] : (uint32_t)i;
    if ((int64_t)r >= n) r = 0;  // only after a timed-out sort (reported by the caller)
    Box<T> x = load_box(b, r);
    uint32_t c = ukey(use_y ? x.y1 : x.x1);
    keys[i] = ((uint64_t)(i / seg) << 32) | c;
    vals[i] = r;
  }
}

// The current top-down order: perm_a or perm_b as *sel says (sel nullptr:
// perm_a; perm_a nullptr: the identity).
__device__ __forceinline__ const uint32_t *cur_perm(const uint32_t *perm_a, const uint32_t *perm_b, const int *sel) {
  return perm_a ? ((sel && *sel) ? perm_b : perm_a) : nullptr;
}

// Top-down level whose runs are sorted one by one (radix_sort_runs) or that
// is one run: the key is the coordinate's order-preserving image alone.  One
// block per 4096 positions (inside one run, since runs are whole tiles)
// counts the digit histograms of every pass on the way, into its run's
// histograms hist[(run * passes + p) * 256 + digit], so the sort does not
// read the keys again to count them.  The order is read and the values
// written at the same positions by the same thread: vals may be the buffer
// the order is read from.  Record r's (x1, y1) is at c[stride * r] (the boxes,
// stride 4, or the compact copy, stride 2); with the identity order the
// kernel can write that compact copy (xy_out), so later levels gather from
// an array a quarter (float) of the boxes' size, which stays in L2.
template <typename T, typename K>
__global__ void __launch_bounds__(256) td_keyrun_kernel(const T *__restrict__ cxy, int stride, const uint32_t *perm_a,
                                                        const uint32_t *perm_b, const int *sel, int64_t n, int use_y,
                                                        int64_t tiles_per_run, K *__restrict__ keys, uint32_t *vals,
                                                        uint32_t *__restrict__ hist, T *__restrict__ xy_out) {
  constexpr int kPasses = (int)sizeof(K);
  constexpr int kPer = (int)(kSortRunTile / 256);
  __shared__ uint32_t sh[kPasses * 256];
  for (int i = threadIdx.x; i < kPasses * 256; i += 256) sh[i] = 0;
  __syncthreads();
  const uint32_t *perm = cur_perm(perm_a, perm_b, sel);
  const T *c = cxy + (use_y ? 1 : 0);
  const int64_t base = (int64_t)blockIdx.x * kSortRunTile + threadIdx.x;
  // all loads of the order first, then all coordinate loads, then the stores
  uint32_t r[kPer];
#pragma unroll
  for (int j = 0; j < kPer; j++) {
    const int64_t i = base + 256 * j;
    r[j] = i < n ? (perm ? perm[i] : (uint32_t)i) : 0u;
    if ((int64_t)r[j] >= n) r[j] = 0;  // only after a timed-out sort (reported by the caller)
  }
  K k[kPer];
#pragma unroll
  for (int j = 0; j < kPer; j++) k[j] = base + 256 * j < n ? (K)ukey(__ldg(&c[stride * (int64_t)r[j]])) : K(0);
  if (xy_out) {  // identity order: record i's (x1, y1), read in order
#pragma unroll
    for (int j = 0; j < kPer; j++) {
      const int64_t i = base + 256 * j;
      if (i < n) {
        xy_out[2 * i] = cxy[stride * i];
        xy_out[2 * i + 1] = cxy[stride * i + 1];
      }
    }
  }
#pragma unroll
  for (int j = 0; j < kPer; j++) {
    const int64_t i = base + 256 * j;
    if (i < n) {
      keys[i] = k[j];
      vals[i] = r[j];
#pragma unroll
      for (int p = 0; p < kPasses; p++) atomicAdd(&sh[p * 256 + (int)((k[j] >> (8 * p)) & 0xFF)], 1u);
    }
  }
  __syncthreads();
  uint32_t *h = hist + (int64_t)(blockIdx.x / tiles_per_run) * kPasses * 256;
  for (int i = threadIdx.x; i < kPasses * 256; i += 256)
    if (sh[i]) atomicAdd(&h[i], sh[i]);
}

// Top-down level, 64-bit coordinates, first stage: key = coordinate, value = position.
template <typename T>
__global__ void td_key64_kernel(const Box<T> *__restrict__ b, const uint32_t *__restrict__ perm, int64_t n,
                                int use_y, uint64_t *__restrict__ keys, uint32_t *__restrict__ vals) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t r = perm ? perm[i] : (uint32_t)i;
    if ((int64_t)r >= n) r = 0;  // only after a timed-out sort (reported by the caller)
    Box<T> x = load_box(b, r);
    keys[i] = ukey(use_y ? x.y1 : x.x1);
    vals[i] = (uint32_t)i;
  }
}

// second stage: key = segment of the original position
__global__ void td_segkey_kernel(const uint32_t *__restrict__ pos, int64_t n, int64_t seg,
                                 uint32_t *__restrict__ keys) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    keys[i] = (uint32_t)(pos[i] / seg);
}

__global__ void gather_u32_kernel(const uint32_t *__restrict__ src, const uint32_t *__restrict__ idx, int64_t n,
                                  uint32_t *__restrict__ dst) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t k = idx[i];
    if ((int64_t)k >= n) k = 0;  // only after a timed-out sort (reported by the caller)
    dst[i] = src ? src[k] : k;
  }
}

__global__ void select_copy_u32_kernel(const uint32_t *a, const uint32_t *b, const int *sel, int64_t n,
                                       uint32_t *dst) {
  const uint32_t *src = *sel ? b : a;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

// ------------------------------------------------------------------ top-down, short runs

// The top-down levels whose runs hold at most kTdLocal records (the last
// levels of the build: run lengths F^k <= 4096, each dividing the one before)
// are sorted together, tile by tile, in shared memory: one CTA takes as many
// whole runs of the first such level as fit in a tile of kTdLocal records (in
// the current order), gathers each record's (x1, y1) once, and sorts the tile
// level by level.  A level with runs longer than F sorts stably by (run
// within the tile, key - the tile's smallest key) with an LSD radix sort in
// shared memory over only the bits that needs, 8 bits per pass, each pass
// ranked by the warp multisplit (lanes with the same digit from one ballot
// per digit bit); the last level (runs of F <= 32) places each record by
// counting the run's smaller keys.  The tile's index order is the current
// order, so equal keys keep it, as each level's stable sort requires; each
// item's run travels with it.  One read and one write of the order replace
// 4-7 global passes per level.
constexpr int kTdLocal = 4096;
#ifndef PRT_TD_THREADS
// 512 threads of 8 records (64 registers, 2 CTAs of 16 warps per SM) against
// 256 of 16 (80 registers with a spill, 3 CTAs of 8 warps): the top-down
// build of 10M boxes (F = 16) 2.18 -> 2.07 ms
#define PRT_TD_THREADS 512
#endif
constexpr int kTdThreads = PRT_TD_THREADS;     // per CTA
constexpr int kTdWarps = kTdThreads / 32;
constexpr int kTdItems = kTdLocal / kTdThreads;  // per thread
constexpr int kTdMaxLocal = 12;           // local levels one launch sorts (4096 = 2^12)

__device__ __forceinline__ uint32_t lane_lt() {
  uint32_t m;
  asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Shared memory of one tile: the items in the current order (run << 16 |
// slot, double-buffered; slot = the item's position in the tile's input
// order), the (x1, y1) of every slot, gathered once for all levels, and the
// ranking scratch.
template <typename T>
struct TdLocalSmem {
  uint32_t item[2][kTdLocal];
  T xy[kTdLocal][2];
  uint32_t wh[kTdWarps][256];
  uint32_t dstart[256];
  uint32_t wsum[8];
  unsigned long long red[2][kTdWarps];
};

// The local levels, in order: run length and axis (0: x1, 1: y1) of each.
struct TdLocalLevels {
  int64_t seg[kTdMaxLocal];
  int use_y[kTdMaxLocal];
  int count;
};

// The last level's runs (F records) are short: each record's new position in
// its run is the number of the run's records with a smaller key, or an equal
// key at an earlier position (a stable sort by counting), seg comparisons
// per record instead of the radix passes.
constexpr int kTdRankMax = 32;

__device__ __forceinline__ int bit_length(uint32_t x) { return 32 - __clz(x); }
__device__ __forceinline__ int bit_length(uint64_t x) { return 64 - __clzll((long long)x); }

// Each level sorts the tile stably by (run, key - the tile's smallest key):
// only the bits that difference needs, with the run index directly above
// them, in 8-bit digits (the last one narrower).  Subtracting one constant
// from every key keeps their order, so this is the order of a stable sort by
// key within each run.
template <typename T, int kStride>
__global__ void __launch_bounds__(kTdThreads, kTdThreads == 256 ? (sizeof(T) == 4 ? 3 : 2) : (sizeof(T) == 4 ? 2 : 1))
    td_local_sort_kernel(
    const T *__restrict__ c, const uint32_t *__restrict__ perm_a, const uint32_t *__restrict__ perm_b,
    const int *__restrict__ sel, int64_t n, TdLocalLevels lv, uint32_t *__restrict__ perm_out) {
  using K = typename std::conditional<sizeof(T) == 8, uint64_t, uint32_t>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TdLocalSmem<T> &S = *reinterpret_cast<TdLocalSmem<T> *>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t chunk = (kTdLocal / lv.seg[0]) * lv.seg[0];  // whole runs of the first local level
  const int64_t base = blockIdx.x * chunk;
  const int m = (int)min(chunk, n - base);
  const uint32_t *perm_in = cur_perm(perm_a, perm_b, sel);
  for (int i = tid; i < m; i += kTdThreads) {
    uint32_t r = perm_in ? perm_in[base + i] : (uint32_t)(base + i);
    if ((int64_t)r >= n) r = 0;  // only after a timed-out sort (reported by the caller)
    S.xy[i][0] = __ldg(&c[kStride * (int64_t)r]);
    S.xy[i][1] = __ldg(&c[kStride * (int64_t)r + 1]);
    S.item[0][i] = (uint32_t)i;
  }
  const uint32_t lt = lane_lt();
  int cur = 0;
  for (int level = 0; level < lv.count; level++) {
    const int seg = (int)min(lv.seg[level], (int64_t)kTdLocal);
    const int axis = lv.use_y[level];
    __syncthreads();
    if (level == lv.count - 1 && seg <= kTdRankMax) {
      // keys into the (x1, y1) array's space (no later level reads it)
      K kq[kTdItems];
#pragma unroll
      for (int q = 0; q < kTdItems; q++) {
        const int i = tid + kTdThreads * q;
        kq[q] = i < m ? (K)ukey(S.xy[S.item[cur][i] & 0xFFFFu][axis]) : K(0);
      }
      __syncthreads();
      K *key = reinterpret_cast<K *>(&S.xy[0][0]);
#pragma unroll
      for (int q = 0; q < kTdItems; q++) {
        const int i = tid + kTdThreads * q;
        if (i < m) key[i] = kq[q];
      }
      __syncthreads();
#pragma unroll
      for (int q = 0; q < kTdItems; q++) {
        const int i = tid + kTdThreads * q;
        if (i < m) {
          const int r0 = (i / seg) * seg, r1 = min(r0 + seg, m);
          int rank = 0;
          for (int j = r0; j < r1; j++) {
            const K kj = key[j];
            rank += (kj < kq[q] || (kj == kq[q] && j < i)) ? 1 : 0;
          }
          S.item[1 - cur][r0 + rank] = S.item[cur][i];
        }
      }
      cur = 1 - cur;
      continue;
    }
    // the run of each item from its position in the order the previous level
    // left, and the tile's key range
    K lo = ~K(0), hi = 0;
    for (int i = tid; i < m; i += kTdThreads) {
      const uint32_t slot = S.item[cur][i] & 0xFFFFu;
      S.item[cur][i] = (uint32_t)(i / seg) << 16 | slot;
      const K k = (K)ukey(S.xy[slot][axis]);
      lo = k < lo ? k : lo;
      hi = k > hi ? k : hi;
    }
    for (int o = 16; o; o >>= 1) {
      const K a = __shfl_xor_sync(0xffffffffu, lo, o), z = __shfl_xor_sync(0xffffffffu, hi, o);
      lo = a < lo ? a : lo;
      hi = z > hi ? z : hi;
    }
    if (lane == 0) {
      S.red[0][warp] = lo;
      S.red[1][warp] = hi;
    }
    __syncthreads();
#pragma unroll
    for (int w = 0; w < kTdWarps; w++) {
      const K a = (K)S.red[0][w], z = (K)S.red[1][w];
      lo = a < lo ? a : lo;
      hi = z > hi ? z : hi;
    }
    const int key_bits = hi > lo ? bit_length(hi - lo) : 0;
    int run_bits = 0;
    while ((1 << run_bits) < (m + seg - 1) / seg) run_bits++;
    const int total_bits = key_bits + run_bits;
    for (int shift = 0; shift < total_bits; shift += 8) {
      const int width = min(8, total_bits - shift);
      __syncthreads();
      for (int i = tid; i < kTdWarps * 256; i += kTdThreads) (&S.wh[0][0])[i] = 0;
      __syncthreads();
      uint32_t it[kTdItems];
      int dg[kTdItems];
      uint32_t rk[kTdItems];
      uint32_t *wh = S.wh[warp];
#pragma unroll
      for (int j = 0; j < kTdItems; j++) {
        const int i = warp * (32 * kTdItems) + j * 32 + lane;
        const bool ok = i < m;
        int d = 256 + lane;
        it[j] = 0;
        if (ok) {
          // digit: bits [shift, shift + width) of (run << key_bits | key - lo)
          const uint32_t x = S.item[cur][i];
          const uint32_t run = x >> 16;
          const K rel = (K)ukey(S.xy[x & 0xFFFFu][axis]) - lo;
          uint32_t v;
          if (shift < key_bits) {
            v = (uint32_t)(rel >> shift);
            if (shift + 8 > key_bits) v |= run << (key_bits - shift);
          } else {
            v = run >> (shift - key_bits);
          }
          d = (int)(v & ((1u << width) - 1u));
          it[j] = x;
        }
        // eight ballots whatever the width: a live item's bits above it are 0
        uint32_t peers = __ballot_sync(0xffffffffu, ok);
#pragma unroll
        for (int bit = 0; bit < 8; bit++) {
          const uint32_t bm = __ballot_sync(0xffffffffu, (d >> bit) & 1);
          peers &= ((d >> bit) & 1) ? bm : ~bm;
        }
        if (!ok) peers = 1u << lane;
        const int leader = __ffs(peers) - 1;
        uint32_t cnt = 0;
        if (lane == leader && ok) {
          cnt = wh[d];
          wh[d] = cnt + __popc(peers);
        }
        cnt = __shfl_sync(0xffffffffu, cnt, leader);
        dg[j] = d;
        rk[j] = cnt + __popc(peers & lt);
        __syncwarp();
      }
      __syncthreads();
      // thread d < 256: exclusive prefix of digit d over the warps, then over
      // digits (warps 0-7; the others wait at the barriers)
      uint32_t tot = 0, incl = 0;
      if (tid < 256) {
#pragma unroll
        for (int w = 0; w < kTdWarps; w++) {
          const uint32_t x = S.wh[w][tid];
          S.wh[w][tid] = tot;
          tot += x;
        }
        incl = tot;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += y;
        }
        if (lane == 31) S.wsum[warp] = incl;
      }
      __syncthreads();
      if (tid < 256) {
        uint32_t woff = 0;
#pragma unroll
        for (int w = 0; w < 8; w++) woff += w < warp ? S.wsum[w] : 0u;
        S.dstart[tid] = woff + incl - tot;
      }
      __syncthreads();
#pragma unroll
      for (int j = 0; j < kTdItems; j++) {
        const int i = warp * (32 * kTdItems) + j * 32 + lane;
        if (i < m) S.item[1 - cur][S.dstart[dg[j]] + S.wh[warp][dg[j]] + rk[j]] = it[j];
      }
      cur = 1 - cur;
    }
  }
  __syncthreads();
  for (int i = tid; i < m; i += kTdThreads) {
    const uint32_t slot = S.item[cur][i] & 0xFFFFu;
    uint32_t r = perm_in ? perm_in[base + slot] : (uint32_t)(base + slot);
    if ((int64_t)r >= n) r = 0;
    perm_out[base + i] = r;
  }
}

// Launches the short-run sort of the local levels lv (first run length at
// most kTdLocal, each next one dividing it).
template <typename T>
int td_local_levels(const T *cxy, int stride, const uint32_t *perm_a, const uint32_t *perm_b, const int *sel,
                    int64_t n, const TdLocalLevels &lv, uint32_t *perm_out, cudaStream_t s) {
  const int64_t chunk = (kTdLocal / lv.seg[0]) * lv.seg[0];
  const size_t smem = sizeof(TdLocalSmem<T>);
  static bool attr_done[256] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 256 || !attr_done[dev]) {
    PRT_CUDA(cudaFuncSetAttribute(td_local_sort_kernel<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    PRT_CUDA(cudaFuncSetAttribute(td_local_sort_kernel<T, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (dev >= 0 && dev < 256) attr_done[dev] = true;
  }
  const int64_t blocks = (n + chunk - 1) / chunk;
  {
    PRT_PROF("td_local_sort", s);
    if (stride == 2)
      td_local_sort_kernel<T, 2><<<(unsigned)blocks, kTdThreads, smem, s>>>(cxy, perm_a, perm_b, sel, n, lv, perm_out);
    else
      td_local_sort_kernel<T, 4><<<(unsigned)blocks, kTdThreads, smem, s>>>(cxy, perm_a, perm_b, sel, n, lv, perm_out);
  }
  PRT_CUDA(cudaGetLastError());
  return PRT_OK;
}

// ------------------------------------------------------------------ packing

// Leaf level: gather the records in leaf order (coalesced writes), their ids,
// and when F divides 32, the leaf-node unions for level 1 by shuffles.  The
// gather by sort index is random, so each warp takes kLeafUnroll chunks of 32
// consecutive leaves at a time and issues all their index loads, then all
// their box loads, before using any: more independent loads in flight.
constexpr int kLeafUnroll = 4;

template <typename T, int F>
__global__ void __launch_bounds__(256) pack_leaf_kernel(const Box<T> *__restrict__ b, const int32_t *__restrict__ ids,
                                 const uint32_t *__restrict__ perm_a, const uint32_t *__restrict__ perm_b,
                                 const int *__restrict__ sel, int64_t n, int64_t padded, Box<T> *__restrict__ lv0,
                                 int32_t *__restrict__ leaf_id, Box<T> *__restrict__ lv1) {
  const uint32_t *perm = (sel && *sel) ? perm_b : perm_a;
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  constexpr int64_t kChunk = 32 * kLeafUnroll;
  for (int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; c * kChunk < padded; c += nwarps) {
    uint32_t r[kLeafUnroll];
#pragma unroll
    for (int k = 0; k < kLeafUnroll; k++) {
      const int64_t j = c * kChunk + 32 * k + lane;
      r[k] = j < n ? perm[j] : 0u;
      if ((int64_t)r[k] >= n) r[k] = 0;  // only after a timed-out sort (reported by the caller)
    }
    Box<T> x[kLeafUnroll];
#pragma unroll
    for (int k = 0; k < kLeafUnroll; k++) {
      const int64_t j = c * kChunk + 32 * k + lane;
      x[k] = j < n ? load_box(b, r[k]) : empty_box<T>();
    }
#pragma unroll
    for (int k = 0; k < kLeafUnroll; k++) {
      const int64_t j = c * kChunk + 32 * k + lane;
      if (j < n) leaf_id[j] = ids ? ids[r[k]] : (int32_t)r[k];
      else if (j < padded) leaf_id[j] = -1;
      if (j < padded) store_box(lv0, j, x[k]);
      if constexpr (F > 0) {
        Box<T> u = x[k];
#pragma unroll
        for (int o = F / 2; o > 0; o >>= 1) {
          u.x1 = tmin(u.x1, __shfl_xor_sync(0xffffffffu, u.x1, o));
          u.y1 = tmin(u.y1, __shfl_xor_sync(0xffffffffu, u.y1, o));
          u.x2 = tmax(u.x2, __shfl_xor_sync(0xffffffffu, u.x2, o));
          u.y2 = tmax(u.y2, __shfl_xor_sync(0xffffffffu, u.y2, o));
        }
        if ((j % F) == 0 && j < n) store_box(lv1, j / F, u);
      }
    }
  }
}

// Upper level: entry j of level l+1 = union of node j of level l.
template <typename T>
__global__ void pack_level_kernel(const Box<T> *__restrict__ lo, int64_t n_lo, int fanout, Box<T> *__restrict__ hi,
                                  int64_t n_hi, int64_t padded_hi) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < padded_hi; j += (int64_t)gridDim.x * blockDim.x) {
    if (j >= n_hi) {
      store_box(hi, j, empty_box<T>());
      continue;
    }
    int64_t a = j * fanout, e = min(a + fanout, n_lo);
    Box<T> u = load_box(lo, a);
    for (int64_t k = a + 1; k < e; k++) {
      Box<T> x = load_box(lo, k);
      u.x1 = tmin(u.x1, x.x1);
      u.y1 = tmin(u.y1, x.y1);
      u.x2 = tmax(u.x2, x.x2);
      u.y2 = tmax(u.y2, x.y2);
    }
    store_box(hi, j, u);
  }
}

// padding of level 1 when the leaf kernel wrote the unions
template <typename T>
__global__ void pad_level_kernel(Box<T> *__restrict__ lv, int64_t n, int64_t padded) {
  int64_t j = n + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j < padded) store_box(lv, j, empty_box<T>());
}

template <typename T>
int pack_tree(prt_tree *t, const void *d_boxes, const int32_t *d_ids, const uint32_t *perm_a,
              const uint32_t *perm_b, const int *d_sel, cudaStream_t s) {
  const TreeLevels &L = t->lv;
  const Box<T> *b = reinterpret_cast<const Box<T> *>(d_boxes);
  Box<T> *mbr = reinterpret_cast<Box<T> *>(t->d_mbr);
  Box<T> *lv1 = L.levels > 1 ? mbr + L.offset[1] : nullptr;
  const int block = 256;
  int g = grid_for((L.padded[0] + kLeafUnroll - 1) / kLeafUnroll, block, 8);
  bool fused = false;
  switch (L.levels > 1 ? t->fanout : 0) {
#define PRT_LEAF_CASE(F)                                                                                 \
  case F: {                                                                                              \
    PRT_PROF("pack_leaf", s);                                                                            \
    pack_leaf_kernel<T, F><<<g, block, 0, s>>>(b, d_ids, perm_a, perm_b, d_sel, t->n, L.padded[0], mbr, \
                                               t->d_leaf_id, lv1 ? lv1 : mbr);                           \
    fused = lv1 != nullptr;                                                                              \
    break;                                                                                               \
  }
    PRT_LEAF_CASE(2)
    PRT_LEAF_CASE(4)
    PRT_LEAF_CASE(8)
    PRT_LEAF_CASE(16)
    PRT_LEAF_CASE(32)
#undef PRT_LEAF_CASE
    default:
      {
        PRT_PROF("pack_leaf", s);
        pack_leaf_kernel<T, 0><<<g, block, 0, s>>>(b, d_ids, perm_a, perm_b, d_sel, t->n, L.padded[0], mbr,
                                                 t->d_leaf_id, nullptr);
      }
  }
  for (int l = 1; l < L.levels; l++) {
    if (l == 1 && fused) {
      int64_t pad = L.padded[1] - L.count[1];
      if (pad > 0) {
        PRT_PROF("pad_level", s);
        pad_level_kernel<T><<<1, 64, 0, s>>>(lv1, L.count[1], L.padded[1]);
      }
      continue;
    }
    {
      PRT_PROF("pack_level", s);
      pack_level_kernel<T><<<grid_for(L.padded[l], block, 16), block, 0, s>>>(
        mbr + L.offset[l - 1], L.count[l - 1], t->fanout, mbr + L.offset[l], L.count[l], L.padded[l]);
    }
  }
  PRT_CUDA(cudaGetLastError());
  return PRT_OK;
}

int new_tree(const void *d_boxes, int coord, int64_t n, int fanout, int kind, int key_mode, cudaStream_t s,
             prt_tree **out) {
  PRT_CHECK(out != nullptr, PRT_ERR_INVALID, "out is NULL");
  *out = nullptr;
  PRT_CHECK(d_boxes != nullptr || n == 0, PRT_ERR_INVALID, "d_boxes is NULL");
  PRT_CHECK((reinterpret_cast<uintptr_t>(d_boxes) & 15) == 0, PRT_ERR_INVALID,
            "d_boxes must be 16-byte aligned (boxes are read as 16-byte vectors)");
  PRT_CHECK(n >= 1 && n < (1ll << 30), PRT_ERR_INVALID, "n=%lld outside [1, 2^30)", (long long)n);
  PRT_CHECK(fanout >= 2 && fanout <= 32, PRT_ERR_INVALID, "fanout %d outside [2, 32]", fanout);
  PRT_CHECK(coord >= 0 && coord <= 3, PRT_ERR_INVALID, "coordinate type %d", coord);
  prt_tree *t = new prt_tree();
  t->kind = kind;
  t->coord = coord;
  t->fanout = fanout;
  t->key_mode = key_mode;
  t->n = n;
  t->lv = level_layout(n, fanout);
  cudaGetDevice(&t->device);
  size_t bs = 4 * coord_size(coord);
  int rc = dmalloc(&t->d_mbr, bs * t->lv.total, s);
  if (!rc) rc = dalloc(&t->d_leaf_id, t->lv.padded[0], s);
  if (rc) {
    dfree(t->d_mbr, s);
    dfree(t->d_leaf_id, s);
    delete t;
    return rc;
  }
  *out = t;
  return PRT_OK;
}

int finish(unsigned *d_err, cudaStream_t s, int rc) {
  unsigned herr = 0;
  if (rc == PRT_OK) {
    cudaError_t e = cudaMemcpyAsync(&herr, d_err, sizeof herr, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = cuda_status(e, "build");
  }
  if (rc == PRT_OK && (herr & kErrTimeout)) {
    set_error("radix sort look-back wait timed out");
    rc = PRT_ERR_TIMEOUT;
  }
  return rc;
}

}  // namespace

// Enqueues the bottom-up build of `t` (allocated by tree_alloc) from d_boxes
// without any host synchronisation, so it can be captured in a CUDA graph;
// *d_err (device, zeroed by the caller) receives kErrTimeout if a sort
// look-back wait gives up.
int bu_enqueue(prt_tree *t, const void *d_boxes, const int32_t *d_ids, unsigned *err, cudaStream_t s) {
  const int64_t n = t->n;
  // scratch: ext (4 x 8), err, sel, digit histograms (4 x 256), keys0/1, vals0/1
  unsigned char *scr = nullptr;
  size_t kb = t->key_mode == PRT_KEY_REF64 ? 8 : 4;
  size_t need = 64 + 4096 + 2 * kb * n + 2 * 4 * n + 64;
  int rc = dmalloc(reinterpret_cast<void **>(&scr), need, s);
  if (rc) return rc;
  unsigned long long *ext = reinterpret_cast<unsigned long long *>(scr);
  int *sel = reinterpret_cast<int *>(scr + 36);
  uint32_t *hist = reinterpret_cast<uint32_t *>(scr + 64);
  unsigned char *kp = scr + 64 + 4096;
  void *keys0 = kp, *keys1 = kp + kb * n;
  uint32_t *vals0 = reinterpret_cast<uint32_t *>(kp + 2 * kb * n);
  uint32_t *vals1 = vals0 + n;
  cudaError_t e = cudaSuccess;
  int g = grid_for(n, 256, 16);
  if (e == cudaSuccess) {
    if (t->key_mode == PRT_KEY_MORTON32) {
      e = cudaMemsetAsync(hist, 0, 4096, s);
      if (e != cudaSuccess) {
        dfree(scr, s);
        return cuda_status(e, "memset");
      }
      {
        PRT_PROF("extent_init", s);
        extent_init_kernel<<<1, 1, 0, s>>>(ext);
      }
      rc = dispatch_coord(t->coord, [&](auto tag) {
        using T = decltype(tag);
        const Box<T> *b = reinterpret_cast<const Box<T> *>(d_boxes);
        {
          PRT_PROF("extent_f64", s);
          // 16 blocks per SM: enough loads in flight to stream the boxes
          extent_f64_kernel<T><<<grid_for(n, 256, 16), 256, 0, s>>>(b, n, ext);
        }
        {
          PRT_PROF("morton32", s);
          morton32_kernel<T><<<g, 256, 0, s>>>(b, n, ext, reinterpret_cast<uint32_t *>(keys0), vals0, hist);
        }
        return PRT_OK;
      });
      if (!rc)
        rc = radix_sort_pairs<uint32_t>(reinterpret_cast<uint32_t *>(keys0), vals0,
                                        reinterpret_cast<uint32_t *>(keys1), vals1, n, 32, sel, err, s, hist);
    } else {
      long long *ei = reinterpret_cast<long long *>(ext);
      const Box<int64_t> *b = reinterpret_cast<const Box<int64_t> *>(d_boxes);
      {
        PRT_PROF("extent_i64_init", s);
        extent_i64_init_kernel<<<1, 1, 0, s>>>(ei);
      }
      {
        PRT_PROF("extent_i64", s);
        extent_i64_kernel<<<grid_for(n, 256, 4), 256, 0, s>>>(b, n, ei);
      }
      {
        PRT_PROF("ref64", s);
        ref64_kernel<<<g, 256, 0, s>>>(b, n, ei, reinterpret_cast<uint64_t *>(keys0), vals0);
      }
      rc = radix_sort_pairs<uint64_t>(reinterpret_cast<uint64_t *>(keys0), vals0,
                                      reinterpret_cast<uint64_t *>(keys1), vals1, n, 64, sel, err, s);
    }
  } else {
    rc = cuda_status(e, "memset");
  }
  if (!rc) rc = dispatch_coord(t->coord, [&](auto tag) {
    using T = decltype(tag);
    return pack_tree<T>(t, d_boxes, d_ids, vals0, vals1, sel, s);
  });
  dfree(scr, s);
  return rc;
}

int tree_alloc(const void *d_boxes, int coord, int64_t n, int fanout, int kind, int key_mode, cudaStream_t s,
               prt_tree **out) {
  return new_tree(d_boxes, coord, n, fanout, kind, key_mode, s, out);
}

}  // namespace prt

using namespace prt;

extern "C" {

const char *prt_last_error(void) { return g_err.c_str(); }
int prt_version(void) { return 1; }

int prt_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

int prt_build_bottomup(const void *d_boxes, int coord_type, const int32_t *d_ids, int64_t n, int fanout,
                       int key_mode, void *stream, prt_tree **out) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  PRT_CHECK(key_mode == PRT_KEY_MORTON32 || key_mode == PRT_KEY_REF64, PRT_ERR_INVALID, "key mode %d",
            key_mode);
  PRT_CHECK(key_mode != PRT_KEY_REF64 || coord_type == PRT_COORD_I64, PRT_ERR_INVALID,
            "REF64 keys need int64 boxes");
  prt_tree *t = nullptr;
  int rc = new_tree(d_boxes, coord_type, n, fanout, PRT_BOTTOM_UP, key_mode, s, &t);
  if (rc) return rc;
  unsigned *err = nullptr;
  rc = dalloc(&err, 2, s);
  if (!rc) {
    cudaError_t e = cudaMemsetAsync(err, 0, 8, s);
    if (e != cudaSuccess) rc = cuda_status(e, "memset");
  }
  if (!rc) rc = bu_enqueue(t, d_boxes, d_ids, err, s);
  rc = finish(err, s, rc);
  dfree(err, s);
  if (rc) {
    prt_tree_free(t);
    return rc;
  }
  *out = t;
  return PRT_OK;
}

int prt_build_topdown(const void *d_boxes, int coord_type, const int32_t *d_ids, int64_t n, int fanout,
                      void *stream, prt_tree **out) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  prt_tree *t = nullptr;
  int rc = new_tree(d_boxes, coord_type, n, fanout, PRT_TOP_DOWN, -1, s, &t);
  if (rc) return rc;
  const int H = t->lv.levels;
  const bool wide = coord_size(coord_type) == 8;
  unsigned char *scr = nullptr;
  // per-run digit histograms: at most one run per sort tile, 8 passes
  const size_t hist_words = (size_t)((n + kSortRunTile - 1) / kSortRunTile) * 8 * 256;
  // and the compact (x1, y1) copy the first level writes
  const size_t csize = (size_t)coord_size(coord_type);
  size_t need = 64 + 2 * 8 * n + 4 * 4 * n + 4 * hist_words + 2 * csize * n + 64;
  rc = dmalloc(reinterpret_cast<void **>(&scr), need, s);
  if (rc) {
    prt_tree_free(t);
    return rc;
  }
  unsigned *err = reinterpret_cast<unsigned *>(scr);
  int *sel = reinterpret_cast<int *>(scr + 8);
  uint64_t *k0 = reinterpret_cast<uint64_t *>(scr + 64);
  uint64_t *k1 = k0 + n;
  uint32_t *v0 = reinterpret_cast<uint32_t *>(k1 + n);
  uint32_t *v1 = v0 + n;
  uint32_t *perm = v1 + n;  // current leaf order (when materialised)
  uint32_t *tmp = perm + n;  // scratch
  uint32_t *hist = tmp + n;
  void *xyc = hist + hist_words;
  // where the levels read record r's (x1, y1): d_boxes[4 r], or the compact
  // copy at xyc[2 r] once a level has written it
  const void *cxy = d_boxes;
  int cstride = 4;
  cudaError_t e = cudaMemsetAsync(err, 0, 8, s);
  if (e != cudaSuccess) rc = cuda_status(e, "memset");
  const int g = grid_for(n, 256, 16);
  // the current order: pa or pb as *psel says (psel nullptr: pa; pa nullptr:
  // the identity).  A sort leaves it in (v0, v1, sel) and the next level
  // reads it there; paths that need one array copy it into perm first.
  const uint32_t *pa = nullptr, *pb = nullptr;
  const int *psel = nullptr;
  auto materialise = [&]() -> const uint32_t * {
    if (psel && !rc) {
      PRT_PROF("select_copy_u32", s);
      select_copy_u32_kernel<<<g, 256, 0, s>>>(pa, pb, psel, n, perm);
      pa = pb = perm;
      psel = nullptr;
    }
    return pa;
  };
  for (int p = 0; p < H && !rc; p++) {
    // segment size fanout^(H-p), saturated at n
    int64_t seg = 1;
    for (int k = 0; k < H - p; k++) {
      seg *= fanout;
      if (seg >= n) {
        seg = n;
        break;
      }
    }
    int64_t nseg = (n + seg - 1) / seg;
    int seg_bits = 0;
    while ((1ll << seg_bits) < nseg) seg_bits++;
    const int use_y = p & 1;
    if (seg <= kTdLocal) {
      // this and every later level have short runs: all of them sorted in
      // shared memory by one launch
      TdLocalLevels lv;
      lv.count = 0;
      for (int q = p; q < H && lv.count < kTdMaxLocal; q++) {
        // run length fanout^(H-q), saturated at n like seg (only when all n
        // records fit in one tile)
        int64_t sq = 1;
        for (int k = 0; k < H - q && sq < n; k++) sq *= fanout;
        if (sq > n) sq = n;
        lv.seg[lv.count] = sq;
        lv.use_y[lv.count] = q & 1;
        lv.count++;
      }
      uint32_t *out = (pa == tmp || pb == tmp) ? perm : tmp;
      rc = dispatch_coord(coord_type, [&](auto tag) {
        using T = decltype(tag);
        return td_local_levels<T>(reinterpret_cast<const T *>(cxy), cstride, pa, pb, psel, n, lv, out, s);
      });
      pa = pb = out;
      psel = nullptr;
      p += lv.count - 1;  // the loop's p++ moves past the last local level
    } else if (seg % kSortRunTile == 0 || seg == n) {
      // runs of whole sort tiles (or one run): every run sorted on its own by
      // the coordinate alone, 4 (32-bit) or 8 (64-bit) passes; the key kernel
      // counts the digit histograms
      rc = dispatch_coord(coord_type, [&](auto tag) {
        using T = decltype(tag);
        using K = typename std::conditional<sizeof(T) == 8, uint64_t, uint32_t>::type;
        K *kk0 = reinterpret_cast<K *>(k0), *kk1 = reinterpret_cast<K *>(k1);
        const int64_t tiles = (n + kSortRunTile - 1) / kSortRunTile;
        const int64_t tpr = seg == n ? tiles : seg / kSortRunTile;
        PRT_CUDA(cudaMemsetAsync(hist, 0, sizeof(uint32_t) * (size_t)((tiles + tpr - 1) / tpr) * sizeof(K) * 256, s));
        // the identity order reads the boxes in order: write the compact copy
        T *xy_out = (pa == nullptr && cstride == 4) ? reinterpret_cast<T *>(xyc) : nullptr;
        {
          PRT_PROF("td_key", s);
          td_keyrun_kernel<T, K><<<(unsigned)tiles, 256, 0, s>>>(reinterpret_cast<const T *>(cxy), cstride, pa, pb,
                                                                 psel, n, use_y, tpr, kk0, v0, hist, xy_out);
        }
        if (xy_out) {
          cxy = xy_out;
          cstride = 2;
        }
        PRT_CUDA(cudaGetLastError());
        return seg == n ? radix_sort_pairs<K>(kk0, v0, kk1, v1, n, 8 * (int)sizeof(K), sel, err, s, hist)
                        : radix_sort_runs<K>(kk0, v0, kk1, v1, n, seg, sel, err, s, hist);
      });
      pa = v0;
      pb = v1;
      psel = sel;
    } else if (!wide) {
      const uint32_t *cur = materialise();
      rc = dispatch_coord(coord_type, [&](auto tag) {
        using T = decltype(tag);
        if constexpr (sizeof(T) == 4) {
          {
            PRT_PROF("td_key32", s);
            td_key32_kernel<T><<<g, 256, 0, s>>>(reinterpret_cast<const Box<T> *>(d_boxes), cur, n, seg, use_y, k0,
                                               v0);
          }
        }
        return PRT_OK;
      });
      if (!rc) rc = radix_sort_pairs<uint64_t>(k0, v0, k1, v1, n, 32 + seg_bits, sel, err, s);
      pa = v0;
      pb = v1;
      psel = sel;
    } else {
      const uint32_t *cur = materialise();
      rc = dispatch_coord(coord_type, [&](auto tag) {
        using T = decltype(tag);
        if constexpr (sizeof(T) == 8) {
          {
            PRT_PROF("td_key64", s);
            td_key64_kernel<T><<<g, 256, 0, s>>>(reinterpret_cast<const Box<T> *>(d_boxes), cur, n, use_y, k0, v0);
          }
        }
        return PRT_OK;
      });
      if (!rc) rc = radix_sort_pairs<uint64_t>(k0, v0, k1, v1, n, 64, sel, err, s);
      if (!rc) {
        // positions, in coordinate order
        PRT_PROF("select_copy_u32", s);
        select_copy_u32_kernel<<<g, 256, 0, s>>>(v0, v1, sel, n, tmp);
      }
      if (!rc && seg_bits > 0) {
        uint32_t *sk0 = reinterpret_cast<uint32_t *>(k0), *sk1 = reinterpret_cast<uint32_t *>(k1);
        {
          PRT_PROF("td_segkey", s);
          td_segkey_kernel<<<g, 256, 0, s>>>(tmp, n, seg, sk0);
        }
        rc = radix_sort_pairs<uint32_t>(sk0, tmp, sk1, v1, n, seg_bits, sel, err, s);
        if (!rc) {
          PRT_PROF("select_copy_u32", s);
          select_copy_u32_kernel<<<g, 256, 0, s>>>(tmp, v1, sel, n, v0);
        }
        if (!rc) {
          cudaMemcpyAsync(tmp, v0, 4 * n, cudaMemcpyDeviceToDevice, s);
        }
      }
      // positions -> records (gathered into v0 first: cur may alias perm)
      if (!rc) {
        {
          PRT_PROF("gather_u32", s);
          gather_u32_kernel<<<g, 256, 0, s>>>(cur, tmp, n, v0);
        }
        cudaMemcpyAsync(perm, v0, 4 * n, cudaMemcpyDeviceToDevice, s);
      }
      pa = pb = perm;
      psel = nullptr;
    }
  }
  if (!rc) rc = dispatch_coord(coord_type, [&](auto tag) {
    using T = decltype(tag);
    return pack_tree<T>(t, d_boxes, d_ids, pa, pb, psel, s);
  });
  rc = finish(err, s, rc);
  dfree(scr, s);
  if (rc) {
    prt_tree_free(t);
    return rc;
  }
  *out = t;
  return PRT_OK;
}

// Stream-ordered release on the legacy default stream (which orders itself
// after all blocking streams): no device-wide synchronisation.
int prt_tree_free(prt_tree *t) {
  if (!t) return PRT_OK;
  cudaFreeAsync(t->d_mbr, 0);
  cudaFreeAsync(t->d_leaf_id, 0);
  cudaGetLastError();
  delete t;
  return PRT_OK;
}

int prt_tree_info(const prt_tree *t, int64_t *info) {
  PRT_CHECK(t && info, PRT_ERR_INVALID, "NULL argument");
  for (int i = 0; i < 8 + PRT_MAX_LEVELS; i++) info[i] = 0;
  info[0] = t->n;
  info[1] = t->fanout;
  info[2] = t->lv.levels;
  info[3] = t->kind;
  info[4] = t->coord;
  info[5] = t->key_mode;
  for (int l = 0; l < t->lv.levels; l++) info[8 + l] = t->lv.count[l];
  return PRT_OK;
}

int prt_tree_level_mbr(const prt_tree *t, int level, double *h_out) {
  PRT_CHECK(t && h_out, PRT_ERR_INVALID, "NULL argument");
  PRT_CHECK(level >= 0 && level < t->lv.levels, PRT_ERR_INVALID, "level %d", level);
  const int64_t cnt = t->lv.count[level];
  size_t cs = coord_size(t->coord);
  std::string buf(cnt * 4 * cs, '\0');
  PRT_CUDA(cudaDeviceSynchronize());
  PRT_CUDA(cudaMemcpy(&buf[0], reinterpret_cast<const char *>(t->d_mbr) + t->lv.offset[level] * 4 * cs,
                      cnt * 4 * cs, cudaMemcpyDeviceToHost));
  for (int64_t i = 0; i < 4 * cnt; i++) {
    const char *p = buf.data() + i * cs;
    switch (t->coord) {
      case PRT_COORD_I64: h_out[i] = (double)reinterpret_cast<const int64_t *>(p)[0]; break;
      case PRT_COORD_F32: h_out[i] = (double)reinterpret_cast<const float *>(p)[0]; break;
      case PRT_COORD_F64: h_out[i] = reinterpret_cast<const double *>(p)[0]; break;
      default: h_out[i] = (double)reinterpret_cast<const int32_t *>(p)[0]; break;
    }
  }
  return PRT_OK;
}

int prt_tree_leaf_order(const prt_tree *t, int32_t *d_out, void *stream) {
  PRT_CHECK(t && d_out, PRT_ERR_INVALID, "NULL argument");
  PRT_CUDA(cudaMemcpyAsync(d_out, t->d_leaf_id, sizeof(int32_t) * t->n, cudaMemcpyDeviceToDevice,
                           reinterpret_cast<cudaStream_t>(stream)));
  return PRT_OK;
}

int prt_tree_export_bu_size(const prt_tree *t, int64_t *n_nodes) {
  PRT_CHECK(t && n_nodes, PRT_ERR_INVALID, "NULL argument");
  int64_t nn = 0;
  for (int l = 0; l < t->lv.levels; l++) nn += (t->lv.count[l] + t->fanout - 1) / t->fanout;
  *n_nodes = nn;
  return PRT_OK;
}

// Reference node order: node levels bottom-up, nodes in level order; the
// children of node j of level l+1 are nodes jF.. of level l.
int prt_tree_export_bu(const prt_tree *t, int32_t *h_flag, int32_t *h_num, double *h_mbr, int32_t *h_children,
                       int32_t *h_data, int32_t *h_root) {
  PRT_CHECK(t && h_flag && h_num && h_mbr && h_children && h_data && h_root, PRT_ERR_INVALID, "NULL argument");
  const int F = t->fanout;
  std::vector<int64_t> first(t->lv.levels + 1, 0);
  for (int l = 0; l < t->lv.levels; l++) first[l + 1] = first[l] + (t->lv.count[l] + F - 1) / F;
  std::vector<int32_t> ids(t->n);
  PRT_CUDA(cudaDeviceSynchronize());
  PRT_CUDA(cudaMemcpy(ids.data(), t->d_leaf_id, sizeof(int32_t) * t->n, cudaMemcpyDeviceToHost));
  for (int l = 0; l < t->lv.levels; l++) {
    std::vector<double> m(4 * t->lv.count[l]);
    int rc = prt_tree_level_mbr(t, l, m.data());
    if (rc) return rc;
    int64_t nodes = first[l + 1] - first[l];
    for (int64_t j = 0; j < nodes; j++) {
      int64_t k = first[l] + j;
      int64_t a = j * F, e = std::min<int64_t>(a + F, t->lv.count[l]);
      h_flag[k] = l == 0 ? 0 : 1;
      h_num[k] = (int32_t)(e - a);
      for (int s2 = 0; s2 < F; s2++) {
        int64_t q = a + s2;
        bool live = q < e;
        for (int c = 0; c < 4; c++) h_mbr[(k * F + s2) * 4 + c] = live ? m[4 * q + c] : 0.0;
        h_children[k * F + s2] = live && l > 0 ? (int32_t)(first[l - 1] + q) : -1;
        h_data[k * F + s2] = live && l == 0 ? ids[q] : -1;
      }
    }
  }
  *h_root = (int32_t)(first[t->lv.levels] - 1);
  return PRT_OK;
}

int prt_tree_export_td_size(const prt_tree *t, int64_t *n_slots, int32_t *n_offsets) {
  PRT_CHECK(t && n_slots && n_offsets, PRT_ERR_INVALID, "NULL argument");
  int64_t s = 0;
  for (int l = 0; l < t->lv.levels; l++) s += t->lv.padded[l];
  *n_slots = s;
  *n_offsets = t->lv.levels + 1;
  return PRT_OK;
}

// Reference slot order: levels top-down (root slots first); slot i of a level
// points at the first slot of node i of the level below.
int prt_tree_export_td(const prt_tree *t, int32_t *h_nodes_index, double *h_nodes_mbr, int32_t *h_offsets) {
  PRT_CHECK(t && h_nodes_index && h_nodes_mbr && h_offsets, PRT_ERR_INVALID, "NULL argument");
  const int L = t->lv.levels;
  std::vector<int64_t> off(L + 1, 0);
  for (int p = 0; p < L; p++) off[p + 1] = off[p] + t->lv.padded[L - 1 - p];
  for (int p = 0; p <= L; p++) h_offsets[p] = (int32_t)off[p];
  for (int p = 0; p < L; p++) {
    int l = L - 1 - p;
    std::vector<double> m(4 * t->lv.count[l]);
    int rc = prt_tree_level_mbr(t, l, m.data());
    if (rc) return rc;
    for (int64_t i = 0; i < t->lv.padded[l]; i++) {
      int64_t s = off[p] + i;
      bool live = i < t->lv.count[l];
      h_nodes_index[s] = !live ? 0 : (l == 0 ? (int32_t)(-i - 1) : (int32_t)(off[p + 1] + i * t->fanout));
      for (int c = 0; c < 4; c++) h_nodes_mbr[4 * s + c] = live ? m[4 * i + c] : 0.0;
    }
  }
  return PRT_OK;
}

}  // extern "C"
