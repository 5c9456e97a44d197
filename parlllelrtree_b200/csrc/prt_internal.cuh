// Internal helpers shared by the library's CUDA translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <string>

#include "../../include/prt.h"

namespace prt {

// ---- error reporting -------------------------------------------------------
void set_error(const char *fmt, ...);
int cuda_status(cudaError_t e, const char *what);

#define PRT_CUDA(call)                                             \
  do {                                                             \
    cudaError_t prt_e_ = (call);                                   \
    if (prt_e_ != cudaSuccess) return ::prt::cuda_status(prt_e_, #call); \
  } while (0)

#define PRT_CHECK(cond, code, ...)        \
  do {                                    \
    if (!(cond)) {                        \
      ::prt::set_error(__VA_ARGS__);      \
      return (code);                      \
    }                                     \
  } while (0)

// The device-side error word: bit 0 capacity, bit 1 timeout, bit 2 invalid.
enum : unsigned { kErrCapacity = 1u, kErrTimeout = 2u, kErrInvalid = 4u };

// Bounded spin limit for decoupled look-back waits: every wait on another
// CTA's flag gives up after this many polls and records kErrTimeout.
constexpr int kSpinLimit = 1 << 22;

// The wait limit the next sorts use: kSpinLimit polls unless a test lowered
// it with prt_debug_wait_limit, which can also make every look-back see no
// predecessor published, so that each wait runs to its limit and the
// timeout path is exercised without a hang or a fault.
struct WaitLimit {
  int polls;
  int blind;
};
WaitLimit wait_limit();

constexpr int kSMs = 148;

// ---- launch profiler ---------------------------------------------------------
// When enabled (prt_profile_enable), every kernel launch wrapped in PRT_PROF
// is bracketed by two CUDA events on its own stream; prt_profile_read sums the
// device durations per kernel name.  Disabled, a scope costs one branch.
extern bool g_prof_on;
void prof_begin(const char *name, cudaStream_t s, void **token);
void prof_end(void *token, cudaStream_t s);
struct ProfScope {
  void *token = nullptr;
  cudaStream_t s;
  ProfScope(const char *name, cudaStream_t st) : s(st) {
    if (g_prof_on) prof_begin(name, st, &token);
  }
  ~ProfScope() {
    if (token) prof_end(token, s);
  }
};
#define PRT_PROF_CAT2(a, b) a##b
#define PRT_PROF_CAT(a, b) PRT_PROF_CAT2(a, b)
#define PRT_PROF(name, s) ::prt::ProfScope PRT_PROF_CAT(prt_prof_, __LINE__)(name, s)

// ---- stream-ordered scratch ------------------------------------------------
int dmalloc(void **p, size_t bytes, cudaStream_t s);
void dfree(void *p, cudaStream_t s);

template <typename T>
int dalloc(T **p, size_t count, cudaStream_t s) {
  return dmalloc(reinterpret_cast<void **>(p), count * sizeof(T), s);
}

// ---- coordinate traits -----------------------------------------------------
template <typename T>
struct Box {
  T x1, y1, x2, y2;
};

template <typename T>
struct CoordLimits;
template <>
struct CoordLimits<float> {
  __host__ __device__ static float lo() { return -3.402823466e38f; }
  __host__ __device__ static float hi() { return 3.402823466e38f; }
};
template <>
struct CoordLimits<double> {
  __host__ __device__ static double lo() { return -1.7976931348623157e308; }
  __host__ __device__ static double hi() { return 1.7976931348623157e308; }
};
template <>
struct CoordLimits<int64_t> {
  __host__ __device__ static int64_t lo() { return INT64_MIN; }
  __host__ __device__ static int64_t hi() { return INT64_MAX; }
};
template <>
struct CoordLimits<int32_t> {
  __host__ __device__ static int32_t lo() { return INT32_MIN; }
  __host__ __device__ static int32_t hi() { return INT32_MAX; }
};

// An entry that intersects nothing: fills the padded slots of a node.
template <typename T>
__host__ __device__ inline Box<T> empty_box() {
  return Box<T>{CoordLimits<T>::hi(), CoordLimits<T>::hi(), CoordLimits<T>::lo(), CoordLimits<T>::lo()};
}

// Closed-interval intersection; equals the reference's
// "width_a + width_b + 1e-8 < union width => disjoint" test for valid boxes
// (BotomUp-rtree.cu:496-506, TopDown-rtree.cu:26-39).
template <typename T>
__host__ __device__ inline bool overlaps(const Box<T> &a, const Box<T> &b) {
  return a.x1 <= b.x2 && b.x1 <= a.x2 && a.y1 <= b.y2 && b.y1 <= a.y2;
}

template <typename T>
__device__ inline T tmin(T a, T b) { return b < a ? b : a; }
template <typename T>
__device__ inline T tmax(T a, T b) { return b > a ? b : a; }

template <typename T>
__device__ inline Box<T> load_box(const Box<T> *p, int64_t i);

template <>
__device__ inline Box<float> load_box(const Box<float> *p, int64_t i) {
  float4 v = __ldg(reinterpret_cast<const float4 *>(p) + i);
  return Box<float>{v.x, v.y, v.z, v.w};
}
template <>
__device__ inline Box<int32_t> load_box(const Box<int32_t> *p, int64_t i) {
  int4 v = __ldg(reinterpret_cast<const int4 *>(p) + i);
  return Box<int32_t>{v.x, v.y, v.z, v.w};
}
template <>
__device__ inline Box<double> load_box(const Box<double> *p, int64_t i) {
  const double2 *q = reinterpret_cast<const double2 *>(p) + 2 * i;
  double2 a = __ldg(q), b = __ldg(q + 1);
  return Box<double>{a.x, a.y, b.x, b.y};
}
template <>
__device__ inline Box<int64_t> load_box(const Box<int64_t> *p, int64_t i) {
  const longlong2 *q = reinterpret_cast<const longlong2 *>(p) + 2 * i;
  longlong2 a = __ldg(q), b = __ldg(q + 1);
  return Box<int64_t>{a.x, a.y, b.x, b.y};
}

template <typename T>
__device__ inline void store_box(Box<T> *p, int64_t i, const Box<T> &b) {
  p[i] = b;
}
template <>
__device__ inline void store_box(Box<float> *p, int64_t i, const Box<float> &b) {
  reinterpret_cast<float4 *>(p)[i] = make_float4(b.x1, b.y1, b.x2, b.y2);
}

inline size_t coord_size(int coord) {
  return coord == PRT_COORD_F32 || coord == PRT_COORD_I32 ? 4 : 8;
}

// Dispatch a templated functor on the coordinate type.
template <typename F>
int dispatch_coord(int coord, F &&f) {
  switch (coord) {
    case PRT_COORD_I64: return f(int64_t{});
    case PRT_COORD_F32: return f(float{});
    case PRT_COORD_F64: return f(double{});
    case PRT_COORD_I32: return f(int32_t{});
    default:
      set_error("unknown coordinate type %d", coord);
      return PRT_ERR_INVALID;
  }
}

inline int grid_for(int64_t work, int block, int per_sm = 8) {
  int64_t g = (work + block - 1) / block;
  int64_t cap = (int64_t)kSMs * per_sm;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

// ---- radix sort --------------------------------------------------------------
// Stable LSD sort of (key, value) pairs; keys are KeyT (uint32_t or
// uint64_t), values uint32_t.  Bits [0, key_bits) are sorted.  The sorted data
// ends in either the input or the alternate buffers; *d_sel (device) receives
// 0 when it is in (keys0, vals0) and 1 for (keys1, vals1).  d_hist, when
// given, holds the 8-bit digit histograms of every pass (passes x 256, as a
// key generator can count them while it writes the keys); otherwise the sort
// reads the keys once to count them.
template <typename KeyT>
int radix_sort_pairs(KeyT *keys0, uint32_t *vals0, KeyT *keys1, uint32_t *vals1, int64_t n,
                     int key_bits, int *d_sel, unsigned *d_err, cudaStream_t s,
                     const uint32_t *d_hist = nullptr);

// The same sort applied to every run of run_len consecutive pairs
// independently (all bits of the keys; the last run may be shorter): each run
// ends sorted in place of itself.  run_len must be a multiple of the sort's
// 4096-key tile.  d_hist, when given, holds every run's digit histograms
// (runs x passes x 256).
template <typename KeyT>
int radix_sort_runs(KeyT *keys0, uint32_t *vals0, KeyT *keys1, uint32_t *vals1, int64_t n, int64_t run_len,
                    int *d_sel, unsigned *d_err, cudaStream_t s, const uint32_t *d_hist = nullptr);
constexpr int64_t kSortRunTile = 4096;

// Exclusive prefix sum of n values into d_out (int64); *d_total (device,
// optional) receives the sum.
template <typename InT>
int exclusive_scan(const InT *d_in, int64_t n, int64_t *d_out, int64_t *d_total, cudaStream_t s);

// ---- tree ----------------------------------------------------------------------
struct TreeLevels {
  int levels;                        // L: level 0 = records
  int64_t count[PRT_MAX_LEVELS];     // entries per level
  int64_t padded[PRT_MAX_LEVELS];    // rounded up to a multiple of fanout
  int64_t offset[PRT_MAX_LEVELS];    // first entry of each level in the box array
  int64_t total;                     // entries over all levels, padded
};

TreeLevels level_layout(int64_t n, int fanout);

}  // namespace prt

struct prt_tree;

namespace prt {

// Capture-safe pieces of the pipeline (no host synchronisation inside):
// tree_alloc allocates a tree's storage for n boxes; bu_enqueue enqueues its
// bottom-up build; join_enqueue enqueues a breadth-first join with caller-owned
// frontier buffers and counters (counters: PRT_MAX_LEVELS + 2 uint64, zeroed by
// the caller; [l] = frontier items entering node level l-1, [PRT_MAX_LEVELS] =
// pairs found, all counted even past the capacities).
int tree_alloc(const void *d_boxes, int coord, int64_t n, int fanout, int kind, int key_mode, cudaStream_t s,
               prt_tree **out);
int bu_enqueue(prt_tree *t, const void *d_boxes, const int32_t *d_ids, unsigned *d_err, cudaStream_t s);
int join_enqueue(const prt_tree *t, const void *d_queries, int64_t nq, uint2 *d_pairs, int64_t cap, uint2 *fr0,
                 uint2 *fr1, int64_t fcap, unsigned long long *d_counters, cudaStream_t s);

}  // namespace prt

struct prt_tree {
  int kind;
  int coord;
  int fanout;
  int key_mode;
  int64_t n;
  prt::TreeLevels lv;
  void *d_mbr;          // Box<T>[lv.total], level after level
  int32_t *d_leaf_id;   // record id per leaf entry
  int device;
};
