// Pair sources shared by the overlay and the area kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "prt_internal.cuh"

namespace prt {

struct LayerDev {
  const int64_t *poly_ring;
  const int64_t *ring_vert;
  const int32_t *ring_hole;
  const double *xy;
  int64_t n_poly;
};

// Candidate pairs: either (nodeid, queryid) records resolved through the leaf
// order (base = leaf_to_poly[nodeid - offset], overlay = queryid), or two
// direct polygon-id arrays pa / pb.
struct PairSrc {
  const uint2 *pairs;
  const int32_t *pa;
  const int32_t *pb;
  int32_t offset;
  const int32_t *leaf_to_poly;
  LayerDev base, over;
  int op;
};

inline LayerDev layer_dev(const prt_layer *l) {
  LayerDev d;
  d.poly_ring = l->poly_ring;
  d.ring_vert = l->ring_vert;
  d.ring_hole = l->ring_hole;
  d.xy = l->xy;
  d.n_poly = l->n_poly;
  return d;
}

// Clips all pairs.  d_area != nullptr: area-only mode (per-pair area, no
// results object); otherwise *out receives the results.
int overlay_impl(const PairSrc &S, int64_t n, int sched, double *d_area, cudaStream_t s, prt_results **out);

}  // namespace prt

namespace prt {

// Resident warps per SM of the persistent batched clip launch (its launch
// bounds); a schedule's warps_per_sm is capped at it.
constexpr int kLptWarpsPerSM = 12;
// Resident warps per SM of the same launch when no pair is clipped by a warp.
constexpr int kLptThreadWarpsPerSM = 24;

// Bins of the batched schedule, size-descending: bin b holds sorted positions
// [begin[b], end[b]).  Warps [warp0[g], warp0[g+1]) start on bin g with
// region[g] bytes of arena each (one pair of any later bin in warp mode, or
// 32 pairs in thread mode) and move to the later bins as bins drain; the
// planner puts every warp in group 0, so all warps take the largest pairs
// first.
struct BinPlan {
  int64_t begin[PRT_MAX_BINS], end[PRT_MAX_BINS];
  int64_t warp0[PRT_MAX_BINS + 1];
  int64_t region[PRT_MAX_BINS];
  int64_t arena_off[PRT_MAX_BINS];
  int32_t warp_mode[PRT_MAX_BINS];
  int64_t n_pairs;  // pair indices in the order array are below this (others are skipped)
  int nbins;
  int wcap;         // AET slots per warp (warp mode)
  int thread_only;  // no bin with pairs in warp mode: the thread-only kernel
};

// The schedule of the calling process (prt_schedule_set).
prt_schedule current_schedule();
// PRT_OK, or PRT_ERR_INVALID with the reason as the last error.
int schedule_valid(const prt_schedule &s);
// Fills plan for bins with at most counts[b] pairs of at most maxnv[b]
// vertices, arena limited to `budget` bytes; returns the arena bytes and the
// dynamic shared memory per block in *smem.  With thread_kernel, a plan with
// no warp-mode pairs is marked for the thread-only kernel (and sized for its
// resident warps).
size_t plan_bins(const prt_schedule &sc, const int64_t *counts, const int64_t *maxnv, size_t budget, BinPlan &plan,
                 size_t *smem, int scale = 1, bool thread_kernel = false);

// Allows the persistent clip kernel `smem` bytes of dynamic shared memory.
int prepare_lpt_launch(size_t smem);

// Buffers of the capture-safe (CUDA graph) overlay: everything preallocated
// for at most cap_pairs pairs, sizes read from device memory at run time.
struct GraphOverlay {
  int64_t cap_pairs = 0;
  uint32_t *k0 = nullptr, *k1 = nullptr, *v0 = nullptr, *v1 = nullptr, *order = nullptr;
  int *sel = nullptr;
  unsigned *err = nullptr;
  int64_t *ranges = nullptr;              // [2 * bins] begin/end per bin (device)
  int64_t *thresholds = nullptr;          // [bins] vertex-count upper bounds (device)
  unsigned long long *tickets = nullptr;  // [bins]
  unsigned long long *totals = nullptr;   // [4] contours, vertices, non-empty, failed pairs
  unsigned char *arena = nullptr;
  size_t arena_bytes = 0;
  BinPlan plan;
  size_t smem = 0;
  // results
  int32_t *status = nullptr;
  int64_t *pair_cstart = nullptr;
  int32_t *pair_ncont = nullptr;
  int64_t *cont_vstart = nullptr;
  int32_t *cont_nverts = nullptr;
  int32_t *cont_hole = nullptr;
  double *xy = nullptr;
  unsigned long long *pool = nullptr;     // [2] contours, vertices reserved
  int64_t cap_c = 0, cap_v = 0;
};

// Enqueues the batched overlay of the first *d_npairs pairs (at most
// G.cap_pairs) with no host synchronisation: zero the counters, size keys,
// size sort, bin ranges, one longest-first persistent launch, result totals.
int overlay_graph_enqueue(const PairSrc &S, const unsigned long long *d_npairs, GraphOverlay &G, cudaStream_t s);

}  // namespace prt

// A result set (the reference's per-pair gpc_polygon array): pair i owns
// contours [pair_cstart[i], + pair_ncont[i]) of the pools, contour c owns
// vertices [cont_vstart[c], + cont_nverts[c]) of xy.  Pools are filled by
// atomic reservations, so they are not in pair order.
struct prt_results {
  int64_t n_pairs, n_cont, n_vert, nonempty, retried;
  int64_t *pair_cstart;
  int32_t *pair_ncont;
  int32_t *status;
  int64_t *cont_vstart;
  int32_t *cont_nverts;
  int32_t *cont_hole;
  double *xy;
  unsigned long long *pool;
};
