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
