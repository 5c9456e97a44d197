// Intersection area and its adjoint.
//
// Forward: area(A_i ∩ B_i) from the GPC clip of each pair (prt_overlay.cu,
// area-only mode: the clip result is reduced to its shoelace area in place and
// never written out).
//
// Backward: d area / d vertex by the boundary integral, recomputed from the
// input polygons rather than stored by the forward pass.  The boundary of
// A∩B is made of the pieces of A's edges inside B and of B's edges inside A
// (even-odd fill, GPC's parity rule).  For an edge p -> q traversed with the
// material on its left (ring orientation sign s: +1 for CCW outer rings and CW
// holes), outward normal N = s (q.y - p.y, p.x - q.x), and inside parameter
// intervals [t0, t1]:
//     d area / d q += N sum (t1^2 - t0^2) / 2
//     d area / d p += N sum ((t1 - t0) - (t1^2 - t0^2) / 2)
// One warp per pair: lanes take edges of A (then of B); each lane walks its
// edge's crossings with the other polygon in increasing t (a min-search per
// step, so no per-lane list) and classifies each interval by an even-odd test
// of its midpoint.  Contributions are scaled by the upstream gradient and
// accumulated with atomicAdd, since a polygon may appear in many pairs.
#include <cuda_runtime.h>

#include "prt_internal.cuh"
#include "prt_overlay.cuh"

namespace prt {
namespace {

struct Poly {
  const int64_t *ring_vert;
  const int32_t *ring_hole;
  const double *xy;
  int64_t r0, r1;
};

__device__ inline bool inside_evenodd(const Poly &P, double px, double py) {
  bool c = false;
  for (int64_t r = P.r0; r < P.r1; r++) {
    const int64_t v0 = P.ring_vert[r], v1 = P.ring_vert[r + 1];
    const int64_t n = v1 - v0;
    for (int64_t i = 0; i < n; i++) {
      const int64_t j = (i + 1 == n) ? 0 : i + 1;
      const double ax = __ldg(&P.xy[2 * (v0 + i)]), ay = __ldg(&P.xy[2 * (v0 + i) + 1]);
      const double bx = __ldg(&P.xy[2 * (v0 + j)]), by = __ldg(&P.xy[2 * (v0 + j) + 1]);
      if ((ay > py) != (by > py)) {
        const double xi = ax + (py - ay) * (bx - ax) / (by - ay);
        if (px < xi) c = !c;
      }
    }
  }
  return c;
}

// smallest crossing parameter t of p + t r with the edges of P, t in (t_lo, 1)
__device__ inline double next_crossing(const Poly &P, double px, double py, double rx, double ry, double t_lo) {
  double best = 1.0;
  for (int64_t r = P.r0; r < P.r1; r++) {
    const int64_t v0 = P.ring_vert[r], v1 = P.ring_vert[r + 1];
    const int64_t n = v1 - v0;
    for (int64_t k = 0; k < n; k++) {
      const int64_t l = (k + 1 == n) ? 0 : k + 1;
      const double ax = __ldg(&P.xy[2 * (v0 + k)]), ay = __ldg(&P.xy[2 * (v0 + k) + 1]);
      const double sx = __ldg(&P.xy[2 * (v0 + l)]) - ax, sy = __ldg(&P.xy[2 * (v0 + l) + 1]) - ay;
      const double den = rx * sy - ry * sx;
      if (den == 0.0) continue;
      const double apx = ax - px, apy = ay - py;
      const double t = (apx * sy - apy * sx) / den;
      const double u = (apx * ry - apy * rx) / den;
      if (t > 0.0 && t < 1.0 && u >= 0.0 && u <= 1.0 && t > t_lo && t < best) best = t;
    }
  }
  return best;
}

// Pieces of A's boundary inside B, for the edges handled by this lane.
__device__ void pieces(const Poly &A, const Poly &B, double w, double *grad, int lane) {
  for (int64_t r = A.r0; r < A.r1; r++) {
    const int64_t v0 = A.ring_vert[r], v1 = A.ring_vert[r + 1];
    const int64_t n = v1 - v0;
    if (n < 2) continue;
    // ring orientation (warp-cooperative shoelace)
    double sa = 0.0;
    for (int64_t i = lane; i < n; i += 32) {
      const int64_t j = (i + 1 == n) ? 0 : i + 1;
      sa += A.xy[2 * (v0 + i)] * A.xy[2 * (v0 + j) + 1] - A.xy[2 * (v0 + j)] * A.xy[2 * (v0 + i) + 1];
    }
    for (int o = 16; o; o >>= 1) sa += __shfl_xor_sync(0xffffffffu, sa, o);
    // material on the left: CCW outer rings and CW hole rings (s = +1)
    const bool hole = A.ring_hole && A.ring_hole[r];
    const double s = (sa >= 0.0 ? 1.0 : -1.0) * (hole ? -1.0 : 1.0);
    for (int64_t i = lane; i < n; i += 32) {
      const int64_t j = (i + 1 == n) ? 0 : i + 1;
      const double px = A.xy[2 * (v0 + i)], py = A.xy[2 * (v0 + i) + 1];
      const double qx = A.xy[2 * (v0 + j)], qy = A.xy[2 * (v0 + j) + 1];
      const double rx = qx - px, ry = qy - py;
      double it = 0.0, i1 = 0.0;
      double t0 = 0.0;
      for (;;) {
        const double t1 = next_crossing(B, px, py, rx, ry, t0);
        const double tm = 0.5 * (t0 + t1);
        if (t1 > t0 && inside_evenodd(B, px + tm * rx, py + tm * ry)) {
          const double a = 0.5 * (t1 * t1 - t0 * t0);
          it += a;
          i1 += (t1 - t0) - a;
        }
        if (t1 >= 1.0) break;
        t0 = t1;
      }
      if (it != 0.0 || i1 != 0.0) {
        const double nx = w * s * ry, ny = -w * s * rx;
        atomicAdd(&grad[2 * (v0 + j)], nx * it);
        atomicAdd(&grad[2 * (v0 + j) + 1], ny * it);
        atomicAdd(&grad[2 * (v0 + i)], nx * i1);
        atomicAdd(&grad[2 * (v0 + i) + 1], ny * i1);
      }
    }
  }
}

__global__ void __launch_bounds__(256) area_bwd_kernel(const int32_t *__restrict__ pa, const int32_t *__restrict__ pb,
                                                       int64_t n, LayerDev base, LayerDev over,
                                                       const double *__restrict__ upstream, double *grad_base,
                                                       double *grad_over) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i = warp; i < n; i += nw) {
    const int64_t a = pa[i], b = pb[i];
    if (a < 0 || a >= base.n_poly || b < 0 || b >= over.n_poly) continue;
    const double w = upstream ? upstream[i] : 1.0;
    Poly A{base.ring_vert, base.ring_hole, base.xy, base.poly_ring[a], base.poly_ring[a + 1]};
    Poly B{over.ring_vert, over.ring_hole, over.xy, over.poly_ring[b], over.poly_ring[b + 1]};
    pieces(A, B, w, grad_base, lane);
    pieces(B, A, w, grad_over, lane);
  }
}

}  // namespace
}  // namespace prt

using namespace prt;

extern "C" {

int prt_area_fwd(const int32_t *d_pair_a, const int32_t *d_pair_b, int64_t n_pairs, const prt_layer *base,
                 const prt_layer *overlay, double *d_area, void *stream) {
  PRT_CHECK(base && overlay && d_area && (n_pairs == 0 || (d_pair_a && d_pair_b)), PRT_ERR_INVALID,
            "NULL argument");
  PairSrc S;
  memset(&S, 0, sizeof S);
  S.pa = d_pair_a;
  S.pb = d_pair_b;
  S.base = layer_dev(base);
  S.over = layer_dev(overlay);
  S.op = PRT_GPC_INT;
  return overlay_impl(S, n_pairs, PRT_SCHED_BATCHED, d_area, reinterpret_cast<cudaStream_t>(stream), nullptr);
}

int prt_area_bwd(const int32_t *d_pair_a, const int32_t *d_pair_b, int64_t n_pairs, const prt_layer *base,
                 const prt_layer *overlay, const double *d_upstream, double *d_grad_base, double *d_grad_overlay,
                 void *stream) {
  PRT_CHECK(base && overlay && d_grad_base && d_grad_overlay && (n_pairs == 0 || (d_pair_a && d_pair_b)),
            PRT_ERR_INVALID, "NULL argument");
  if (n_pairs == 0) return PRT_OK;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int blocks = grid_for(n_pairs * 32, 256, 8);
  {
    PRT_PROF("area_bwd", s);
    area_bwd_kernel<<<blocks, 256, 0, s>>>(d_pair_a, d_pair_b, n_pairs, layer_dev(base), layer_dev(overlay), d_upstream,
                                         d_grad_base, d_grad_overlay);
  }
  PRT_CUDA(cudaGetLastError());
  return PRT_OK;
}

}  // extern "C"
