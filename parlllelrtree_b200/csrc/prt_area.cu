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
// One warp per pair: lanes take edges of A (then of B); each lane finds its
// edge's crossings with the other polygon, in increasing t, and classifies
// each interval by an even-odd test of its midpoint.  Contributions are scaled by the upstream gradient and
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

// ---- shared-memory adjoint (pairs up to kBwdMaxV vertices per polygon) ----
// The same boundary pieces with both polygons staged in shared memory.  Each
// lane takes one edge (the edges of A and of B in one pass) and runs over the
// edges of the other polygon in the same order as its neighbours, so the
// loads are broadcasts and the lanes do not diverge.  A conservative float
// bounding box (rounded outwards) rejects most edges before any double
// arithmetic; the exact crossing expression runs only for the rest.  The
// crossing parameters are sorted and deduplicated, which gives the intervals
// of next_crossing's repeated minimum search, and a second pass tests every
// interval midpoint (inside_evenodd's expression, behind a float y-range
// check).  Pairs with larger polygons, and edges with more than kBwdMaxT
// crossings, take the global-memory path (pieces / next_crossing).
constexpr int kBwdMaxV = 128;
constexpr int kBwdMaxT = 16;
constexpr int kBwdWarps = 4;

struct BwdPoly {  // one polygon in shared memory
  float4 bb[kBwdMaxV];     // edge k's box (x_lo, y_lo, x_hi, y_hi), rounded outwards
  double x[kBwdMaxV], y[kBwdMaxV];
  int8_t sgn[kBwdMaxV];    // orientation sign of edge k (0: ring of < 2 vertices)
  uint8_t nxt[kBwdMaxV];   // end vertex of edge k
};

// Loads a polygon into shared memory with its ring links, orientation signs
// and edge boxes; returns its vertex count (all lanes).  Nothing is loaded
// when the polygon has more than kBwdMaxV vertices.
__device__ inline int bwd_load(const LayerDev &L, int64_t poly, BwdPoly &Q) {
  const int lane = threadIdx.x & 31;
  const int64_t r0 = L.poly_ring[poly], r1 = L.poly_ring[poly + 1];
  const int64_t vbase = L.ring_vert[r0];
  const int nv = (int)(L.ring_vert[r1] - vbase);
  if (nv > kBwdMaxV) return nv;
  for (int64_t r = r0; r < r1; r++) {
    const int v0 = (int)(L.ring_vert[r] - vbase), n = (int)(L.ring_vert[r + 1] - L.ring_vert[r]);
    double sa = 0.0;
    for (int i = lane; i < n; i += 32) {
      const int j = (i + 1 == n) ? 0 : i + 1;
      const double xi = L.xy[2 * (vbase + v0 + i)], yi = L.xy[2 * (vbase + v0 + i) + 1];
      const double xj = L.xy[2 * (vbase + v0 + j)], yj = L.xy[2 * (vbase + v0 + j) + 1];
      sa += xi * yj - xj * yi;
      Q.x[v0 + i] = xi;
      Q.y[v0 + i] = yi;
      Q.nxt[v0 + i] = (uint8_t)(v0 + j);
      Q.bb[v0 + i] = make_float4(__double2float_rd(fmin(xi, xj)), __double2float_rd(fmin(yi, yj)),
                                 __double2float_ru(fmax(xi, xj)), __double2float_ru(fmax(yi, yj)));
    }
    for (int o = 16; o; o >>= 1) sa += __shfl_xor_sync(0xffffffffu, sa, o);
    const bool hole = L.ring_hole && L.ring_hole[r];
    const int8_t sg = n < 2 ? 0 : (int8_t)((sa >= 0.0 ? 1 : -1) * (hole ? -1 : 1));
    for (int i = lane; i < n; i += 32) Q.sgn[v0 + i] = sg;
  }
  __syncwarp();
  return nv;
}

// One edge whose crossings overflow the per-lane list: the global-memory path.
__device__ __noinline__ void bwd_edge_global(const Poly &Qg, double px, double py, double rx, double ry, double *it,
                                             double *i1) {
  double t0 = 0.0;
  for (;;) {
    const double t1 = next_crossing(Qg, px, py, rx, ry, t0);
    const double tm = 0.5 * (t0 + t1);
    if (t1 > t0 && inside_evenodd(Qg, px + tm * rx, py + tm * ry)) {
      const double a = 0.5 * (t1 * t1 - t0 * t0);
      *it += a;
      *i1 += (t1 - t0) - a;
    }
    if (t1 >= 1.0) break;
    t0 = t1;
  }
}

// pieces() for both polygons of a staged pair: lane edge e < na is edge e of
// A (against B), e >= na edge e - na of B (against A).
__device__ inline void bwd_pair(const BwdPoly *M, int na, int nb, double w, double *ga, double *gb, int64_t va,
                                int64_t vb, const Poly &Ag, const Poly &Bg) {
  const int lane = threadIdx.x & 31;
  const int nk = na > nb ? na : nb;
  for (int e0 = 0; e0 < na + nb; e0 += 32) {
    const int e = e0 + lane;
    const int side = e < na ? 0 : 1;
    const int i = side ? e - na : e;
    const BwdPoly &P = M[side], &Q = M[1 - side];
    const int nq = side ? na : nb;
    const bool valid = e < na + nb && P.sgn[i] != 0;
    double px = 0.0, py = 0.0, qx = 0.0, qy = 0.0;
    if (valid) {
      const int j = P.nxt[i];
      px = P.x[i];
      py = P.y[i];
      qx = P.x[j];
      qy = P.y[j];
    }
    const double rx = qx - px, ry = qy - py;
    const float fx0 = __double2float_rd(fmin(px, qx)), fy0 = __double2float_rd(fmin(py, qy));
    const float fx1 = __double2float_ru(fmax(px, qx)), fy1 = __double2float_ru(fmax(py, qy));
    // one uniform pass: candidate masks (bit k: edge k of Q) for crossings
    // (boxes overlap) and for the midpoint tests (y ranges overlap)
    unsigned mc[kBwdMaxV / 32], my[kBwdMaxV / 32];
#pragma unroll
    for (int c = 0; c < kBwdMaxV / 32; c++) {
      unsigned wc = 0, wy = 0;
      if (c * 32 < nk) {
        for (int kk = 0; kk < 32; kk++) {
          const int k = c * 32 + kk;
          if (k >= nk) break;
          const float4 b = Q.bb[k];
          const bool yo = k < nq && !(b.w < fy0 || b.y > fy1);
          const bool xo = !(b.z < fx0 || b.x > fx1);
          wy |= (unsigned)yo << kk;
          wc |= (unsigned)(yo && xo) << kk;
        }
      }
      mc[c] = valid ? wc : 0u;
      my[c] = valid ? wy : 0u;
    }
    double ts[kBwdMaxT];
    int nt = 0;
    bool over = false;
#pragma unroll
    for (int c = 0; c < kBwdMaxV / 32; c++) {
      unsigned bits = mc[c];
      while (bits) {
        const int k = c * 32 + __ffs(bits) - 1;
        bits &= bits - 1;
        const int l = Q.nxt[k];
        const double ax = Q.x[k], ay = Q.y[k], bx = Q.x[l], by = Q.y[l];
        const double sx = bx - ax, sy = by - ay;
        const double den = rx * sy - ry * sx;
        if (den == 0.0) continue;
        const double apx = ax - px, apy = ay - py;
        const double t = (apx * sy - apy * sx) / den;
        const double u = (apx * ry - apy * rx) / den;
        if (t > 0.0 && t < 1.0 && u >= 0.0 && u <= 1.0) {
          if (nt < kBwdMaxT) ts[nt++] = t;
          else over = true;
        }
      }
    }
    for (int a = 1; a < nt; a++) {  // sort, then drop duplicates
      const double v = ts[a];
      int b = a - 1;
      while (b >= 0 && ts[b] > v) {
        ts[b + 1] = ts[b];
        b--;
      }
      ts[b + 1] = v;
    }
    int m = 0;
    for (int a = 0; a < nt; a++)
      if (m == 0 || ts[a] > ts[m - 1]) ts[m++] = ts[a];
    // interval a = [b_a, b_{a+1}] with b_0 = 0, b_{m+1} = 1; bit a of `in`:
    // its midpoint is inside the other polygon.  Every midpoint lies in the
    // edge's y range, so only edges of Q overlapping that range can toggle.
    const int nint = valid && !over ? m + 1 : 0;
    unsigned in = 0;
#pragma unroll
    for (int c = 0; c < kBwdMaxV / 32; c++) {
      unsigned bits = nint ? my[c] : 0u;
      while (bits) {
        const int k = c * 32 + __ffs(bits) - 1;
        bits &= bits - 1;
        const int l = Q.nxt[k];
        const double ax = Q.x[k], ay = Q.y[k], bx = Q.x[l], by = Q.y[l];
        for (int a = 0; a < nint; a++) {
          const double t0 = a == 0 ? 0.0 : ts[a - 1], t1 = a < m ? ts[a] : 1.0;
          const double tm = 0.5 * (t0 + t1);
          const double mx = px + tm * rx, my2 = py + tm * ry;
          if ((ay > my2) != (by > my2)) {
            const double xi = ax + (my2 - ay) * (bx - ax) / (by - ay);
            if (mx < xi) in ^= 1u << a;
          }
        }
      }
    }
    double it = 0.0, i1 = 0.0;
    if (over) {
      bwd_edge_global(side ? Ag : Bg, px, py, rx, ry, &it, &i1);
    } else {
      for (int a = 0; a < nint; a++) {
        const double t0 = a == 0 ? 0.0 : ts[a - 1], t1 = a < m ? ts[a] : 1.0;
        if ((in >> a) & 1u) {
          const double aa = 0.5 * (t1 * t1 - t0 * t0);
          it += aa;
          i1 += (t1 - t0) - aa;
        }
      }
    }
    if (valid && (it != 0.0 || i1 != 0.0)) {
      const double s = P.sgn[i];
      const int j = P.nxt[i];
      const double nx = w * s * ry, ny = -w * s * rx;
      double *g = side ? gb : ga;
      const int64_t vbase = side ? vb : va;
      atomicAdd(&g[2 * (vbase + j)], nx * it);
      atomicAdd(&g[2 * (vbase + j) + 1], ny * it);
      atomicAdd(&g[2 * (vbase + i)], nx * i1);
      atomicAdd(&g[2 * (vbase + i) + 1], ny * i1);
    }
  }
}

// Pairs with a polygon above kBwdMaxV vertices: the global-memory path.
__device__ __noinline__ void bwd_pair_global(const Poly &A, const Poly &B, double w, double *ga, double *gb) {
  const int lane = threadIdx.x & 31;
  pieces(A, B, w, ga, lane);
  pieces(B, A, w, gb, lane);
}

__global__ void __launch_bounds__(32 * kBwdWarps) area_bwd_kernel(
    const int32_t *__restrict__ pa, const int32_t *__restrict__ pb, int64_t n, LayerDev base, LayerDev over,
    const double *__restrict__ upstream, double *grad_base, double *grad_over) {
  __shared__ BwdPoly sm[kBwdWarps][2];
  BwdPoly *M = sm[threadIdx.x >> 5];
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i = warp; i < n; i += nw) {
    const int64_t a = pa[i], b = pb[i];
    if (a < 0 || a >= base.n_poly || b < 0 || b >= over.n_poly) continue;
    const double w = upstream ? upstream[i] : 1.0;
    Poly A{base.ring_vert, base.ring_hole, base.xy, base.poly_ring[a], base.poly_ring[a + 1]};
    Poly B{over.ring_vert, over.ring_hole, over.xy, over.poly_ring[b], over.poly_ring[b + 1]};
    const int na = bwd_load(base, a, M[0]);
    const int nb = bwd_load(over, b, M[1]);
    if (na <= kBwdMaxV && nb <= kBwdMaxV) {
      bwd_pair(M, na, nb, w, grad_base, grad_over, base.ring_vert[A.r0], over.ring_vert[B.r0], A, B);
    } else {
      bwd_pair_global(A, B, w, grad_base, grad_over);
    }
    __syncwarp();
  }
}

}  // namespace
}  // namespace prt

using namespace prt;

extern "C" {

int prt_area_fwd(const int32_t *d_pair_a, const int32_t *d_pair_b, int64_t n_pairs, const prt_layer *base,
                 const prt_layer *overlay, double *d_area, void *stream) {
  PRT_CHECK(base && overlay && (n_pairs == 0 || (d_area && d_pair_a && d_pair_b)), PRT_ERR_INVALID,
            "NULL argument");
  if (n_pairs == 0) return PRT_OK;
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
  PRT_CHECK(base && overlay && (n_pairs == 0 || (d_grad_base && d_grad_overlay && d_pair_a && d_pair_b)),
            PRT_ERR_INVALID, "NULL argument");
  if (n_pairs == 0) return PRT_OK;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  {
    PRT_PROF("area_bwd", s);
    // exactly the resident blocks (each warp loops over pairs): no tail wave
    static int per_sm = 0;
    if (per_sm == 0) {
      int b = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, area_bwd_kernel, 32 * kBwdWarps, 0) != cudaSuccess || b < 1)
        b = 4;
      per_sm = b;
    }
    const int blocks = grid_for(n_pairs * 32, 32 * kBwdWarps, per_sm);
    area_bwd_kernel<<<blocks, 32 * kBwdWarps, 0, s>>>(d_pair_a, d_pair_b, n_pairs, layer_dev(base),
                                                      layer_dev(overlay), d_upstream, d_grad_base, d_grad_overlay);
  }
  PRT_CUDA(cudaGetLastError());
  return PRT_OK;
}

}  // extern "C"
