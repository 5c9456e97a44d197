// Intersection area and its adjoint.
//
// Forward: area(A_i ∩ B_i) = the shoelace sum over the boundary of A∩B, i.e.
// over the pieces of A's edges inside B and of B's edges inside A, found by
// the same slab / parity pass as the adjoint below (area mode).  Pairs whose
// crossings are not all clean, whose polygons do not fit the shared-memory
// staging, or whose area the crossing-rounding bound does not pin to 1e-10 are
// clipped by GPC instead (prt_overlay.cu, area-only mode: the clip result is
// reduced to its shoelace area in place and never written out).  The fast
// path assumes what GPC's output implies for map layers: the rings of a
// polygon do not cross each other or themselves, and hole rings are flagged.
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
// the intervals between them (by crossing parity along the ring, or by the
// even-odd test of each midpoint when a crossing is not clean; see
// pair_boundary).  Contributions are scaled by the upstream gradient and
// accumulated with atomicAdd, since a polygon may appear in many pairs.  Both
// directions run in two stages: polygons of up to 64 vertices staged in
// shared memory first, the pairs that do not fit listed for a 128-vertex
// staging, larger ones on a global-memory path (backward) or the GPC clip
// (forward).
#include <cuda_runtime.h>

#include <atomic>

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
// The same boundary pieces with both polygons staged in shared memory, and
// the candidate edges of the other polygon found through y slabs instead of
// a scan over all of its edges.  The pair's common y range (float, rounded
// outwards) is cut into kSlabs slabs; slab s of polygon Q holds a bitmask of
// Q's edges whose float box reaches slab s (built by a warp bit transpose of
// each edge's slab range).  The slab index is a monotone function of the
// float y, so two y ranges that overlap always share a slab and the masks
// never drop a candidate:
//   crossings of an edge: the OR of the slab masks over its y range, then the
//     float box test and the exact FP64 crossing expression of
//     next_crossing, so the crossing set equals the exhaustive scan's;
//   midpoint of an interval: only edges whose y range holds the midpoint's y
//     can straddle it, and they all sit in the midpoint's slab; the even-odd
//     test is inside_evenodd's expression.
// Each lane takes one edge (the edges of A and of B in one pass); the
// crossing parameters are sorted and deduplicated, which gives the intervals
// of next_crossing's repeated minimum search.  The two gradient contributions
// a vertex receives (as the end of one edge, as the start of the next) are
// summed across neighbouring lanes before the atomics.  Edges with more than
// kBwdMaxT crossings take the global-memory path (next_crossing).
constexpr int kBwdMaxV = 128;
constexpr int kBwdSmallV = 64;
constexpr int kBwdMaxT = 16;
constexpr int kBwdWarps = 4;
constexpr int kSlabs = 32;
constexpr unsigned kFullMask = 0xffffffffu;

template <int V>
struct BwdPoly {  // one polygon in shared memory (up to V vertices)
  float4 bb[V];                    // edge k's box (x_lo, y_lo, x_hi, y_hi), rounded outwards
  double x[V], y[V];
  uint32_t slab[V / 32][kSlabs];   // y slabs: word c of slab s, bit k = edge 32 c + k reaches slab s
  uint32_t xslab[V / 32][kSlabs];  // the same for x slabs
  int16_t ringv[33];                      // first vertex of ring r; ringv[rings] = the vertex count
  int8_t sgn[V];                   // orientation sign of edge k (0: ring of < 2 vertices)
  uint8_t nxt[V];                  // end vertex of edge k
  uint8_t rst[V];                  // first vertex of edge k's ring
};

// coordinate -> slab: monotone non-decreasing (round-to-nearest float steps
// and a clamp), which is what makes the slab masks conservative.
struct SlabGrid {
  float v0, scale;
  __device__ int operator()(float v) const {
    const float f = __fmul_rn(__fsub_rn(v, v0), scale);
    return (int)fminf(fmaxf(f, 0.0f), (float)(kSlabs - 1));
  }
};

__device__ inline SlabGrid slab_grid(float lo, float hi) {
  const float span = __fsub_rn(hi, lo);
  return SlabGrid{lo, span > 1e-30f ? __fdiv_rn((float)kSlabs, span) : 0.0f};
}

// Stages both polygons of a pair (A from rings [ra0, ra1) of LA, B from
// [rb0, rb1) of LB) with their ring links, orientation signs and edge boxes;
// the loads of the two are issued together.  nv[p] is polygon p's vertex
// count, vb[p] its first vertex, ext[p] the float extent of its edge boxes.
// Returns false (nothing staged) when a polygon has more than V
// vertices or more than 31 rings.
template <int V>
__device__ inline bool bwd_load_pair(const LayerDev &LA, int64_t ra0, int64_t ra1, const LayerDev &LB, int64_t rb0,
                                     int64_t rb1, BwdPoly<V> *M, int *nv, int64_t *vb, float4 *ext) {
  const int lane = threadIdx.x & 31;
  const int nr[2] = {(int)(ra1 - ra0), (int)(rb1 - rb0)};
  if (nr[0] > 31 || nr[1] > 31) return false;
  int64_t rv[2] = {0, 0};
  int hl[2] = {0, 0};
  if (lane <= nr[0]) rv[0] = LA.ring_vert[ra0 + lane];
  if (lane <= nr[1]) rv[1] = LB.ring_vert[rb0 + lane];
  if (lane < nr[0] && LA.ring_hole) hl[0] = LA.ring_hole[ra0 + lane];
  if (lane < nr[1] && LB.ring_hole) hl[1] = LB.ring_hole[rb0 + lane];
#pragma unroll
  for (int p = 0; p < 2; p++) {
    vb[p] = __shfl_sync(kFullMask, rv[p], 0);
    nv[p] = (int)(__shfl_sync(kFullMask, rv[p], nr[p]) - vb[p]);
  }
  if (nv[0] > V || nv[1] > V) return false;
#pragma unroll
  for (int p = 0; p < 2; p++)
    if (lane <= nr[p]) M[p].ringv[lane] = (int16_t)(rv[p] - vb[p]);
  __syncwarp();
  const float inf = __int_as_float(0x7f800000);
  float4 e[2] = {make_float4(inf, inf, -inf, -inf), make_float4(inf, inf, -inf, -inf)};
  double term[2][V / 32];  // shoelace terms of this lane's vertices
  int rix[2][V / 32];      // and their rings
#pragma unroll
  for (int t = 0; t < V / 32; t++) {
#pragma unroll
    for (int p = 0; p < 2; p++) {
      const LayerDev &L = p ? LB : LA;
      BwdPoly<V> &Q = M[p];
      const int i = 32 * t + lane;
      term[p][t] = 0.0;
      rix[p][t] = -1;
      if (i < nv[p]) {
        int r = 0;
        while (Q.ringv[r + 1] <= i) r++;
        const int v0 = Q.ringv[r], j = i + 1 == Q.ringv[r + 1] ? v0 : i + 1;
        const double xi = L.xy[2 * (vb[p] + i)], yi = L.xy[2 * (vb[p] + i) + 1];
        const double xj = L.xy[2 * (vb[p] + j)], yj = L.xy[2 * (vb[p] + j) + 1];
        term[p][t] = xi * yj - xj * yi;
        rix[p][t] = r;
        Q.x[i] = xi;
        Q.y[i] = yi;
        Q.nxt[i] = (uint8_t)j;
        Q.rst[i] = (uint8_t)v0;
        const float4 b = make_float4(__double2float_rd(fmin(xi, xj)), __double2float_rd(fmin(yi, yj)),
                                     __double2float_ru(fmax(xi, xj)), __double2float_ru(fmax(yi, yj)));
        Q.bb[i] = b;
        e[p] = make_float4(fminf(e[p].x, b.x), fminf(e[p].y, b.y), fmaxf(e[p].z, b.z), fmaxf(e[p].w, b.w));
      }
    }
  }
  // ring orientations: material on the left for CCW outer rings and CW holes
#pragma unroll
  for (int p = 0; p < 2; p++) {
    for (int r = 0; r < nr[p]; r++) {
      double sa = 0.0;
#pragma unroll
      for (int t = 0; t < V / 32; t++) sa += rix[p][t] == r ? term[p][t] : 0.0;
      for (int o = 16; o; o >>= 1) sa += __shfl_xor_sync(kFullMask, sa, o);
      const bool hole = __shfl_sync(kFullMask, hl[p], r) != 0;
      const int n = M[p].ringv[r + 1] - M[p].ringv[r];
      const int8_t sg = n < 2 ? 0 : (int8_t)((sa >= 0.0 ? 1 : -1) * (hole ? -1 : 1));
#pragma unroll
      for (int t = 0; t < V / 32; t++)
        if (rix[p][t] == r) M[p].sgn[32 * t + lane] = sg;
    }
    for (int o = 16; o; o >>= 1) {
      e[p].x = fminf(e[p].x, __shfl_xor_sync(kFullMask, e[p].x, o));
      e[p].y = fminf(e[p].y, __shfl_xor_sync(kFullMask, e[p].y, o));
      e[p].z = fmaxf(e[p].z, __shfl_xor_sync(kFullMask, e[p].z, o));
      e[p].w = fmaxf(e[p].w, __shfl_xor_sync(kFullMask, e[p].w, o));
    }
    ext[p] = e[p];
  }
  __syncwarp();
  return true;
}

// 32 x 32 bit matrix transpose across the warp: bit i of lane l's result is
// bit l of lane i's input (recursive exchange of off-diagonal blocks).
__device__ inline uint32_t bit_transpose(uint32_t x) {
  const int lane = threadIdx.x & 31;
  uint32_t m = 0x0000ffffu;
#pragma unroll
  for (int j = 16; j; j >>= 1, m ^= m << j) {
    const uint32_t t = __shfl_xor_sync(kFullMask, x, j);
    x = (lane & j) ? ((x & ~m) | ((t >> j) & m)) : ((x & m) | ((t << j) & ~m));
  }
  return x;
}

// y and x slab masks of both staged polygons (four independent transposes
// per word).
template <int V>
__device__ inline void bwd_slabs(BwdPoly<V> *M, const int *nv, const SlabGrid &gy, const SlabGrid &gx) {
  const int lane = threadIdx.x & 31;
  const int nw = ((nv[0] > nv[1] ? nv[0] : nv[1]) + 31) / 32;
  for (int c = 0; c < nw; c++) {
    uint32_t ry[2], rx[2];
#pragma unroll
    for (int p = 0; p < 2; p++) {
      const int k = 32 * c + lane;
      ry[p] = rx[p] = 0;
      if (k < nv[p]) {
        const float4 b = M[p].bb[k];
        ry[p] = (kFullMask >> (31 - gy(b.w))) & (kFullMask << gy(b.y));
        rx[p] = (kFullMask >> (31 - gx(b.z))) & (kFullMask << gx(b.x));
      }
    }
#pragma unroll
    for (int p = 0; p < 2; p++) {
      M[p].slab[c][lane] = bit_transpose(ry[p]);
      M[p].xslab[c][lane] = bit_transpose(rx[p]);
    }
  }
  __syncwarp();
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

// Even-odd test of (mx, my) against staged polygon Q through the slab of
// my: inside_evenodd's expression over the edges that can straddle my.
template <int V>
__device__ inline bool bwd_inside(const BwdPoly<V> &Q, int nwq, const float4 &qe, const SlabGrid &g, double mx,
                                  double my) {
  const float fy = __double2float_rn(my);
  if (fy < qe.y || fy > qe.w) return false;  // no edge of Q straddles my
  const int s = g(fy);
  bool in = false;
  for (int c = 0; c < nwq; c++) {
    uint32_t bits = Q.slab[c][s];
    while (bits) {
      const int k = 32 * c + __ffs(bits) - 1;
      bits &= bits - 1;
      const int l = Q.nxt[k];
      const double ay = Q.y[k], by = Q.y[l];
      if ((ay > my) != (by > my)) {
        const double ax = Q.x[k], bx = Q.x[l];
        const double xi = ax + (my - ay) * (bx - ax) / (by - ay);
        if (mx < xi) in = !in;
      }
    }
  }
  return in;
}

// Candidate edges of Q (mask word c) for an edge whose box covers y slabs
// [s0, s1] and x slabs [x0, x1].
template <int V>
__device__ inline uint32_t bwd_cands(const BwdPoly<V> &Q, int c, int s0, int s1, int x0, int x1) {
  uint32_t ybits = 0, xbits = 0;
  for (int s = s0; s <= s1; s++) ybits |= Q.slab[c][s];
  for (int s = x0; s <= x1; s++) xbits |= Q.xslab[c][s];
  return ybits & xbits;
}

// One edge p -> p + r against staged polygon Q by the definition: every
// crossing by next_crossing's test (kBwdMaxT at most, else the global-memory
// path), sorted and deduplicated, and every interval by its midpoint.
template <int V>
__device__ __noinline__ void bwd_edge_exact(const BwdPoly<V> &Q, int nwq, const float4 &qe, const SlabGrid &g,
                                            const SlabGrid &gx, const float4 &pb, double px, double py, double rx,
                                            double ry, const Poly &Qg, double *it_out, double *i1_out) {
  double ts[kBwdMaxT];
  int nt = 0;
  bool over = false;
  const int s0 = g(pb.y), s1 = g(pb.w), x0 = gx(pb.x), x1 = gx(pb.z);
  for (int c = 0; c < nwq; c++) {
    uint32_t bits = bwd_cands(Q, c, s0, s1, x0, x1);
    while (bits) {
      const int k = 32 * c + __ffs(bits) - 1;
      bits &= bits - 1;
      const float4 b = Q.bb[k];
      if (b.w < pb.y || b.y > pb.w || b.z < pb.x || b.x > pb.z) continue;
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
  double it = 0.0, i1 = 0.0;
  if (over) {
    bwd_edge_global(Qg, px, py, rx, ry, &it, &i1);
  } else {
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
    for (int a = 0; a <= m; a++) {
      const double t0 = a == 0 ? 0.0 : ts[a - 1], t1 = a < m ? ts[a] : 1.0;
      const double tm = 0.5 * (t0 + t1);
      if (bwd_inside(Q, nwq, qe, g, px + tm * rx, py + tm * ry)) {
        const double aa = 0.5 * (t1 * t1 - t0 * t0);
        it += aa;
        i1 += (t1 - t0) - aa;
      }
    }
  }
  *it_out = it;
  *i1_out = i1;
}

// pieces() for both polygons of a staged pair: lane edge e < na is edge e of
// A (against B), e >= na edge e - na of B (against A); rounds of 32 edges.
// ext[0], ext[1]: the float extents of A and B.
//
// Which intervals are inside: the midpoint of each interval (the
// definition, bwd_edge_exact), or, while the pair's crossings are all clean,
// by parity: a ring's first interval by its midpoint, every later interval of
// the ring flips at each crossing (prefix XOR of the crossing counts over the
// ring's edges, carried between rounds).  A crossing is clean when it is well
// inside both edges (t and u at least 1e-9 from 0 and 1) and the edges are
// not nearly parallel; collinear overlapping edges, two coinciding crossings
// on an edge and an edge with more crossings than the list below holds are
// not clean.
// From the first round with an unclean edge on, the pair goes by the
// definition.  Clean crossings flip the inside state exactly where the
// midpoints change and pass next_crossing's test, so the two give the same
// intervals.  The clean path keeps an edge's crossings sorted in registers.
// Clean crossings kept per edge: 4 in gradient mode, 6 in area mode (1M
// pairs of 16-64-vertex stars: 0.5% of the pairs have an edge with 5 or 6
// crossings; in area mode they would go to the GPC clip, 3,670 pairs against
// 119 with 6, while the gradient mode runs faster with the shorter list and
// the definition for those pairs).
constexpr int kBwdFast = 4;
constexpr int kFwdFast = 6;

// Area mode of the same pass (the forward): per edge, the inside length
// L = sum (t1 - t0) over its inside intervals contributes
//     s * L * cross(p - O, q - p) / 2
// to area(A∩B) (the shoelace term of each inside piece, about a pair-local
// origin O), and every clean crossing adds a bound on how far GPC's own
// vertex can lie from it: a vertex error of ~eps * max|coordinate| /
// sin(angle) times the two edges' lengths,
//     (|r|_1 + |s|_1) * |r|_1 * |s|_1 / |r x s|  (times eps * max|coordinate|).
struct AreaSum {
  double area;  // twice the area, summed over the warp by the caller
  double err;   // the crossing error bound above, without its eps * max|coordinate| factor
};

// Returns false in area mode as soon as any crossing of the pair is unclean
// (the caller then clips the pair with GPC); in gradient mode it always runs
// to the end, by the definition from the first unclean crossing on.
template <bool kArea, int V>
__device__ inline bool pair_boundary(const BwdPoly<V> *M, const float4 *ext, int na, int nb, const SlabGrid &g,
                                     const SlabGrid &gx, double w, double *ga, double *gb, int64_t va, int64_t vb,
                                     const Poly &Ag, const Poly &Bg, double ox, double oy, AreaSum *acc) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  bool exact = false;  // by the definition from here on (sticky)
  bool carry = false;  // inside state after the last edge of the previous round
  double area2 = 0.0, err = 0.0;
  for (int e0 = 0; e0 < na + nb; e0 += 32) {
    const int e = e0 + lane;
    const int side = e < na ? 0 : 1;
    const int i = side ? e - na : e;
    const BwdPoly<V> &P = M[side], &Q = M[1 - side];
    const int nwq = ((side ? na : nb) + 31) >> 5;
    const bool valid = e < na + nb && P.sgn[i] != 0;
    const int j = valid ? P.nxt[i] : 0;
    double px = 0.0, py = 0.0, qx = 0.0, qy = 0.0;
    float4 pb = make_float4(0.f, 0.f, 0.f, 0.f);
    if (valid) {
      px = P.x[i];
      py = P.y[i];
      qx = P.x[j];
      qy = P.y[j];
      pb = P.bb[i];
    }
    const double rx = qx - px, ry = qy - py;
    // clean crossings, ascending (2.0 = empty)
    constexpr int kFast = kArea ? kFwdFast : kBwdFast;
    double tc[kFast];
#pragma unroll
    for (int q = 0; q < kFast; q++) tc[q] = 2.0;
    int m = 0;
    bool unclean = false;
    if (valid && !exact) {
      const double rl = fabs(rx) + fabs(ry);
      const int s0 = g(pb.y), s1 = g(pb.w), x0 = gx(pb.x), x1 = gx(pb.z);
      for (int c = 0; c < nwq; c++) {
        uint32_t bits = bwd_cands(Q, c, s0, s1, x0, x1);
        while (bits) {
          const int k = 32 * c + __ffs(bits) - 1;
          bits &= bits - 1;
          const float4 b = Q.bb[k];
          if (b.w < pb.y || b.y > pb.w || b.z < pb.x || b.x > pb.z) continue;
          const int l = Q.nxt[k];
          const double ax = Q.x[k], ay = Q.y[k], bx = Q.x[l], by = Q.y[l];
          const double sx = bx - ax, sy = by - ay;
          const double den = rx * sy - ry * sx;
          const double apx = ax - px, apy = ay - py;
          const double tn = apx * sy - apy * sx;
          if (den == 0.0) {
            unclean |= tn == 0.0;  // collinear
            continue;
          }
          const double un = apx * ry - apy * rx;
          // t = tn / den and u = un / den, with the signs of den folded in
          const double d = fabs(den), tol = 1e-9 * d;
          const double tt = den > 0.0 ? tn : -tn, uu = den > 0.0 ? un : -un;
          if (tt < -tol || tt > d + tol || uu < -tol || uu > d + tol) continue;  // next_crossing rejects it
          if (!(tt > tol && tt < d - tol && uu > tol && uu < d - tol && d > 1e-6 * rl * (fabs(sx) + fabs(sy))) ||
              m == kFast) {
            unclean = true;
            continue;
          }
          if constexpr (kArea) {
            const double sl = fabs(sx) + fabs(sy);
            err += (rl + sl) * rl * sl / d;
          }
          double v = (apx * sy - apy * sx) / den;  // next_crossing's t
          // sorted insert into the register list
#pragma unroll
          for (int q = 0; q < kFast; q++)
            if (v < tc[q]) {
              const double x = tc[q];
              tc[q] = v;
              v = x;
            }
          m++;
        }
      }
#pragma unroll
      for (int q = 1; q < kFast; q++) unclean |= m > q && tc[q - 1] == tc[q];
    }
    exact = __any_sync(kFullMask, unclean) || exact;
    if constexpr (kArea) {
      if (exact) return false;
    }
    double it = 0.0, i1 = 0.0;
    if (exact) {
      if (valid)
        bwd_edge_exact(Q, nwq, ext[1 - side], g, gx, pb, px, py, rx, ry, side ? Ag : Bg, &it, &i1);
    } else {
      const int rs = valid ? (side ? na : 0) + P.rst[i] : e;  // this edge's ring starts at edge rs
      // the first interval of each ring starting in this round, by its
      // midpoint: the whole warp tests it against all edges of the other polygon
      const bool rstart = valid && rs == e;
      double mx0 = 0.0, my0 = 0.0;
      if (rstart) {
        const double tm = 0.5 * (m > 0 ? tc[0] : 1.0);
        mx0 = px + tm * rx;
        my0 = py + tm * ry;
      }
      bool first = false;
      for (unsigned q = __ballot_sync(kFullMask, rstart); q; q &= q - 1) {
        const int L = __ffs(q) - 1;
        const double mxl = __shfl_sync(kFullMask, mx0, L), myl = __shfl_sync(kFullMask, my0, L);
        const int sl = e0 + L < na ? 0 : 1;
        const BwdPoly<V> &QL = M[1 - sl];
        const int nql = sl ? na : nb;
        bool in = false;
        for (int k = lane; k < nql; k += 32) {
          const int l = QL.nxt[k];
          const double ay = QL.y[k], by = QL.y[l];
          if ((ay > myl) != (by > myl)) {
            const double ax = QL.x[k], bx = QL.x[l];
            const double xi = ax + (myl - ay) * (bx - ax) / (by - ay);
            if (mxl < xi) in = !in;
          }
        }
        const bool inside = (__popc(__ballot_sync(kFullMask, in)) & 1) != 0;
        if (lane == L) first = inside;
      }
      const unsigned odd = __ballot_sync(kFullMask, (m & 1) != 0);
      const int from = rs > e0 ? rs - e0 : 0;
      const int par = __popc(odd & lt & ~((1u << from) - 1u)) & 1;
      const bool sf = __shfl_sync(kFullMask, first, from);
      const bool st = (rs >= e0 ? sf : carry) != (par != 0);  // inside state at the edge's start
      carry = __shfl_sync(kFullMask, st != ((m & 1) != 0), 31);
      // intervals [0, tc[0]], [tc[0], tc[1]], ..., [tc[m-1], 1], alternately inside
      if (valid) {
        bool in = st;
        double a0 = 0.0;
#pragma unroll
        for (int a = 0; a <= kFast; a++) {
          if (a <= m) {
            const double a1 = a < m ? tc[a < kFast ? a : kFast - 1] : 1.0;
            if (in) {
              const double aa = 0.5 * (a1 * a1 - a0 * a0);
              it += aa;
              i1 += (a1 - a0) - aa;
            }
            a0 = a1;
            in = !in;
          }
        }
      }
    }
    if constexpr (kArea) {
      // it + i1 = sum (t1 - t0) over the inside intervals
      if (valid) area2 += P.sgn[i] * (it + i1) * ((px - ox) * ry - (py - oy) * rx);
      continue;
    }
    // contributions: it to the end vertex j, i1 to the start vertex i; the
    // lane of the next edge of the ring hands its start contribution over so
    // the shared vertex takes one atomic per coordinate
    double gxj = 0.0, gyj = 0.0, gxi = 0.0, gyi = 0.0;
    if (valid) {
      const double s = P.sgn[i];
      const double nx = w * s * ry, ny = -w * s * rx;
      gxj = nx * it;
      gyj = ny * it;
      gxi = nx * i1;
      gyi = ny * i1;
    }
    const int key = valid ? (side << 8) | i : -1;           // this edge's start vertex
    const int kend = valid ? (side << 8) | j : -2;          // its end vertex
    const int knext = __shfl_down_sync(kFullMask, key, 1);  // start vertex of the next lane's edge
    const int kprev = __shfl_up_sync(kFullMask, kend, 1);   // end vertex of the previous lane's edge
    const double hx = __shfl_down_sync(kFullMask, gxi, 1), hy = __shfl_down_sync(kFullMask, gyi, 1);
    const bool take = lane < 31 && knext == kend;  // the next lane's i1 part goes with mine
    const bool given = lane > 0 && kprev == key;   // mine went to the previous lane
    if (take) {
      gxj += hx;
      gyj += hy;
    }
    double *gr = side ? gb : ga;
    const int64_t vbase = side ? vb : va;
    if (valid && (gxj != 0.0 || gyj != 0.0)) {
      atomicAdd(&gr[2 * (vbase + j)], gxj);
      atomicAdd(&gr[2 * (vbase + j) + 1], gyj);
    }
    if (valid && !given && (gxi != 0.0 || gyi != 0.0)) {
      atomicAdd(&gr[2 * (vbase + i)], gxi);
      atomicAdd(&gr[2 * (vbase + i) + 1], gyi);
    }
  }
  if constexpr (kArea) {
    acc->area = area2;
    acc->err = err;
  }
  return true;
}

// Pairs with a polygon above V vertices: the global-memory path.
__device__ __noinline__ void bwd_pair_global(const Poly &A, const Poly &B, double w, double *ga, double *gb) {
  const int lane = threadIdx.x & 31;
  pieces(A, B, w, ga, lane);
  pieces(B, A, w, gb, lane);
}

// Pair lists of the two-stage launches: the first stage (V = kBwdSmallV)
// takes every pair and lists those with a polygon above V vertices (or 31
// rings) in `defer`; the second stage (V = kBwdMaxV) takes only the listed
// pairs (`sel`, *sel_count of them).
struct PairList {
  const int32_t *sel;                   // items of this launch (nullptr: pairs 0 .. n-1)
  const unsigned long long *sel_count;  // how many (device)
  int32_t *defer;                       // pairs this stage cannot stage (nullptr: none deferred)
  unsigned long long *defer_count;
};

__device__ __forceinline__ int64_t list_items(const PairList &L, int64_t n) {
  return L.sel ? (int64_t)min((unsigned long long)n, *L.sel_count) : n;
}

// 4 blocks of 4 warps per SM (120 registers, no spills; measured at 1M
// pairs of 16-64-vertex stars, 5 blocks of the V = 64 kernel spill and run
// 10% slower).
template <int V>
__global__ void __launch_bounds__(32 * kBwdWarps, 4) area_bwd_kernel(
    const int32_t *__restrict__ pa, const int32_t *__restrict__ pb, int64_t n, LayerDev base, LayerDev over,
    const double *__restrict__ upstream, double *grad_base, double *grad_over, PairList PL) {
  __shared__ BwdPoly<V> sm[kBwdWarps][2];
  BwdPoly<V> *M = sm[threadIdx.x >> 5];
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t items = list_items(PL, n);
  // a pair's ids are read one pair ahead and its ring ranges half a pair
  // ahead, so the staging of a pair waits only for its ring starts and
  // vertices
  auto ids = [&](int64_t k, int64_t *i, int64_t *a, int64_t *b) {
    *i = -1;
    *a = -1;
    *b = -1;
    if (k < items) {
      const int64_t j = PL.sel ? PL.sel[k] : k;
      if (j >= 0 && j < n) {
        const int64_t x = pa[j], y = pb[j];
        if (x >= 0 && x < base.n_poly && y >= 0 && y < over.n_poly) {
          *i = j;
          *a = x;
          *b = y;
        }
      }
    }
  };
  auto rings = [&](int64_t a, int64_t b, int64_t *r) {
    r[0] = r[1] = r[2] = r[3] = 0;
    if (a >= 0) {
      r[0] = base.poly_ring[a];
      r[1] = base.poly_ring[a + 1];
      r[2] = over.poly_ring[b];
      r[3] = over.poly_ring[b + 1];
    }
  };
  int64_t i, a, b, rr[4];
  ids(warp, &i, &a, &b);
  rings(a, b, rr);
  for (int64_t k = warp; k < items; k += nw) {
    int64_t in, an, bn, rn[4];
    ids(k + nw, &in, &an, &bn);
    bool fetched = false;
    if (a >= 0) {
      int nv[2];
      int64_t vb[2];
      float4 ext[2];
      const bool staged = bwd_load_pair(base, rr[0], rr[1], over, rr[2], rr[3], M, nv, vb, ext);
      rings(an, bn, rn);
      fetched = true;
      if (staged) {
        const double w = upstream ? upstream[i] : 1.0;
        // boxes apart: no crossings and no midpoint inside the other polygon
        const float x0 = fmaxf(ext[0].x, ext[1].x), x1 = fminf(ext[0].z, ext[1].z);
        const float y0 = fmaxf(ext[0].y, ext[1].y), y1 = fminf(ext[0].w, ext[1].w);
        if (!(x0 > x1 || y0 > y1)) {
          const SlabGrid gy = slab_grid(y0, y1), gx = slab_grid(x0, x1);
          bwd_slabs(M, nv, gy, gx);
          Poly A{base.ring_vert, base.ring_hole, base.xy, rr[0], rr[1]};
          Poly B{over.ring_vert, over.ring_hole, over.xy, rr[2], rr[3]};
          pair_boundary<false>(M, ext, nv[0], nv[1], gy, gx, w, grad_base, grad_over, vb[0], vb[1], A, B, 0.0,
                               0.0, nullptr);
        }
      } else if (PL.defer) {
        if ((threadIdx.x & 31) == 0) PL.defer[atomicAdd(PL.defer_count, 1ull)] = (int32_t)i;
      } else {
        const double w = upstream ? upstream[i] : 1.0;
        Poly A{base.ring_vert, base.ring_hole, base.xy, rr[0], rr[1]};
        Poly B{over.ring_vert, over.ring_hole, over.xy, rr[2], rr[3]};
        bwd_pair_global(A, B, w, grad_base, grad_over);
      }
    }
    if (!fetched) rings(an, bn, rn);
    i = in;
    a = an;
    b = bn;
    for (int q = 0; q < 4; q++) rr[q] = rn[q];
    __syncwarp();
  }
}

// Forward: one warp per pair, staged as in the backward.  A pair gets its
// area from pair_boundary's area mode when every crossing is clean and the
// crossing error bound stays below kFwdTol of the area; every other pair
// (polygons above V vertices or 31 rings, unclean crossings, slivers
// whose area the bound does not pin to kFwdTol, ids out of range) is listed in
// fb[] for the GPC clip.  GPC intersects the same edges, so for a clean pair
// the two areas differ only by where each side rounds the crossing vertices:
// a vertex moves by at most ~2 eps max|coordinate| / sin(angle), which moves
// the area by that times the crossing edges' lengths.  pair_boundary sums
// (|r|_1 + |s|_1) / sin over the crossings as seen from both edges (each
// crossing twice, and 1-norms, which are at least the lengths), so
// 2 eps max|coordinate| times the sum bounds the difference; a pair is kept
// when that is below kFwdTol of its area, ten times inside the 1e-9 the
// forward promises.
constexpr double kFwdTol = 1e-10;

// Pairs the last forward call listed for the GPC clip (prt_area_fwd_fallbacks).
std::atomic<int64_t> g_fwd_fallbacks{0};

// V = 64: 5 blocks of 4 warps per SM (96 registers: a few spills, 10% faster
// than 4 blocks at 1M pairs of 16-64-vertex stars).
template <int V>
__global__ void __launch_bounds__(32 * kBwdWarps, V <= kBwdSmallV ? 5 : 4) area_fwd_kernel(
    const int32_t *__restrict__ pa, const int32_t *__restrict__ pb, int64_t n, LayerDev base, LayerDev over,
    double *__restrict__ area, int32_t *__restrict__ fb, unsigned long long *__restrict__ fb_count, PairList PL) {
  __shared__ BwdPoly<V> sm[kBwdWarps][2];
  BwdPoly<V> *M = sm[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t items = list_items(PL, n);
  auto fallback = [&](int64_t i) {
    if (lane == 0) fb[atomicAdd(fb_count, 1ull)] = (int32_t)i;
  };
  for (int64_t k = warp; k < items; k += nw) {
    const int64_t i = PL.sel ? PL.sel[k] : k;
    if (i < 0 || i >= n) continue;
    const int64_t a = pa[i], b = pb[i];
    if (a < 0 || a >= base.n_poly || b < 0 || b >= over.n_poly) {
      fallback(i);  // the clip reports the bad id
      continue;
    }
    const int64_t ra0 = base.poly_ring[a], ra1 = base.poly_ring[a + 1];
    const int64_t rb0 = over.poly_ring[b], rb1 = over.poly_ring[b + 1];
    int nv[2];
    int64_t vb[2];
    float4 ext[2];
    const bool staged = bwd_load_pair(base, ra0, ra1, over, rb0, rb1, M, nv, vb, ext);
    if (!staged) {
      if (PL.defer) {
        if (lane == 0) PL.defer[atomicAdd(PL.defer_count, 1ull)] = (int32_t)i;
      } else {
        fallback(i);
      }
      __syncwarp();
      continue;
    }
    const float x0 = fmaxf(ext[0].x, ext[1].x), x1 = fminf(ext[0].z, ext[1].z);
    const float y0 = fmaxf(ext[0].y, ext[1].y), y1 = fminf(ext[0].w, ext[1].w);
    if (x0 > x1 || y0 > y1 || nv[0] == 0 || nv[1] == 0) {
      // boxes apart: no crossing, no point of one inside the other
      if (lane == 0) area[i] = 0.0;
      __syncwarp();
      continue;
    }
    const SlabGrid gy = slab_grid(y0, y1), gx = slab_grid(x0, x1);
    bwd_slabs(M, nv, gy, gx);
    Poly A{base.ring_vert, base.ring_hole, base.xy, ra0, ra1};
    Poly B{over.ring_vert, over.ring_hole, over.xy, rb0, rb1};
    AreaSum acc{0.0, 0.0};
    const double ox = M[0].x[0], oy = M[0].y[0];  // the pair-local origin
    const bool ok = pair_boundary<true>(M, ext, nv[0], nv[1], gy, gx, 1.0, nullptr, nullptr, vb[0], vb[1], A, B,
                                        ox, oy, &acc);
    if (ok) {
      double a2 = acc.area, er = acc.err;
      for (int o = 16; o; o >>= 1) {
        a2 += __shfl_xor_sync(kFullMask, a2, o);
        er += __shfl_xor_sync(kFullMask, er, o);
      }
      const float cmax = fmaxf(fmaxf(fmaxf(fabsf(ext[0].x), fabsf(ext[0].y)), fmaxf(fabsf(ext[0].z), fabsf(ext[0].w))),
                               fmaxf(fmaxf(fabsf(ext[1].x), fabsf(ext[1].y)), fmaxf(fabsf(ext[1].z), fabsf(ext[1].w))));
      const double bound = 2.0 * 2.220446049250313e-16 * (double)cmax * er;
      const double ar = 0.5 * a2;
      if (bound <= kFwdTol * fabs(ar)) {
        if (lane == 0) area[i] = ar;
      } else {
        fallback(i);
      }
    } else {
      fallback(i);
    }
    __syncwarp();
  }
}

__global__ void gather_pairs_kernel(const int32_t *__restrict__ fb, int64_t m, const int32_t *__restrict__ pa,
                                    const int32_t *__restrict__ pb, int32_t *__restrict__ qa,
                                    int32_t *__restrict__ qb) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x) {
    qa[k] = pa[fb[k]];
    qb[k] = pb[fb[k]];
  }
}

__global__ void scatter_area_kernel(const int32_t *__restrict__ fb, int64_t m, const double *__restrict__ src,
                                    double *__restrict__ area) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x)
    area[fb[k]] = src[k];
}

int area_blocks(int64_t n_pairs, const void *kernel) {
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, 32 * kBwdWarps, 0) != cudaSuccess || b < 1) {
    cudaGetLastError();
    b = 4;
  }
  // exactly the resident blocks (each warp loops over pairs): no tail wave
  return grid_for(n_pairs * 32, 32 * kBwdWarps, b);
}

}  // namespace
}  // namespace prt

using namespace prt;

extern "C" {

int prt_area_fwd(const int32_t *d_pair_a, const int32_t *d_pair_b, int64_t n_pairs, const prt_layer *base,
                 const prt_layer *overlay, double *d_area, void *stream) {
  PRT_CHECK(base && overlay && (n_pairs == 0 || (d_area && d_pair_a && d_pair_b)), PRT_ERR_INVALID,
            "NULL argument");
  PRT_CHECK(n_pairs >= 0 && n_pairs < (1ll << 31), PRT_ERR_INVALID, "n_pairs=%lld", (long long)n_pairs);
  if (n_pairs == 0) return PRT_OK;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  // boundary integral for the clean pairs, the list of the others; pairs
  // with a polygon above kBwdSmallV vertices go through the second stage
  unsigned char *scr = nullptr;
  int rc = dmalloc(reinterpret_cast<void **>(&scr), 64 + 8 * (size_t)n_pairs, s);
  if (rc) return rc;
  unsigned long long *cnt = reinterpret_cast<unsigned long long *>(scr);
  unsigned long long *dcnt = cnt + 1;
  int32_t *fb = reinterpret_cast<int32_t *>(scr + 64);
  int32_t *defer = fb + n_pairs;
  cudaError_t e = cudaMemsetAsync(cnt, 0, 16, s);
  if (e == cudaSuccess) {
    PRT_PROF("area_fwd", s);
    area_fwd_kernel<kBwdSmallV><<<area_blocks(n_pairs, (const void *)area_fwd_kernel<kBwdSmallV>), 32 * kBwdWarps,
                                  0, s>>>(d_pair_a, d_pair_b, n_pairs, layer_dev(base), layer_dev(overlay), d_area, fb,
                                          cnt, PairList{nullptr, nullptr, defer, dcnt});
    area_fwd_kernel<kBwdMaxV><<<area_blocks(n_pairs, (const void *)area_fwd_kernel<kBwdMaxV>), 32 * kBwdWarps, 0,
                                s>>>(d_pair_a, d_pair_b, n_pairs, layer_dev(base), layer_dev(overlay), d_area, fb,
                                     cnt, PairList{defer, dcnt, nullptr, nullptr});
    e = cudaGetLastError();
  }
  unsigned long long m = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&m, cnt, 8, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    dfree(scr, s);
    return cuda_status(e, "area forward");
  }
  g_fwd_fallbacks.store((int64_t)m);
  if (m > 0) {
    // the listed pairs: GPC clip, area of its result (area-only mode)
    int32_t *q = nullptr;
    double *ar = nullptr;
    rc = dalloc(&q, 2 * m, s);
    if (!rc) rc = dalloc(&ar, m, s);
    if (!rc) {
      {
        PRT_PROF("gather_pairs", s);
        gather_pairs_kernel<<<grid_for((int64_t)m, 256, 8), 256, 0, s>>>(fb, (int64_t)m, d_pair_a, d_pair_b, q,
                                                                           q + m);
      }
      PairSrc S;
      memset(&S, 0, sizeof S);
      S.pa = q;
      S.pb = q + m;
      S.base = layer_dev(base);
      S.over = layer_dev(overlay);
      S.op = PRT_GPC_INT;
      rc = overlay_impl(S, (int64_t)m, PRT_SCHED_BATCHED, ar, s, nullptr);
    }
    if (!rc) {
      PRT_PROF("scatter_area", s);
      scatter_area_kernel<<<grid_for((int64_t)m, 256, 8), 256, 0, s>>>(fb, (int64_t)m, ar, d_area);
      e = cudaGetLastError();
      if (e != cudaSuccess) rc = cuda_status(e, "area scatter");
    }
    dfree(q, s);
    dfree(ar, s);
  }
  dfree(scr, s);
  return rc;
}

int prt_area_fwd_fallbacks(int64_t *h_count) {
  PRT_CHECK(h_count, PRT_ERR_INVALID, "NULL argument");
  *h_count = g_fwd_fallbacks.load();
  return PRT_OK;
}

int prt_area_bwd(const int32_t *d_pair_a, const int32_t *d_pair_b, int64_t n_pairs, const prt_layer *base,
                 const prt_layer *overlay, const double *d_upstream, double *d_grad_base, double *d_grad_overlay,
                 void *stream) {
  PRT_CHECK(base && overlay && (n_pairs == 0 || (d_grad_base && d_grad_overlay && d_pair_a && d_pair_b)),
            PRT_ERR_INVALID, "NULL argument");
  if (n_pairs == 0) return PRT_OK;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  // pairs with a polygon above kBwdSmallV vertices: listed by the first
  // stage, taken by the second
  unsigned char *scr = nullptr;
  int rc = dmalloc(reinterpret_cast<void **>(&scr), 64 + 4 * (size_t)n_pairs, s);
  if (rc) return rc;
  unsigned long long *dcnt = reinterpret_cast<unsigned long long *>(scr);
  int32_t *defer = reinterpret_cast<int32_t *>(scr + 64);
  cudaError_t e = cudaMemsetAsync(dcnt, 0, 8, s);
  if (e == cudaSuccess) {
    PRT_PROF("area_bwd", s);
    area_bwd_kernel<kBwdSmallV><<<area_blocks(n_pairs, (const void *)area_bwd_kernel<kBwdSmallV>), 32 * kBwdWarps,
                                  0, s>>>(d_pair_a, d_pair_b, n_pairs, layer_dev(base), layer_dev(overlay),
                                          d_upstream, d_grad_base, d_grad_overlay,
                                          PairList{nullptr, nullptr, defer, dcnt});
    area_bwd_kernel<kBwdMaxV><<<area_blocks(n_pairs, (const void *)area_bwd_kernel<kBwdMaxV>), 32 * kBwdWarps, 0,
                                s>>>(d_pair_a, d_pair_b, n_pairs, layer_dev(base), layer_dev(overlay), d_upstream,
                                     d_grad_base, d_grad_overlay, PairList{defer, dcnt, nullptr, nullptr});
    e = cudaGetLastError();
  }
  dfree(scr, s);
  if (e != cudaSuccess) return cuda_status(e, "area backward");
  return PRT_OK;
}

}  // extern "C"
