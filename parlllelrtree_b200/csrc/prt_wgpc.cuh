// Warp-cooperative GPC clipper: ONE pair per warp, same output as the thread
// clipper in prt_gpc.cuh (contours, hole flags, vertex order and the order of
// the contour list), which restates gpc_polygon_clip
// (vector_map_overlay_gpc_kernel.cu:115-750).
//
// The thread clipper walks the active edge table (AET) as an index-linked list
// in global memory several times per scanbeam; for pairs with thousands of
// vertices that is a chain of dependent loads per edge per pass.  Here the AET
// is an ARRAY of slots in shared memory, in AET order, and every per-beam pass
// is data-parallel over the slots:
//   insertion of the beam's local minima    ballot for the insertion point, shift
//   bundle detection (GPC:371-393)           segmented XOR over the edges that
//                                            do not end at yb
//   parity and horizontal state (GPC:395-423) popcounts of ballots (the state
//                                            changes only at one-sided edges)
//   vertex classes                           per slot from that state
//   output (GPC:425-570)                     continuing edges in parallel; the
//                                            events (vertices, local minima and
//                                            maxima) on lane 0 in AET order; a
//                                            contour merge's redirect by the warp
//   next scanbeam, deletion, xt (GPC:426-459) warp min and ballot compaction
//   intersection test (GPC:461-485)          fast check that the ST insertion
//                                            would record no intersection; a beam
//                                            that has intersections spills the
//                                            slots to the linked form and runs the
//                                            thread clipper's intersect_beam
//   successor edges (GPC:661-693)            per slot
// The build is parallel too: ring staging by ballot, bound edges written by
// the whole warp, the local-minima table sorted by a stable warp radix sort.
// No scanbeam table is sorted: every vertex y is a local minimum or the top
// of an edge, so the next beam is the lower of the next local minimum and the
// lowest top of an active edge, which walks the same sorted unique ys as
// GPC's table (build_sbt, GPC:1019-1085).  An active edge table larger than
// the shared-memory slots moves to the pair's arena; only an AET list the
// intersection step leaves malformed or more rings than the ring scratch
// holds make the caller rerun the pair with the thread clipper, so the result
// is always the thread clipper's.
#pragma once
#include "prt_gpc.cuh"

namespace prt {
namespace gpc {

constexpr unsigned kFull = 0xffffffffu;
constexpr double kInf = __builtin_huge_val();

// Slot flag bits.
enum : uint32_t {
  W_TYPE = 1u,         // SUBJ edge
  W_BA = 1,            // bits 1-2: bundle[ABOVE][CLIP], [SUBJ]
  W_BB = 3,            // bits 3-4: bundle[BELOW]
  W_SIDE = 5,          // bits 5-6: bside[CLIP], bside[SUBJ]
  W_STA = 7,           // bits 7-8: bstate[ABOVE]
  W_STB = 9,           // bits 9-10: bstate[BELOW]
  W_VC = 11,           // bits 11-14: vertex class
  W_CONTRIB = 1u << 15,
  W_STARTS = 1u << 16,  // the edge starts at yb
  W_PXNE = 1u << 17,    // xb differs from GPC's px (the x of the last output event before it)
};

__device__ inline int fbits(uint32_t f, int sh) { return (int)((f >> sh) & 3u); }
__device__ inline uint32_t fset(uint32_t f, int sh, int v) { return (f & ~(3u << sh)) | ((uint32_t)v << sh); }

struct WSlot {
  double xb, xt, dx, ty, bx, by, tx;
  int32_t edge, outA, outB, succ;
  uint32_t fl;
};

// Dynamic shared memory of the block (one warp per block): the warp
// clipper's slot arrays, then the radix counters and the cached output
// polygon nodes.
extern __shared__ __align__(16) unsigned char prt_wsm[];

// Output polygon nodes kept in shared memory per warp.
constexpr int kWarpPolyNodes = 128;

// Bytes of the slot arrays for cap slots: 7 double arrays, 6 int arrays,
// cap/32 event masks.
__host__ __device__ inline size_t wslot_bytes(int cap) {
  return (size_t)cap * (7 * 8 + 6 * 4) + (size_t)(cap / 32) * 4;
}

// Dynamic shared memory per warp: slots, 256 radix counters, polygon nodes.
__host__ __device__ inline size_t waet_bytes(int cap) {
  return wslot_bytes(cap) + 256 * 4 + sizeof(PolyNode) * kWarpPolyNodes;
}

// Arena of one pair in warp mode: the thread clipper's arena, then room for
// an active edge table as large as the pair's edge count, where the slots go
// when they outgrow shared memory.
__host__ __device__ inline size_t warp_arena_bytes(const Caps &c) {
  return arena_bytes(c) + align16(wslot_bytes((c.e + 31) / 32 * 32));
}

// Slot arrays of one warp (structure of arrays): the dynamic state of each
// active edge and the static fields every beam reads (bottom, top x,
// successor), so no pass over the slots reads the edge table.  `base` is the
// block's shared memory until the table outgrows it, then the arena.
struct WAet {
  unsigned char *base;
  int cap;     // slots at base
  int scap;    // slots of the shared-memory layout (fixed at launch)
  int spcap;   // polygon nodes in shared memory
  __device__ double *dbl(int k) const { return reinterpret_cast<double *>(base) + k * cap; }
  __device__ int32_t *i32(int k) const { return reinterpret_cast<int32_t *>(base + 56 * (size_t)cap) + k * cap; }
  __device__ double *xb() const { return dbl(0); }
  __device__ double *xt() const { return dbl(1); }
  __device__ double *dx() const { return dbl(2); }
  __device__ double *ty() const { return dbl(3); }
  __device__ double *bx() const { return dbl(4); }
  __device__ double *by() const { return dbl(5); }
  __device__ double *tx() const { return dbl(6); }
  __device__ int32_t *edge() const { return i32(0); }
  __device__ int32_t *outA() const { return i32(1); }
  __device__ int32_t *outB() const { return i32(2); }
  __device__ int32_t *succ() const { return i32(3); }
  __device__ int32_t *ord() const { return i32(4); }
  __device__ uint32_t *fl() const { return reinterpret_cast<uint32_t *>(i32(5)); }
  __device__ uint32_t *cmask() const { return reinterpret_cast<uint32_t *>(i32(6)); }
};

__device__ inline uint32_t *wsm_counters(int scap) { return reinterpret_cast<uint32_t *>(prt_wsm + wslot_bytes(scap)); }
__device__ inline PolyNode *wsm_polys(int scap) { return reinterpret_cast<PolyNode *>(wsm_counters(scap) + 256); }

__device__ inline WAet waet_carve(int cap) {
  WAet w;
  w.base = prt_wsm;
  w.cap = cap;
  w.scap = cap;
  w.spcap = kWarpPolyNodes;
  return w;
}

__device__ inline WSlot wload(const WAet &w, int s) {
  WSlot v;
  v.xb = w.xb()[s];
  v.xt = w.xt()[s];
  v.dx = w.dx()[s];
  v.ty = w.ty()[s];
  v.bx = w.bx()[s];
  v.by = w.by()[s];
  v.tx = w.tx()[s];
  v.edge = w.edge()[s];
  v.outA = w.outA()[s];
  v.outB = w.outB()[s];
  v.succ = w.succ()[s];
  v.fl = w.fl()[s];
  return v;
}

__device__ inline void wstore(const WAet &w, int s, const WSlot &v) {
  w.xb()[s] = v.xb;
  w.xt()[s] = v.xt;
  w.dx()[s] = v.dx;
  w.ty()[s] = v.ty;
  w.bx()[s] = v.bx;
  w.by()[s] = v.by;
  w.tx()[s] = v.tx;
  w.edge()[s] = v.edge;
  w.outA()[s] = v.outA;
  w.outB()[s] = v.outB;
  w.succ()[s] = v.succ;
  w.fl()[s] = v.fl;
}

// A slot holding edge e with the edge's stored state.
__device__ inline WSlot wslot_of(const Arena &A, int e) {
  const Edge &E = A.E[e];
  WSlot v;
  v.edge = e;
  v.xb = E.xb;
  v.xt = E.xt;
  v.dx = E.dx;
  v.ty = E.ty;
  v.bx = E.bx;
  v.by = E.by;
  v.tx = E.tx;
  v.succ = E.succ;
  v.outA = E.outp[ABOVE];
  v.outB = E.outp[BELOW];
  v.fl = (E.type ? W_TYPE : 0u) | ((uint32_t)(E.bundle[ABOVE][CLIP] | (E.bundle[ABOVE][SUBJ] << 1)) << W_BA) |
         ((uint32_t)(E.bundle[BELOW][CLIP] | (E.bundle[BELOW][SUBJ] << 1)) << W_BB) |
         ((uint32_t)(E.bside[CLIP] | (E.bside[SUBJ] << 1)) << W_SIDE) | ((uint32_t)E.bstate[ABOVE] << W_STA) |
         ((uint32_t)E.bstate[BELOW] << W_STB);
  return v;
}

// Writes a slot's state back to its edge, linked between prev and next.
__device__ inline void wspill(Arena &A, const WSlot &v, int prev, int next) {
  Edge &E = A.E[v.edge];
  E.xb = v.xb;
  E.xt = v.xt;
  E.outp[ABOVE] = v.outA;
  E.outp[BELOW] = v.outB;
  const int ba = fbits(v.fl, W_BA), bb = fbits(v.fl, W_BB), sd = fbits(v.fl, W_SIDE);
  E.bundle[ABOVE][CLIP] = (int8_t)(ba & 1);
  E.bundle[ABOVE][SUBJ] = (int8_t)(ba >> 1);
  E.bundle[BELOW][CLIP] = (int8_t)(bb & 1);
  E.bundle[BELOW][SUBJ] = (int8_t)(bb >> 1);
  E.bside[CLIP] = (int8_t)(sd & 1);
  E.bside[SUBJ] = (int8_t)(sd >> 1);
  E.bstate[ABOVE] = (int8_t)fbits(v.fl, W_STA);
  E.bstate[BELOW] = (int8_t)fbits(v.fl, W_STB);
  E.prev = prev;
  E.next = next;
}

__device__ inline unsigned lanemask_lt() { return (1u << (threadIdx.x & 31)) - 1u; }

// ---------------------------------------------------------------- warp radix sort
// Order-preserving 64-bit image of a double (-0.0 and +0.0 map to one key, as
// they compare equal).
__device__ inline uint64_t dkey(double v) {
  uint64_t u = (uint64_t)__double_as_longlong(v + 0.0);
  return (u >> 63) ? ~u : (u | (1ull << 63));
}

// Stable LSD radix sort of a[0, n) by key(a[i]) (8 passes of 8 bits), moving
// elements between a and b; passes whose digit is the same for every element
// are skipped.  Returns the buffer that holds the sorted data.
template <typename T, typename KeyF>
__device__ T *warp_radix(T *a, T *b, int n, KeyF key, uint32_t *cnt) {
  const int lane = threadIdx.x & 31;
  for (int p = 0; p < 8; p++) {
    const int sh = 8 * p;
    for (int i = lane; i < 256; i += 32) cnt[i] = 0;
    __syncwarp();
    for (int i = lane; i < n; i += 32) atomicAdd(&cnt[(uint32_t)(key(a[i]) >> sh) & 255u], 1u);
    __syncwarp();
    bool same = false;
    for (int i = lane; i < 256; i += 32) same |= cnt[i] == (uint32_t)n;
    if (__any_sync(kFull, same)) continue;
    uint32_t c[8], tot = 0;
    for (int j = 0; j < 8; j++) {
      c[j] = cnt[8 * lane + j];
      tot += c[j];
    }
    uint32_t incl = tot;
    for (int d = 1; d < 32; d <<= 1) {
      uint32_t t = __shfl_up_sync(kFull, incl, d);
      if (lane >= d) incl += t;
    }
    uint32_t run = incl - tot;
    __syncwarp();
    for (int j = 0; j < 8; j++) {
      cnt[8 * lane + j] = run;
      run += c[j];
    }
    __syncwarp();
    for (int base = 0; base < n; base += 32) {
      const int i = base + lane;
      const bool valid = i < n;
      T v;
      uint32_t d = 256u + (uint32_t)lane;
      if (valid) {
        v = a[i];
        d = (uint32_t)(key(v) >> sh) & 255u;
      }
      const unsigned peers = __match_any_sync(kFull, d);
      const int leader = __ffs(peers) - 1;
      const int rank = __popc(peers & lanemask_lt());
      uint32_t off = 0;
      if (valid && lane == leader) off = cnt[d];
      off = __shfl_sync(kFull, off, leader);
      if (valid) b[off + rank] = v;
      __syncwarp();
      if (valid && lane == leader) cnt[d] = off + (uint32_t)__popc(peers);
      __syncwarp();
    }
    T *t = a;
    a = b;
    b = t;
  }
  return a;
}

template <typename T>
__device__ inline void warp_copy(T *dst, const T *src, int n) {
  for (int i = threadIdx.x & 31; i < n; i += 32) dst[i] = src[i];
  __syncwarp();
}

// ---------------------------------------------------------------- build
// Bounds of ring r (build_lmt, GPC:1175-1307) with the whole warp: the optimal
// vertices are staged by ballot, each local minimum's bound is measured by a
// warp-wide walk and its edges are written in parallel.  Edges and bounds
// come out in the thread clipper's order.
__device__ inline void wbuild_ring(Arena &A, const PolyView &p, int64_t r, int type, int op, double *sx,
                                   double *sy) {
  const int lane = threadIdx.x & 31;
  const int64_t v0 = p.ring_vert[r];
  const int n = (int)(p.ring_vert[r + 1] - v0);
  const double *xy = p.xy + 2 * v0;
  int k = 0;
  for (int c = 0; c < n; c += 32) {
    const int i = c + lane;
    bool opt = false;
    double x = 0.0, y = 0.0;
    if (i < n) {
      const int ip = (i + n - 1) % n, in = (i + 1) % n;
      y = xy[2 * i + 1];
      x = xy[2 * i];
      opt = xy[2 * ip + 1] != y || xy[2 * in + 1] != y;
    }
    const unsigned m = __ballot_sync(kFull, opt);
    if (opt) {
      const int kk = k + __popc(m & lanemask_lt());
      sx[kk] = x;
      sy[kk] = y;
    }
    k += __popc(m);
  }
  __syncwarp();
  for (int dir = 0; dir < 2; dir++) {
    for (int c = 0; c < k; c += 32) {
      const int mn = c + lane;
      bool is_min = false;
      if (mn < k) {
        const int pv = (mn + k - 1) % k, nx = (mn + 1) % k;
        is_min = dir == 0 ? (sy[pv] >= sy[mn] && sy[nx] > sy[mn]) : (sy[pv] > sy[mn] && sy[nx] >= sy[mn]);
      }
      unsigned m = __ballot_sync(kFull, is_min);
      while (m) {
        const int m0 = c + __ffs(m) - 1;
        m &= m - 1;
        // ne = 1 + the rising steps after the first edge
        int ne = 0;
        for (int q = 1; ne == 0; q += 32) {
          const int i = q + lane;  // step i goes from vertex w_i to w_{i+1}
          bool stop = true;
          if (i < k) {
            const int wi = dir == 0 ? (m0 + i) % k : ((m0 - i) % k + k) % k;
            const int wn = dir == 0 ? (wi + 1) % k : (wi + k - 1) % k;
            stop = !(sy[wn] > sy[wi]);
          }
          const unsigned sm = __ballot_sync(kFull, stop);
          if (sm) ne = q + __ffs(sm) - 1;
        }
        if (A.ne + ne > A.cap.e || A.nb >= A.cap.b) {
          A.status = kClipCapacity;
          return;
        }
        const int base = A.ne;
        for (int i = lane; i < ne; i += 32) {
          const int w = dir == 0 ? (m0 + i) % k : ((m0 - i) % k + k) % k;
          const int w2 = dir == 0 ? (w + 1) % k : (w + k - 1) % k;
          Edge &e = A.E[base + i];
          e.xb = sx[w];
          e.bx = sx[w];
          e.by = sy[w];
          e.tx = sx[w2];
          e.ty = sy[w2];
          e.dx = (sx[w2] - e.bx) / (e.ty - e.by);
          e.xt = 0.0;
          e.type = (int8_t)type;
          e.outp[0] = e.outp[1] = -1;
          e.prev = e.next = -1;
          e.succ = (ne > 1 && i < ne - 1) ? base + i + 1 : -1;
          e.bside[CLIP] = (int8_t)(op == OP_DIFF ? RIGHT : LEFT);
          e.bside[SUBJ] = LEFT;
          e.bundle[0][0] = e.bundle[0][1] = e.bundle[1][0] = e.bundle[1][1] = 0;
          e.bstate[0] = e.bstate[1] = UNBUNDLED;
        }
        if (lane == 0) {
          const int w1 = dir == 0 ? (m0 + 1) % k : (m0 + k - 1) % k;
          Bound &b = A.B[A.nb];
          b.y = sy[m0];
          b.x = sx[m0];
          b.dx = (sx[w1] - sx[m0]) / (sy[w1] - sy[m0]);
          b.edge = base;
          b.order = A.nb;
        }
        A.ne += ne;
        A.nb++;
      }
    }
  }
  __syncwarp();
}

// Ring contributions (minimax_test, GPC:1656-1709), all bounds, and the
// sorted local-minima table.  Returns false when the pair has more rings
// than the ring scratch holds.
__device__ inline bool wbuild(Arena &A, int op, const PolyView &subj, const PolyView &clip, const WAet &W) {
  const int lane = threadIdx.x & 31;
  const int sn = (int)(subj.r1 - subj.r0), cn = (int)(clip.r1 - clip.r0);
  const bool minimax = (op == OP_INT || op == OP_DIFF) && sn > 0 && cn > 0;
  double *rbb = reinterpret_cast<double *>(A.ST);  // ring boxes: subject rings, then clip rings
  if (minimax) {
    if ((size_t)(sn + cn) * 4 * sizeof(double) > sizeof(StNode) * (size_t)A.cap.st) return false;
    for (int rr = 0; rr < sn + cn; rr++) {
      const PolyView &p = rr < sn ? subj : clip;
      const int64_t r = rr < sn ? subj.r0 + rr : clip.r0 + (rr - sn);
      double b0 = kDblMax, b1 = kDblMax, b2 = -kDblMax, b3 = -kDblMax;
      for (int64_t v = p.ring_vert[r] + lane; v < p.ring_vert[r + 1]; v += 32) {
        const double x = p.xy[2 * v], y = p.xy[2 * v + 1];
        b0 = x < b0 ? x : b0;
        b1 = y < b1 ? y : b1;
        b2 = x > b2 ? x : b2;
        b3 = y > b3 ? y : b3;
      }
      for (int o = 16; o; o >>= 1) {
        double t;
        t = __shfl_xor_sync(kFull, b0, o);
        b0 = t < b0 ? t : b0;
        t = __shfl_xor_sync(kFull, b1, o);
        b1 = t < b1 ? t : b1;
        t = __shfl_xor_sync(kFull, b2, o);
        b2 = t > b2 ? t : b2;
        t = __shfl_xor_sync(kFull, b3, o);
        b3 = t > b3 ? t : b3;
      }
      if (lane == 0) {
        rbb[4 * rr] = b0;
        rbb[4 * rr + 1] = b1;
        rbb[4 * rr + 2] = b2;
        rbb[4 * rr + 3] = b3;
      }
    }
    __syncwarp();
  }
  // staged vertices of one ring: the vertex-node area, free until the beams
  double *sx = reinterpret_cast<double *>(A.V);
  double *sy = sx + A.cap.e;
  for (int pass = 0; pass < 2 && !A.status; pass++) {
    const PolyView &p = pass == 0 ? subj : clip;
    const int type = pass == 0 ? SUBJ : CLIP;
    const int nr = pass == 0 ? sn : cn;
    for (int j = 0; j < nr && !A.status; j++) {
      if (minimax && (pass == 1 || op == OP_INT)) {
        const double *own = rbb + 4 * (pass == 0 ? j : sn + j);
        const int no = pass == 0 ? cn : sn;
        bool hit = false;
        for (int k = lane; k < no; k += 32) {
          const double *oth = rbb + 4 * (pass == 0 ? sn + k : k);
          hit |= pass == 0 ? bbox_overlap(own, oth) : bbox_overlap(oth, own);
        }
        if (!__any_sync(kFull, hit)) continue;
      }
      wbuild_ring(A, p, p.r0 + j, type, op, sx, sy);
    }
  }
  if (A.status || A.nb == 0) return true;
  // local-minima table: (y, x, dx), ties in creation order
  if (A.nb <= 32) {
    // one bound per lane, placed at its rank
    const bool v = lane < A.nb;
    Bound b;
    uint64_t ky = 0, kx = 0, kd = 0;
    if (v) {
      b = A.B[lane];
      ky = dkey(b.y);
      kx = dkey(b.x);
      kd = dkey(b.dx);
    }
    int rank = 0;
    for (int k = 0; k < A.nb; k++) {
      const uint64_t oy = __shfl_sync(kFull, ky, k), ox = __shfl_sync(kFull, kx, k), od = __shfl_sync(kFull, kd, k);
      rank += oy < ky || (oy == ky && (ox < kx || (ox == kx && (od < kd || (od == kd && k < lane)))));
    }
    __syncwarp();
    if (v) A.B[rank] = b;
    __syncwarp();
    return true;
  }
  // more: three stable radix sorts, least significant key first
  uint32_t *cnt = wsm_counters(W.scap);
  Bound *bs = reinterpret_cast<Bound *>(A.IT);
  Bound *cur = warp_radix(A.B, bs, A.nb, [](const Bound &b) { return dkey(b.dx); }, cnt);
  Bound *oth = cur == A.B ? bs : A.B;
  cur = warp_radix(cur, oth, A.nb, [](const Bound &b) { return dkey(b.x); }, cnt);
  oth = cur == A.B ? bs : A.B;
  cur = warp_radix(cur, oth, A.nb, [](const Bound &b) { return dkey(b.y); }, cnt);
  if (cur != A.B) warp_copy(A.B, cur, A.nb);
  return true;
}

// ---------------------------------------------------------------- output polygons
// Output polygon nodes of the warp clipper: node k lives in shared memory
// when k < spcap, else in the arena.  The functions below are the thread
// clipper's add_local_min / add_left / add_right / merge_* (GPC:1506-1621)
// over this split store.
struct WPoly {
  PolyNode *sp;
  PolyNode *gp;
  int spcap;
  __device__ PolyNode &operator[](int k) const { return k < spcap ? sp[k] : gp[k]; }
};

__device__ inline int wp_local_min(Arena &A, const WPoly &P, int &out_poly, double x, double y) {
  if (A.np >= A.cap.p) {
    A.status = kClipCapacity;
    return -1;
  }
  int v = new_vertex(A, x, y, -1);
  if (v < 0) return -1;
  int k = A.np++;
  PolyNode &p = P[k];
  p.active = 1;
  p.hole = 0;
  p.next = out_poly;
  p.proxy = k;
  p.vl = v;
  p.vr = v;
  out_poly = k;
  return k;
}

__device__ inline void wp_add_left(Arena &A, const WPoly &P, int p, double x, double y) {
  if (p < 0) return;
  PolyNode &q = P[P[p].proxy];
  int v = new_vertex(A, x, y, q.vl);
  if (v >= 0) q.vl = v;
}

__device__ inline void wp_add_right(Arena &A, const WPoly &P, int p, double x, double y) {
  if (p < 0) return;
  PolyNode &q = P[P[p].proxy];
  int v = new_vertex(A, x, y, -1);
  if (v < 0) return;
  A.V[q.vr].next = v;
  q.vr = v;
}

// merge_left / merge_right without the redirect: returns the proxy to
// redirect (*to receives its replacement), or -1.  The redirect itself
// (every node whose proxy is the old one becomes inactive and takes the new
// one) touches every node of the output list, which holds all nodes ever
// created (nodes are only prepended); the warp does it as one parallel pass
// over the node array (wp_redirect_all), in any order, as the update is the
// same for every node.
__device__ inline int wp_merge_left(Arena &A, const WPoly &P, int p, int q, int *to) {
  if (p < 0 || q < 0) return -1;
  int pp = P[p].proxy, qp = P[q].proxy;
  P[qp].hole = 1;
  if (pp == qp) return -1;
  A.V[P[pp].vr].next = P[qp].vl;
  P[qp].vl = P[pp].vl;
  *to = qp;
  return pp;
}

__device__ inline int wp_merge_right(Arena &A, const WPoly &P, int p, int q, int *to) {
  if (p < 0 || q < 0) return -1;
  int pp = P[p].proxy, qp = P[q].proxy;
  P[qp].hole = 0;
  if (pp == qp) return -1;
  A.V[P[qp].vr].next = P[pp].vl;
  P[qp].vr = P[pp].vr;
  *to = qp;
  return pp;
}

// All lanes: nodes [0, np) whose proxy is `target` become inactive and point
// at `to` (redirect, GPC:1529-1540 / 1574-1585).
__device__ inline void wp_redirect_all(const WPoly &P, int np, int target, int to) {
  for (int k = threadIdx.x & 31; k < np; k += 32) {
    PolyNode &n = P[k];
    if (n.proxy == target) {
      n.active = 0;
      n.proxy = to;
    }
  }
  __syncwarp();
}

// Copies the shared-memory nodes to the arena (dir 0) or back (dir 1); np
// is lane 0's count.
__device__ inline void wp_sync(const WPoly &P, int np, int dir) {
  np = __shfl_sync(kFull, np, 0);
  const int m = np < P.spcap ? np : P.spcap;
  for (int k = threadIdx.x & 31; k < m; k += 32) {
    if (dir == 0) P.gp[k] = P.sp[k];
    else P.sp[k] = P.gp[k];
  }
  __syncwarp();
}

enum : int { kWarpOk = 0, kWarpFallback = 1 };

// Horizontal state before each lane's slot and after the chunk (hstate_*):
// one-sided edges (exists 1 or 2) move NH to BH/TH and BH/TH back to NH;
// two-sided edges (exists 3) swap BH and TH; `x` is the state a one-sided
// edge gives when it leaves NH.
__device__ inline int hstate_before(int carry, unsigned m1, unsigned m2, int x) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = lanemask_lt();
  const unsigned l1 = m1 & lt;
  const int j = l1 ? 31 - __clz(l1) : lane;
  const int xj = __shfl_sync(kFull, x, j);
  const bool nonNH = (carry != NH) ^ (__popc(l1) & 1);
  if (!nonNH) return NH;
  const int from = l1 ? xj : carry;
  const unsigned between = l1 ? (m2 & lt & ~((2u << j) - 1u)) : (m2 & lt);
  return (__popc(between) & 1) ? 3 - from : from;
}

__device__ inline int hstate_after(int carry, unsigned m1, unsigned m2, int x) {
  const int last = m1 ? 31 - __clz(m1) : -1;
  const int xl = __shfl_sync(kFull, x, last < 0 ? 0 : last);
  const bool nonNH = (carry != NH) ^ (__popc(m1) & 1);
  if (!nonNH) return NH;
  const int from = last >= 0 ? xl : carry;
  const unsigned between = last >= 0 ? (m2 & ~((2u << last) - 1u)) : m2;
  return (__popc(between) & 1) ? 3 - from : from;
}

// GPC's output step for one contributing slot (GPC:425-570), on one lane:
// vertex class from the slot's flags, xb its bottom x; oa / ob are the
// slot's above / below output polygons, cf the current fragment.  A contour
// merge returns in rt the proxy to redirect and in rto its replacement.
__device__ inline void wout_event(Arena &A, const WPoly &P, uint32_t fl, double xb, double yb, int &oa, int &ob, int &cf,
                                  int &out_poly, int &rt, int &rto) {
  const int vclass = (int)((fl >> W_VC) & 15u);
  const bool pxne = (fl & W_PXNE) != 0;
  switch (vclass) {
    case EMN:
    case IMN: {
      const int k = wp_local_min(A, P, out_poly, xb, yb);
      if (k >= 0) oa = k;
      cf = oa;
      break;
    }
    case ERI:
      if (pxne) wp_add_right(A, P, cf, xb, yb);
      oa = cf;
      cf = -1;
      break;
    case ELI:
      wp_add_left(A, P, ob, xb, yb);
      cf = ob;
      break;
    case EMX:
      if (pxne) wp_add_left(A, P, cf, xb, yb);
      rt = wp_merge_right(A, P, cf, ob, &rto);
      cf = -1;
      break;
    case ILI:
      if (pxne) wp_add_left(A, P, cf, xb, yb);
      oa = cf;
      cf = -1;
      break;
    case IRI:
      wp_add_right(A, P, ob, xb, yb);
      cf = ob;
      ob = -1;
      break;
    case IMX:
      if (pxne) wp_add_right(A, P, cf, xb, yb);
      rt = wp_merge_left(A, P, cf, ob, &rto);
      cf = -1;
      ob = -1;
      break;
    case IMM: {
      if (pxne) wp_add_right(A, P, cf, xb, yb);
      rt = wp_merge_left(A, P, cf, ob, &rto);
      ob = -1;
      const int k = wp_local_min(A, P, out_poly, xb, yb);
      if (k >= 0) oa = k;
      cf = oa;
      break;
    }
    case EMM: {
      if (pxne) wp_add_left(A, P, cf, xb, yb);
      rt = wp_merge_right(A, P, cf, ob, &rto);
      ob = -1;
      const int k = wp_local_min(A, P, out_poly, xb, yb);
      if (k >= 0) oa = k;
      cf = oa;
      break;
    }
    case LED:
      if (fl & W_STARTS) wp_add_left(A, P, ob, xb, yb);
      oa = ob;
      break;
    case RED:
      if (fl & W_STARTS) wp_add_right(A, P, ob, xb, yb);
      oa = ob;
      break;
    default:
      break;
  }
}

// Bundle fix-ups of deleted bundle heads (GPC:426-459), in AET order, on one
// lane.
__device__ inline void wfixups(const WAet &W, int n, double yb) {
  for (int d = 0; d < n; d++) {
    if (!(W.ty()[d] == yb && fbits(W.fl()[d], W_STB) == BUNDLE_HEAD)) continue;
    int pe = d - 1;
    while (pe >= 0 && W.ty()[pe] == yb) pe--;
    if (pe < 0) continue;
    if (fbits(W.fl()[pe], W_STB) == BUNDLE_TAIL) {
      W.outB()[pe] = W.outB()[d];
      W.fl()[pe] = fset(W.fl()[pe], W_STB, UNBUNDLED);
      int pp = pe - 1;
      while (pp >= 0 && W.ty()[pp] == yb) pp--;
      if (pp >= 0 && fbits(W.fl()[pp], W_STB) == BUNDLE_TAIL) W.fl()[pe] = fset(W.fl()[pe], W_STB, BUNDLE_HEAD);
    }
  }
}

// A beam with intersections (GPC:461-659): the slots are spilled to the
// linked form, the thread clipper's intersect_beam runs on lane 0 and the
// slots are rebuilt in the new AET order.  Returns nonzero (A.status set, or
// *mode = kWarpFallback for an AET list it leaves malformed) on failure.
__device__ __noinline__ int wintersect(Arena &A, const WAet &W, const WPoly &P, int op, int n, double yb, double dy,
                                       int &out_poly, int *mode) {
  const int lane = threadIdx.x & 31;
  for (int c = 0; c < n; c += 32) {
    const int s = c + lane;
    if (s < n) wspill(A, wload(W, s), s > 0 ? W.edge()[s - 1] : -1, s + 1 < n ? W.edge()[s + 1] : -1);
  }
  __syncwarp();
  wp_sync(P, A.np, 0);
  int bad = 0;
  if (lane == 0) {
    int aet = W.edge()[0];
    intersect_beam(A, op, aet, out_poly, yb, dy);
    if (!A.status) {
      int cur = aet, k = 0;
      while (cur >= 0 && k < n) {
        W.ord()[k++] = cur;
        cur = A.E[cur].next;
      }
      bad = (k != n || cur >= 0) ? 1 : 0;
    }
  }
  __syncwarp();
  A.status = __shfl_sync(kFull, A.status, 0);
  out_poly = __shfl_sync(kFull, out_poly, 0);
  bad = __shfl_sync(kFull, bad, 0);
  wp_sync(P, A.np, 1);
  if (bad) {
    *mode = kWarpFallback;
    return 1;
  }
  if (A.status) return 1;
  for (int c = 0; c < n; c += 32) {
    const int s = c + lane;
    WSlot v;
    if (s < n) v = wslot_of(A, W.ord()[s]);
    __syncwarp();
    if (s < n) wstore(W, s, v);
  }
  __syncwarp();
  return 0;
}

// All fields of lane src's slot (wshfl) or of the lane below (wshfl_up).
__device__ inline WSlot wshfl(const WSlot &v, int src) {
  WSlot r;
  r.xb = __shfl_sync(kFull, v.xb, src);
  r.xt = __shfl_sync(kFull, v.xt, src);
  r.dx = __shfl_sync(kFull, v.dx, src);
  r.ty = __shfl_sync(kFull, v.ty, src);
  r.bx = __shfl_sync(kFull, v.bx, src);
  r.by = __shfl_sync(kFull, v.by, src);
  r.tx = __shfl_sync(kFull, v.tx, src);
  r.edge = __shfl_sync(kFull, v.edge, src);
  r.outA = __shfl_sync(kFull, v.outA, src);
  r.outB = __shfl_sync(kFull, v.outB, src);
  r.succ = __shfl_sync(kFull, v.succ, src);
  r.fl = __shfl_sync(kFull, v.fl, src);
  return r;
}

__device__ inline WSlot wshfl_up(const WSlot &v) {
  WSlot r;
  r.xb = __shfl_up_sync(kFull, v.xb, 1);
  r.xt = __shfl_up_sync(kFull, v.xt, 1);
  r.dx = __shfl_up_sync(kFull, v.dx, 1);
  r.ty = __shfl_up_sync(kFull, v.ty, 1);
  r.bx = __shfl_up_sync(kFull, v.bx, 1);
  r.by = __shfl_up_sync(kFull, v.by, 1);
  r.tx = __shfl_up_sync(kFull, v.tx, 1);
  r.edge = __shfl_up_sync(kFull, v.edge, 1);
  r.outA = __shfl_up_sync(kFull, v.outA, 1);
  r.outB = __shfl_up_sync(kFull, v.outB, 1);
  r.succ = __shfl_up_sync(kFull, v.succ, 1);
  r.fl = __shfl_up_sync(kFull, v.fl, 1);
  return r;
}

// Source lane of each slot after GPC's swap of two crossing bundles
// (GPC:622-657): the bundle of slot l0 (with the tail slots before it, when
// l0 is a bundle head; GPC steps over l0's predecessor, then over tails) moves
// to just after slot l1, and the slots between move down.  tails: the lanes
// whose edges are bundle tails; sta0: slot l0's bundle state.
__device__ inline int wswap_src(unsigned tails, int sta0, int l0, int l1) {
  const int lane = threadIdx.x & 31;
  int b0 = l0;
  if (sta0 == BUNDLE_HEAD) {
    const unsigned others = ~tails & (l0 >= 1 ? (1u << (l0 - 1)) - 1u : 0u);
    b0 = others ? 32 - __clz(others) : 0;
  }
  const int len2 = l1 - l0;
  if (lane < b0 || lane > l1) return lane;
  return lane < b0 + len2 ? l0 + 1 + (lane - b0) : b0 + (lane - b0 - len2);
}

// GPC's output at one crossing of two contributing edges (GPC:487-619), on
// one lane: f0 / f1 are the flags of the left and right edge, o0 / o1 their
// output polygons above (updated).  A contour merge returns in rt the proxy
// to redirect and in rto its replacement.
template <int op>
__device__ inline void wcross_event(Arena &A, const WPoly &P, uint32_t f0, uint32_t f1, double ix, double iy, int &o0,
                                    int &o1, int &out_poly, int &rt, int &rto) {
  const int ba0 = fbits(f0, W_BA), ba1 = fbits(f1, W_BA), s0 = fbits(f0, W_SIDE), s1 = fbits(f1, W_SIDE);
  const int b0C = ba0 & 1, b0S = ba0 >> 1, b1C = ba1 & 1, b1S = ba1 >> 1;
  const int s0C = s0 & 1, s0S = s0 >> 1, s1C = s1 & 1, s1S = s1 >> 1;
  const int inC = (b0C && !s0C) || (b1C && s1C) || (!b0C && !b1C && s0C && s1C);
  const int inS = (b0S && !s0S) || (b1S && s1S) || (!b0S && !b1S && s0S && s1S);
  int tr, tl, br, bl;
  if (op == OP_DIFF || op == OP_INT) {
    tr = inC && inS;
    tl = (inC ^ b1C) && (inS ^ b1S);
    br = (inC ^ b0C) && (inS ^ b0S);
    bl = (inC ^ b1C ^ b0C) && (inS ^ b1S ^ b0S);
  } else if (op == OP_XOR) {
    tr = inC ^ inS;
    tl = (inC ^ b1C) ^ (inS ^ b1S);
    br = (inC ^ b0C) ^ (inS ^ b0S);
    bl = (inC ^ b1C ^ b0C) ^ (inS ^ b1S ^ b0S);
  } else {
    tr = inC || inS;
    tl = (inC ^ b1C) || (inS ^ b1S);
    br = (inC ^ b0C) || (inS ^ b0S);
    bl = (inC ^ b1C ^ b0C) || (inS ^ b1S ^ b0S);
  }
  const int p = o0, q = o1;
  switch (tr + (tl << 1) + (br << 2) + (bl << 3)) {
    case EMN:
    case IMN: {
      const int k = wp_local_min(A, P, out_poly, ix, iy);
      if (k >= 0) o0 = k;
      o1 = o0;
      break;
    }
    case ERI:
      if (p >= 0) {
        wp_add_right(A, P, p, ix, iy);
        o1 = p;
        o0 = -1;
      }
      break;
    case ELI:
      if (q >= 0) {
        wp_add_left(A, P, q, ix, iy);
        o0 = q;
        o1 = -1;
      }
      break;
    case EMX:
      if (p >= 0 && q >= 0) {
        wp_add_left(A, P, p, ix, iy);
        rt = wp_merge_right(A, P, p, q, &rto);
        o0 = -1;
        o1 = -1;
      }
      break;
    case ILI:
      if (p >= 0) {
        wp_add_left(A, P, p, ix, iy);
        o1 = p;
        o0 = -1;
      }
      break;
    case IRI:
      if (q >= 0) {
        wp_add_right(A, P, q, ix, iy);
        o0 = q;
        o1 = -1;
      }
      break;
    case IMX:
      if (p >= 0 && q >= 0) {
        wp_add_right(A, P, p, ix, iy);
        rt = wp_merge_left(A, P, p, q, &rto);
        o0 = -1;
        o1 = -1;
      }
      break;
    case IMM:
      if (p >= 0 && q >= 0) {
        wp_add_right(A, P, p, ix, iy);
        rt = wp_merge_left(A, P, p, q, &rto);
        const int k = wp_local_min(A, P, out_poly, ix, iy);
        if (k >= 0) o0 = k;
        o1 = o0;
      }
      break;
    case EMM:
      if (p >= 0 && q >= 0) {
        wp_add_left(A, P, p, ix, iy);
        rt = wp_merge_right(A, P, p, q, &rto);
        const int k = wp_local_min(A, P, out_poly, ix, iy);
        if (k >= 0) o0 = k;
        o1 = o0;
      }
      break;
    default:
      break;
  }
}

// Position of the k-th (0-based) set bit of m; m has more than k set bits.
__device__ inline int nth_bit(unsigned m, int k) {
  int pos = 0;
#pragma unroll
  for (int w = 16; w; w >>= 1) {
    const unsigned lo = m & ((1u << w) - 1u);
    const int c = __popc(lo);
    if (k >= c) {
      k -= c;
      m >>= w;
      pos += w;
    } else {
      m = lo;
    }
  }
  return pos;
}

// Beam-loop state handed between the shared-memory and the register loops.
struct WBeams {
  double yb, yt, dy, bwin;
  int n, lmin, cf, out_poly, bbase;
};

enum : int { kBeamsDone = 0, kBeamsGrow = 1, kBeamsFail = -1 };

// The scanbeam loop while the AET has at most 32 edges: slot k lives in the
// registers of lane k, so every per-slot step of the shared-memory loop in
// wclip_impl (the same steps, for one chunk of 32) runs on registers, with
// ballots and shuffles for the neighbours.  The loop starts at a beam's
// insertion step with the slots in W.  Returns kBeamsDone after the last
// beam, kBeamsFail on failure (A.status or *mode set), and kBeamsGrow when an
// insertion would make a 33rd slot: the slots are then back in W and the
// shared-memory loop goes on with the same insertion.
template <int op>
__device__ __noinline__ int wbeams_reg(Arena &A, const WAet &W, const WPoly &P, WBeams &S, int *mode) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = lanemask_lt();
  const int pC0 = op == OP_DIFF ? RIGHT : LEFT;
  // the initial sides of every edge (bside[CLIP], bside[SUBJ])
  constexpr uint32_t kSides = (uint32_t)((op == OP_DIFF ? RIGHT : LEFT) | (LEFT << 1)) << W_SIDE;
  int n = S.n, lmin = S.lmin, cf = S.cf, out_poly = S.out_poly, bbase = S.bbase;
  double yb = S.yb, yt = S.yt, dy = S.dy;
  // local-minima window: bound bbase + lane and the static fields of its
  // first edge, read 32 at a time
  double bwin = 0.0, wx = 0.0, wdx = 0.0, wtx = 0.0, wty = 0.0;
  int wedge = -1, wsucc = -1, wtype = 0;
  auto load_win = [&]() {
    const int k = bbase + lane;
    bwin = 0.0;
    if (k < A.nb) {
      const Bound &b = A.B[k];
      bwin = b.y;
      wx = b.x;
      wdx = b.dx;
      wedge = b.edge;
      const Edge &E = A.E[wedge];
      wtx = E.tx;
      wty = E.ty;
      wsucc = E.succ;
      wtype = E.type;
    }
  };
  load_win();
  auto bys = [&](int i) -> double {
    if (i - bbase >= 32) {
      bbase += 32 * ((i - bbase) / 32);
      load_win();
    }
    return __shfl_sync(kFull, bwin, i - bbase);
  };
  WSlot R;
  if (lane < n) R = wload(W, lane);
  int ret = kBeamsDone;
  for (;;) {
    // ---- local minima at yb into the AET
    bool grow = false;
    while (lmin < A.nb && bys(lmin) == yb) {
      if (n == 32) {
        grow = true;
        break;
      }
      // the bound's first edge as wslot_of would read it: an edge that has
      // not been active keeps the build's values (xb = bx = the bound's x,
      // by = its y, the bound's dx, xt = 0, no output polygons or bundles,
      // the initial sides)
      const int sl = lmin++ - bbase;
      WSlot ns;
      ns.edge = __shfl_sync(kFull, wedge, sl);
      ns.xb = ns.bx = __shfl_sync(kFull, wx, sl);
      ns.by = __shfl_sync(kFull, bwin, sl);
      ns.dx = __shfl_sync(kFull, wdx, sl);
      ns.tx = __shfl_sync(kFull, wtx, sl);
      ns.ty = __shfl_sync(kFull, wty, sl);
      ns.succ = __shfl_sync(kFull, wsucc, sl);
      ns.xt = 0.0;
      ns.outA = ns.outB = -1;
      ns.fl = (__shfl_sync(kFull, wtype, sl) ? W_TYPE : 0u) | kSides;
      const unsigned m = __ballot_sync(kFull, lane < n && (ns.xb < R.xb || (ns.xb == R.xb && ns.dx < R.dx)));
      const int pos = m ? __ffs(m) - 1 : n;
      const WSlot up = wshfl_up(R);
      if (lane > pos) R = up;
      if (lane == pos) R = ns;
      n++;
    }
    if (grow) {
      wstore(W, lane, R);
      __syncwarp();
      ret = kBeamsGrow;
      break;
    }
    if (n == 0) {
      if (lmin >= A.nb) break;
      yb = bys(lmin);
      continue;
    }
    const bool valid = lane < n;

    // ---- bundles above yb
    {
      const bool f = valid && R.ty != yb;
      const unsigned mf = __ballot_sync(kFull, f);
      const unsigned lower = mf & lt;
      const int pj = lower ? 31 - __clz(lower) : lane;
      const double pxb = __shfl_sync(kFull, R.xb, pj), pdx = __shfl_sync(kFull, R.dx, pj);
      const bool link = f && lower && fabs(pxb - R.xb) <= kEps && fabs(pdx - R.dx) <= kEps;
      const unsigned ml = __ballot_sync(kFull, link);
      int acc = f ? (1 << (R.fl & W_TYPE)) : 0;
      if (ml) {
        int ptr = link ? pj : -1;
        for (int d = 0; d < 5; d++) {
          const int src = ptr >= 0 ? ptr : lane;
          const int a2 = __shfl_sync(kFull, acc, src);
          const int p2 = __shfl_sync(kFull, ptr, src);
          if (ptr >= 0) {
            acc ^= a2;
            ptr = p2;
          }
        }
      }
      const unsigned upper = mf & ~lt & ~(1u << lane);
      const int nj = upper ? __ffs(upper) - 1 : -1;
      const bool tail = f && nj >= 0 && ((ml >> nj) & 1u);
      if (valid) {
        int ba, st;
        if (tail) {
          ba = 0;
          st = BUNDLE_TAIL;
        } else if (link) {
          ba = acc;
          st = BUNDLE_HEAD;
        } else {
          ba = acc;
          st = UNBUNDLED;
        }
        R.fl = fset(fset(R.fl, W_BA, ba), W_STA, st);
      }
    }

    // ---- parity, horizontal state, vertex classes
    unsigned mc;
    bool any_fix;
    {
      uint32_t fl = valid ? R.fl : 0u;
      const int ba = fbits(fl, W_BA), bb = fbits(fl, W_BB);
      const int aC = ba & 1, aS = ba >> 1, bC = bb & 1, bS = bb >> 1;
      const int exC = aC + (bC << 1), exS = aS + (bS << 1);
      const unsigned maC = __ballot_sync(kFull, aC), maS = __ballot_sync(kFull, aS);
      const int pCb = pC0 ^ (__popc(maC & lt) & 1), pSb = LEFT ^ (__popc(maS & lt) & 1);
      const int pCa = pCb ^ aC, pSa = pSb ^ aS;
      const unsigned m1C = __ballot_sync(kFull, exC == 1 || exC == 2), m2C = __ballot_sync(kFull, exC == 3);
      const unsigned m1S = __ballot_sync(kFull, exS == 1 || exS == 2), m2S = __ballot_sync(kFull, exS == 3);
      const int xC = ((exC == 2) ^ pCa) ? TH : BH, xS = ((exS == 2) ^ pSa) ? TH : BH;
      const int horC = hstate_before(NH, m1C, m2C, xC), horS = hstate_before(NH, m1S, m2S, xS);
      const bool exists = valid && (exC || exS);
      bool contributing = false;
      int vclass = 0;
      if (exists) {
        const int hc = horC != NH, hs = horS != NH;
        int br = 0, bl = 0, tr = 0, tl = 0;
        if (op == OP_DIFF || op == OP_INT) {
          contributing = (exC && (pSb || horS)) || (exS && (pCb || horC)) || (exC && exS && (pCb == pSb));
          br = pCb && pSb;
          bl = (pCb ^ aC) && (pSb ^ aS);
          tr = (pCb ^ hc) && (pSb ^ hs);
          tl = (pCb ^ hc ^ bC) && (pSb ^ hs ^ bS);
        } else if (op == OP_XOR) {
          contributing = exC || exS;
          br = pCb ^ pSb;
          bl = (pCb ^ aC) ^ (pSb ^ aS);
          tr = (pCb ^ hc) ^ (pSb ^ hs);
          tl = (pCb ^ hc ^ bC) ^ (pSb ^ hs ^ bS);
        } else {
          contributing = (exC && (!pSb || horS)) || (exS && (!pCb || horC)) || (exC && exS && (pCb == pSb));
          br = pCb || pSb;
          bl = (pCb ^ aC) || (pSb ^ aS);
          tr = (pCb ^ hc) || (pSb ^ hs);
          tl = (pCb ^ hc ^ bC) || (pSb ^ hs ^ bS);
        }
        vclass = tr + (tl << 1) + (br << 2) + (bl << 3);
        fl = fset(fl, W_SIDE, pCb | (pSb << 1));
        fl = (fl & ~(15u << W_VC) & ~W_STARTS & ~W_PXNE) | ((uint32_t)vclass << W_VC);
        if (contributing && (vclass == LED || vclass == RED) && R.by == yb) fl |= W_STARTS;
      }
      const bool handled = contributing && vclass != NUL && vclass != TED && vclass != BED && vclass != FUL;
      const unsigned lh = __ballot_sync(kFull, handled) & lt;
      const double xbs = valid ? R.xb : 0.0;
      const double pxl = __shfl_sync(kFull, xbs, lh ? 31 - __clz(lh) : lane);
      const double px_before = lh ? pxl : -kDblMax;
      const bool copy = contributing && (vclass == LED || vclass == RED) && !(fl & W_STARTS);
      if (exists) {
        if (xbs != px_before) fl |= W_PXNE;
        R.fl = fl;
        if (copy) R.outA = R.outB;
      }
      mc = __ballot_sync(kFull, contributing && !copy);
      any_fix = __any_sync(kFull, valid && R.ty == yb && fbits(fl, W_STB) == BUNDLE_HEAD);
    }

    // ---- output, in AET order: lane 0 runs the events, the warp the redirects
    if (mc) {
      for (unsigned m = mc; m; m &= m - 1) {
        const int s = __ffs(m) - 1;
        const uint32_t fl = __shfl_sync(kFull, R.fl, s);
        const double xb = __shfl_sync(kFull, R.xb, s);
        int oa = __shfl_sync(kFull, R.outA, s), ob = __shfl_sync(kFull, R.outB, s);
        int rt = -1, rto = -1;
        if (lane == 0 && !A.status) wout_event(A, P, fl, xb, yb, oa, ob, cf, out_poly, rt, rto);
        oa = __shfl_sync(kFull, oa, 0);
        ob = __shfl_sync(kFull, ob, 0);
        if (lane == s) {
          R.outA = oa;
          R.outB = ob;
        }
        rt = __shfl_sync(kFull, rt, 0);
        if (rt >= 0) wp_redirect_all(P, __shfl_sync(kFull, A.np, 0), rt, __shfl_sync(kFull, rto, 0));
      }
      __syncwarp();
      A.status = __shfl_sync(kFull, A.status, 0);
      out_poly = __shfl_sync(kFull, out_poly, 0);
      if (A.status) {
        ret = kBeamsFail;
        break;
      }
    }

    // ---- next scanbeam, delete edges ending at yb, compute xt
    if (any_fix) {
      if (valid) wstore(W, lane, R);
      __syncwarp();
      if (lane == 0) wfixups(W, n, yb);
      __syncwarp();
      if (valid) R = wload(W, lane);
    }
    double ny = lmin < A.nb ? bys(lmin) : kInf;
    {
      double m = valid && R.ty != yb ? R.ty : kInf;
      for (int o = 16; o; o >>= 1) {
        const double t = __shfl_xor_sync(kFull, m, o);
        m = t < m ? t : m;
      }
      ny = m < ny ? m : ny;
    }
    if (!(ny < kInf)) break;  // the last beam
    yt = ny;
    dy = yt - yb;
    {
      const bool keep = valid && R.ty != yb;
      const unsigned km = __ballot_sync(kFull, keep), vm = __ballot_sync(kFull, valid);
      if (keep) R.xt = R.ty == yt ? R.tx : R.bx + R.dx * (yt - R.by);
      if (km != vm) R = wshfl(R, lane < __popc(km) ? nth_bit(km, lane) : lane);
      n = __popc(km);
    }

    // ---- intersections
    {
      const bool v2 = lane < n;
      const bool el = v2 && (fbits(R.fl, W_STA) == BUNDLE_HEAD || fbits(R.fl, W_BA) != 0);
      const unsigned lower = __ballot_sync(kFull, el) & lt;
      const int pj = lower ? 31 - __clz(lower) : lane;
      const double qxb = __shfl_sync(kFull, R.xb, pj), qxt = __shfl_sync(kFull, R.xt, pj),
                   qdx = __shfl_sync(kFull, R.dx, pj);
      bool good = true;
      if (el && lower) {
        const double den = (qxt - qxb) - (R.xt - R.xb);
        good = R.xt >= qxt || R.dx == qdx || fabs(den) <= kEps;
      }
      if (!__all_sync(kFull, good)) {
        // the intersection table (build_intersection_table, GPC:1309-1471):
        // eligible slots enter the sorted edge table (ST) in AET order; an
        // entering edge walks the ST from its head and records a crossing
        // with every member it passes, up to the first member it stops at.
        // ST positions live in the lanes (0 = head), the stop is found with
        // one OR-reduction per entering edge.  Crossing i (in recording
        // order) goes to entry i of the slot arrays W, unused in this loop:
        // x in xb, the beam-relative y in xt, the two edges in edge / outA.
        int pos = -1, k = 0, nrec = 0;
        bool many = false;  // more than 32 crossings
        for (unsigned todo = __ballot_sync(kFull, el); todo; todo &= todo - 1) {
          const int le = __ffs(todo) - 1;
          const double exb = __shfl_sync(kFull, R.xb, le), ext = __shfl_sync(kFull, R.xt, le),
                       edx = __shfl_sync(kFull, R.dx, le);
          const int eid = __shfl_sync(kFull, R.edge, le);
          double den = 0.0;
          bool stop = false;
          if (pos >= 0) {
            den = (R.xt - R.xb) - (ext - exb);
            stop = ext >= R.xt || edx == R.dx || fabs(den) <= kEps;
          }
          const unsigned sm = __reduce_or_sync(kFull, pos >= 0 && stop ? 1u << pos : 0u);
          const int q = sm ? __ffs(sm) - 1 : k;
          if (nrec + q > 32) {
            many = true;
            break;
          }
          if (pos >= 0 && pos < q) {
            const double rr = (exb - R.xb) / den;
            const int i = nrec + pos;
            W.xb()[i] = R.xb + rr * (R.xt - R.xb);
            W.xt()[i] = rr * dy;
            W.edge()[i] = R.edge;
            W.outA()[i] = eid;
          }
          nrec += q;
          if (pos >= q) pos++;
          if (lane == le) pos = q;
          k++;
        }
        __syncwarp();
        // the table in y order, ties in recording order (add_intersection):
        // crossing `lane` has rank `rk`
        bool regular = !many;
        double cy = 0.0;
        int c0 = -1, c1 = -1, rk = 0;
        if (regular) {
          if (lane < nrec) {
            cy = W.xt()[lane];
            c0 = W.edge()[lane];
            c1 = W.outA()[lane];
          }
          for (int j = 0; j < nrec; j++) {
            const double oy = __shfl_sync(kFull, cy, j);
            rk += oy < cy || (oy == cy && j < lane);
          }
          // dry run on the edge ids and bundle states: each crossing's left
          // edge must still be left of its right edge when its turn comes
          int eid = lane < n ? R.edge : -1, sta = lane < n ? fbits(R.fl, W_STA) : 0;
          for (int r = 0; r < nrec && regular; r++) {
            const int cl = __ffs(__ballot_sync(kFull, lane < nrec && rk == r)) - 1;
            const int e0 = __shfl_sync(kFull, c0, cl), e1 = __shfl_sync(kFull, c1, cl);
            const int l0 = __ffs(__ballot_sync(kFull, eid == e0)) - 1, l1 = __ffs(__ballot_sync(kFull, eid == e1)) - 1;
            if (l0 < 0 || l1 <= l0) {
              regular = false;
              break;
            }
            const int src = wswap_src(__ballot_sync(kFull, sta == BUNDLE_TAIL), __shfl_sync(kFull, sta, l0), l0, l1);
            eid = __shfl_sync(kFull, eid, src);
            sta = __shfl_sync(kFull, sta, src);
          }
        }
        if (regular) {
          // each crossing in turn (GPC:487-657): the output event when both
          // edges contribute, the side flips, the swap of the two bundles
          bool failed = false;
          for (int r = 0; r < nrec; r++) {
            const int cl = __ffs(__ballot_sync(kFull, lane < nrec && rk == r)) - 1;
            const int e0 = __shfl_sync(kFull, c0, cl), e1 = __shfl_sync(kFull, c1, cl);
            const int l0 = __ffs(__ballot_sync(kFull, lane < n && R.edge == e0)) - 1;
            const int l1 = __ffs(__ballot_sync(kFull, lane < n && R.edge == e1)) - 1;
            const uint32_t f0 = __shfl_sync(kFull, R.fl, l0), f1 = __shfl_sync(kFull, R.fl, l1);
            int o0 = __shfl_sync(kFull, R.outA, l0), o1 = __shfl_sync(kFull, R.outA, l1);
            const double ix = W.xb()[cl], iy = __shfl_sync(kFull, cy, cl) + yb;
            const int ba0 = fbits(f0, W_BA), ba1 = fbits(f1, W_BA);
            int rt = -1, rto = -1;
            if (ba0 && ba1 && lane == 0 && !A.status) wcross_event<op>(A, P, f0, f1, ix, iy, o0, o1, out_poly, rt, rto);
            o0 = __shfl_sync(kFull, o0, 0);
            o1 = __shfl_sync(kFull, o1, 0);
            rt = __shfl_sync(kFull, rt, 0);
            if (rt >= 0) wp_redirect_all(P, __shfl_sync(kFull, A.np, 0), rt, __shfl_sync(kFull, rto, 0));
            A.status = __shfl_sync(kFull, A.status, 0);
            out_poly = __shfl_sync(kFull, out_poly, 0);
            if (A.status) {
              failed = true;
              break;
            }
            // outputs above, sides flipped by the other edge's bundle
            if (lane == l0) {
              R.outA = o0;
              R.fl ^= (uint32_t)ba1 << W_SIDE;
            }
            if (lane == l1) {
              R.outA = o1;
              R.fl ^= (uint32_t)ba0 << W_SIDE;
            }
            const unsigned tails = __ballot_sync(kFull, lane < n && fbits(R.fl, W_STA) == BUNDLE_TAIL);
            R = wshfl(R, wswap_src(tails, fbits(f0, W_STA), l0, l1));
          }
          if (failed) {
            ret = kBeamsFail;
            break;
          }
        } else {
          if (v2) wstore(W, lane, R);
          __syncwarp();
          if (wintersect(A, W, P, op, n, yb, dy, out_poly, mode)) {
            ret = kBeamsFail;
            break;
          }
          if (v2) R = wload(W, lane);
        }
      }
    }

    // ---- successors of edges ending at yt; state below := state above
    if (lane < n) {
      const int oa = R.outA, sta = fbits(R.fl, W_STA), ba = fbits(R.fl, W_BA);
      const int sc = R.ty == yt ? R.succ : -1;
      if (sc >= 0) {
        WSlot v = wslot_of(A, sc);
        v.outB = oa;
        v.fl = fset(fset(v.fl, W_STB, sta), W_BB, ba);
        v.outA = -1;
        R = v;
      } else {
        R.outB = oa;
        R.fl = fset(fset(R.fl, W_STB, sta), W_BB, ba);
        R.xb = R.xt;
        R.outA = -1;
      }
    }
    yb = yt;
  }
  S.yb = yb;
  S.yt = yt;
  S.dy = dy;
  S.bwin = bwin;  // bound bbase + lane's y: the shared-memory loop's window
  S.n = n;
  S.lmin = lmin;
  S.cf = cf;
  S.out_poly = out_poly;
  S.bbase = bbase;
  return ret;
}

template <int op>
__device__ __noinline__ int wclip_impl(Arena &A, const PolyView &subj, const PolyView &clip, WAet &W, int *mode) {
  const int lane = threadIdx.x & 31;
  *mode = kWarpOk;
  const int sn = (int)(subj.r1 - subj.r0), cn = (int)(clip.r1 - clip.r0);
  if ((sn == 0 && cn == 0) || (sn == 0 && (op == OP_INT || op == OP_DIFF)) || (cn == 0 && op == OP_INT)) return -1;
  if (!wbuild(A, op, subj, clip, W)) {
    *mode = kWarpFallback;
    return -1;
  }
  if (A.status || A.nb == 0) return -1;

  const int pC0 = op == OP_DIFF ? RIGHT : LEFT;
  const WPoly P{wsm_polys(W.scap), A.P, W.spcap};
  int n = 0;  // active edges (slots)
  int out_poly = -1, lmin = 0;
  int cf = -1;  // current output fragment; lane 0 only, carried across beams as in GPC
  double yt = 0.0, dy = 0.0;
  // the next 32 local-minimum ys, one per lane
  int bbase = 0;
  double bwin = lane < A.nb ? A.B[lane].y : 0.0;
  auto bys = [&](int i) -> double {
    if (i - bbase >= 32) {
      bbase += 32 * ((i - bbase) / 32);
      bwin = bbase + lane < A.nb ? A.B[bbase + lane].y : 0.0;
    }
    return __shfl_sync(kFull, bwin, i - bbase);
  };
  double yb = bys(0);  // the lowest vertex is a local minimum
  bool grown = false;  // this beam's insertion outgrew the register loop
  for (;;) {
    if (n <= 32 && !grown) {
      WBeams S{yb, yt, dy, bwin, n, lmin, cf, out_poly, bbase};
      const int r = wbeams_reg<op>(A, W, P, S, mode);
      yb = S.yb;
      yt = S.yt;
      dy = S.dy;
      bwin = S.bwin;
      n = S.n;
      lmin = S.lmin;
      cf = S.cf;
      out_poly = S.out_poly;
      bbase = S.bbase;
      if (r == kBeamsDone) break;
      if (r == kBeamsFail) return -1;
      grown = true;  // kBeamsGrow: the insertion goes on below
    }
    // ---- local minima at yb into the AET (add_edge_to_aet)
    while (lmin < A.nb && bys(lmin) == yb) {
      const int e = A.B[lmin++].edge;
      if (n >= W.cap) {
        // the table outgrows its slots: move it to the arena's overflow area,
        // sized for every edge of the pair
        const int big = (A.cap.e + 31) / 32 * 32;
        if (n >= big || W.base != prt_wsm) {
          *mode = kWarpFallback;
          return -1;
        }
        WAet G = W;
        G.base = reinterpret_cast<unsigned char *>(A.E) + arena_bytes(A.cap);
        G.cap = big;
        for (int k = lane; k < n; k += 32) wstore(G, k, wload(W, k));
        __syncwarp();
        W = G;
      }
      const WSlot ns = wslot_of(A, e);
      int pos = n;
      for (int c = 0; c < n; c += 32) {
        const int s = c + lane;
        bool hit = false;
        if (s < n) {
          const double sxb = W.xb()[s];
          hit = ns.xb < sxb || (ns.xb == sxb && ns.dx < W.dx()[s]);
        }
        const unsigned m = __ballot_sync(kFull, hit);
        if (m) {
          pos = c + __ffs(m) - 1;
          break;
        }
      }
      for (int c = (n - pos + 31) / 32 - 1; c >= 0; c--) {
        const int s = pos + 32 * c + lane;
        WSlot v;
        if (s < n) v = wload(W, s);
        __syncwarp();
        if (s < n) wstore(W, s + 1, v);
        __syncwarp();
      }
      if (lane == 0) wstore(W, pos, ns);
      __syncwarp();
      n++;
    }
    if (n == 0) {
      if (lmin >= A.nb) break;
      yb = bys(lmin);
      continue;
    }

    // ---- bundles above yb (GPC:371-393)
    {
      int cj = -1;   // last slot so far whose edge does not end at yb
      int cacc = 0;  // its accumulated bundle bits
      double cxb = 0.0, cdx = 0.0;
      for (int c = 0; c < n; c += 32) {
        const int s = c + lane;
        const bool valid = s < n;
        double xb = 0.0, dx = 0.0, ty = 0.0;
        uint32_t fl = 0;
        if (valid) {
          xb = W.xb()[s];
          dx = W.dx()[s];
          ty = W.ty()[s];
          fl = W.fl()[s];
        }
        const bool f = valid && ty != yb;
        const unsigned mf = __ballot_sync(kFull, f);
        const unsigned lower = mf & lanemask_lt();
        const int pj = lower ? 31 - __clz(lower) : lane;
        const double pxb = __shfl_sync(kFull, xb, pj), pdx = __shfl_sync(kFull, dx, pj);
        bool pf;
        double zxb, zdx;
        if (lower) {
          pf = true;
          zxb = pxb;
          zdx = pdx;
        } else {
          pf = cj >= 0;
          zxb = cxb;
          zdx = cdx;
        }
        const bool link = f && s > 0 && pf && fabs(zxb - xb) <= kEps && fabs(zdx - dx) <= kEps;
        const unsigned ml = __ballot_sync(kFull, link);
        // accumulated bits: XOR of onehot(type) along linked chains
        int acc = f ? (1 << (fl & W_TYPE)) : 0;
        if (ml) {
          int ptr = link ? (lower ? pj : 32) : -1;  // 32 = the carried slot of earlier chunks
          for (int d = 0; d < 5; d++) {
            const int src = (ptr >= 0 && ptr < 32) ? ptr : lane;
            const int a2 = __shfl_sync(kFull, acc, src);
            const int p2 = __shfl_sync(kFull, ptr, src);
            if (ptr >= 0 && ptr < 32) {
              acc ^= a2;
              ptr = p2;
            }
          }
          if (ptr == 32) acc ^= cacc;
        }
        // a linked successor within the chunk makes this slot a tail
        const unsigned upper = mf & ~lanemask_lt() & ~(1u << lane);
        const int nj = upper ? __ffs(upper) - 1 : -1;
        const bool tail = f && nj >= 0 && ((ml >> nj) & 1u);
        if (valid) {
          int ba, st;
          if (tail) {
            ba = 0;
            st = BUNDLE_TAIL;
          } else if (link) {
            ba = acc;
            st = BUNDLE_HEAD;
          } else {
            ba = acc;
            st = UNBUNDLED;
          }
          W.fl()[s] = fset(fset(fl, W_BA, ba), W_STA, st);
        }
        // the first linked slot of this chunk makes the carried slot a tail
        if (mf && cj >= 0) {
          const int first = __ffs(mf) - 1;
          if (((ml >> first) & 1u) && lane == 0) W.fl()[cj] = fset(fset(W.fl()[cj], W_BA, 0), W_STA, BUNDLE_TAIL);
        }
        if (mf) {
          const int lj = 31 - __clz(mf);
          cj = c + lj;
          cacc = __shfl_sync(kFull, acc, lj);
          cxb = __shfl_sync(kFull, xb, lj);
          cdx = __shfl_sync(kFull, dx, lj);
        }
        __syncwarp();
      }
    }

    // ---- parity, horizontal state, vertex classes (GPC:395-423)
    // Parity before a slot is the XOR of the above-bundle bits before it (a
    // popcount of a ballot); the horizontal state follows from the last
    // one-sided edge before it and the two-sided edges in between.
    bool any_contrib = false, any_fix = false;
    {
      int parC = pC0, parS = LEFT;
      int hC = NH, hS = NH;
      double cpx = -kDblMax;  // GPC's px carried across chunks
      for (int c = 0; c < n; c += 32) {
        const int s = c + lane;
        const bool valid = s < n;
        uint32_t fl = valid ? W.fl()[s] : 0u;
        const int ba = fbits(fl, W_BA), bb = fbits(fl, W_BB);
        const int aC = ba & 1, aS = ba >> 1, bC = bb & 1, bS = bb >> 1;
        const int exC = aC + (bC << 1), exS = aS + (bS << 1);
        const unsigned lt = lanemask_lt();
        const unsigned maC = __ballot_sync(kFull, aC), maS = __ballot_sync(kFull, aS);
        const int pCb = parC ^ (__popc(maC & lt) & 1), pSb = parS ^ (__popc(maS & lt) & 1);
        const int pCa = pCb ^ aC, pSa = pSb ^ aS;
        const unsigned m1C = __ballot_sync(kFull, exC == 1 || exC == 2), m2C = __ballot_sync(kFull, exC == 3);
        const unsigned m1S = __ballot_sync(kFull, exS == 1 || exS == 2), m2S = __ballot_sync(kFull, exS == 3);
        const int xC = ((exC == 2) ^ pCa) ? TH : BH, xS = ((exS == 2) ^ pSa) ? TH : BH;
        const int horC = hstate_before(hC, m1C, m2C, xC), horS = hstate_before(hS, m1S, m2S, xS);
        const bool exists = valid && (exC || exS);
        bool contributing = false;
        int vclass = 0;
        if (exists) {
          const int hc = horC != NH, hs = horS != NH;
          int br = 0, bl = 0, tr = 0, tl = 0;
          if (op == OP_DIFF || op == OP_INT) {
            contributing = (exC && (pSb || horS)) || (exS && (pCb || horC)) || (exC && exS && (pCb == pSb));
            br = pCb && pSb;
            bl = (pCb ^ aC) && (pSb ^ aS);
            tr = (pCb ^ hc) && (pSb ^ hs);
            tl = (pCb ^ hc ^ bC) && (pSb ^ hs ^ bS);
          } else if (op == OP_XOR) {
            contributing = exC || exS;
            br = pCb ^ pSb;
            bl = (pCb ^ aC) ^ (pSb ^ aS);
            tr = (pCb ^ hc) ^ (pSb ^ hs);
            tl = (pCb ^ hc ^ bC) ^ (pSb ^ hs ^ bS);
          } else {
            contributing = (exC && (!pSb || horS)) || (exS && (!pCb || horC)) || (exC && exS && (pCb == pSb));
            br = pCb || pSb;
            bl = (pCb ^ aC) || (pSb ^ aS);
            tr = (pCb ^ hc) || (pSb ^ hs);
            tl = (pCb ^ hc ^ bC) || (pSb ^ hs ^ bS);
          }
          vclass = tr + (tl << 1) + (br << 2) + (bl << 3);
          fl = fset(fl, W_SIDE, pCb | (pSb << 1));
          fl = (fl & ~(15u << W_VC) & ~W_STARTS & ~W_PXNE) | ((uint32_t)vclass << W_VC);
          if (contributing && (vclass == LED || vclass == RED) && W.by()[s] == yb) fl |= W_STARTS;
        }
        // GPC's px before a slot: the xb of the last contributing slot before
        // it whose class the output step handles (each of those leaves px = xb)
        const bool handled = contributing && vclass != NUL && vclass != TED && vclass != BED && vclass != FUL;
        const unsigned mh = __ballot_sync(kFull, handled);
        const unsigned lh = mh & lt;
        const double xbs = valid ? W.xb()[s] : 0.0;
        const double pxl = __shfl_sync(kFull, xbs, lh ? 31 - __clz(lh) : lane);
        const double px_before = lh ? pxl : cpx;
        if (mh) cpx = __shfl_sync(kFull, xbs, 31 - __clz(mh));
        // continuing left / right edges only pass their output polygon up:
        // done here; the rest are events for the serial step
        const bool copy = contributing && (vclass == LED || vclass == RED) && !(fl & W_STARTS);
        if (exists) {
          if (xbs != px_before) fl |= W_PXNE;
          W.fl()[s] = fl;
          if (copy) W.outA()[s] = W.outB()[s];
        }
        const unsigned mc = __ballot_sync(kFull, contributing && !copy);
        if (lane == 0) W.cmask()[c >> 5] = mc;
        any_contrib |= mc != 0;
        any_fix |= __any_sync(kFull, valid && W.ty()[s] == yb && fbits(fl, W_STB) == BUNDLE_HEAD);
        parC ^= __popc(maC) & 1;
        parS ^= __popc(maS) & 1;
        hC = hstate_after(hC, m1C, m2C, xC);
        hS = hstate_after(hS, m1S, m2S, xS);
        __syncwarp();
      }
    }

    // ---- output, in AET order (GPC:425-570): lane 0 runs GPC's serial
    // bookkeeping for the event slots; a contour merge's redirect runs on the
    // whole warp
    if (any_contrib) {
      for (int c = 0; c < n; c += 32) {
        unsigned m = W.cmask()[c >> 5];
        while (m) {
          const int s = c + __ffs(m) - 1;
          m &= m - 1;
          int rt = -1, rto = -1;
          if (lane == 0 && !A.status) wout_event(A, P, W.fl()[s], W.xb()[s], yb, W.outA()[s], W.outB()[s], cf, out_poly, rt, rto);
          rt = __shfl_sync(kFull, rt, 0);
          if (rt >= 0) {
            // the new local minimum of IMM / EMM (if any) is past the old list
            // and never has proxy rt, so the pass may include it
            wp_redirect_all(P, __shfl_sync(kFull, A.np, 0), rt, __shfl_sync(kFull, rto, 0));
          }
        }
      }
      __syncwarp();
      A.status = __shfl_sync(kFull, A.status, 0);
      out_poly = __shfl_sync(kFull, out_poly, 0);
      if (A.status) return -1;
    }

    // ---- next scanbeam, delete edges ending at yb, compute xt (GPC:426-459)
    bool last;
    {
      if (any_fix) {
        // bundle fix-ups of deleted bundle heads, in AET order (lane 0)
        if (lane == 0) wfixups(W, n, yb);
        __syncwarp();
      }
      // the next scanbeam y: the lowest top of the edges that go on, or the
      // next local minimum
      double ny = lmin < A.nb ? bys(lmin) : kInf;
      for (int c = 0; c < n; c += 32) {
        const int s = c + lane;
        const double ty = s < n ? W.ty()[s] : kInf;
        double m = ty != yb ? ty : kInf;
        for (int o = 16; o; o >>= 1) {
          const double t = __shfl_xor_sync(kFull, m, o);
          m = t < m ? t : m;
        }
        ny = m < ny ? m : ny;
      }
      last = !(ny < kInf);
      if (!last) {
        yt = ny;
        dy = yt - yb;
      }
      int kept = 0;
      for (int c = 0; c < n; c += 32) {
        const int s = c + lane;
        const bool valid = s < n;
        const double ty = valid ? W.ty()[s] : 0.0;
        const bool keep = valid && ty != yb;
        const unsigned m = __ballot_sync(kFull, keep);
        const unsigned vm = __ballot_sync(kFull, valid);
        double xt = 0.0;
        if (keep) {
          if (ty == yt) xt = W.tx()[s];
          else xt = W.bx()[s] + W.dx()[s] * (yt - W.by()[s]);
        }
        if (kept == c && m == vm) {
          if (keep) W.xt()[s] = xt;  // nothing deleted so far: in place
        } else {
          WSlot v;
          if (keep) {
            v = wload(W, s);
            v.xt = xt;
          }
          __syncwarp();
          if (keep) wstore(W, kept + __popc(m & lanemask_lt()), v);
        }
        kept += __popc(m);
        __syncwarp();
      }
      n = kept;
    }
    if (last) break;

    // ---- intersections (GPC:461-659)
    {
      bool ok = true;
      bool hp = false;  // an eligible slot was seen in earlier chunks
      double hxb = 0.0, hxt = 0.0, hdx = 0.0;
      for (int c = 0; c < n; c += 32) {
        const int s = c + lane;
        bool el = false;
        double xb = 0.0, xt = 0.0, dx = 0.0;
        if (s < n) {
          const uint32_t fl = W.fl()[s];
          el = fbits(fl, W_STA) == BUNDLE_HEAD || fbits(fl, W_BA) != 0;
          xb = W.xb()[s];
          xt = W.xt()[s];
          dx = W.dx()[s];
        }
        const unsigned me = __ballot_sync(kFull, el);
        const unsigned lower = me & lanemask_lt();
        const int pj = lower ? 31 - __clz(lower) : lane;
        const double qxb = __shfl_sync(kFull, xb, pj), qxt = __shfl_sync(kFull, xt, pj),
                     qdx = __shfl_sync(kFull, dx, pj);
        bool has = lower != 0;
        double sxb = qxb, sxt = qxt, sdx = qdx;
        if (!lower) {
          has = hp;
          sxb = hxb;
          sxt = hxt;
          sdx = hdx;
        }
        bool good = true;
        if (el && has) {
          const double den = (sxt - sxb) - (xt - xb);
          good = xt >= sxt || dx == sdx || fabs(den) <= kEps;
        }
        ok &= __all_sync(kFull, good);
        if (me) {
          const int lj = 31 - __clz(me);
          hp = true;
          hxb = __shfl_sync(kFull, xb, lj);
          hxt = __shfl_sync(kFull, xt, lj);
          hdx = __shfl_sync(kFull, dx, lj);
        }
      }
      if (!ok && wintersect(A, W, P, op, n, yb, dy, out_poly, mode)) return -1;
    }

    // ---- successors of edges ending at yt; state below := state above (GPC:661-693)
    for (int c = 0; c < n; c += 32) {
      const int s = c + lane;
      if (s < n) {
        const uint32_t fl = W.fl()[s];
        const int oa = W.outA()[s], sta = fbits(fl, W_STA), ba = fbits(fl, W_BA);
        const int sc = W.ty()[s] == yt ? W.succ()[s] : -1;
        if (sc >= 0) {
          WSlot v = wslot_of(A, sc);
          v.outB = oa;
          v.fl = fset(fset(v.fl, W_STB, sta), W_BB, ba);
          v.outA = -1;
          wstore(W, s, v);
        } else {
          W.outB()[s] = oa;
          W.fl()[s] = fset(fset(fl, W_STB, sta), W_BB, ba);
          W.xb()[s] = W.xt()[s];
          W.outA()[s] = -1;
        }
      }
    }
    __syncwarp();
    yb = yt;
    grown = false;
  }
  wp_sync(P, A.np, 0);  // the result readers use the arena's nodes
  return out_poly;
}

// Clips subj against clip with the calling warp (all 32 lanes, converged).
// Returns the output polygon list head on every lane; A.status is valid on
// every lane, the output counters (np, nvx) on lane 0.  *mode =
// kWarpFallback when the pair needs the thread clipper (the arena is then in
// an undefined state).
__device__ inline int wclip_pair(Arena &A, int op, const PolyView &subj, const PolyView &clip, WAet &W, int *mode) {
  switch (op) {
    case OP_DIFF: return wclip_impl<OP_DIFF>(A, subj, clip, W, mode);
    case OP_INT: return wclip_impl<OP_INT>(A, subj, clip, W, mode);
    case OP_XOR: return wclip_impl<OP_XOR>(A, subj, clip, W, mode);
    default: return wclip_impl<OP_UNION>(A, subj, clip, W, mode);
  }
}

}  // namespace gpc
}  // namespace prt
