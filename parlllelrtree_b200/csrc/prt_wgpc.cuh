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
//   insertion of the beam's local minima   ballot for the insertion point, shift
//   bundle detection (GPC:371-393)          segmented XOR scan over the edges
//                                           that do not end at yb
//   parity and horizontal state (GPC:395-423) XOR scans and a scan of the
//                                           3-state transition functions
//   vertex classes                          per slot from the scanned state
//   output (GPC:425-570)                    lane 0, only for contributing slots,
//                                           in AET order (the output lists are
//                                           the reference's linked structure)
//   deletion of terminating edges, xt       ballot compaction
//   intersection test (GPC:461-485)         fast check that the ST insertion
//                                           would record no intersection; a beam
//                                           that has intersections spills the
//                                           slots to the linked form and runs the
//                                           thread clipper's intersect_beam
//   successor edges (GPC:661-693)           per slot
// The build phase (local-minima table, scanbeam table) is parallel too: ring
// staging by ballot, bound edges written by the whole warp, stable warp radix
// sorts instead of the heap sort.  Any case the slot array cannot hold (more
// active edges than slots, an AET list the intersection step left malformed,
// more rings than the ring scratch holds) makes the caller rerun the pair with
// the thread clipper, so the result is always the thread clipper's.
#pragma once
#include "prt_gpc.cuh"

namespace prt {
namespace gpc {

constexpr unsigned kFull = 0xffffffffu;

// Slot flag bits.
enum : uint32_t {
  W_TYPE = 1u,             // SUBJ edge
  W_BA = 1,                // bits 1-2: bundle[ABOVE][CLIP], [SUBJ]
  W_BB = 3,                // bits 3-4: bundle[BELOW]
  W_SIDE = 5,              // bits 5-6: bside[CLIP], bside[SUBJ]
  W_STA = 7,               // bits 7-8: bstate[ABOVE]
  W_STB = 9,               // bits 9-10: bstate[BELOW]
  W_VC = 11,               // bits 11-14: vertex class
  W_CONTRIB = 1u << 15,
  W_STARTS = 1u << 16,     // the edge starts at yb
};

__device__ inline int fbits(uint32_t f, int sh) { return (int)((f >> sh) & 3u); }
__device__ inline uint32_t fset(uint32_t f, int sh, int v) { return (f & ~(3u << sh)) | ((uint32_t)v << sh); }

struct WSlot {
  double xb, xt, dx, ty;
  int32_t edge, outA, outB;
  uint32_t fl;
};

// Shared-memory slot arrays of one warp (structure of arrays).
struct WAet {
  double *xb, *xt, *dx, *ty;
  int32_t *edge, *outA, *outB, *ord;
  uint32_t *fl;
  uint32_t *cnt;  // 256 radix counters
  int cap;
};

__host__ __device__ inline size_t waet_bytes(int cap) { return (size_t)cap * (4 * 8 + 5 * 4) + 256 * 4; }

__device__ inline WAet waet_carve(unsigned char *smem, int cap) {
  WAet w;
  w.cap = cap;
  double *d = reinterpret_cast<double *>(smem);
  w.xb = d;
  w.xt = d + cap;
  w.dx = d + 2 * cap;
  w.ty = d + 3 * cap;
  int32_t *i = reinterpret_cast<int32_t *>(d + 4 * cap);
  w.edge = i;
  w.outA = i + cap;
  w.outB = i + 2 * cap;
  w.ord = i + 3 * cap;
  w.fl = reinterpret_cast<uint32_t *>(i + 4 * cap);
  w.cnt = w.fl + cap;
  return w;
}

__device__ inline WSlot wload(const WAet &w, int s) {
  WSlot v;
  v.xb = w.xb[s];
  v.xt = w.xt[s];
  v.dx = w.dx[s];
  v.ty = w.ty[s];
  v.edge = w.edge[s];
  v.outA = w.outA[s];
  v.outB = w.outB[s];
  v.fl = w.fl[s];
  return v;
}

__device__ inline void wstore(const WAet &w, int s, const WSlot &v) {
  w.xb[s] = v.xb;
  w.xt[s] = v.xt;
  w.dx[s] = v.dx;
  w.ty[s] = v.ty;
  w.edge[s] = v.edge;
  w.outA[s] = v.outA;
  w.outB[s] = v.outB;
  w.fl[s] = v.fl;
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
// warp-wide walk and its edges are written in parallel.  Edges, bounds and
// scanbeam entries come out in the thread clipper's order.
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
      if (A.ny + kk < A.cap.y) {
        A.Y[A.ny + kk].y = y;
        A.Y[A.ny + kk].order = A.ny + kk;
      }
    }
    k += __popc(m);
  }
  if (A.ny + k > A.cap.y) {
    A.status = kClipCapacity;
    return;
  }
  A.ny += k;
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

// Ring contributions (minimax_test, GPC:1656-1709) and all bounds; then the
// sorted local-minima table and the sorted unique scanbeam table.  Returns
// false when the pair has more rings than the ring scratch holds.
__device__ inline bool wbuild(Arena &A, int op, const PolyView &subj, const PolyView &clip, WAet &W, int *nsbt) {
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
  // local-minima table: (y, x, dx), ties in creation order = three stable
  // passes, least significant key first
  Bound *bs = reinterpret_cast<Bound *>(A.IT);
  Bound *cur = warp_radix(A.B, bs, A.nb, [](const Bound &b) { return dkey(b.dx); }, W.cnt);
  Bound *oth = cur == A.B ? bs : A.B;
  cur = warp_radix(cur, oth, A.nb, [](const Bound &b) { return dkey(b.x); }, W.cnt);
  oth = cur == A.B ? bs : A.B;
  cur = warp_radix(cur, oth, A.nb, [](const Bound &b) { return dkey(b.y); }, W.cnt);
  if (cur != A.B) warp_copy(A.B, cur, A.nb);
  YKey *ys = reinterpret_cast<YKey *>(A.ST);
  YKey *yc = warp_radix(A.Y, ys, A.ny, [](const YKey &k) { return dkey(k.y); }, W.cnt);
  if (yc != A.Y) warp_copy(A.Y, yc, A.ny);
  // unique y, compacted in place
  int cnt = 0;
  double last = 0.0;
  for (int c = 0; c < A.ny; c += 32) {
    const int i = c + lane;
    double y = 0.0, prev = 0.0;
    if (i < A.ny) y = A.Y[i].y;
    prev = __shfl_up_sync(kFull, y, 1);
    if (lane == 0) prev = last;
    const bool keep = i < A.ny && (i == 0 || y > prev);
    const unsigned m = __ballot_sync(kFull, keep);
    last = __shfl_sync(kFull, y, 31);
    __syncwarp();
    if (keep) A.Y[cnt + __popc(m & lanemask_lt())].y = y;
    cnt += __popc(m);
    __syncwarp();
  }
  *nsbt = cnt;
  return true;
}

__constant__ int8_t c_wnext_h[3][6] = {{BH, TH, TH, BH, NH, NH}, {NH, NH, NH, NH, TH, TH}, {NH, NH, NH, NH, BH, BH}};

// 3-state transition function packed as 2 bits per state.
__device__ inline uint32_t hf_apply(uint32_t f, int h) { return (f >> (2 * h)) & 3u; }
__device__ inline uint32_t hf_compose(uint32_t later, uint32_t earlier) {  // later(earlier(h))
  return hf_apply(later, (int)hf_apply(earlier, 0)) | (hf_apply(later, (int)hf_apply(earlier, 1)) << 2) |
         (hf_apply(later, (int)hf_apply(earlier, 2)) << 4);
}
constexpr uint32_t kHfIdentity = 0u | (1u << 2) | (2u << 4);

__device__ inline int w_add_local_min(Arena &A, int &out_poly, double x, double y) {
  if (A.np >= A.cap.p) {
    A.status = kClipCapacity;
    return -1;
  }
  int v = new_vertex(A, x, y, -1);
  if (v < 0) return -1;
  int k = A.np++;
  PolyNode &p = A.P[k];
  p.active = 1;
  p.hole = 0;
  p.next = out_poly;
  p.proxy = k;
  p.vl = v;
  p.vr = v;
  out_poly = k;
  return k;
}

enum : int { kWarpOk = 0, kWarpFallback = 1 };

// Clips subj against clip with the calling warp (all 32 lanes, converged).
// Returns the output polygon list head on every lane; A.status and the
// output counters are valid on every lane.  *mode = kWarpFallback when the
// pair needs the thread clipper (the arena is then in an undefined state).
__device__ int wclip_pair(Arena &A, int op, const PolyView &subj, const PolyView &clip, WAet &W, int *mode) {
  const int lane = threadIdx.x & 31;
  *mode = kWarpOk;
  const int sn = (int)(subj.r1 - subj.r0), cn = (int)(clip.r1 - clip.r0);
  if ((sn == 0 && cn == 0) || (sn == 0 && (op == OP_INT || op == OP_DIFF)) || (cn == 0 && op == OP_INT)) return -1;
  int nsbt = 0;
  if (!wbuild(A, op, subj, clip, W, &nsbt)) {
    *mode = kWarpFallback;
    return -1;
  }
  if (A.status || A.nb == 0) return -1;

  const int pC0 = op == OP_DIFF ? RIGHT : LEFT;
  int n = 0;  // active edges (slots)
  int out_poly = -1, lmin = 0, scanbeam = 0;
  int cf = -1;  // current output fragment; lane 0 only, carried across beams as in GPC
  double yb, yt = 0.0, dy = 0.0;
  while (scanbeam < nsbt) {
    yb = A.Y[scanbeam++].y;
    if (scanbeam < nsbt) {
      yt = A.Y[scanbeam].y;
      dy = yt - yb;
    }
    // ---- local minima at yb into the AET (add_edge_to_aet)
    while (lmin < A.nb && A.B[lmin].y == yb) {
      const int e = A.B[lmin++].edge;
      if (n >= W.cap) {
        *mode = kWarpFallback;
        return -1;
      }
      const WSlot ns = wslot_of(A, e);
      int pos = n;
      for (int c = 0; c < n; c += 32) {
        const int s = c + lane;
        bool hit = false;
        if (s < n) {
          const double sxb = W.xb[s];
          hit = ns.xb < sxb || (ns.xb == sxb && ns.dx < W.dx[s]);
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
    if (n == 0) continue;

    // ---- bundles above yb (GPC:371-393)
    {
      int cj = -1;       // last slot so far whose edge does not end at yb
      int cacc = 0;      // its accumulated bundle bits
      double cxb = 0.0, cdx = 0.0;
      for (int c = 0; c < n; c += 32) {
        const int s = c + lane;
        const bool valid = s < n;
        double xb = 0.0, dx = 0.0, ty = 0.0;
        uint32_t fl = 0;
        if (valid) {
          xb = W.xb[s];
          dx = W.dx[s];
          ty = W.ty[s];
          fl = W.fl[s];
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
          W.fl[s] = fset(fset(fl, W_BA, ba), W_STA, st);
        }
        // the first linked slot of this chunk makes the carried slot a tail
        if (mf && cj >= 0) {
          const int first = __ffs(mf) - 1;
          if (((ml >> first) & 1u) && lane == 0) W.fl[cj] = fset(fset(W.fl[cj], W_BA, 0), W_STA, BUNDLE_TAIL);
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
    unsigned any_contrib = 0;
    {
      int parC = pC0, parS = LEFT;
      int hC = NH, hS = NH;
      for (int c = 0; c < n; c += 32) {
        const int s = c + lane;
        const bool valid = s < n;
        uint32_t fl = valid ? W.fl[s] : 0u;
        const int ba = fbits(fl, W_BA), bb = fbits(fl, W_BB);
        const int aC = ba & 1, aS = ba >> 1, bC = bb & 1, bS = bb >> 1;
        const int exC = aC + (bC << 1), exS = aS + (bS << 1);
        // exclusive XOR scans of the parities
        int xC = aC, xS = aS;
        for (int d = 1; d < 32; d <<= 1) {
          const int tC = __shfl_up_sync(kFull, xC, d), tS = __shfl_up_sync(kFull, xS, d);
          if (lane >= d) {
            xC ^= tC;
            xS ^= tS;
          }
        }
        const int pCb = parC ^ xC ^ aC, pSb = parS ^ xS ^ aS;  // before this slot
        const int pCa = pCb ^ aC, pSa = pSb ^ aS;              // after it
        // horizontal-state transitions, composed by an inclusive scan
        uint32_t fC = kHfIdentity, fS = kHfIdentity;
        if (exC) {
          const int col = ((exC - 1) << 1) + pCa;
          fC = (uint32_t)c_wnext_h[0][col] | ((uint32_t)c_wnext_h[1][col] << 2) | ((uint32_t)c_wnext_h[2][col] << 4);
        }
        if (exS) {
          const int col = ((exS - 1) << 1) + pSa;
          fS = (uint32_t)c_wnext_h[0][col] | ((uint32_t)c_wnext_h[1][col] << 2) | ((uint32_t)c_wnext_h[2][col] << 4);
        }
        for (int d = 1; d < 32; d <<= 1) {
          const uint32_t tC = __shfl_up_sync(kFull, fC, d), tS = __shfl_up_sync(kFull, fS, d);
          if (lane >= d) {
            fC = hf_compose(fC, tC);
            fS = hf_compose(fS, tS);
          }
        }
        uint32_t eC = __shfl_up_sync(kFull, fC, 1), eS = __shfl_up_sync(kFull, fS, 1);
        if (lane == 0) {
          eC = kHfIdentity;
          eS = kHfIdentity;
        }
        const int horC = (int)hf_apply(eC, hC), horS = (int)hf_apply(eS, hS);
        const bool exists = valid && (exC || exS);
        bool contributing = false;
        if (exists) {
          const int hc = horC != NH, hs = horS != NH;
          int br = 0, bl = 0, tr = 0, tl = 0;
          switch (op) {
            case OP_DIFF:
            case OP_INT:
              contributing = (exC && (pSb || horS)) || (exS && (pCb || horC)) || (exC && exS && (pCb == pSb));
              br = pCb && pSb;
              bl = (pCb ^ aC) && (pSb ^ aS);
              tr = (pCb ^ hc) && (pSb ^ hs);
              tl = (pCb ^ hc ^ bC) && (pSb ^ hs ^ bS);
              break;
            case OP_XOR:
              contributing = exC || exS;
              br = pCb ^ pSb;
              bl = (pCb ^ aC) ^ (pSb ^ aS);
              tr = (pCb ^ hc) ^ (pSb ^ hs);
              tl = (pCb ^ hc ^ bC) ^ (pSb ^ hs ^ bS);
              break;
            default:
              contributing = (exC && (!pSb || horS)) || (exS && (!pCb || horC)) || (exC && exS && (pCb == pSb));
              br = pCb || pSb;
              bl = (pCb ^ aC) || (pSb ^ aS);
              tr = (pCb ^ hc) || (pSb ^ hs);
              tl = (pCb ^ hc ^ bC) || (pSb ^ hs ^ bS);
              break;
          }
          const int vclass = tr + (tl << 1) + (br << 2) + (bl << 3);
          fl = fset(fl, W_SIDE, pCb | (pSb << 1));
          fl = (fl & ~(15u << W_VC) & ~W_CONTRIB & ~W_STARTS) | ((uint32_t)vclass << W_VC);
          if (contributing) {
            fl |= W_CONTRIB;
            if ((vclass == LED || vclass == RED) && A.E[W.edge[s]].by == yb) fl |= W_STARTS;
          }
          W.fl[s] = fl;
        } else if (valid) {
          W.fl[s] = fl & ~W_CONTRIB;
        }
        any_contrib |= __ballot_sync(kFull, contributing);
        const int lastC = __shfl_sync(kFull, pCa, 31), lastS = __shfl_sync(kFull, pSa, 31);
        const uint32_t gC = __shfl_sync(kFull, fC, 31), gS = __shfl_sync(kFull, fS, 31);
        parC = lastC;
        parS = lastS;
        hC = (int)hf_apply(gC, hC);
        hS = (int)hf_apply(gS, hS);
        __syncwarp();
      }
    }

    // ---- output, in AET order (lane 0; GPC:425-570)
    if (any_contrib) {
      if (lane == 0) {
        double px = -kDblMax;
        for (int s = 0; s < n && !A.status; s++) {
          const uint32_t fl = W.fl[s];
          if (!(fl & W_CONTRIB)) continue;
          const int vclass = (int)((fl >> W_VC) & 15u);
          const double xb = W.xb[s];
          int &oa = W.outA[s];
          int &ob = W.outB[s];
          switch (vclass) {
            case EMN:
            case IMN: {
              const int k = w_add_local_min(A, out_poly, xb, yb);
              if (k >= 0) oa = k;
              px = xb;
              cf = oa;
              break;
            }
            case ERI:
              if (xb != px) {
                add_right(A, cf, xb, yb);
                px = xb;
              }
              oa = cf;
              cf = -1;
              break;
            case ELI:
              add_left(A, ob, xb, yb);
              px = xb;
              cf = ob;
              break;
            case EMX:
              if (xb != px) {
                add_left(A, cf, xb, yb);
                px = xb;
              }
              merge_right(A, cf, ob, out_poly);
              cf = -1;
              break;
            case ILI:
              if (xb != px) {
                add_left(A, cf, xb, yb);
                px = xb;
              }
              oa = cf;
              cf = -1;
              break;
            case IRI:
              add_right(A, ob, xb, yb);
              px = xb;
              cf = ob;
              ob = -1;
              break;
            case IMX:
              if (xb != px) {
                add_right(A, cf, xb, yb);
                px = xb;
              }
              merge_left(A, cf, ob, out_poly);
              cf = -1;
              ob = -1;
              break;
            case IMM: {
              if (xb != px) {
                add_right(A, cf, xb, yb);
                px = xb;
              }
              merge_left(A, cf, ob, out_poly);
              ob = -1;
              const int k = w_add_local_min(A, out_poly, xb, yb);
              if (k >= 0) oa = k;
              cf = oa;
              break;
            }
            case EMM: {
              if (xb != px) {
                add_left(A, cf, xb, yb);
                px = xb;
              }
              merge_right(A, cf, ob, out_poly);
              ob = -1;
              const int k = w_add_local_min(A, out_poly, xb, yb);
              if (k >= 0) oa = k;
              cf = oa;
              break;
            }
            case LED:
              if (fl & W_STARTS) add_left(A, ob, xb, yb);
              oa = ob;
              px = xb;
              break;
            case RED:
              if (fl & W_STARTS) add_right(A, ob, xb, yb);
              oa = ob;
              px = xb;
              break;
            default:
              break;
          }
        }
      }
      __syncwarp();
      A.status = __shfl_sync(kFull, A.status, 0);
      out_poly = __shfl_sync(kFull, out_poly, 0);
      if (A.status) return -1;
    }

    // ---- delete edges ending at yb, compute xt (GPC:426-459)
    {
      // bundle fix-ups of deleted bundle heads, in AET order (lane 0)
      bool fix = false;
      for (int c = 0; c < n; c += 32) {
        const int s = c + lane;
        fix |= s < n && W.ty[s] == yb && fbits(W.fl[s], W_STB) == BUNDLE_HEAD;
      }
      if (__any_sync(kFull, fix)) {
        if (lane == 0) {
          for (int d = 0; d < n; d++) {
            if (!(W.ty[d] == yb && fbits(W.fl[d], W_STB) == BUNDLE_HEAD)) continue;
            int pe = d - 1;
            while (pe >= 0 && W.ty[pe] == yb) pe--;
            if (pe < 0) continue;
            if (fbits(W.fl[pe], W_STB) == BUNDLE_TAIL) {
              W.outB[pe] = W.outB[d];
              W.fl[pe] = fset(W.fl[pe], W_STB, UNBUNDLED);
              int pp = pe - 1;
              while (pp >= 0 && W.ty[pp] == yb) pp--;
              if (pp >= 0 && fbits(W.fl[pp], W_STB) == BUNDLE_TAIL) W.fl[pe] = fset(W.fl[pe], W_STB, BUNDLE_HEAD);
            }
          }
        }
        __syncwarp();
      }
      int kept = 0;
      for (int c = 0; c < n; c += 32) {
        const int s = c + lane;
        WSlot v;
        bool keep = false;
        if (s < n) {
          v = wload(W, s);
          keep = v.ty != yb;
          if (keep) {
            const Edge &E = A.E[v.edge];
            if (v.ty == yt) v.xt = E.tx;
            else v.xt = E.bx + v.dx * (yt - E.by);
          }
        }
        const unsigned m = __ballot_sync(kFull, keep);
        __syncwarp();
        if (keep) wstore(W, kept + __popc(m & lanemask_lt()), v);
        kept += __popc(m);
        __syncwarp();
      }
      n = kept;
    }
    if (scanbeam >= nsbt) continue;

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
          const uint32_t fl = W.fl[s];
          el = fbits(fl, W_STA) == BUNDLE_HEAD || fbits(fl, W_BA) != 0;
          xb = W.xb[s];
          xt = W.xt[s];
          dx = W.dx[s];
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
      if (!ok) {
        // spill to the linked form, run the thread clipper's step, reload
        for (int c = 0; c < n; c += 32) {
          const int s = c + lane;
          if (s < n) wspill(A, wload(W, s), s > 0 ? W.edge[s - 1] : -1, s + 1 < n ? W.edge[s + 1] : -1);
        }
        __syncwarp();
        int bad = 0;
        if (lane == 0) {
          int aet = W.edge[0];
          intersect_beam(A, op, aet, out_poly, yb, dy);
          if (!A.status) {
            int cur = aet, k = 0;
            while (cur >= 0 && k < n) {
              W.ord[k++] = cur;
              cur = A.E[cur].next;
            }
            bad = (k != n || cur >= 0) ? 1 : 0;
          }
        }
        __syncwarp();
        A.status = __shfl_sync(kFull, A.status, 0);
        out_poly = __shfl_sync(kFull, out_poly, 0);
        bad = __shfl_sync(kFull, bad, 0);
        if (bad) {
          *mode = kWarpFallback;
          return -1;
        }
        if (A.status) return -1;
        for (int c = 0; c < n; c += 32) {
          const int s = c + lane;
          WSlot v;
          if (s < n) v = wslot_of(A, W.ord[s]);
          __syncwarp();
          if (s < n) wstore(W, s, v);
        }
        __syncwarp();
      }
    }

    // ---- successors of edges ending at yt; state below := state above (GPC:661-693)
    for (int c = 0; c < n; c += 32) {
      const int s = c + lane;
      if (s < n) {
        WSlot v = wload(W, s);
        const int oa = v.outA, sta = fbits(v.fl, W_STA), ba = fbits(v.fl, W_BA);
        const int sc = v.ty == yt ? A.E[v.edge].succ : -1;
        if (sc >= 0) {
          v = wslot_of(A, sc);
        } else {
          v.xb = v.xt;
        }
        v.outB = oa;
        v.fl = fset(fset(v.fl, W_STB, sta), W_BB, ba);
        v.outA = -1;
        wstore(W, s, v);
      }
    }
    __syncwarp();
  }
  return out_poly;
}

}  // namespace gpc
}  // namespace prt
