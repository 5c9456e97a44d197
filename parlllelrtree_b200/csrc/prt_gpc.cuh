// Device GPC clipper: the Vatti scanbeam algorithm of the General Polygon
// Clipper with the reference's semantics (vector_map_overlay_gpc_kernel.cu:
// 115-750, helpers 890-1709), for ONE pair per calling thread.
//
// The reference builds linked lists with device malloc per node; here every
// list lives in a fixed-capacity arena slice owned by the thread and is linked
// by int32 indices:
//   E   edge table (bounds are contiguous runs, successor = index + 1)
//   B   local-minimum table: bounds ordered by (y, bot.x, dx), ties in
//       creation order (insert_bound / bound_list, GPC:929-1015)
//   Y   scanbeam table: sorted unique vertex y (add_to_sbtree/build_sbt,
//       GPC:1019-1085 -- a sorted array instead of an unbalanced BST)
//   IT  intersection table of the current scanbeam, ordered by y, ties
//       appended (add_intersection GPC:1357-1393)
//   ST  sorted edge table of the current scanbeam (add_st_edge GPC:1395-1445)
//   P/V output polygons and vertex lists (GPC:1506-1621)
// Every arithmetic expression is the reference's, evaluated in FP64 without
// contraction (the file is compiled with -fmad=false), so contours, hole flags
// and vertex order equal the reference's.  A full arena sets
// kClipCapacity in the pair status instead of corrupting memory; the host
// retries such pairs with larger slices.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace prt {
namespace gpc {

enum : int { LEFT = 0, RIGHT = 1, ABOVE = 0, BELOW = 1, CLIP = 0, SUBJ = 1 };
enum : int { OP_DIFF = 0, OP_INT = 1, OP_XOR = 2, OP_UNION = 3 };
enum : int { NUL = 0, EMX, ELI, TED, ERI, RED, IMM, IMN, EMN, EMM, LED, ILI, BED, IRI, IMX, FUL };
enum : int { NH = 0, BH = 1, TH = 2 };
enum : int { UNBUNDLED = 0, BUNDLE_HEAD = 1, BUNDLE_TAIL = 2 };

constexpr double kEps = 2.2204460492503131e-16;  // DBL_EPSILON
constexpr double kDblMax = 1.7976931348623157e308;

enum : int { kClipOk = 0, kClipCapacity = 1, kClipInvalid = 2 };

struct Edge {
  double bx, by, tx, ty;
  double xb, xt, dx;
  int32_t outp[2];
  int32_t prev, next, succ;
  int8_t type;
  int8_t bundle[2][2];
  int8_t bside[2];
  int8_t bstate[2];
};

struct Bound {
  double y, x, dx;
  int32_t edge, order;
};

struct YKey {
  double y;
  int32_t order, pad;
};

struct ItNode {
  double x, y;
  int32_t e0, e1, next, pad;
};

struct StNode {
  double xb, xt, dx;
  int32_t edge, prev;
};

struct PolyNode {
  int32_t active, hole, vl, vr, next, proxy;
};

struct VertNode {
  double x, y;
  int32_t next, pad;
};

// Capacities of one arena slice, derived from the pair's vertex count.
struct Caps {
  int32_t e, b, y, it, st, p, v;
};

__host__ __device__ inline Caps caps_for(int64_t nv, int scale) {
  Caps c;
  int32_t n = (int32_t)(nv < 4 ? 4 : nv);
  c.e = n;
  c.b = n;
  c.y = n;
  c.st = n;
  c.it = scale * (n < 32 ? 32 : n);
  c.p = scale * (n / 2 + 16);
  c.v = scale * (2 * n + 32);
  return c;
}

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

// Bytes of one slice.
__host__ __device__ inline size_t arena_bytes(const Caps &c) {
  return align16(sizeof(Edge) * c.e) + align16(sizeof(Bound) * c.b) + align16(sizeof(YKey) * c.y) +
         align16(sizeof(ItNode) * c.it) + align16(sizeof(StNode) * c.st) + align16(sizeof(PolyNode) * c.p) +
         align16(sizeof(VertNode) * c.v);
}

struct Arena {
  Caps cap;
  Edge *E;
  Bound *B;
  YKey *Y;
  ItNode *IT;
  StNode *ST;
  PolyNode *P;
  VertNode *V;
  int32_t ne, nb, ny, nit, nst, np, nvx;
  int status;
};

__device__ inline void arena_init(Arena &a, unsigned char *base, const Caps &c) {
  a.cap = c;
  size_t o = 0;
  a.E = reinterpret_cast<Edge *>(base + o);
  o += align16(sizeof(Edge) * c.e);
  a.B = reinterpret_cast<Bound *>(base + o);
  o += align16(sizeof(Bound) * c.b);
  a.Y = reinterpret_cast<YKey *>(base + o);
  o += align16(sizeof(YKey) * c.y);
  a.IT = reinterpret_cast<ItNode *>(base + o);
  o += align16(sizeof(ItNode) * c.it);
  a.ST = reinterpret_cast<StNode *>(base + o);
  o += align16(sizeof(StNode) * c.st);
  a.P = reinterpret_cast<PolyNode *>(base + o);
  o += align16(sizeof(PolyNode) * c.p);
  a.V = reinterpret_cast<VertNode *>(base + o);
  a.ne = a.nb = a.ny = a.nit = a.nst = a.np = a.nvx = 0;
  a.status = kClipOk;
}

// One input polygon: rings [r0, r1) of a ring CSR.
struct PolyView {
  const int64_t *ring_vert;
  const double *xy;  // (x, y) pairs
  int64_t r0, r1;
};

// ---------------------------------------------------------------- sorting
__device__ inline bool bound_less(const Bound &a, const Bound &b) {
  if (a.y < b.y) return true;
  if (a.y > b.y) return false;
  if (a.x < b.x) return true;
  if (a.x > b.x) return false;
  if (a.dx < b.dx) return true;
  if (a.dx > b.dx) return false;
  return a.order < b.order;
}
__device__ inline bool y_less(const YKey &a, const YKey &b) {
  if (a.y < b.y) return true;
  if (a.y > b.y) return false;
  return a.order < b.order;
}

template <typename T, typename Less>
__device__ void heap_sort(T *a, int n, Less less) {
  for (int start = n / 2 - 1; start >= 0; start--) {
    int root = start;
    for (;;) {
      int child = 2 * root + 1;
      if (child >= n) break;
      if (child + 1 < n && less(a[child], a[child + 1])) child++;
      if (!less(a[root], a[child])) break;
      T t = a[root];
      a[root] = a[child];
      a[child] = t;
      root = child;
    }
  }
  for (int end = n - 1; end > 0; end--) {
    T t = a[0];
    a[0] = a[end];
    a[end] = t;
    int root = 0;
    for (;;) {
      int child = 2 * root + 1;
      if (child >= end) break;
      if (child + 1 < end && less(a[child], a[child + 1])) child++;
      if (!less(a[root], a[child])) break;
      T u = a[root];
      a[root] = a[child];
      a[child] = u;
      root = child;
    }
  }
}

// Insertion sort for short runs (stable with the order tie-break anyway).
template <typename T, typename Less>
__device__ void small_sort(T *a, int n, Less less) {
  for (int i = 1; i < n; i++) {
    T x = a[i];
    int j = i - 1;
    while (j >= 0 && less(x, a[j])) {
      a[j + 1] = a[j];
      j--;
    }
    a[j + 1] = x;
  }
}

template <typename T, typename Less>
__device__ void sort_any(T *a, int n, Less less) {
  if (n <= 24) small_sort(a, n, less);
  else heap_sort(a, n, less);
}

// ---------------------------------------------------------------- output lists
__device__ inline int new_vertex(Arena &A, double x, double y, int next) {
  if (A.nvx >= A.cap.v) {
    A.status = kClipCapacity;
    return -1;
  }
  VertNode &v = A.V[A.nvx];
  v.x = x;
  v.y = y;
  v.next = next;
  return A.nvx++;
}

__device__ inline void add_local_min(Arena &A, int &out_poly, int edge, double x, double y) {
  if (A.np >= A.cap.p) {
    A.status = kClipCapacity;
    return;
  }
  int v = new_vertex(A, x, y, -1);
  if (v < 0) return;
  int k = A.np++;
  PolyNode &p = A.P[k];
  p.active = 1;
  p.hole = 0;
  p.next = out_poly;
  p.proxy = k;
  p.vl = v;
  p.vr = v;
  out_poly = k;
  A.E[edge].outp[ABOVE] = k;
}

__device__ inline void add_left(Arena &A, int p, double x, double y) {
  if (p < 0) return;
  int px = A.P[p].proxy;
  int v = new_vertex(A, x, y, A.P[px].vl);
  if (v >= 0) A.P[px].vl = v;
}

__device__ inline void add_right(Arena &A, int p, double x, double y) {
  if (p < 0) return;
  int px = A.P[p].proxy;
  int v = new_vertex(A, x, y, -1);
  if (v < 0) return;
  A.V[A.P[px].vr].next = v;
  A.P[px].vr = v;
}

// Every walk over an index-linked list is bounded by the number of nodes that
// list can hold: a malformed list ends the pair with kClipInvalid instead of
// looping on the GPU.
#define PRT_GUARD(counter, limit)    \
  if (++(counter) > (limit) + 1) {   \
    A.status = kClipInvalid;         \
    break;                           \
  }

__device__ inline void redirect(Arena &A, int target, int to, int list) {
  int g = 0;
  for (int l = list; l >= 0; l = A.P[l].next) {
    PRT_GUARD(g, A.np)
    if (A.P[l].proxy == target) {
      A.P[l].active = 0;
      A.P[l].proxy = to;
    }
  }
}

__device__ inline void merge_left(Arena &A, int p, int q, int list) {
  if (p < 0 || q < 0) return;
  int pp = A.P[p].proxy, qp = A.P[q].proxy;
  A.P[qp].hole = 1;
  if (pp != qp) {
    A.V[A.P[pp].vr].next = A.P[qp].vl;
    A.P[qp].vl = A.P[pp].vl;
    redirect(A, pp, qp, list);
  }
}

__device__ inline void merge_right(Arena &A, int p, int q, int list) {
  if (p < 0 || q < 0) return;
  int pp = A.P[p].proxy, qp = A.P[q].proxy;
  A.P[qp].hole = 0;
  if (pp != qp) {
    A.V[A.P[qp].vr].next = A.P[pp].vl;
    A.P[qp].vr = A.P[pp].vr;
    redirect(A, pp, qp, list);
  }
}

// ---------------------------------------------------------------- LMT / SBT
__device__ inline void ring_bbox(const PolyView &p, int64_t r, double *bb) {
  bb[0] = kDblMax;
  bb[1] = kDblMax;
  bb[2] = -kDblMax;
  bb[3] = -kDblMax;
  for (int64_t v = p.ring_vert[r]; v < p.ring_vert[r + 1]; v++) {
    double x = p.xy[2 * v], y = p.xy[2 * v + 1];
    if (x < bb[0]) bb[0] = x;
    if (y < bb[1]) bb[1] = y;
    if (x > bb[2]) bb[2] = x;
    if (y > bb[3]) bb[3] = y;
  }
}

__device__ inline bool bbox_overlap(const double *s, const double *c) {
  return !((s[2] < c[0]) || (s[0] > c[2])) && !((s[3] < c[1]) || (s[1] > c[3]));
}

// Does ring r of `a` overlap (by contour bbox) any ring of `b`? (minimax_test)
__device__ inline bool ring_contributes(const PolyView &a, int64_t r, const PolyView &b, bool a_is_subj) {
  double ra[4], rb[4];
  ring_bbox(a, r, ra);
  for (int64_t k = b.r0; k < b.r1; k++) {
    ring_bbox(b, k, rb);
    if (a_is_subj ? bbox_overlap(ra, rb) : bbox_overlap(rb, ra)) return true;
  }
  return false;
}

// Stages the optimal vertices of ring r in the Y array region reserved by the
// caller (vx/vy scratch inside V), then creates the forward and reverse
// bounds.  Mirrors build_lmt (GPC:1175-1307).
__device__ inline void build_ring_bounds(Arena &A, const PolyView &p, int64_t r, int type, int op,
                                         double *sx, double *sy) {
  const int64_t v0 = p.ring_vert[r];
  const int n = (int)(p.ring_vert[r + 1] - v0);
  const double *xy = p.xy + 2 * v0;
  int k = 0;
  for (int i = 0; i < n; i++) {
    int ip = (i + n - 1) % n, in = (i + 1) % n;
    if (xy[2 * ip + 1] != xy[2 * i + 1] || xy[2 * in + 1] != xy[2 * i + 1]) {
      sx[k] = xy[2 * i];
      sy[k] = xy[2 * i + 1];
      if (A.ny >= A.cap.y) {
        A.status = kClipCapacity;
        return;
      }
      A.Y[A.ny].y = sy[k];
      A.Y[A.ny].order = A.ny;
      A.ny++;
      k++;
    }
  }
  for (int dir = 0; dir < 2; dir++) {
    for (int mn = 0; mn < k; mn++) {
      int pv = (mn + k - 1) % k, nx = (mn + 1) % k;
      bool is_min = dir == 0 ? (sy[pv] >= sy[mn] && sy[nx] > sy[mn]) : (sy[pv] > sy[mn] && sy[nx] >= sy[mn]);
      if (!is_min) continue;
      int ne = 1;
      int mx = dir == 0 ? nx : pv;
      for (;;) {
        int t = dir == 0 ? (mx + 1) % k : (mx + k - 1) % k;
        if (!(sy[t] > sy[mx])) break;
        ne++;
        mx = t;
      }
      if (A.ne + ne > A.cap.e || A.nb >= A.cap.b) {
        A.status = kClipCapacity;
        return;
      }
      int base = A.ne;
      int v = mn;
      for (int i = 0; i < ne; i++) {
        Edge &e = A.E[base + i];
        e.xb = sx[v];
        e.bx = sx[v];
        e.by = sy[v];
        v = dir == 0 ? (v + 1) % k : (v + k - 1) % k;
        e.tx = sx[v];
        e.ty = sy[v];
        e.dx = (sx[v] - e.bx) / (e.ty - e.by);
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
      A.ne += ne;
      Bound &b = A.B[A.nb];
      b.y = sy[mn];
      b.x = sx[mn];
      b.dx = A.E[base].dx;
      b.edge = base;
      b.order = A.nb;
      A.nb++;
    }
  }
}

// ---------------------------------------------------------------- AET / ST / IT
__device__ inline void add_edge_to_aet(Arena &A, int &aet, int e) {
  Edge *E = A.E;
  int prev = -1, cur = aet, g = 0;
  while (cur >= 0) {
    PRT_GUARD(g, A.ne)
    if (E[e].xb < E[cur].xb || (E[e].xb == E[cur].xb && E[e].dx < E[cur].dx)) break;
    prev = cur;
    cur = E[cur].next;
  }
  E[e].prev = prev;
  E[e].next = cur;
  if (cur >= 0) E[cur].prev = e;
  if (prev >= 0) E[prev].next = e;
  else aet = e;
}

__device__ inline void add_intersection(Arena &A, int &it, int e0, int e1, double x, double y) {
  if (A.nit >= A.cap.it) {
    A.status = kClipCapacity;
    return;
  }
  int owner = -1, cur = it, g = 0;
  while (cur >= 0 && !(A.IT[cur].y > y)) {
    PRT_GUARD(g, A.nit)
    owner = cur;
    cur = A.IT[cur].next;
  }
  int k = A.nit++;
  ItNode &n = A.IT[k];
  n.e0 = e0;
  n.e1 = e1;
  n.x = x;
  n.y = y;
  n.next = cur;
  if (owner < 0) it = k;
  else A.IT[owner].next = k;
}

__device__ inline void add_st_edge(Arena &A, int &st, int &it, int e, double dy) {
  const Edge &E = A.E[e];
  int owner = -1, g = 0;
  for (;;) {
    PRT_GUARD(g, A.nst)
    int cur = owner < 0 ? st : A.ST[owner].prev;
    bool insert = cur < 0;
    if (!insert) {
      const StNode &s = A.ST[cur];
      double den = (s.xt - s.xb) - (E.xt - E.xb);
      if (E.xt >= s.xt || E.dx == s.dx || fabs(den) <= kEps) {
        insert = true;
      } else {
        double r = (E.xb - s.xb) / den;
        double x = s.xb + r * (s.xt - s.xb);
        double y = r * dy;
        add_intersection(A, it, s.edge, e, x, y);
        if (A.status) return;
        owner = cur;
        continue;
      }
    }
    if (A.nst >= A.cap.st) {
      A.status = kClipCapacity;
      return;
    }
    int k = A.nst++;
    StNode &n = A.ST[k];
    n.edge = e;
    n.xb = E.xb;
    n.xt = E.xt;
    n.dx = E.dx;
    n.prev = cur;
    if (owner < 0) st = k;
    else A.ST[owner].prev = k;
    return;
  }
}

__device__ inline void build_intersection_table(Arena &A, int &it, int aet, double dy) {
  A.nit = 0;
  A.nst = 0;
  it = -1;
  int st = -1;
  int g = 0;
  for (int e = aet; e >= 0 && !A.status; e = A.E[e].next) {
    PRT_GUARD(g, A.ne)
    const Edge &E = A.E[e];
    if (E.bstate[ABOVE] == BUNDLE_HEAD || E.bundle[ABOVE][CLIP] || E.bundle[ABOVE][SUBJ]) add_st_edge(A, st, it, e, dy);
  }
}

// Intersections of one scanbeam (GPC:461-659): builds the intersection table
// of the AET for beam height dy, then processes each intersection in y order:
// output vertices at the crossing and the swap of the two bundles in the AET.
// Shared by the thread and the warp clippers.
__device__ inline void intersect_beam(Arena &A, int op, int &aet, int &out_poly, double yb, double dy) {
  Edge *E = A.E;
  int it = -1;
  int in[2];
  build_intersection_table(A, it, aet, dy);
  if (A.status) return;
  int g4 = 0;
  for (int in_ = it; in_ >= 0 && !A.status; in_ = A.IT[in_].next) {
    PRT_GUARD(g4, A.nit)
    const int a0 = A.IT[in_].e0, a1 = A.IT[in_].e1;
    Edge &x0 = E[a0];
    Edge &x1 = E[a1];
    if ((x0.bundle[ABOVE][CLIP] || x0.bundle[ABOVE][SUBJ]) && (x1.bundle[ABOVE][CLIP] || x1.bundle[ABOVE][SUBJ])) {
      const int p = x0.outp[ABOVE], q = x1.outp[ABOVE];
      const double ix = A.IT[in_].x;
      const double iy = A.IT[in_].y + yb;
      const int b0C = x0.bundle[ABOVE][CLIP], b0S = x0.bundle[ABOVE][SUBJ];
      const int b1C = x1.bundle[ABOVE][CLIP], b1S = x1.bundle[ABOVE][SUBJ];
      in[CLIP] = (b0C && !x0.bside[CLIP]) || (b1C && x1.bside[CLIP]) ||
                 (!b0C && !b1C && x0.bside[CLIP] && x1.bside[CLIP]);
      in[SUBJ] = (b0S && !x0.bside[SUBJ]) || (b1S && x1.bside[SUBJ]) ||
                 (!b0S && !b1S && x0.bside[SUBJ] && x1.bside[SUBJ]);
      int tr = 0, tl = 0, br = 0, bl = 0;
      switch (op) {
        case OP_DIFF:
        case OP_INT:
          tr = in[CLIP] && in[SUBJ];
          tl = (in[CLIP] ^ b1C) && (in[SUBJ] ^ b1S);
          br = (in[CLIP] ^ b0C) && (in[SUBJ] ^ b0S);
          bl = (in[CLIP] ^ b1C ^ b0C) && (in[SUBJ] ^ b1S ^ b0S);
          break;
        case OP_XOR:
          tr = in[CLIP] ^ in[SUBJ];
          tl = (in[CLIP] ^ b1C) ^ (in[SUBJ] ^ b1S);
          br = (in[CLIP] ^ b0C) ^ (in[SUBJ] ^ b0S);
          bl = (in[CLIP] ^ b1C ^ b0C) ^ (in[SUBJ] ^ b1S ^ b0S);
          break;
        default:
          tr = in[CLIP] || in[SUBJ];
          tl = (in[CLIP] ^ b1C) || (in[SUBJ] ^ b1S);
          br = (in[CLIP] ^ b0C) || (in[SUBJ] ^ b0S);
          bl = (in[CLIP] ^ b1C ^ b0C) || (in[SUBJ] ^ b1S ^ b0S);
          break;
      }
      const int vclass = tr + (tl << 1) + (br << 2) + (bl << 3);
      switch (vclass) {
        case EMN:
        case IMN:
          add_local_min(A, out_poly, a0, ix, iy);
          x1.outp[ABOVE] = x0.outp[ABOVE];
          break;
        case ERI:
          if (p >= 0) {
            add_right(A, p, ix, iy);
            x1.outp[ABOVE] = p;
            x0.outp[ABOVE] = -1;
          }
          break;
        case ELI:
          if (q >= 0) {
            add_left(A, q, ix, iy);
            x0.outp[ABOVE] = q;
            x1.outp[ABOVE] = -1;
          }
          break;
        case EMX:
          if (p >= 0 && q >= 0) {
            add_left(A, p, ix, iy);
            merge_right(A, p, q, out_poly);
            x0.outp[ABOVE] = -1;
            x1.outp[ABOVE] = -1;
          }
          break;
        case ILI:
          if (p >= 0) {
            add_left(A, p, ix, iy);
            x1.outp[ABOVE] = p;
            x0.outp[ABOVE] = -1;
          }
          break;
        case IRI:
          if (q >= 0) {
            add_right(A, q, ix, iy);
            x0.outp[ABOVE] = q;
            x1.outp[ABOVE] = -1;
          }
          break;
        case IMX:
          if (p >= 0 && q >= 0) {
            add_right(A, p, ix, iy);
            merge_left(A, p, q, out_poly);
            x0.outp[ABOVE] = -1;
            x1.outp[ABOVE] = -1;
          }
          break;
        case IMM:
          if (p >= 0 && q >= 0) {
            add_right(A, p, ix, iy);
            merge_left(A, p, q, out_poly);
            add_local_min(A, out_poly, a0, ix, iy);
            x1.outp[ABOVE] = x0.outp[ABOVE];
          }
          break;
        case EMM:
          if (p >= 0 && q >= 0) {
            add_left(A, p, ix, iy);
            merge_right(A, p, q, out_poly);
            add_local_min(A, out_poly, a0, ix, iy);
            x1.outp[ABOVE] = x0.outp[ABOVE];
          }
          break;
        default:
          break;
      }
    }
    if (x0.bundle[ABOVE][CLIP]) x1.bside[CLIP] = !x1.bside[CLIP];
    if (x1.bundle[ABOVE][CLIP]) x0.bside[CLIP] = !x0.bside[CLIP];
    if (x0.bundle[ABOVE][SUBJ]) x1.bside[SUBJ] = !x1.bside[SUBJ];
    if (x1.bundle[ABOVE][SUBJ]) x0.bside[SUBJ] = !x0.bside[SUBJ];
    // swap the e0 and e1 bundles in the AET (GPC:622-657)
    int pe = x0.prev, nx = x1.next;
    if (nx >= 0) E[nx].prev = a0;
    if (x0.bstate[ABOVE] == BUNDLE_HEAD) {
      bool search = true;
      int g5 = 0;
      while (search) {
        PRT_GUARD(g5, A.ne)
        if (pe < 0) break;
        pe = E[pe].prev;
        if (pe >= 0) {
          if (E[pe].bstate[ABOVE] != BUNDLE_TAIL) search = false;
        } else {
          search = false;
        }
      }
    }
    if (pe < 0) {
      E[aet].prev = a1;
      x1.next = aet;
      aet = x0.next;
    } else {
      E[E[pe].next].prev = a1;
      x1.next = E[pe].next;
      E[pe].next = x0.next;
    }
    if (x0.next >= 0) E[x0.next].prev = pe;
    if (x1.next >= 0) E[x1.next].prev = a1;
    x0.next = nx;
  }
}

__constant__ int8_t c_next_h[3][6] = {{BH, TH, TH, BH, NH, NH}, {NH, NH, NH, NH, TH, TH}, {NH, NH, NH, NH, BH, BH}};

// Clips subj against clip.  Returns the head of the output polygon list
// (-1 for an empty result); read it with count_result / write_result /
// result_area.  A.status != kClipOk means the arena was too small.
static __device__ __noinline__ int clip_pair(Arena &A, int op, const PolyView &subj, const PolyView &clip) {
  const int sn = (int)(subj.r1 - subj.r0), cn = (int)(clip.r1 - clip.r0);
  if ((sn == 0 && cn == 0) || (sn == 0 && (op == OP_INT || op == OP_DIFF)) || (cn == 0 && op == OP_INT)) return -1;

  // scratch for staged ring vertices: the tail of the vertex-node area,
  // which is free until the scanbeam loop starts
  double *sx = reinterpret_cast<double *>(A.V);
  double *sy = sx + A.cap.e;  // cap.v >= 2 cap.e + 32 VertNodes = plenty of doubles
  const bool minimax = (op == OP_INT || op == OP_DIFF) && sn > 0 && cn > 0;
  for (int pass = 0; pass < 2 && !A.status; pass++) {
    const PolyView &p = pass == 0 ? subj : clip;
    const PolyView &o = pass == 0 ? clip : subj;
    const int type = pass == 0 ? SUBJ : CLIP;
    for (int64_t r = p.r0; r < p.r1 && !A.status; r++) {
      // contributing contours: clip rings always filtered for INT/DIFF,
      // subject rings only for INT (minimax_test GPC:1656-1709)
      if (minimax && (pass == 1 || op == OP_INT) && !ring_contributes(p, r, o, pass == 0)) continue;
      build_ring_bounds(A, p, r, type, op, sx, sy);
    }
  }
  if (A.status || A.nb == 0) return -1;

  sort_any(A.B, A.nb, bound_less);
  sort_any(A.Y, A.ny, y_less);
  int nsbt = 0;
  for (int i = 0; i < A.ny; i++)
    if (nsbt == 0 || A.Y[i].y > A.Y[nsbt - 1].y) A.Y[nsbt++].y = A.Y[i].y;

  Edge *E = A.E;
  int parity[2] = {LEFT, LEFT};
  if (op == OP_DIFF) parity[CLIP] = RIGHT;
  int aet = -1, cf = -1, out_poly = -1;
  int lmin = 0, scanbeam = 0;
  double yb, yt = 0.0, dy = 0.0, px, xb;
  int horiz[2], exists[2];

  while (scanbeam < nsbt) {
    yb = A.Y[scanbeam++].y;
    if (scanbeam < nsbt) {
      yt = A.Y[scanbeam].y;
      dy = yt - yb;
    }
    if (lmin < A.nb && A.B[lmin].y == yb) {
      double ly = A.B[lmin].y;
      while (lmin < A.nb && A.B[lmin].y == ly) add_edge_to_aet(A, aet, A.B[lmin++].edge);
    }
    px = -kDblMax;
    if (aet < 0) continue;
    int e0 = aet;
    {
      Edge &h = E[aet];
      h.bundle[ABOVE][h.type] = (h.ty != yb);
      h.bundle[ABOVE][!h.type] = 0;
      h.bstate[ABOVE] = UNBUNDLED;
    }
    int g1 = 0;
    for (int ne = E[aet].next; ne >= 0; ne = E[ne].next) {
      PRT_GUARD(g1, A.ne)
      Edge &n = E[ne];
      const int t = n.type;
      n.bundle[ABOVE][t] = (n.ty != yb);
      n.bundle[ABOVE][!t] = 0;
      n.bstate[ABOVE] = UNBUNDLED;
      if (n.bundle[ABOVE][t]) {
        Edge &z = E[e0];
        if (fabs(z.xb - n.xb) <= kEps && fabs(z.dx - n.dx) <= kEps && (z.ty != yb)) {
          n.bundle[ABOVE][t] ^= z.bundle[ABOVE][t];
          n.bundle[ABOVE][!t] = z.bundle[ABOVE][!t];
          n.bstate[ABOVE] = BUNDLE_HEAD;
          z.bundle[ABOVE][CLIP] = 0;
          z.bundle[ABOVE][SUBJ] = 0;
          z.bstate[ABOVE] = BUNDLE_TAIL;
        }
        e0 = ne;
      }
    }
    horiz[CLIP] = NH;
    horiz[SUBJ] = NH;
    int g2 = 0;
    for (int edge = aet; edge >= 0 && !A.status; edge = E[edge].next) {
      PRT_GUARD(g2, A.ne)
      Edge &ed = E[edge];
      exists[CLIP] = ed.bundle[ABOVE][CLIP] + (ed.bundle[BELOW][CLIP] << 1);
      exists[SUBJ] = ed.bundle[ABOVE][SUBJ] + (ed.bundle[BELOW][SUBJ] << 1);
      if (!(exists[CLIP] || exists[SUBJ])) continue;
      ed.bside[CLIP] = (int8_t)parity[CLIP];
      ed.bside[SUBJ] = (int8_t)parity[SUBJ];
      int contributing = 0, br = 0, bl = 0, tr = 0, tl = 0;
      const int aC = ed.bundle[ABOVE][CLIP], aS = ed.bundle[ABOVE][SUBJ];
      const int bC = ed.bundle[BELOW][CLIP], bS = ed.bundle[BELOW][SUBJ];
      const int hc = horiz[CLIP] != NH, hs = horiz[SUBJ] != NH;
      switch (op) {
        case OP_DIFF:
        case OP_INT:
          contributing = (exists[CLIP] && (parity[SUBJ] || horiz[SUBJ])) ||
                         (exists[SUBJ] && (parity[CLIP] || horiz[CLIP])) ||
                         (exists[CLIP] && exists[SUBJ] && (parity[CLIP] == parity[SUBJ]));
          br = parity[CLIP] && parity[SUBJ];
          bl = (parity[CLIP] ^ aC) && (parity[SUBJ] ^ aS);
          tr = (parity[CLIP] ^ hc) && (parity[SUBJ] ^ hs);
          tl = (parity[CLIP] ^ hc ^ bC) && (parity[SUBJ] ^ hs ^ bS);
          break;
        case OP_XOR:
          contributing = exists[CLIP] || exists[SUBJ];
          br = parity[CLIP] ^ parity[SUBJ];
          bl = (parity[CLIP] ^ aC) ^ (parity[SUBJ] ^ aS);
          tr = (parity[CLIP] ^ hc) ^ (parity[SUBJ] ^ hs);
          tl = (parity[CLIP] ^ hc ^ bC) ^ (parity[SUBJ] ^ hs ^ bS);
          break;
        default:  // OP_UNION
          contributing = (exists[CLIP] && (!parity[SUBJ] || horiz[SUBJ])) ||
                         (exists[SUBJ] && (!parity[CLIP] || horiz[CLIP])) ||
                         (exists[CLIP] && exists[SUBJ] && (parity[CLIP] == parity[SUBJ]));
          br = parity[CLIP] || parity[SUBJ];
          bl = (parity[CLIP] ^ aC) || (parity[SUBJ] ^ aS);
          tr = (parity[CLIP] ^ hc) || (parity[SUBJ] ^ hs);
          tl = (parity[CLIP] ^ hc ^ bC) || (parity[SUBJ] ^ hs ^ bS);
          break;
      }
      parity[CLIP] ^= aC;
      parity[SUBJ] ^= aS;
      if (exists[CLIP]) horiz[CLIP] = c_next_h[horiz[CLIP]][((exists[CLIP] - 1) << 1) + parity[CLIP]];
      if (exists[SUBJ]) horiz[SUBJ] = c_next_h[horiz[SUBJ]][((exists[SUBJ] - 1) << 1) + parity[SUBJ]];
      const int vclass = tr + (tl << 1) + (br << 2) + (bl << 3);
      if (!contributing) continue;
      xb = ed.xb;
      switch (vclass) {
        case EMN:
        case IMN:
          add_local_min(A, out_poly, edge, xb, yb);
          px = xb;
          cf = ed.outp[ABOVE];
          break;
        case ERI:
          if (xb != px) {
            add_right(A, cf, xb, yb);
            px = xb;
          }
          ed.outp[ABOVE] = cf;
          cf = -1;
          break;
        case ELI:
          add_left(A, ed.outp[BELOW], xb, yb);
          px = xb;
          cf = ed.outp[BELOW];
          break;
        case EMX:
          if (xb != px) {
            add_left(A, cf, xb, yb);
            px = xb;
          }
          merge_right(A, cf, ed.outp[BELOW], out_poly);
          cf = -1;
          break;
        case ILI:
          if (xb != px) {
            add_left(A, cf, xb, yb);
            px = xb;
          }
          ed.outp[ABOVE] = cf;
          cf = -1;
          break;
        case IRI:
          add_right(A, ed.outp[BELOW], xb, yb);
          px = xb;
          cf = ed.outp[BELOW];
          ed.outp[BELOW] = -1;
          break;
        case IMX:
          if (xb != px) {
            add_right(A, cf, xb, yb);
            px = xb;
          }
          merge_left(A, cf, ed.outp[BELOW], out_poly);
          cf = -1;
          ed.outp[BELOW] = -1;
          break;
        case IMM:
          if (xb != px) {
            add_right(A, cf, xb, yb);
            px = xb;
          }
          merge_left(A, cf, ed.outp[BELOW], out_poly);
          ed.outp[BELOW] = -1;
          add_local_min(A, out_poly, edge, xb, yb);
          cf = ed.outp[ABOVE];
          break;
        case EMM:
          if (xb != px) {
            add_left(A, cf, xb, yb);
            px = xb;
          }
          merge_right(A, cf, ed.outp[BELOW], out_poly);
          ed.outp[BELOW] = -1;
          add_local_min(A, out_poly, edge, xb, yb);
          cf = ed.outp[ABOVE];
          break;
        case LED:
          if (ed.by == yb) add_left(A, ed.outp[BELOW], xb, yb);
          ed.outp[ABOVE] = ed.outp[BELOW];
          px = xb;
          break;
        case RED:
          if (ed.by == yb) add_right(A, ed.outp[BELOW], xb, yb);
          ed.outp[ABOVE] = ed.outp[BELOW];
          px = xb;
          break;
        default:
          break;
      }
    }
    if (A.status) return -1;
    // delete terminating edges, compute xt (GPC:426-459)
    int g3 = 0;
    for (int edge = aet; edge >= 0; edge = E[edge].next) {
      PRT_GUARD(g3, A.ne)
      Edge &ed = E[edge];
      if (ed.ty == yb) {
        int pe = ed.prev, ne = ed.next;
        if (pe >= 0) E[pe].next = ne;
        else aet = ne;
        if (ne >= 0) E[ne].prev = pe;
        if (ed.bstate[BELOW] == BUNDLE_HEAD && pe >= 0) {
          if (E[pe].bstate[BELOW] == BUNDLE_TAIL) {
            E[pe].outp[BELOW] = ed.outp[BELOW];
            E[pe].bstate[BELOW] = UNBUNDLED;
            if (E[pe].prev >= 0)
              if (E[E[pe].prev].bstate[BELOW] == BUNDLE_TAIL) E[pe].bstate[BELOW] = BUNDLE_HEAD;
          }
        }
      } else {
        if (ed.ty == yt) ed.xt = ed.tx;
        else ed.xt = ed.bx + ed.dx * (yt - ed.by);
      }
    }
    if (scanbeam < nsbt) {
      intersect_beam(A, op, aet, out_poly, yb, dy);
      if (A.status) return -1;
      // prepare for the next scanbeam (GPC:661-693)
      int nx;
      int g6 = 0;
      for (int edge = aet; edge >= 0; edge = nx) {
        PRT_GUARD(g6, A.ne)
        Edge &ed = E[edge];
        nx = ed.next;
        const int sc = ed.succ;
        if (ed.ty == yt && sc >= 0) {
          Edge &su = E[sc];
          su.outp[BELOW] = ed.outp[ABOVE];
          su.bstate[BELOW] = ed.bstate[ABOVE];
          su.bundle[BELOW][CLIP] = ed.bundle[ABOVE][CLIP];
          su.bundle[BELOW][SUBJ] = ed.bundle[ABOVE][SUBJ];
          int pe = ed.prev;
          if (pe >= 0) E[pe].next = sc;
          else aet = sc;
          if (nx >= 0) E[nx].prev = sc;
          su.prev = pe;
          su.next = nx;
        } else {
          ed.outp[BELOW] = ed.outp[ABOVE];
          ed.bstate[BELOW] = ed.bstate[ABOVE];
          ed.bundle[BELOW][CLIP] = ed.bundle[ABOVE][CLIP];
          ed.bundle[BELOW][SUBJ] = ed.bundle[ABOVE][SUBJ];
          ed.xb = ed.xt;
        }
        ed.outp[ABOVE] = -1;
      }
    }
  }

  return out_poly;
}

// count_contours (GPC:1473-1504): contours with more than two vertices are
// kept; their vertex count is recorded in `active`.
__device__ inline void count_result(Arena &A, int out_poly, int *ncont, int64_t *nvtot) {
  int nc = 0;
  int64_t tot = 0;
  int gp = 0;
  for (int p = out_poly; p >= 0; p = A.P[p].next) {
    PRT_GUARD(gp, A.np)
    if (!A.P[p].active) continue;
    int nv = 0;
    for (int v = A.P[A.P[p].proxy].vl; v >= 0; v = A.V[v].next) {
      PRT_GUARD(nv, A.nvx)
    }
    if (nv > 2) {
      A.P[p].active = nv;
      nc++;
      tot += nv;
    } else {
      A.P[p].active = 0;
    }
  }
  *ncont = nc;
  *nvtot = tot;
}

// Result assembly (GPC:698-741): contours in list order, each contour's
// vertices in reverse order of its left-to-right vertex list.
__device__ inline void write_result(const Arena &A, int out_poly, int32_t *cont_nverts, int32_t *cont_hole,
                                    int64_t *cont_vstart, double *xy, int64_t cbase, int64_t vbase) {
  int64_t c = cbase, off = vbase;
  for (int p = out_poly; p >= 0; p = A.P[p].next) {
    const int nv = A.P[p].active;
    if (!nv) continue;
    const int px2 = A.P[p].proxy;
    cont_nverts[c] = nv;
    cont_hole[c] = A.P[px2].hole;
    cont_vstart[c] = off;
    int64_t k = off + nv - 1;
    for (int v = A.P[px2].vl; v >= 0; v = A.V[v].next) {
      xy[2 * k] = A.V[v].x;
      xy[2 * k + 1] = A.V[v].y;
      k--;
    }
    off += nv;
    c++;
  }
}

// Sum over result contours of |shoelace area|, hole contours negative.  The
// shoelace runs on coordinates relative to the contour's first output vertex
// (the last node of its left-to-right list): the plain form cancels terms of
// size |x||y| down to an area of size r^2 and loses ~|x||y|/r^2 ulps on small
// contours far from the origin.  Terms are summed in list order (the reverse
// of output order), so the value agrees with a sum over the written-out
// contour to rounding (~1e-15 relative), not bit for bit.
__device__ inline double result_area(const Arena &A, int out_poly) {
  double total = 0.0;
  for (int p = out_poly; p >= 0; p = A.P[p].next) {
    if (!A.P[p].active) continue;
    const int px2 = A.P[p].proxy;
    int last = A.P[px2].vl;
    while (A.V[last].next >= 0) last = A.V[last].next;
    const double x0 = A.V[last].x, y0 = A.V[last].y;
    // the walk visits output vertices n-1, n-2, ..., 0; the term of output
    // edge (i, i+1) pairs the visited vertex i with the one visited before it
    double xn = 0.0, yn = 0.0;  // output vertex 0, relative to itself
    double a = 0.0;
    for (int u = A.P[px2].vl; u >= 0; u = A.V[u].next) {
      const double xi = A.V[u].x - x0, yi = A.V[u].y - y0;
      a += xi * yn - xn * yi;
      xn = xi;
      yn = yi;
    }
    a = 0.5 * fabs(a);
    total += A.P[px2].hole ? -a : a;
  }
  return total;
}

}  // namespace gpc
}  // namespace prt
