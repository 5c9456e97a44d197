/* ORACLE — test infrastructure only.  CPU restatement of the reference's GPC
 * intersection clip (vector_map_overlay_gpc_kernel.cu:115-750, helpers
 * :890-1709), the Vatti scanbeam algorithm of the General Polygon Clipper
 * (A. Murta; no version pinned by the reference), plus the shoelace area of a
 * result and the boundary-integral gradient of an intersection area.
 * Used by tests/ and bench.py's CPU baseline as the checker; never linked
 * into the product library.
 *
 * The lists of the reference (LMT, scanbeam tree, AET, sorted edge table,
 * intersection table, output polygons and vertices) are restated as arrays
 * linked by int indices; each step keeps the reference's order of operations
 * and its floating-point expressions (compile with -ffp-contract=off), so the
 * result is the same contour list, hole flags and vertex order:
 *   minimax_test        GPC:1656-1709   contour bbox prefilter
 *   build_lmt           GPC:1175-1307   bounds from local minima, LMT order by
 *                                       (y, bot.x, dx) with ties in creation
 *                                       order (insert_bound GPC:929-978)
 *   build_sbt           GPC:1019-1085   sorted unique vertex y values
 *   scanbeam loop       GPC:183-695     bundling, vertex classes, IT swaps
 *   add_edge_to_aet     GPC:1309-1355
 *   add_st_edge         GPC:1395-1445   intersection rule with DBL_EPSILON
 *   add_intersection    GPC:1357-1393   IT kept ordered by y, ties appended
 *   output polygons     GPC:1473-1621, result assembly GPC:698-741
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define G_LEFT 0
#define G_RIGHT 1
#define G_ABOVE 0
#define G_BELOW 1
#define G_CLIP 0
#define G_SUBJ 1
enum { OP_DIFF = 0, OP_INT = 1, OP_XOR = 2, OP_UNION = 3 };
enum { NUL_, EMX_, ELI_, TED_, ERI_, RED_, IMM_, IMN_, EMN_, EMM_, LED_, ILI_, BED_, IRI_, IMX_, FUL_ };
enum { NH_ = 0, BH_ = 1, TH_ = 2 };
enum { UNB_ = 0, BHEAD_ = 1, BTAIL_ = 2 };

/* next horizontal state [state][((exists - 1) << 1) + parity] (GPC:62) */
static const int k_next_h[3][6] = {{BH_, TH_, TH_, BH_, NH_, NH_},
                                   {NH_, NH_, NH_, NH_, TH_, TH_},
                                   {NH_, NH_, NH_, NH_, BH_, BH_}};

#define GEQ(a, b) (fabs((a) - (b)) <= DBL_EPSILON)

typedef struct { double x, y; } gv;

typedef struct {
  gv bot, top;
  double xb, xt, dx;
  int type;
  int bundle[2][2];
  int bside[2];
  int bstate[2];
  int outp[2];
  int prev, next, pred, succ;
} gedge;

typedef struct { double y, x, dx; int edge, order; } gbound;
typedef struct { int ie0, ie1; double x, y; int next; } git;
typedef struct { int edge; double xb, xt, dx; int prev; } gst;
typedef struct { int active, hole; int vl, vr; int next, proxy; } gpoly;
typedef struct { double x, y; int next; } gvert;

#define VEC(T) struct { T *a; int n, cap; }
#define VPUSH(v, x)                                                     \
  do {                                                                  \
    if ((v).n == (v).cap) {                                             \
      (v).cap = (v).cap ? 2 * (v).cap : 64;                             \
      (v).a = realloc((v).a, sizeof(*(v).a) * (size_t)(v).cap);         \
    }                                                                   \
    (v).a[(v).n++] = (x);                                               \
  } while (0)

typedef struct {
  VEC(gedge) E;
  VEC(gbound) B;
  VEC(double) ys;
  VEC(git) IT;
  VEC(gst) ST;
  VEC(gpoly) P;
  VEC(gvert) V;
  int out_poly;
  /* sizing statistics for the device arenas */
  int max_aet, max_it, max_st;
} gctx;

/* one polygon: ncont rings, nverts[c] vertices each, packed xy */
typedef struct {
  int ncont;
  const int *nverts;
  const double *xy;
  const int64_t *voff; /* first vertex of each ring */
} gpolyin;

/* ---- output polygon lists (GPC:1506-1621) ---- */

static int new_vertex(gctx *g, double x, double y, int next) {
  gvert v = {x, y, next};
  VPUSH(g->V, v);
  return g->V.n - 1;
}

static void add_local_min(gctx *g, int edge, double x, double y) {
  gpoly p;
  p.active = 1;
  p.hole = 0;
  p.next = g->out_poly;
  p.proxy = g->P.n;
  int v = new_vertex(g, x, y, -1);
  p.vl = v;
  p.vr = v;
  VPUSH(g->P, p);
  g->out_poly = g->P.n - 1;
  g->E.a[edge].outp[G_ABOVE] = g->out_poly;
}

static void add_left(gctx *g, int p, double x, double y) {
  if (p < 0) return;
  int px = g->P.a[p].proxy;
  int v = new_vertex(g, x, y, g->P.a[px].vl);
  g->P.a[px].vl = v;
}

static void add_right(gctx *g, int p, double x, double y) {
  if (p < 0) return;
  int px = g->P.a[p].proxy;
  int v = new_vertex(g, x, y, -1);
  g->V.a[g->P.a[px].vr].next = v;
  g->P.a[px].vr = v;
}

static void redirect(gctx *g, int target, int to, int list) {
  for (int l = list; l >= 0; l = g->P.a[l].next) {
    if (g->P.a[l].proxy == target) {
      g->P.a[l].active = 0;
      g->P.a[l].proxy = to;
    }
  }
}

static void merge_left(gctx *g, int p, int q, int list) {
  if (p < 0 || q < 0) return;
  int pp = g->P.a[p].proxy, qp = g->P.a[q].proxy;
  g->P.a[qp].hole = 1;
  if (pp != qp) {
    g->V.a[g->P.a[pp].vr].next = g->P.a[qp].vl;
    g->P.a[qp].vl = g->P.a[pp].vl;
    redirect(g, pp, qp, list);
  }
}

static void merge_right(gctx *g, int p, int q, int list) {
  if (p < 0 || q < 0) return;
  int pp = g->P.a[p].proxy, qp = g->P.a[q].proxy;
  g->P.a[qp].hole = 0;
  if (pp != qp) {
    g->V.a[g->P.a[qp].vr].next = g->P.a[pp].vl;
    g->P.a[qp].vr = g->P.a[pp].vr;
    redirect(g, pp, qp, list);
  }
}

/* ---- LMT / SBT (GPC:929-1307) ---- */

static int cmp_bound(const void *a, const void *b) {
  const gbound *x = (const gbound *)a, *y = (const gbound *)b;
  if (x->y < y->y) return -1;
  if (x->y > y->y) return 1;
  if (x->x < y->x) return -1;
  if (x->x > y->x) return 1;
  if (x->dx < y->dx) return -1;
  if (x->dx > y->dx) return 1;
  return x->order - y->order;
}

typedef struct { double y; int order; } ykey;
static int cmp_ykey(const void *a, const void *b) {
  const ykey *x = (const ykey *)a, *y = (const ykey *)b;
  if (x->y < y->y) return -1;
  if (x->y > y->y) return 1;
  return x->order - y->order;
}

static void build_bounds(gctx *g, const gpolyin *p, const int *contrib, int type, int op) {
  int maxn = 0;
  for (int c = 0; c < p->ncont; c++) if (p->nverts[c] > maxn) maxn = p->nverts[c];
  gv *st = (gv *)malloc(sizeof(gv) * (size_t)(maxn > 0 ? maxn : 1));
  for (int c = 0; c < p->ncont; c++) {
    if (!contrib[c]) continue;
    int n = p->nverts[c];
    const double *xy = p->xy + 2 * p->voff[c];
    int k = 0;
    for (int i = 0; i < n; i++) {
      int ip = (i + n - 1) % n, in = (i + 1) % n;
      if (xy[2 * ip + 1] != xy[2 * i + 1] || xy[2 * in + 1] != xy[2 * i + 1]) {
        st[k].x = xy[2 * i];
        st[k].y = xy[2 * i + 1];
        VPUSH(g->ys, st[k].y);
        k++;
      }
    }
    for (int dir = 0; dir < 2; dir++) {
      for (int mn = 0; mn < k; mn++) {
        int pv = (mn + k - 1) % k, nx = (mn + 1) % k;
        int is_min = dir == 0 ? (st[pv].y >= st[mn].y && st[nx].y > st[mn].y)
                              : (st[pv].y > st[mn].y && st[nx].y >= st[mn].y);
        if (!is_min) continue;
        int ne = 1;
        int mx = dir == 0 ? nx : pv;
        for (;;) {
          int t = dir == 0 ? (mx + 1) % k : (mx + k - 1) % k;
          if (!(st[t].y > st[mx].y)) break;
          ne++;
          mx = t;
        }
        int base = g->E.n;
        int v = mn;
        for (int i = 0; i < ne; i++) {
          gedge e;
          memset(&e, 0, sizeof e);
          e.xb = st[v].x;
          e.bot = st[v];
          v = dir == 0 ? (v + 1) % k : (v + k - 1) % k;
          e.top = st[v];
          e.dx = (st[v].x - e.bot.x) / (e.top.y - e.bot.y);
          e.type = type;
          e.outp[0] = e.outp[1] = -1;
          e.prev = e.next = -1;
          e.succ = (ne > 1 && i < ne - 1) ? base + i + 1 : -1;
          e.pred = (ne > 1 && i > 0) ? base + i - 1 : -1;
          e.bside[G_CLIP] = op == OP_DIFF ? G_RIGHT : G_LEFT;
          e.bside[G_SUBJ] = G_LEFT;
          e.bstate[G_BELOW] = UNB_;
          VPUSH(g->E, e);
        }
        gbound b = {st[mn].y, st[mn].x, g->E.a[base].dx, base, g->B.n};
        VPUSH(g->B, b);
      }
    }
  }
  free(st);
}

static void bbox_of(const gpolyin *p, int c, double *bb) {
  bb[0] = DBL_MAX; bb[1] = DBL_MAX; bb[2] = -DBL_MAX; bb[3] = -DBL_MAX;
  const double *xy = p->xy + 2 * p->voff[c];
  for (int v = 0; v < p->nverts[c]; v++) {
    if (xy[2 * v] < bb[0]) bb[0] = xy[2 * v];
    if (xy[2 * v + 1] < bb[1]) bb[1] = xy[2 * v + 1];
    if (xy[2 * v] > bb[2]) bb[2] = xy[2 * v];
    if (xy[2 * v + 1] > bb[3]) bb[3] = xy[2 * v + 1];
  }
}

/* ---- AET / ST / IT (GPC:1309-1471) ---- */

static void add_edge_to_aet(gctx *g, int *aet, int e) {
  gedge *E = g->E.a;
  int prev = -1, cur = *aet;
  while (cur >= 0) {
    if (E[e].xb < E[cur].xb || (E[e].xb == E[cur].xb && E[e].dx < E[cur].dx)) break;
    prev = cur;
    cur = E[cur].next;
  }
  E[e].prev = prev;
  E[e].next = cur;
  if (cur >= 0) E[cur].prev = e;
  if (prev >= 0) E[prev].next = e; else *aet = e;
}

static void add_intersection(gctx *g, int *it, int e0, int e1, double x, double y) {
  int owner = -1, cur = *it;
  while (cur >= 0 && !(g->IT.a[cur].y > y)) {
    owner = cur;
    cur = g->IT.a[cur].next;
  }
  git n = {e0, e1, x, y, cur};
  VPUSH(g->IT, n);
  if (owner < 0) *it = g->IT.n - 1; else g->IT.a[owner].next = g->IT.n - 1;
}

static void add_st_edge(gctx *g, int *st, int *it, int e, double dy) {
  gedge *E;
  int owner = -1; /* -1: the head link */
  for (;;) {
    int cur = owner < 0 ? *st : g->ST.a[owner].prev;
    E = g->E.a;
    if (cur < 0) {
      gst n = {e, E[e].xb, E[e].xt, E[e].dx, -1};
      VPUSH(g->ST, n);
      if (owner < 0) *st = g->ST.n - 1; else g->ST.a[owner].prev = g->ST.n - 1;
      return;
    }
    gst s = g->ST.a[cur];
    double den = (s.xt - s.xb) - (E[e].xt - E[e].xb);
    if (E[e].xt >= s.xt || E[e].dx == s.dx || fabs(den) <= DBL_EPSILON) {
      gst n = {e, E[e].xb, E[e].xt, E[e].dx, cur};
      VPUSH(g->ST, n);
      if (owner < 0) *st = g->ST.n - 1; else g->ST.a[owner].prev = g->ST.n - 1;
      return;
    }
    double r = (E[e].xb - s.xb) / den;
    double x = s.xb + r * (s.xt - s.xb);
    double y = r * dy;
    add_intersection(g, it, s.edge, e, x, y);
    owner = cur;
  }
}

static void build_intersection_table(gctx *g, int *it, int aet, double dy) {
  g->IT.n = 0;
  g->ST.n = 0;
  *it = -1;
  int st = -1;
  for (int e = aet; e >= 0; e = g->E.a[e].next) {
    gedge *E = g->E.a;
    if (E[e].bstate[G_ABOVE] == BHEAD_ || E[e].bundle[G_ABOVE][G_CLIP] || E[e].bundle[G_ABOVE][G_SUBJ])
      add_st_edge(g, &st, it, e, dy);
  }
  if (g->ST.n > g->max_st) g->max_st = g->ST.n;
  if (g->IT.n > g->max_it) g->max_it = g->IT.n;
}

/* ---- the clip (GPC:115-750) ---- */

typedef struct {
  int ncont;
  int *nverts;
  int *hole;
  double *xy;
  int64_t nv_total;
} gresult;

static void gclip(int op, const gpolyin *subj, const gpolyin *clip, gresult *res, gctx *g) {
  memset(g, 0, sizeof *g);
  g->out_poly = -1;
  res->ncont = 0;
  res->nv_total = 0;
  if ((subj->ncont == 0 && clip->ncont == 0) || (subj->ncont == 0 && (op == OP_INT || op == OP_DIFF)) ||
      (clip->ncont == 0 && op == OP_INT))
    return;
  int *sc = (int *)malloc(sizeof(int) * (size_t)(subj->ncont + 1));
  int *cc = (int *)malloc(sizeof(int) * (size_t)(clip->ncont + 1));
  for (int c = 0; c < subj->ncont; c++) sc[c] = 1;
  for (int c = 0; c < clip->ncont; c++) cc[c] = 1;
  if ((op == OP_INT || op == OP_DIFF) && subj->ncont > 0 && clip->ncont > 0) {
    double *sb = (double *)malloc(sizeof(double) * 4 * (size_t)subj->ncont);
    double *cb = (double *)malloc(sizeof(double) * 4 * (size_t)clip->ncont);
    for (int s = 0; s < subj->ncont; s++) bbox_of(subj, s, sb + 4 * s);
    for (int c = 0; c < clip->ncont; c++) bbox_of(clip, c, cb + 4 * c);
#define OVL(s, c)                                                         \
  (!((sb[4 * (s) + 2] < cb[4 * (c) + 0]) || (sb[4 * (s) + 0] > cb[4 * (c) + 2])) && \
   !((sb[4 * (s) + 3] < cb[4 * (c) + 1]) || (sb[4 * (s) + 1] > cb[4 * (c) + 3])))
    for (int c = 0; c < clip->ncont; c++) {
      int o = 0;
      for (int s = 0; !o && s < subj->ncont; s++) o = OVL(s, c);
      if (!o) cc[c] = 0;
    }
    if (op == OP_INT) {
      for (int s = 0; s < subj->ncont; s++) {
        int o = 0;
        for (int c = 0; !o && c < clip->ncont; c++) o = OVL(s, c);
        if (!o) sc[s] = 0;
      }
    }
#undef OVL
    free(sb);
    free(cb);
  }
  if (subj->ncont > 0) build_bounds(g, subj, sc, G_SUBJ, op);
  if (clip->ncont > 0) build_bounds(g, clip, cc, G_CLIP, op);
  free(sc);
  free(cc);
  if (g->B.n == 0) return;

  /* LMT: bounds ordered by (y, bot.x, dx), ties in creation order */
  qsort(g->B.a, (size_t)g->B.n, sizeof(gbound), cmp_bound);
  /* SBT: sorted unique y (first inserted of equal values is kept) */
  int nys = g->ys.n;
  ykey *yk = (ykey *)malloc(sizeof(ykey) * (size_t)nys);
  for (int i = 0; i < nys; i++) { yk[i].y = g->ys.a[i]; yk[i].order = i; }
  qsort(yk, (size_t)nys, sizeof(ykey), cmp_ykey);
  double *sbt = (double *)malloc(sizeof(double) * (size_t)nys);
  int sbt_entries = 0;
  for (int i = 0; i < nys; i++)
    if (sbt_entries == 0 || yk[i].y > sbt[sbt_entries - 1]) sbt[sbt_entries++] = yk[i].y;
  free(yk);

  int parity[2] = {G_LEFT, G_LEFT};
  if (op == OP_DIFF) parity[G_CLIP] = G_RIGHT;
  int aet = -1, it = -1, cf = -1;
  int lmin = 0;
  int scanbeam = 0;
  double yb, yt = 0.0, dy = 0.0, px, xb, ix, iy;
  int horiz[2], exists[2], in[2];

  while (scanbeam < sbt_entries) {
    yb = sbt[scanbeam++];
    if (scanbeam < sbt_entries) {
      yt = sbt[scanbeam];
      dy = yt - yb;
    }
    if (lmin < g->B.n && g->B.a[lmin].y == yb) {
      double ly = g->B.a[lmin].y;
      while (lmin < g->B.n && g->B.a[lmin].y == ly) add_edge_to_aet(g, &aet, g->B.a[lmin++].edge);
    }
    gedge *E = g->E.a;
    {
      int na = 0;
      for (int e = aet; e >= 0; e = E[e].next) na++;
      if (na > g->max_aet) g->max_aet = na;
    }
    px = -DBL_MAX;
    if (aet < 0) continue; /* the reference dereferences an empty AET here */
    int e0 = aet;
    E[aet].bundle[G_ABOVE][E[aet].type] = (E[aet].top.y != yb);
    E[aet].bundle[G_ABOVE][!E[aet].type] = 0;
    E[aet].bstate[G_ABOVE] = UNB_;
    for (int ne = E[aet].next; ne >= 0; ne = E[ne].next) {
      int t = E[ne].type;
      E[ne].bundle[G_ABOVE][t] = (E[ne].top.y != yb);
      E[ne].bundle[G_ABOVE][!t] = 0;
      E[ne].bstate[G_ABOVE] = UNB_;
      if (E[ne].bundle[G_ABOVE][t]) {
        if (GEQ(E[e0].xb, E[ne].xb) && GEQ(E[e0].dx, E[ne].dx) && (E[e0].top.y != yb)) {
          E[ne].bundle[G_ABOVE][t] ^= E[e0].bundle[G_ABOVE][t];
          E[ne].bundle[G_ABOVE][!t] = E[e0].bundle[G_ABOVE][!t];
          E[ne].bstate[G_ABOVE] = BHEAD_;
          E[e0].bundle[G_ABOVE][G_CLIP] = 0;
          E[e0].bundle[G_ABOVE][G_SUBJ] = 0;
          E[e0].bstate[G_ABOVE] = BTAIL_;
        }
        e0 = ne;
      }
    }
    horiz[G_CLIP] = NH_;
    horiz[G_SUBJ] = NH_;
    for (int edge = aet; edge >= 0; edge = g->E.a[edge].next) {
      E = g->E.a;
      exists[G_CLIP] = E[edge].bundle[G_ABOVE][G_CLIP] + (E[edge].bundle[G_BELOW][G_CLIP] << 1);
      exists[G_SUBJ] = E[edge].bundle[G_ABOVE][G_SUBJ] + (E[edge].bundle[G_BELOW][G_SUBJ] << 1);
      if (!(exists[G_CLIP] || exists[G_SUBJ])) continue;
      E[edge].bside[G_CLIP] = parity[G_CLIP];
      E[edge].bside[G_SUBJ] = parity[G_SUBJ];
      int contributing = 0, br = 0, bl = 0, tr = 0, tl = 0;
      const int *bA = E[edge].bundle[G_ABOVE];
      const int *bB = E[edge].bundle[G_BELOW];
      int hc = horiz[G_CLIP] != NH_, hs = horiz[G_SUBJ] != NH_;
      switch (op) {
        case OP_DIFF:
        case OP_INT:
          contributing = (exists[G_CLIP] && (parity[G_SUBJ] || horiz[G_SUBJ])) ||
                         (exists[G_SUBJ] && (parity[G_CLIP] || horiz[G_CLIP])) ||
                         (exists[G_CLIP] && exists[G_SUBJ] && (parity[G_CLIP] == parity[G_SUBJ]));
          br = parity[G_CLIP] && parity[G_SUBJ];
          bl = (parity[G_CLIP] ^ bA[G_CLIP]) && (parity[G_SUBJ] ^ bA[G_SUBJ]);
          tr = (parity[G_CLIP] ^ hc) && (parity[G_SUBJ] ^ hs);
          tl = (parity[G_CLIP] ^ hc ^ bB[G_CLIP]) && (parity[G_SUBJ] ^ hs ^ bB[G_SUBJ]);
          break;
        case OP_XOR:
          contributing = exists[G_CLIP] || exists[G_SUBJ];
          br = parity[G_CLIP] ^ parity[G_SUBJ];
          bl = (parity[G_CLIP] ^ bA[G_CLIP]) ^ (parity[G_SUBJ] ^ bA[G_SUBJ]);
          tr = (parity[G_CLIP] ^ hc) ^ (parity[G_SUBJ] ^ hs);
          tl = (parity[G_CLIP] ^ hc ^ bB[G_CLIP]) ^ (parity[G_SUBJ] ^ hs ^ bB[G_SUBJ]);
          break;
        case OP_UNION:
          contributing = (exists[G_CLIP] && (!parity[G_SUBJ] || horiz[G_SUBJ])) ||
                         (exists[G_SUBJ] && (!parity[G_CLIP] || horiz[G_CLIP])) ||
                         (exists[G_CLIP] && exists[G_SUBJ] && (parity[G_CLIP] == parity[G_SUBJ]));
          br = parity[G_CLIP] || parity[G_SUBJ];
          bl = (parity[G_CLIP] ^ bA[G_CLIP]) || (parity[G_SUBJ] ^ bA[G_SUBJ]);
          tr = (parity[G_CLIP] ^ hc) || (parity[G_SUBJ] ^ hs);
          tl = (parity[G_CLIP] ^ hc ^ bB[G_CLIP]) || (parity[G_SUBJ] ^ hs ^ bB[G_SUBJ]);
          break;
      }
      parity[G_CLIP] ^= bA[G_CLIP];
      parity[G_SUBJ] ^= bA[G_SUBJ];
      if (exists[G_CLIP]) horiz[G_CLIP] = k_next_h[horiz[G_CLIP]][((exists[G_CLIP] - 1) << 1) + parity[G_CLIP]];
      if (exists[G_SUBJ]) horiz[G_SUBJ] = k_next_h[horiz[G_SUBJ]][((exists[G_SUBJ] - 1) << 1) + parity[G_SUBJ]];
      int vclass = tr + (tl << 1) + (br << 2) + (bl << 3);
      if (!contributing) continue;
      xb = E[edge].xb;
      switch (vclass) {
        case EMN_:
        case IMN_:
          add_local_min(g, edge, xb, yb);
          px = xb;
          cf = g->E.a[edge].outp[G_ABOVE];
          break;
        case ERI_:
          if (xb != px) { add_right(g, cf, xb, yb); px = xb; }
          g->E.a[edge].outp[G_ABOVE] = cf;
          cf = -1;
          break;
        case ELI_:
          add_left(g, g->E.a[edge].outp[G_BELOW], xb, yb);
          px = xb;
          cf = g->E.a[edge].outp[G_BELOW];
          break;
        case EMX_:
          if (xb != px) { add_left(g, cf, xb, yb); px = xb; }
          merge_right(g, cf, g->E.a[edge].outp[G_BELOW], g->out_poly);
          cf = -1;
          break;
        case ILI_:
          if (xb != px) { add_left(g, cf, xb, yb); px = xb; }
          g->E.a[edge].outp[G_ABOVE] = cf;
          cf = -1;
          break;
        case IRI_:
          add_right(g, g->E.a[edge].outp[G_BELOW], xb, yb);
          px = xb;
          cf = g->E.a[edge].outp[G_BELOW];
          g->E.a[edge].outp[G_BELOW] = -1;
          break;
        case IMX_:
          if (xb != px) { add_right(g, cf, xb, yb); px = xb; }
          merge_left(g, cf, g->E.a[edge].outp[G_BELOW], g->out_poly);
          cf = -1;
          g->E.a[edge].outp[G_BELOW] = -1;
          break;
        case IMM_:
          if (xb != px) { add_right(g, cf, xb, yb); px = xb; }
          merge_left(g, cf, g->E.a[edge].outp[G_BELOW], g->out_poly);
          g->E.a[edge].outp[G_BELOW] = -1;
          add_local_min(g, edge, xb, yb);
          cf = g->E.a[edge].outp[G_ABOVE];
          break;
        case EMM_:
          if (xb != px) { add_left(g, cf, xb, yb); px = xb; }
          merge_right(g, cf, g->E.a[edge].outp[G_BELOW], g->out_poly);
          g->E.a[edge].outp[G_BELOW] = -1;
          add_local_min(g, edge, xb, yb);
          cf = g->E.a[edge].outp[G_ABOVE];
          break;
        case LED_:
          if (g->E.a[edge].bot.y == yb) add_left(g, g->E.a[edge].outp[G_BELOW], xb, yb);
          g->E.a[edge].outp[G_ABOVE] = g->E.a[edge].outp[G_BELOW];
          px = xb;
          break;
        case RED_:
          if (g->E.a[edge].bot.y == yb) add_right(g, g->E.a[edge].outp[G_BELOW], xb, yb);
          g->E.a[edge].outp[G_ABOVE] = g->E.a[edge].outp[G_BELOW];
          px = xb;
          break;
        default:
          break;
      }
    }
    /* delete terminating edges, compute xt (GPC:426-459) */
    E = g->E.a;
    for (int edge = aet; edge >= 0; edge = E[edge].next) {
      if (E[edge].top.y == yb) {
        int pe = E[edge].prev, ne = E[edge].next;
        if (pe >= 0) E[pe].next = ne; else aet = ne;
        if (ne >= 0) E[ne].prev = pe;
        if (E[edge].bstate[G_BELOW] == BHEAD_ && pe >= 0) {
          if (E[pe].bstate[G_BELOW] == BTAIL_) {
            E[pe].outp[G_BELOW] = E[edge].outp[G_BELOW];
            E[pe].bstate[G_BELOW] = UNB_;
            if (E[pe].prev >= 0)
              if (E[E[pe].prev].bstate[G_BELOW] == BTAIL_) E[pe].bstate[G_BELOW] = BHEAD_;
          }
        }
      } else {
        if (E[edge].top.y == yt)
          E[edge].xt = E[edge].top.x;
        else
          E[edge].xt = E[edge].bot.x + E[edge].dx * (yt - E[edge].bot.y);
      }
    }
    if (scanbeam < sbt_entries) {
      build_intersection_table(g, &it, aet, dy);
      for (int in_ = it; in_ >= 0; in_ = g->IT.a[in_].next) {
        E = g->E.a;
        int a0 = g->IT.a[in_].ie0, a1 = g->IT.a[in_].ie1;
        if ((E[a0].bundle[G_ABOVE][G_CLIP] || E[a0].bundle[G_ABOVE][G_SUBJ]) &&
            (E[a1].bundle[G_ABOVE][G_CLIP] || E[a1].bundle[G_ABOVE][G_SUBJ])) {
          int p = E[a0].outp[G_ABOVE], q = E[a1].outp[G_ABOVE];
          ix = g->IT.a[in_].x;
          iy = g->IT.a[in_].y + yb;
          const int *b0 = E[a0].bundle[G_ABOVE], *b1 = E[a1].bundle[G_ABOVE];
          in[G_CLIP] = (b0[G_CLIP] && !E[a0].bside[G_CLIP]) || (b1[G_CLIP] && E[a1].bside[G_CLIP]) ||
                       (!b0[G_CLIP] && !b1[G_CLIP] && E[a0].bside[G_CLIP] && E[a1].bside[G_CLIP]);
          in[G_SUBJ] = (b0[G_SUBJ] && !E[a0].bside[G_SUBJ]) || (b1[G_SUBJ] && E[a1].bside[G_SUBJ]) ||
                       (!b0[G_SUBJ] && !b1[G_SUBJ] && E[a0].bside[G_SUBJ] && E[a1].bside[G_SUBJ]);
          int tr = 0, tl = 0, br = 0, bl = 0;
          switch (op) {
            case OP_DIFF:
            case OP_INT:
              tr = in[G_CLIP] && in[G_SUBJ];
              tl = (in[G_CLIP] ^ b1[G_CLIP]) && (in[G_SUBJ] ^ b1[G_SUBJ]);
              br = (in[G_CLIP] ^ b0[G_CLIP]) && (in[G_SUBJ] ^ b0[G_SUBJ]);
              bl = (in[G_CLIP] ^ b1[G_CLIP] ^ b0[G_CLIP]) && (in[G_SUBJ] ^ b1[G_SUBJ] ^ b0[G_SUBJ]);
              break;
            case OP_XOR:
              tr = in[G_CLIP] ^ in[G_SUBJ];
              tl = (in[G_CLIP] ^ b1[G_CLIP]) ^ (in[G_SUBJ] ^ b1[G_SUBJ]);
              br = (in[G_CLIP] ^ b0[G_CLIP]) ^ (in[G_SUBJ] ^ b0[G_SUBJ]);
              bl = (in[G_CLIP] ^ b1[G_CLIP] ^ b0[G_CLIP]) ^ (in[G_SUBJ] ^ b1[G_SUBJ] ^ b0[G_SUBJ]);
              break;
            case OP_UNION:
              tr = in[G_CLIP] || in[G_SUBJ];
              tl = (in[G_CLIP] ^ b1[G_CLIP]) || (in[G_SUBJ] ^ b1[G_SUBJ]);
              br = (in[G_CLIP] ^ b0[G_CLIP]) || (in[G_SUBJ] ^ b0[G_SUBJ]);
              bl = (in[G_CLIP] ^ b1[G_CLIP] ^ b0[G_CLIP]) || (in[G_SUBJ] ^ b1[G_SUBJ] ^ b0[G_SUBJ]);
              break;
          }
          int vclass = tr + (tl << 1) + (br << 2) + (bl << 3);
          switch (vclass) {
            case EMN_:
              add_local_min(g, a0, ix, iy);
              g->E.a[a1].outp[G_ABOVE] = g->E.a[a0].outp[G_ABOVE];
              break;
            case ERI_:
              if (p >= 0) {
                add_right(g, p, ix, iy);
                g->E.a[a1].outp[G_ABOVE] = p;
                g->E.a[a0].outp[G_ABOVE] = -1;
              }
              break;
            case ELI_:
              if (q >= 0) {
                add_left(g, q, ix, iy);
                g->E.a[a0].outp[G_ABOVE] = q;
                g->E.a[a1].outp[G_ABOVE] = -1;
              }
              break;
            case EMX_:
              if (p >= 0 && q >= 0) {
                add_left(g, p, ix, iy);
                merge_right(g, p, q, g->out_poly);
                g->E.a[a0].outp[G_ABOVE] = -1;
                g->E.a[a1].outp[G_ABOVE] = -1;
              }
              break;
            case IMN_:
              add_local_min(g, a0, ix, iy);
              g->E.a[a1].outp[G_ABOVE] = g->E.a[a0].outp[G_ABOVE];
              break;
            case ILI_:
              if (p >= 0) {
                add_left(g, p, ix, iy);
                g->E.a[a1].outp[G_ABOVE] = p;
                g->E.a[a0].outp[G_ABOVE] = -1;
              }
              break;
            case IRI_:
              if (q >= 0) {
                add_right(g, q, ix, iy);
                g->E.a[a0].outp[G_ABOVE] = q;
                g->E.a[a1].outp[G_ABOVE] = -1;
              }
              break;
            case IMX_:
              if (p >= 0 && q >= 0) {
                add_right(g, p, ix, iy);
                merge_left(g, p, q, g->out_poly);
                g->E.a[a0].outp[G_ABOVE] = -1;
                g->E.a[a1].outp[G_ABOVE] = -1;
              }
              break;
            case IMM_:
              if (p >= 0 && q >= 0) {
                add_right(g, p, ix, iy);
                merge_left(g, p, q, g->out_poly);
                add_local_min(g, a0, ix, iy);
                g->E.a[a1].outp[G_ABOVE] = g->E.a[a0].outp[G_ABOVE];
              }
              break;
            case EMM_:
              if (p >= 0 && q >= 0) {
                add_left(g, p, ix, iy);
                merge_right(g, p, q, g->out_poly);
                add_local_min(g, a0, ix, iy);
                g->E.a[a1].outp[G_ABOVE] = g->E.a[a0].outp[G_ABOVE];
              }
              break;
            default:
              break;
          }
        }
        E = g->E.a;
        if (E[a0].bundle[G_ABOVE][G_CLIP]) E[a1].bside[G_CLIP] = !E[a1].bside[G_CLIP];
        if (E[a1].bundle[G_ABOVE][G_CLIP]) E[a0].bside[G_CLIP] = !E[a0].bside[G_CLIP];
        if (E[a0].bundle[G_ABOVE][G_SUBJ]) E[a1].bside[G_SUBJ] = !E[a1].bside[G_SUBJ];
        if (E[a1].bundle[G_ABOVE][G_SUBJ]) E[a0].bside[G_SUBJ] = !E[a0].bside[G_SUBJ];
        /* swap the e0 and e1 bundles in the AET (GPC:622-657) */
        int pe = E[a0].prev, nx = E[a1].next;
        if (nx >= 0) E[nx].prev = a0;
        if (E[a0].bstate[G_ABOVE] == BHEAD_) {
          int search = 1;
          while (search) {
            if (pe < 0) break;
            pe = E[pe].prev;
            if (pe >= 0) {
              if (E[pe].bstate[G_ABOVE] != BTAIL_) search = 0;
            } else {
              search = 0;
            }
          }
        }
        if (pe < 0) {
          E[aet].prev = a1;
          E[a1].next = aet;
          aet = E[a0].next;
        } else {
          E[E[pe].next].prev = a1;
          E[a1].next = E[pe].next;
          E[pe].next = E[a0].next;
        }
        if (E[a0].next >= 0) E[E[a0].next].prev = pe;
        if (E[a1].next >= 0) E[E[a1].next].prev = a1;
        E[a0].next = nx;
      }
      /* prepare for the next scanbeam (GPC:661-693) */
      E = g->E.a;
      int nx;
      for (int edge = aet; edge >= 0; edge = nx) {
        nx = E[edge].next;
        int sc2 = E[edge].succ;
        if (E[edge].top.y == yt && sc2 >= 0) {
          E[sc2].outp[G_BELOW] = E[edge].outp[G_ABOVE];
          E[sc2].bstate[G_BELOW] = E[edge].bstate[G_ABOVE];
          E[sc2].bundle[G_BELOW][G_CLIP] = E[edge].bundle[G_ABOVE][G_CLIP];
          E[sc2].bundle[G_BELOW][G_SUBJ] = E[edge].bundle[G_ABOVE][G_SUBJ];
          int pe = E[edge].prev;
          if (pe >= 0) E[pe].next = sc2; else aet = sc2;
          if (nx >= 0) E[nx].prev = sc2;
          E[sc2].prev = pe;
          E[sc2].next = nx;
        } else {
          E[edge].outp[G_BELOW] = E[edge].outp[G_ABOVE];
          E[edge].bstate[G_BELOW] = E[edge].bstate[G_ABOVE];
          E[edge].bundle[G_BELOW][G_CLIP] = E[edge].bundle[G_ABOVE][G_CLIP];
          E[edge].bundle[G_BELOW][G_SUBJ] = E[edge].bundle[G_ABOVE][G_SUBJ];
          E[edge].xb = E[edge].xt;
        }
        E[edge].outp[G_ABOVE] = -1;
      }
    }
  }
  free(sbt);

  /* result (count_contours GPC:1473-1504, assembly GPC:698-741) */
  int nc = 0;
  int64_t nvt = 0;
  for (int p = g->out_poly; p >= 0; p = g->P.a[p].next) {
    if (!g->P.a[p].active) continue;
    int nv = 0;
    for (int v = g->P.a[g->P.a[p].proxy].vl; v >= 0; v = g->V.a[v].next) nv++;
    if (nv > 2) {
      g->P.a[p].active = nv;
      nc++;
      nvt += nv;
    } else {
      g->P.a[p].active = 0;
    }
  }
  res->ncont = nc;
  res->nv_total = nvt;
  res->nverts = (int *)malloc(sizeof(int) * (size_t)(nc > 0 ? nc : 1));
  res->hole = (int *)malloc(sizeof(int) * (size_t)(nc > 0 ? nc : 1));
  res->xy = (double *)malloc(sizeof(double) * 2 * (size_t)(nvt > 0 ? nvt : 1));
  int c = 0;
  int64_t off = 0;
  for (int p = g->out_poly; p >= 0; p = g->P.a[p].next) {
    if (!g->P.a[p].active) continue;
    int px2 = g->P.a[p].proxy;
    int nv = g->P.a[p].active;
    res->hole[c] = g->P.a[px2].hole;
    res->nverts[c] = nv;
    int v = nv - 1;
    for (int vi = g->P.a[px2].vl; vi >= 0; vi = g->V.a[vi].next) {
      res->xy[2 * (off + v)] = g->V.a[vi].x;
      res->xy[2 * (off + v) + 1] = g->V.a[vi].y;
      v--;
    }
    off += nv;
    c++;
  }
}

static void gctx_free(gctx *g) {
  free(g->E.a); free(g->B.a); free(g->ys.a); free(g->IT.a);
  free(g->ST.a); free(g->P.a); free(g->V.a);
}

static void make_in(gpolyin *p, int ncont, const int *nverts, const double *xy, int64_t *voff) {
  p->ncont = ncont;
  p->nverts = nverts;
  p->xy = xy;
  int64_t o = 0;
  for (int c = 0; c < ncont; c++) { voff[c] = o; o += nverts[c]; }
  p->voff = voff;
}

/* Flat-array entry point.  Returns 0, or -1 when cont_cap / vert_cap are too
 * small (counts are still written).  stats (optional, 3 ints): max AET size,
 * max IT size, max ST size over all scanbeams. */
int orc_gpc_clip(int op, int s_ncont, const int *s_nverts, const double *s_xy,
                 int c_ncont, const int *c_nverts, const double *c_xy,
                 int *out_ncont, int cont_cap, int *out_nverts, int *out_hole,
                 int64_t *out_nv_total, int64_t vert_cap, double *out_xy, int *stats) {
  gpolyin s, c;
  int64_t *so = (int64_t *)malloc(sizeof(int64_t) * (size_t)(s_ncont + 1));
  int64_t *co = (int64_t *)malloc(sizeof(int64_t) * (size_t)(c_ncont + 1));
  make_in(&s, s_ncont, s_nverts, s_xy, so);
  make_in(&c, c_ncont, c_nverts, c_xy, co);
  gresult r = {0, NULL, NULL, NULL, 0};
  gctx g;
  gclip(op, &s, &c, &r, &g);
  *out_ncont = r.ncont;
  *out_nv_total = r.nv_total;
  int rc = 0;
  if (r.ncont > cont_cap || r.nv_total > vert_cap) {
    rc = -1;
  } else {
    for (int k = 0; k < r.ncont; k++) { out_nverts[k] = r.nverts[k]; out_hole[k] = r.hole[k]; }
    if (r.nv_total) memcpy(out_xy, r.xy, sizeof(double) * 2 * (size_t)r.nv_total);
  }
  if (stats) {
    stats[0] = g.max_aet; stats[1] = g.max_it; stats[2] = g.max_st;
    stats[3] = g.P.n; stats[4] = g.V.n; stats[5] = g.E.n;
  }
  free(r.nverts); free(r.hole); free(r.xy);
  gctx_free(&g);
  free(so);
  free(co);
  return rc;
}

/* ---- area of a result ------------------------------------------------------ */

/* Sum over contours of |shoelace area|, negated for hole contours.  The
 * shoelace runs on coordinates relative to the contour's first vertex: for
 * small contours far from the origin the plain form cancels terms of size
 * |x||y| down to an area of size r^2 and loses ~|x||y|/r^2 ulps. */
double orc_result_area(int ncont, const int *nverts, const int *hole, const double *xy) {
  double total = 0.0;
  int64_t off = 0;
  for (int c = 0; c < ncont; c++) {
    int n = nverts[c];
    double a = 0.0;
    const double x0 = xy[2 * off], y0 = xy[2 * off + 1];
    for (int i = 0; i < n; i++) {
      int j = (i + 1) % n;
      a += (xy[2 * (off + i)] - x0) * (xy[2 * (off + j) + 1] - y0) -
           (xy[2 * (off + j)] - x0) * (xy[2 * (off + i) + 1] - y0);
    }
    a = 0.5 * fabs(a);
    total += hole[c] ? -a : a;
    off += n;
  }
  return total;
}
