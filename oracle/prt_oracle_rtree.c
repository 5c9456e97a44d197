/* ORACLE — test infrastructure only.  CPU restatement of the reference's
 * R-tree path, used by tests/ and bench.py's CPU baseline as the checker;
 * never linked into the product library.
 *
 * Restates:
 *   BotomUp-rtree.cu:73-123   key generation (shift, power-of-ten scale,
 *                             4-D 2-bit-chunk interleave of the corners)
 *   BotomUp-rtree.cu:704-716  min shift and scale selection
 *   BotomUp-rtree.cu:780-830  stable sort + bottom-up packing (leaves first)
 *   TopDown-rtree.cu:504-624  top-down build: per level, a stable sort of
 *                             each segment by x1 (even level) or y1 (odd)
 *   BotomUp-rtree.cu:439-483, TopDown-rtree.cu:56-76   DFS query counters
 *   BotomUp-rtree.cu:574-590, TopDown-rtree.cu:78-93   sibling-overlap count
 * plus the project's MORTON32 centre key (no reference counterpart).
 *
 * Coordinates are handled as double, which is exact for float32, float64 and
 * integers below 2^53.  The reference's overlap predicate
 * (width_a + width_b + 1e-8 < union width => disjoint, BU:496-506, TD:26-39)
 * equals the closed-interval intersection test for valid boxes, which is what
 * is used here.
 *
 * Tree representation shared with the product (the reference's node order is
 * derived from it): level 0 holds the N records in leaf order; entry j of level
 * l+1 is the union of entries [jF, min((j+1)F, n_l)) of level l; the root node
 * holds the entries of the first level with n_l <= F.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

enum { ORC_I64 = 0, ORC_F32 = 1, ORC_F64 = 2, ORC_I32 = 3 };

typedef struct { double x1, y1, x2, y2; } obox;

static void load_boxes(const void *src, int ct, int64_t n, obox *out) {
  for (int64_t i = 0; i < n; i++) {
    double v[4];
    for (int c = 0; c < 4; c++) {
      switch (ct) {
        case ORC_I64: v[c] = (double)((const int64_t *)src)[4 * i + c]; break;
        case ORC_F32: v[c] = (double)((const float *)src)[4 * i + c]; break;
        case ORC_F64: v[c] = ((const double *)src)[4 * i + c]; break;
        default: v[c] = (double)((const int32_t *)src)[4 * i + c]; break;
      }
    }
    out[i].x1 = v[0]; out[i].y1 = v[1]; out[i].x2 = v[2]; out[i].y2 = v[3];
  }
}

static int overlaps(const obox *a, const obox *b) {
  return a->x1 <= b->x2 && b->x1 <= a->x2 && a->y1 <= b->y2 && b->y1 <= a->y2;
}

/* ---- keys -------------------------------------------------------------- */

/* Spreads the low 16 bits of v into 2-bit chunks, one chunk per byte
 * (chunk k -> bits 8k..8k+1), by three mask-and-shift rounds (the "binary
 * magic numbers" interleave the reference names at BU:97). */
static uint64_t spread_2bit_chunks(uint64_t v) {
  v = (v | (v << 24)) & 0x000000FF000000FFull;
  v = (v | (v << 12)) & 0x000F000F000F000Full;
  v = (v | (v << 6)) & 0x0303030303030303ull;
  return v;
}

uint64_t orc_interleave4(uint64_t a1, uint64_t a2, uint64_t a3, uint64_t a4) {
  return (spread_2bit_chunks(a1) << 6) | (spread_2bit_chunks(a2) << 4) |
         (spread_2bit_chunks(a3) << 2) | spread_2bit_chunks(a4);
}

/* REF64 keys on int64 boxes (x1,y1,x2,y2): shift by (min x1, min y1), choose
 * scale = 10^k so that the larger extent / scale <= 1e4, integer-divide each
 * corner coordinate by the scale and interleave (BU:682-716, BU:81-92).
 * Returns the scale; shift_out receives (minX, minY). */
int64_t orc_keys_ref64(const int64_t *rects, int64_t n, uint64_t *keys, int64_t *shift_out) {
  int64_t minX = (int64_t)1e17, maxX = 0, minY = (int64_t)1e17, maxY = 0;
  for (int64_t i = 0; i < n; i++) {
    if (rects[4 * i + 0] < minX) minX = rects[4 * i + 0];
    if (rects[4 * i + 2] > maxX) maxX = rects[4 * i + 2];
    if (rects[4 * i + 1] < minY) minY = rects[4 * i + 1];
    if (rects[4 * i + 3] > maxY) maxY = rects[4 * i + 3];
  }
  int64_t ext = (maxX - minX) > (maxY - minY) ? (maxX - minX) : (maxY - minY);
  int64_t scale = 1;
  while (ext > 10000) { scale *= 10; ext /= 10; }
  for (int64_t i = 0; i < n; i++) {
    uint64_t q[4];
    q[0] = (uint64_t)((rects[4 * i + 0] - minX) / scale);
    q[1] = (uint64_t)((rects[4 * i + 1] - minY) / scale);
    q[2] = (uint64_t)((rects[4 * i + 2] - minX) / scale);
    q[3] = (uint64_t)((rects[4 * i + 3] - minY) / scale);
    keys[i] = orc_interleave4(q[0], q[1], q[2], q[3]);
  }
  if (shift_out) { shift_out[0] = minX; shift_out[1] = minY; }
  return scale;
}

static uint32_t part1by1_16(uint32_t v) {
  v &= 0xFFFFu;
  v = (v | (v << 8)) & 0x00FF00FFu;
  v = (v | (v << 4)) & 0x0F0F0F0Fu;
  v = (v | (v << 2)) & 0x33333333u;
  v = (v | (v << 1)) & 0x55555555u;
  return v;
}

/* MORTON32 keys: box centre on a 65536 x 65536 grid spanning the data extent
 * (one scale for both axes, as the reference uses one scale, BU:711), x bits
 * in the even positions.  g = (uint32)((c - min) * (65535 / extent)).  The
 * operation order is fixed so the device kernel reproduces it bit for bit. */
void orc_keys_morton32(const void *boxes, int ct, int64_t n, uint32_t *keys, double *ext_out) {
  obox *b = (obox *)malloc(sizeof(obox) * (size_t)(n > 0 ? n : 1));
  load_boxes(boxes, ct, n, b);
  double minX = INFINITY, minY = INFINITY, maxX = -INFINITY, maxY = -INFINITY;
  for (int64_t i = 0; i < n; i++) {
    if (b[i].x1 < minX) minX = b[i].x1;
    if (b[i].y1 < minY) minY = b[i].y1;
    if (b[i].x2 > maxX) maxX = b[i].x2;
    if (b[i].y2 > maxY) maxY = b[i].y2;
  }
  double ext = (maxX - minX) > (maxY - minY) ? (maxX - minX) : (maxY - minY);
  double inv = ext > 0.0 ? 65535.0 / ext : 0.0;
  for (int64_t i = 0; i < n; i++) {
    double cx = 0.5 * (b[i].x1 + b[i].x2);
    double cy = 0.5 * (b[i].y1 + b[i].y2);
    double tx = (cx - minX) * inv;
    double ty = (cy - minY) * inv;
    uint32_t gx = tx >= 65535.0 ? 65535u : (tx > 0.0 ? (uint32_t)tx : 0u);
    uint32_t gy = ty >= 65535.0 ? 65535u : (ty > 0.0 ? (uint32_t)ty : 0u);
    keys[i] = part1by1_16(gx) | (part1by1_16(gy) << 1);
  }
  if (ext_out) { ext_out[0] = minX; ext_out[1] = minY; ext_out[2] = ext; }
  free(b);
}

/* ---- stable sorts ------------------------------------------------------ */

typedef struct { uint64_t key; int64_t idx; } kidx;
static int cmp_kidx(const void *a, const void *b) {
  const kidx *x = (const kidx *)a, *y = (const kidx *)b;
  if (x->key != y->key) return x->key < y->key ? -1 : 1;
  return x->idx < y->idx ? -1 : (x->idx > y->idx);
}

/* perm[j] = index of the j-th smallest key; ties keep input order. */
void orc_stable_argsort_u64(const uint64_t *keys, int64_t n, int64_t *perm) {
  kidx *t = (kidx *)malloc(sizeof(kidx) * (size_t)(n > 0 ? n : 1));
  for (int64_t i = 0; i < n; i++) { t[i].key = keys[i]; t[i].idx = i; }
  qsort(t, (size_t)n, sizeof(kidx), cmp_kidx);
  for (int64_t i = 0; i < n; i++) perm[i] = t[i].idx;
  free(t);
}

typedef struct { int64_t seg; double c; int64_t pos; int64_t rec; } segrec;
static int cmp_segrec(const void *a, const void *b) {
  const segrec *x = (const segrec *)a, *y = (const segrec *)b;
  if (x->seg != y->seg) return x->seg < y->seg ? -1 : 1;
  if (x->c < y->c) return -1;
  if (x->c > y->c) return 1;
  return x->pos < y->pos ? -1 : (x->pos > y->pos);
}

/* ---- levels -------------------------------------------------------------- */

/* Number of entry levels (level 0 = records) for n records at fanout f:
 * levels continue while the current level holds more than f entries. */
int orc_num_levels(int64_t n, int f) {
  int L = 1;
  int64_t c = n;
  while (c > f) { c = (c + f - 1) / f; L++; }
  return L;
}

int64_t orc_level_count(int64_t n, int f, int l) {
  int64_t c = n;
  for (int i = 0; i < l; i++) c = (c + f - 1) / f;
  return c;
}

/* Packs the tree for a leaf order perm: level_mbr receives, level after level,
 * n_l boxes (x1,y1,x2,y2 as double) for l = 0..L-1 (level 0 = records in leaf
 * order).  Returns the total number of entries written. */
int64_t orc_pack(const void *boxes, int ct, int64_t n, int f, const int64_t *perm, double *level_mbr) {
  obox *b = (obox *)malloc(sizeof(obox) * (size_t)(n > 0 ? n : 1));
  load_boxes(boxes, ct, n, b);
  int L = orc_num_levels(n, f);
  obox *cur = (obox *)level_mbr;
  for (int64_t j = 0; j < n; j++) cur[j] = b[perm[j]];
  int64_t total = n, cnt = n;
  for (int l = 1; l < L; l++) {
    int64_t nc = (cnt + f - 1) / f;
    obox *nxt = cur + cnt;
    for (int64_t j = 0; j < nc; j++) {
      obox u = cur[j * f];
      int64_t end = (j + 1) * f < cnt ? (j + 1) * f : cnt;
      for (int64_t k = j * f + 1; k < end; k++) {
        if (cur[k].x1 < u.x1) u.x1 = cur[k].x1;
        if (cur[k].y1 < u.y1) u.y1 = cur[k].y1;
        if (cur[k].x2 > u.x2) u.x2 = cur[k].x2;
        if (cur[k].y2 > u.y2) u.y2 = cur[k].y2;
      }
      nxt[j] = u;
    }
    total += nc;
    cur = nxt;
    cnt = nc;
  }
  free(b);
  return total;
}

/* Top-down leaf order (TD:575-624 with the CPU key (segment, coordinate),
 * TD:577-587): with H levels and S_p = f^(H-p), level p = 0..H-1 stably sorts
 * each run of S_p consecutive records by x1 (p even) or y1 (p odd). */
void orc_td_order(const void *boxes, int ct, int64_t n, int f, int64_t *perm) {
  obox *b = (obox *)malloc(sizeof(obox) * (size_t)(n > 0 ? n : 1));
  load_boxes(boxes, ct, n, b);
  int H = orc_num_levels(n, f);
  segrec *t = (segrec *)malloc(sizeof(segrec) * (size_t)(n > 0 ? n : 1));
  for (int64_t i = 0; i < n; i++) perm[i] = i;
  for (int p = 0; p < H; p++) {
    /* S_p = f^(H-p); int64 arithmetic with saturation at n */
    int64_t seg = 1;
    for (int k = 0; k < H - p; k++) { seg *= f; if (seg >= n) { seg = n > 0 ? n : 1; break; } }
    for (int64_t i = 0; i < n; i++) {
      const obox *r = &b[perm[i]];
      t[i].seg = i / seg;
      t[i].c = (p & 1) ? r->y1 : r->x1;
      t[i].pos = i;
      t[i].rec = perm[i];
    }
    qsort(t, (size_t)n, sizeof(segrec), cmp_segrec);
    for (int64_t i = 0; i < n; i++) perm[i] = t[i].rec;
  }
  free(t);
  free(b);
}

/* ---- queries --------------------------------------------------------------- */

typedef struct {
  int f, L;
  int64_t cnt[40];
  const obox *lv[40];
} otree;

static void otree_init(otree *t, const double *level_mbr, int64_t n, int f) {
  t->f = f;
  t->L = orc_num_levels(n, f);
  const obox *p = (const obox *)level_mbr;
  for (int l = 0; l < t->L; l++) {
    t->cnt[l] = orc_level_count(n, f, l);
    t->lv[l] = p;
    p += t->cnt[l];
  }
}

typedef struct {
  int64_t examined;  /* entries looked at: node fill (BU) or f per node (TD) */
  int64_t count;     /* sum over visited nodes of max(0, overlapping - 1) */
  int64_t hits;      /* overlapping leaf entries */
} qcount;

/* DFS from node `node` of node level l (node level l groups entries of level l). */
static void dfs(const otree *t, int l, int64_t node, const obox *q, int td_slots,
                qcount *c, int64_t *pairs, int64_t *npairs, int64_t cap, int64_t qid) {
  int64_t first = node * t->f;
  int64_t last = first + t->f < t->cnt[l] ? first + t->f : t->cnt[l];
  c->examined += td_slots ? t->f : (last - first);
  int64_t k = 0;
  for (int64_t e = first; e < last; e++) {
    if (!overlaps(&t->lv[l][e], q)) continue;
    k++;
    if (l == 0) {
      c->hits++;
      if (pairs) {
        if (*npairs < cap) { pairs[2 * *npairs] = e; pairs[2 * *npairs + 1] = qid; }
        (*npairs)++;
      }
    } else {
      dfs(t, l - 1, e, q, td_slots, c, pairs, npairs, cap, qid);
    }
  }
  if (k > 1) c->count += k - 1;
}

/* Per-query reference counters (RtreeSearch semantics) for nq query boxes;
 * out[3*i..] = (examined, count, hits).  td_slots=1 counts f slots per node as
 * TopDown-rtree.cu:58-59 does. */
void orc_query_counts(const double *level_mbr, int64_t n, int f, const void *qboxes, int qct,
                      int64_t nq, int td_slots, int64_t *out) {
  otree t;
  otree_init(&t, level_mbr, n, f);
  obox *q = (obox *)malloc(sizeof(obox) * (size_t)(nq > 0 ? nq : 1));
  load_boxes(qboxes, qct, nq, q);
  for (int64_t i = 0; i < nq; i++) {
    qcount c = {0, 0, 0};
    dfs(&t, t.L - 1, 0, &q[i], td_slots, &c, NULL, NULL, 0, i);
    out[3 * i] = c.examined;
    out[3 * i + 1] = c.count;
    out[3 * i + 2] = c.hits;
  }
  free(q);
}

/* Candidate pairs (leaf position, query id) of a join, in DFS order per query.
 * Returns the pair count (pairs beyond cap are counted, not written). */
int64_t orc_join_pairs(const double *level_mbr, int64_t n, int f, const void *qboxes, int qct,
                       int64_t nq, int64_t *pairs, int64_t cap) {
  otree t;
  otree_init(&t, level_mbr, n, f);
  obox *q = (obox *)malloc(sizeof(obox) * (size_t)(nq > 0 ? nq : 1));
  load_boxes(qboxes, qct, nq, q);
  int64_t np = 0;
  for (int64_t i = 0; i < nq; i++) {
    qcount c = {0, 0, 0};
    dfs(&t, t.L - 1, 0, &q[i], 0, &c, pairs, &np, cap, i);
  }
  free(q);
  return np;
}

/* Pairs of overlapping sibling entries over all nodes (RtreeSearch1). */
int64_t orc_sibling_overlaps(const double *level_mbr, int64_t n, int f) {
  otree t;
  otree_init(&t, level_mbr, n, f);
  int64_t total = 0;
  for (int l = 0; l < t.L; l++) {
    int64_t nodes = (t.cnt[l] + f - 1) / f;
    for (int64_t nd = 0; nd < nodes; nd++) {
      int64_t first = nd * f;
      int64_t last = first + f < t.cnt[l] ? first + f : t.cnt[l];
      for (int64_t i = first + 1; i < last; i++)
        for (int64_t j = first; j < i; j++)
          if (overlaps(&t.lv[l][i], &t.lv[l][j])) total++;
    }
  }
  return total;
}
