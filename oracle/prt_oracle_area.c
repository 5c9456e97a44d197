/* ORACLE — test infrastructure only.  CPU reference gradient of the
 * intersection area of two polygons (even-odd fill, the fill rule GPC's
 * parity tracking implements), used to check the device adjoint kernel.
 *
 * Boundary-integral form: the boundary of A∩B is made of the pieces of A's
 * edges inside B and of B's edges inside A.  For an edge p -> q of a ring
 * traversed with the material on its left (orientation sign s = +1; outer
 * rings CCW and hole rings CW give s = +1, the opposite orientation s = -1),
 * with outward normal N = s * (q.y - p.y, p.x - q.x) and inside parameter
 * intervals [t0, t1] along the edge,
 *     d area / d q += N * sum (t1^2 - t0^2) / 2
 *     d area / d p += N * sum ((t1 - t0) - (t1^2 - t0^2) / 2)
 *     area         += s * sum (x(t0) y(t1) - x(t1) y(t0)) / 2      (Green)
 * Degenerate contacts (collinear overlapping edges, vertices exactly on the
 * other boundary) have measure zero and are not treated specially.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

typedef struct {
  int ncont;
  const int *nverts;
  const int *hole;
  const double *xy;
} apoly;

static int inside_evenodd(const apoly *p, double px, double py) {
  int c = 0;
  int64_t off = 0;
  for (int r = 0; r < p->ncont; r++) {
    int n = p->nverts[r];
    const double *v = p->xy + 2 * off;
    for (int i = 0; i < n; i++) {
      int j = (i + 1) % n;
      double ax = v[2 * i], ay = v[2 * i + 1], bx = v[2 * j], by = v[2 * j + 1];
      if ((ay > py) != (by > py)) {
        double xi = ax + (py - ay) * (bx - ax) / (by - ay);
        if (px < xi) c ^= 1;
      }
    }
    off += n;
  }
  return c;
}

static int cmp_dbl(const void *a, const void *b) {
  double x = *(const double *)a, y = *(const double *)b;
  return (x > y) - (x < y);
}

/* Accumulates the boundary pieces of `a` inside `b` into ga (2 per vertex of
 * a); returns their Green's-theorem area contribution. */
static double pieces(const apoly *a, const apoly *b, double *ga) {
  int64_t nb = 0;
  for (int r = 0; r < b->ncont; r++) nb += b->nverts[r];
  double *ts = (double *)malloc(sizeof(double) * (size_t)(nb + 2));
  double area = 0.0;
  int64_t off = 0;
  for (int r = 0; r < a->ncont; r++) {
    int n = a->nverts[r];
    const double *v = a->xy + 2 * off;
    double sa = 0.0;
    for (int i = 0; i < n; i++) {
      int j = (i + 1) % n;
      sa += v[2 * i] * v[2 * j + 1] - v[2 * j] * v[2 * i + 1];
    }
    double s = (sa >= 0.0 ? 1.0 : -1.0) * ((a->hole && a->hole[r]) ? -1.0 : 1.0);
    for (int i = 0; i < n; i++) {
      int j = (i + 1) % n;
      double px = v[2 * i], py = v[2 * i + 1], qx = v[2 * j], qy = v[2 * j + 1];
      double rx = qx - px, ry = qy - py;
      int nt = 0;
      ts[nt++] = 0.0;
      int64_t boff = 0;
      for (int rb = 0; rb < b->ncont; rb++) {
        int m = b->nverts[rb];
        const double *w = b->xy + 2 * boff;
        for (int k = 0; k < m; k++) {
          int l = (k + 1) % m;
          double ax = w[2 * k], ay = w[2 * k + 1];
          double sx = w[2 * l] - ax, sy = w[2 * l + 1] - ay;
          double den = rx * sy - ry * sx;
          if (den == 0.0) continue;
          double apx = ax - px, apy = ay - py;
          double t = (apx * sy - apy * sx) / den;
          double u = (apx * ry - apy * rx) / den;
          if (t > 0.0 && t < 1.0 && u >= 0.0 && u <= 1.0) ts[nt++] = t;
        }
        boff += m;
      }
      ts[nt++] = 1.0;
      qsort(ts + 1, (size_t)(nt - 2), sizeof(double), cmp_dbl);
      double nx = s * ry, ny = -s * rx;
      for (int k = 0; k + 1 < nt; k++) {
        double t0 = ts[k], t1 = ts[k + 1];
        if (!(t1 > t0)) continue;
        double tm = 0.5 * (t0 + t1);
        if (!inside_evenodd(b, px + tm * rx, py + tm * ry)) continue;
        double it = 0.5 * (t1 * t1 - t0 * t0);
        double i1 = (t1 - t0) - it;
        ga[2 * (off + j)] += nx * it;
        ga[2 * (off + j) + 1] += ny * it;
        ga[2 * (off + i)] += nx * i1;
        ga[2 * (off + i) + 1] += ny * i1;
        double x0 = px + t0 * rx, y0 = py + t0 * ry, x1 = px + t1 * rx, y1 = py + t1 * ry;
        area += s * 0.5 * (x0 * y1 - x1 * y0);
      }
    }
    off += n;
  }
  free(ts);
  return area;
}

/* Gradient of area(A ∩ B) with respect to every vertex of A (ga) and B (gb);
 * ga and gb are overwritten.  Returns the area computed from the same pieces. */
double orc_area_grad(int a_ncont, const int *a_nverts, const int *a_hole, const double *a_xy,
                     int b_ncont, const int *b_nverts, const int *b_hole, const double *b_xy,
                     double *ga, double *gb) {
  apoly A = {a_ncont, a_nverts, a_hole, a_xy};
  apoly B = {b_ncont, b_nverts, b_hole, b_xy};
  int64_t na = 0, nb = 0;
  for (int r = 0; r < a_ncont; r++) na += a_nverts[r];
  for (int r = 0; r < b_ncont; r++) nb += b_nverts[r];
  for (int64_t i = 0; i < 2 * na; i++) ga[i] = 0.0;
  for (int64_t i = 0; i < 2 * nb; i++) gb[i] = 0.0;
  return pieces(&A, &B, ga) + pieces(&B, &A, gb);
}
