/* Harness around the reference's GPC clip core
 * (vector_map_overlay_gpc_kernel.cu:115-750 and 890-1709, sliced by
 * build_ref.sh and compiled for the host with gpc_shim.h).
 *
 * Test infrastructure only: ref_gpc_clip() plays the part of Execute
 * (GPC:81-113) for one pair, on flat ring arrays instead of the device CSR.
 */
#include "gpc_shim.h"

/* the horizontal-state table that run() uploads (GPC:62) */
h_state next_h_state[3][6] = {{BH, TH, TH, BH, NH, NH},
                              {NH, NH, NH, NH, TH, TH},
                              {NH, NH, NH, NH, BH, BH}};

#include "gpc_core.slice.inc"

static void make_polygon(gpc_polygon *p, int ncont, const int *nverts,
                         const int *hole, const double *xy) {
  p->num_contours = ncont;
  p->hole = ncont ? (int *)malloc(sizeof(int) * ncont) : NULL;
  p->contour = ncont ? (gpc_vertex_list *)malloc(sizeof(gpc_vertex_list) * ncont) : NULL;
  long long off = 0;
  for (int c = 0; c < ncont; c++) {
    p->hole[c] = hole ? hole[c] : 0;
    p->contour[c].num_vertices = nverts[c];
    p->contour[c].vertex = (gpc_vertex *)malloc(sizeof(gpc_vertex) * (nverts[c] > 0 ? nverts[c] : 1));
    for (int v = 0; v < nverts[c]; v++) {
      p->contour[c].vertex[v].x = xy[2 * (off + v)];
      p->contour[c].vertex[v].y = xy[2 * (off + v) + 1];
    }
    off += nverts[c];
  }
}

extern "C" {

/* Clips subject by clip with operation op (0 DIFF, 1 INT, 2 XOR, 3 UNION).
 * Output: *out_ncont contours with out_nverts[c], out_hole[c] and vertices
 * packed in out_xy.  Returns 0, or -1 when a capacity is too small (the
 * counts are still written so the caller can retry).
 */
int ref_gpc_clip(int op,
                 int s_ncont, const int *s_nverts, const int *s_hole, const double *s_xy,
                 int c_ncont, const int *c_nverts, const int *c_hole, const double *c_xy,
                 int *out_ncont, int cont_cap, int *out_nverts, int *out_hole,
                 long long *out_nv_total, long long vert_cap, double *out_xy) {
  gpc_polygon subj, clip, result;
  make_polygon(&subj, s_ncont, s_nverts, s_hole, s_xy);
  make_polygon(&clip, c_ncont, c_nverts, c_hole, c_xy);
  gpc_polygon_clip((gpc_op)op, &subj, &clip, &result);
  long long total = 0;
  for (int c = 0; c < result.num_contours; c++) total += result.contour[c].num_vertices;
  *out_ncont = result.num_contours;
  *out_nv_total = total;
  int rc = 0;
  if (result.num_contours > cont_cap || total > vert_cap) {
    rc = -1;
  } else {
    long long off = 0;
    for (int c = 0; c < result.num_contours; c++) {
      out_nverts[c] = result.contour[c].num_vertices;
      out_hole[c] = result.hole[c];
      for (int v = 0; v < result.contour[c].num_vertices; v++) {
        out_xy[2 * (off + v)] = result.contour[c].vertex[v].x;
        out_xy[2 * (off + v) + 1] = result.contour[c].vertex[v].y;
      }
      off += result.contour[c].num_vertices;
    }
  }
  gpc_free_polygon(&result);
  gpc_free_polygon(&subj);
  gpc_free_polygon(&clip);
  return rc;
}

}  /* extern "C" */
