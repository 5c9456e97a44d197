/* Harness around the reference's readData (vector_map_overlay_gpc_kernel.cu:
 * 752-888, sliced by build_ref.sh): the reader of the base and overlay
 * polygon files, compiled for the host.
 *
 * Test infrastructure only.  readData allocates its arrays with MALLOC_CPU
 * (from the reference's missing common.h) and uploads the vertices with
 * cudaMalloc / cudaMemcpy; here those are plain host allocations and copies,
 * so every array it returns is host memory that ref_read_data copies out.
 */
#include <stdint.h>

#include "gpc_shim.h"

#define MALLOC_CPU(p, b, s, t) \
  do { (p) = (t *)malloc((b) > 0 ? (size_t)(b) : 1); } while (0)
#define FREE_CPU(p) do { free(p); } while (0)
enum prt_shim_memcpy_kind { cudaMemcpyHostToDevice = 1 };
static int cudaMalloc(void **p, size_t b) {
  *p = malloc(b ? b : 1);
  return 0;
}
static int cudaMemcpy(void *d, const void *s, size_t b, prt_shim_memcpy_kind) {
  memcpy(d, s, b);
  return 0;
}

#include "readdata.slice.inc"

extern "C" {

/* Runs readData on the two files and copies its outputs: counts[0..1] the
 * polygon counts, counts[2..3] the vertex counts (base, overlay).  Per layer
 * L (0 base, 1 overlay): num, prefix (int64), hole, rect (P x 4: readData's
 * rect1..rect4 / rect*_query) and the vertices (x, y).  min_xy: readData's
 * minX / minY, which start at the values passed in.  Returns -1 (counts set,
 * nothing copied) when a layer exceeds its caps. */
int ref_read_data(const char *base, const char *overlay, int64_t *counts, int32_t *num0, int64_t *prefix0,
                  int32_t *hole0, int32_t *rect0, double *vert0, int32_t *num1, int64_t *prefix1, int32_t *hole1,
                  int32_t *rect1o, double *vert1, int64_t poly_cap, int64_t vert_cap, int32_t *min_xy) {
  int *r1, *r2, *r3, *r4, *q1, *q2, *q3, *q4, *nb, *no, *hb, *ho;
  long int *pb, *po;
  gpc_vertex *vb, *vo;
  int np0 = 0, np1 = 0;
  int mx = min_xy[0], my = min_xy[1];
  readData((char *)base, (char *)overlay, &r1, &r2, &r3, &r4, &np0, &q1, &q2, &q3, &q4, &np1, &nb, &pb, &vb, &no,
           &po, &vo, &mx, &my, &hb, &ho);
  const int64_t nv0 = np0 ? (int64_t)pb[np0 - 1] + nb[np0 - 1] : 0;
  const int64_t nv1 = np1 ? (int64_t)po[np1 - 1] + no[np1 - 1] : 0;
  counts[0] = np0;
  counts[1] = np1;
  counts[2] = nv0;
  counts[3] = nv1;
  min_xy[0] = mx;
  min_xy[1] = my;
  int rc = 0;
  if (np0 > poly_cap || np1 > poly_cap || nv0 > vert_cap || nv1 > vert_cap) {
    rc = -1;
  } else {
    for (int i = 0; i < np0; i++) {
      num0[i] = nb[i];
      prefix0[i] = pb[i];
      hole0[i] = hb[i];
      rect0[4 * i] = r1[i];
      rect0[4 * i + 1] = r2[i];
      rect0[4 * i + 2] = r3[i];
      rect0[4 * i + 3] = r4[i];
    }
    for (int i = 0; i < np1; i++) {
      num1[i] = no[i];
      prefix1[i] = po[i];
      hole1[i] = ho[i];
      rect1o[4 * i] = q1[i];
      rect1o[4 * i + 1] = q2[i];
      rect1o[4 * i + 2] = q3[i];
      rect1o[4 * i + 3] = q4[i];
    }
    for (int64_t v = 0; v < nv0; v++) {
      vert0[2 * v] = vb[v].x;
      vert0[2 * v + 1] = vb[v].y;
    }
    for (int64_t v = 0; v < nv1; v++) {
      vert1[2 * v] = vo[v].x;
      vert1[2 * v + 1] = vo[v].y;
    }
  }
  free(r1); free(r2); free(r3); free(r4);
  free(q1); free(q2); free(q3); free(q4);
  free(nb); free(no); free(hb); free(ho);
  free(pb); free(po); free(vb); free(vo);
  return rc;
}

}  // extern "C"
