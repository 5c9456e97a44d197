/* Harness around the reference's bottom-up CPU path (BotomUp-rtree.cu).
 *
 * Test infrastructure only.  The reference code itself comes from slices of
 * BotomUp-rtree.cu made by build_ref.sh; this file only supplies what the
 * reference's main() does around them (reading boxes, the min/max scan of
 * BU:682-693, and the digest loop of BU:999-1018) so the slices can run on
 * arrays instead of data/Rect1024.txt.  Compiled once per fanout (-Dm=F).
 */
#include "cuda_host_shim.h"
#include <stdint.h>
#include <time.h>

#define printf(...) ((void)0)
#include "bu_defs.slice.inc"
#undef printf

static double now_ms(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
}

extern "C" {

int ref_bu_fanout(void) { return m; }

/* Runs the reference's CPU build and CPU self-join query over n boxes.
 *   rects   n x 4 int64 in (x1, y1, x2, y2) order; ids: bounding_box.data.
 *   keys_out       n zOrderValue, input order (CalcuateZOrderValue on the
 *                  shifted boxes, BU:704-721 then BU:769).
 *   scale_out      the power-of-ten scale of BU:711-716.
 *   nodes (flag, num, mbr[m*4], children[m], data[m]) for up to nn_cap nodes,
 *   in the reference's node order (leaves first, root last).
 *   sorted_ids_out n ids in qsort order (BU:780).
 *   digests        sum, sum1, sum2 (BU:1023-1025), sum3 (BU:1026).
 *   ms             [0] qsort + packing (BU:776-833), [1] DFS query loop.
 * Returns the node count, or -1 if nn_cap is too small.
 */
long long ref_bu_run(const long long *rects, const int *ids, int n,
                     unsigned long long *keys_out, long long *scale_out,
                     int nn_cap, int *flag, int *num, long long *mbr,
                     int *children, int *data, int *root_out,
                     int *sorted_ids_out, long long *digests, double *ms,
                     int do_query) {
  int num_contours = n;
  bounding_box *pointers = (bounding_box *)calloc((size_t)n, sizeof(bounding_box));
  rtree_node *nodes = (rtree_node *)calloc((size_t)nn_cap, sizeof(rtree_node));
  if (!pointers || !nodes) { free(pointers); free(nodes); return -1; }
  long long minX = (long long)1e17, maxX = 0, minY = (long long)1e17, maxY = 0;
  int i;
  for (i = 0; i < n; i++) {
    long long x1 = rects[4 * i + 0], y1 = rects[4 * i + 1];
    long long x2 = rects[4 * i + 2], y2 = rects[4 * i + 3];
    if (x1 < minX) minX = x1;
    if (x2 > maxX) maxX = x2;
    if (y1 < minY) minY = y1;
    if (y2 > maxY) maxY = y2;
    pointers[i].rect[0] = x1;
    pointers[i].rect[1] = y1;
    pointers[i].rect[2] = x2;
    pointers[i].rect[3] = y2;
    pointers[i].data = ids ? ids[i] : i;
  }
  {
#define printf(...) ((void)0)
#include "bu_shift.slice.inc"
#undef printf
  }
  *scale_out = maxY;
  CalcuateZOrderValue(pointers, num_contours, (int)minX, (int)minY, maxY);
  for (i = 0; i < n; i++) keys_out[i] = pointers[i].zOrderValue;

  /* the reference sizes nodes as 3*N/m (BU:674); the caller passes a bound */
  long long n_nodes = 0;
  int root = 0;
  double t0 = now_ms();
  {
#include "bu_pack.slice.inc"
    n_nodes = index;
    root = index - numOfGroup;
  }
  double t1 = now_ms();
  ms[0] = t1 - t0;
  if (n_nodes > nn_cap) { free(pointers); free(nodes); return -1; }
  for (long long k = 0; k < n_nodes; k++) {
    flag[k] = nodes[k].flag;
    num[k] = nodes[k].num;
    for (int e = 0; e < m; e++) {
      for (int c = 0; c < 4; c++) mbr[(k * m + e) * 4 + c] = nodes[k].mbr[e].rect[c];
      children[k * m + e] = nodes[k].children[e];
      data[k * m + e] = nodes[k].data[e];
    }
  }
  *root_out = root;
  for (i = 0; i < n; i++) sorted_ids_out[i] = pointers[i].data;

  long long sum = 0, sum1 = 0, sum2 = 0;
  double t2 = now_ms();
  if (do_query) {
    for (i = 0; i < n; i++) {
      rtree_rectangle temp;
      int numq = 0, num2 = 0;
      temp.rect[0] = pointers[i].rect[0];
      temp.rect[1] = pointers[i].rect[1];
      temp.rect[2] = pointers[i].rect[2];
      temp.rect[3] = pointers[i].rect[3];
      int count = RtreeSearch(nodes, root, temp, pointers[i].data, &numq, num2);
      sum1 += count;
      sum += numq;
      sum2 += num2;
    }
    sum2 /= 2;
  }
  ms[1] = now_ms() - t2;
  digests[0] = sum;
  digests[1] = sum1;
  digests[2] = sum2;
  digests[3] = RtreeSearch1(nodes, root);
  free(pointers);
  free(nodes);
  return n_nodes;
}

/* The reference's Interleave (BU:98-123) on four values. */
unsigned long long ref_bu_interleave(unsigned long long a1, unsigned long long a2,
                                     unsigned long long a3, unsigned long long a4) {
  return Interleave(a1, a2, a3, a4);
}

/* The reference's CPU Overlap predicate (BU:496-506) on two (x1,y1,x2,y2) boxes. */
int ref_bu_overlap(const long long *a, const long long *b) {
  rtree_rectangle ra, rb;
  for (int c = 0; c < 4; c++) { ra.rect[c] = a[c]; rb.rect[c] = b[c]; }
  return Overlap(ra, rb);
}

}  /* extern "C" */
