/* Harness around the reference's top-down CPU path (TopDown-rtree.cu).
 *
 * Test infrastructure only.  The reference code comes from slices of
 * TopDown-rtree.cu made by build_ref.sh (level offsets TD:504-524, CPU build
 * TD:575-624, RtreeSearch / RtreeSearch1 TD:56-93); this file supplies the
 * box array that main() reads from data/Rect1024.txt (TD:486-503) and the
 * digest loop of TD:777-798.  Compiled once per fanout (-DM=F).
 */
#include "cuda_host_shim.h"
#include <stdint.h>
#include <time.h>

#include "td_defs.slice.inc"

static double now_ms(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
}

extern "C" {

int ref_td_fanout(void) { return M; }

/* Runs the reference's CPU top-down build and CPU self-join query.
 *   rects  n x 4 int64 in (x1, y1, x2, y2) order.
 *   nodes_index / nodes_mbr (x1, y1, x2, y2 per slot) for up to slots_cap
 *   slots; empty slots keep index 0 and a zero MBR.
 *   level_offsets_out  the offset vector (up to 64 entries).
 *   sorted_rects_out   n x 4, the final record order (the leaf order).
 *   digests  sum, sum1, sum2 (TD:794-796), sum3 (TD:797).
 *   ms       [0] CPU build (TD:572-627), [1] DFS query loop (TD:776-793).
 * Returns the slot count, or -1 if slots_cap is too small.
 */
long long ref_td_run(const long long *rects, int n, long long slots_cap,
                     int *nodes_index, long long *nodes_mbr,
                     int *level_offsets_out, int *n_offsets_out,
                     long long *sorted_rects_out, long long *digests, double *ms,
                     int do_query) {
  int size = n;
  vector<int> offset;
  MBR *nums = (MBR *)calloc((size_t)n, sizeof(MBR));
  for (int i = 0; i < n; i++) {
    nums[i].x1 = rects[4 * i + 0];
    nums[i].y1 = rects[4 * i + 1];
    nums[i].x2 = rects[4 * i + 2];
    nums[i].y2 = rects[4 * i + 3];
  }
#include "td_offsets.slice.inc"
  long long n_slots = offset.back();
  if (n_slots > slots_cap || (long long)offset.size() > 64) { free(nums); return -1; }
  MBR *nodes_mbr_c = (MBR *)calloc((size_t)n_slots, sizeof(MBR));
  int *nodes_index_c = (int *)calloc((size_t)n_slots, sizeof(int));
  int p = 0;
  int a = b;
  double t0 = now_ms();
#include "td_build.slice.inc"
  ms[0] = now_ms() - t0;
  for (long long s = 0; s < n_slots; s++) {
    nodes_index[s] = nodes_index_c[s];
    nodes_mbr[4 * s + 0] = nodes_mbr_c[s].x1;
    nodes_mbr[4 * s + 1] = nodes_mbr_c[s].y1;
    nodes_mbr[4 * s + 2] = nodes_mbr_c[s].x2;
    nodes_mbr[4 * s + 3] = nodes_mbr_c[s].y2;
  }
  for (size_t k = 0; k < offset.size(); k++) level_offsets_out[k] = offset[k];
  *n_offsets_out = (int)offset.size();
  for (int i = 0; i < n; i++) {
    sorted_rects_out[4 * i + 0] = nums[i].x1;
    sorted_rects_out[4 * i + 1] = nums[i].y1;
    sorted_rects_out[4 * i + 2] = nums[i].x2;
    sorted_rects_out[4 * i + 3] = nums[i].y2;
  }
  long long sum = 0, sum1 = 0, sum2 = 0;
  double t1 = now_ms();
  if (do_query) {
    for (int i = 0; i < size; i++) {
      int numq = 0, num2 = 0;
      int num1 = RtreeSearch(nodes_index_c, nodes_mbr_c, 0, nums[i], i, &numq, num2);
      sum += numq;
      sum1 += num1;
      sum2 += num2;
    }
    sum2 /= 2;
  }
  ms[1] = now_ms() - t1;
  digests[0] = sum;
  digests[1] = sum1;
  digests[2] = sum2;
  digests[3] = RtreeSearch1(nodes_index_c, nodes_mbr_c, 0);
  free(nums);
  free(nodes_mbr_c);
  free(nodes_index_c);
  return n_slots;
}

/* The reference's TD Overlap predicate (TD:26-39). */
int ref_td_overlap(const long long *a, const long long *b) {
  MBR ra, rb;
  ra.x1 = a[0]; ra.y1 = a[1]; ra.x2 = a[2]; ra.y2 = a[3];
  rb.x1 = b[0]; rb.y1 = b[1]; rb.x2 = b[2]; rb.y2 = b[3];
  return Overlap(ra, rb);
}

}  /* extern "C" */
