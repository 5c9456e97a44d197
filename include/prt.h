/* prt.h — C ABI of the B200 filter-and-refine spatial join and polygon overlay.
 *
 * Drop-in for the R-tree / overlay path of ParlllelRtree.  Every entry point
 * takes plain pointers and sizes; device pointers are named d_*, host
 * pointers h_*; `stream` is a cudaStream_t passed as void* (NULL = default
 * stream).  Every call returns a status (PRT_OK = 0); prt_last_error() gives a
 * thread-local message for the last failure.  The library never exits the
 * process and never falls back to the CPU: without a usable CUDA device every
 * compute call returns PRT_ERR_CUDA.
 *
 * Reference interfaces replaced (file:line in the reference project):
 *   prt_build_bottomup   CalcuateZOrderValue + LocalSort/scan1/scan2/Reorder +
 *                        Construction_init/Construction1 and their host loop
 *                        (BotomUp-rtree.cu:73-266, 373-426, 756-874)
 *   prt_build_topdown    changeX/changeY + fun, prefix*, sort + fun/fun1/fun2
 *                        (TopDown-rtree.cu:162-353, 465-481, 504-524, 629-687)
 *   prt_tree_export_bu   the rtree_node array the BU program copies back
 *                        (BotomUp-rtree.cu:47-54, 890)
 *   prt_tree_export_td   nodes_index / nodes_mbr slot arrays
 *                        (TopDown-rtree.cu:15-20, 689-690)
 *   prt_tree_leaf_order  the leaf-order -> record remap zOrder[].index used by
 *                        Execute (vector_map_overlay_gpc_kernel.cu:89)
 *   prt_join             init + query1 BFS batches (BotomUp-rtree.cu:592-630,
 *                        914-987; TopDown-rtree.cu:355-377, 450-463, 694-758),
 *                        emitting the rtree_search {nodeid, queryid} pairs the
 *                        overlay consumes (vector_map_overlay_gpc_kernel.cu:89-90)
 *   prt_query_counts     RtreeSearch / RtreeSearchHelp counters
 *                        (BotomUp-rtree.cu:439-483, TopDown-rtree.cu:56-76)
 *   prt_overlay_run      run() + Execute + gpc_polygon_clip
 *                        (vector_map_overlay_gpc_kernel.cu:61-750)
 *   prt_results_*        the gpc_polygon result array of run()
 *                        (vector_map_overlay_gpc_kernel.cu:64-65, 698-741)
 *   prt_clip_pair_host   gpc_polygon_clip on one host pair (for tests; the
 *                        clip still runs on the device)
 */
#ifndef PRT_H
#define PRT_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define PRT_OK 0
#define PRT_ERR_INVALID 1  /* bad argument */
#define PRT_ERR_CAPACITY 2 /* an output buffer was too small; counts are still reported */
#define PRT_ERR_TIMEOUT 3  /* a bounded device-side wait gave up */
#define PRT_ERR_CUDA 4     /* CUDA runtime error (or no device) */
#define PRT_ERR_NOMEM 5    /* device allocation failed */

/* ---- box coordinate types: boxes are (x1, y1, x2, y2) per record ---- */
#define PRT_COORD_I64 0 /* int64, the reference's bounding_box.rect / MBR */
#define PRT_COORD_F32 1
#define PRT_COORD_F64 2
#define PRT_COORD_I32 3 /* the overlay's quantised MBRs */

/* ---- bottom-up key modes ---- */
#define PRT_KEY_REF64 0    /* the reference's 4-D corner interleave (int64 boxes only) */
#define PRT_KEY_MORTON32 1 /* 2-D Morton code of box centres on a 65536^2 grid */

#define PRT_BOTTOM_UP 0
#define PRT_TOP_DOWN 1

/* ---- GPC operations (the reference hard-codes intersection) ---- */
#define PRT_GPC_DIFF 0
#define PRT_GPC_INT 1
#define PRT_GPC_XOR 2
#define PRT_GPC_UNION 3

/* ---- overlay schedules ---- */
#define PRT_SCHED_PLAIN 0   /* one thread per pair, pairs in input order */
#define PRT_SCHED_BATCHED 1 /* size-binned pairs, persistent work-stealing launch */

#define PRT_MAX_LEVELS 40

typedef struct prt_tree prt_tree;
typedef struct prt_results prt_results;

/* Candidate pair: leaf entry position (the reference's nodeid - offset) and
 * query record id (vector_map_overlay_gpc_kernel.cu:89-90). */
typedef struct {
  int32_t nodeid;
  int32_t queryid;
} prt_pair;

const char *prt_last_error(void);
int prt_version(void);
/* Number of CUDA devices visible to the library (0 when none). */
int prt_device_count(void);

/* ---------------------------------------------------------------- build */

/* Bulk-loads an R-tree bottom-up: keys (key_mode) -> stable radix sort ->
 * leaves of `fanout` consecutive records -> each upper level groups `fanout`
 * consecutive nodes; root = the single node of the top level.
 * d_boxes: n records of 4 coordinates (coord_type); d_ids: optional record ids
 * stored in the leaves (NULL = 0..n-1).  fanout in [2, 32]. */
int prt_build_bottomup(const void *d_boxes, int coord_type, const int32_t *d_ids, int64_t n,
                       int fanout, int key_mode, void *stream, prt_tree **out);

/* Bulk-loads an R-tree top-down: with H node levels, level p = 0..H-1 stably
 * sorts every run of fanout^(H-p) consecutive records by x1 (p even) or y1
 * (p odd), then packs like the bottom-up build. */
int prt_build_topdown(const void *d_boxes, int coord_type, const int32_t *d_ids, int64_t n,
                      int fanout, void *stream, prt_tree **out);

int prt_tree_free(prt_tree *t);

/* info[0] n, [1] fanout, [2] levels L (level 0 = records), [3] kind,
 * [4] coord type, [5] key mode, [8 + l] entries at level l (l < L).
 * `info` holds at least 8 + PRT_MAX_LEVELS int64. */
int prt_tree_info(const prt_tree *t, int64_t *info);

/* Entry boxes of one level, converted to double (exact for float32, float64
 * and integers below 2^53), n_l x 4 into host memory. */
int prt_tree_level_mbr(const prt_tree *t, int level, double *h_out);

/* Record id (d_ids[i], or i) of every leaf entry in leaf order: the zOrder
 * remap; n int32 into device memory. */
int prt_tree_leaf_order(const prt_tree *t, int32_t *d_out, void *stream);

/* The reference's bottom-up node array (BotomUp-rtree.cu:47-54): leaves
 * first, root last; per node flag (0 leaf, 1 internal), num, mbr[fanout][4]
 * (as double), children[fanout] (node index, -1 in leaves), data[fanout]
 * (record id, -1 in internal nodes).  Host buffers sized by
 * prt_tree_export_bu_size(). */
int prt_tree_export_bu_size(const prt_tree *t, int64_t *n_nodes);
int prt_tree_export_bu(const prt_tree *t, int32_t *h_flag, int32_t *h_num, double *h_mbr,
                       int32_t *h_children, int32_t *h_data, int32_t *h_root);

/* The reference's top-down slot arrays (TopDown-rtree.cu:504-524, 575-624):
 * root slots first; nodes_index > 0 is the child's first slot, < 0 is
 * -(leaf position)-1, 0 is empty; nodes_mbr (x1, y1, x2, y2) as double, zero
 * for empty slots.  offsets: the level offset vector (n_levels + 1 values). */
int prt_tree_export_td_size(const prt_tree *t, int64_t *n_slots, int32_t *n_offsets);
int prt_tree_export_td(const prt_tree *t, int32_t *h_nodes_index, double *h_nodes_mbr,
                       int32_t *h_offsets);

/* ---------------------------------------------------------------- join */

/* All (leaf entry, query) pairs whose boxes intersect (closed intervals: boxes
 * that touch intersect, as the reference's Overlap).  Breadth-first over the
 * levels for all queries at once.  Writes up to `cap` pairs to d_pairs in no
 * particular order and the total count to *h_count; returns
 * PRT_ERR_CAPACITY (count still exact) when cap is too small. */
int prt_join(const prt_tree *t, const void *d_queries, int coord_type, int64_t nq,
             prt_pair *d_pairs, int64_t cap, int64_t *h_count, void *stream);

/* prt_join without any device allocation (no counterpart in the reference).
 * For callers that may not allocate device memory when they join: a host
 * process whose own pool owns the whole device memory budget (a serving
 * process or a framework allocator that treats any allocation outside its
 * pool as a failure), or an embedding that forbids the library from calling
 * cudaMalloc / cudaMallocAsync at all.  The frontier scratch lives in a fixed
 * array of the library (64 MiB + 512 B, reserved on every GPU that loads the
 * library until the process exits): a level frontier above 4,194,304
 * (query, node) items returns PRT_ERR_CAPACITY with a message, as does a pair
 * count above `cap` (the count is still reported).  The call waits for
 * `stream` once at its end, to read the level and pair counts.  The first
 * call on a device looks the array's device address up and keeps it for the
 * process; make that first call before any stream capture, and do not call
 * this entry point again on a device after cudaDeviceReset.  Calls share the
 * array and its contents stay from one call to the next (the counters are
 * cleared by every call): calls that can overlap on the GPU race and must be
 * serialised by the caller. */
int prt_join_noalloc(const prt_tree *t, const void *d_queries, int coord_type, int64_t nq,
                     prt_pair *d_pairs, int64_t cap, int64_t *h_count, void *stream);

/* Same as prt_join, with the pairs sorted by (queryid, nodeid). */
int prt_join_sorted(const prt_tree *t, const void *d_queries, int coord_type, int64_t nq,
                    prt_pair *d_pairs, int64_t cap, int64_t *h_count, void *stream);

/* Per-query counters of the reference's DFS search, d_counts nq x 3 int64:
 * entries examined (node fill, or fanout per node when td_slots != 0 as the
 * top-down program counts), sum over visited nodes of max(0, overlapping
 * entries - 1) (the RtreeSearch return value), overlapping leaf entries. */
int prt_query_counts(const prt_tree *t, const void *d_queries, int coord_type, int64_t nq,
                     int td_slots, int64_t *d_counts, void *stream);

/* Pairs of overlapping sibling entries summed over every node of the tree:
 * the reference's tree-quality digest sum3 (RtreeSearch1,
 * BotomUp-rtree.cu:574-590, TopDown-rtree.cu:78-93). */
int prt_tree_sibling_overlaps(const prt_tree *t, int64_t *h_count, void *stream);

/* ---------------------------------------------------------------- overlay */

/* A polygon layer in device memory (ring CSR):
 *   poly_ring[P+1]  ring offsets per polygon
 *   ring_vert[R+1]  vertex offsets per ring
 *   ring_hole[R]    hole flag per ring (informational; the clip uses even-odd parity)
 *   xy[V]           vertices (x, y) as double pairs */
typedef struct {
  const int64_t *poly_ring;
  const int64_t *ring_vert;
  const int32_t *ring_hole;
  const double *xy;
  int64_t n_poly;
} prt_layer;

/* Clips every pair: subject = base polygon leaf_to_poly[nodeid - offset]
 * (or nodeid - offset when leaf_to_poly is NULL), clip = overlay polygon
 * queryid, with GPC semantics for `op`.  The result set (one gpc_polygon per
 * pair, device resident) is returned in *out.  sched: PRT_SCHED_*. */
int prt_overlay_run(const prt_pair *d_pairs, int64_t n_pairs, int32_t offset,
                    const int32_t *d_leaf_to_poly, const prt_layer *base, const prt_layer *overlay,
                    int op, int sched, void *stream, prt_results **out);

/* The reference's single-contour CSR (readData, vector_map_overlay_gpc_kernel.cu:752-888):
 * num[] vertex count, prefix[] first vertex (int64), vertex[] (x, y) doubles,
 * hole[] flag, per polygon. */
int prt_overlay_run_ref(const prt_pair *d_pairs, int64_t n_pairs, int32_t offset,
                        const int32_t *d_leaf_to_poly,
                        const int32_t *d_num_base, const int64_t *d_prefix_base,
                        const double *d_vertex_base, const int32_t *d_hole_base, int64_t n_base,
                        const int32_t *d_num_overlay, const int64_t *d_prefix_overlay,
                        const double *d_vertex_overlay, const int32_t *d_hole_overlay,
                        int64_t n_overlay, int op, int sched, void *stream, prt_results **out);

/* sizes[0] pairs, [1] contours, [2] vertices, [3] non-empty results,
 * [4] pairs retried with larger arenas. */
int prt_results_sizes(const prt_results *r, int64_t *sizes);
/* Device views of the result arrays (valid until prt_results_free).  Like the
 * reference's gpc_polygon array, each pair points at its own contours:
 * pair i owns contours [pair_cont_start[i], + pair_ncont[i]); contour c owns
 * vertices [cont_vert_start[c], + cont_nverts[c]) of xy (x, y pairs). */
int prt_results_device(const prt_results *r, const int64_t **pair_cont_start,
                       const int32_t **pair_ncont, const int64_t **cont_vert_start,
                       const int32_t **cont_nverts, const int32_t **cont_hole, const double **xy);
/* Copies the results to host buffers in pair order (CSR): h_pair_cont_off
 * [pairs+1], h_cont_nverts / h_cont_hole [contours], h_xy [2*vertices]. */
int prt_results_copy(const prt_results *r, int64_t *h_pair_cont_off, int32_t *h_cont_nverts,
                     int32_t *h_cont_hole, double *h_xy);
/* Copies the results of the k pairs listed in h_pairs (pair indices) to host
 * buffers in list order: h_pair_cont_off [k+1], h_cont_nverts / h_cont_hole
 * [cont_cap], h_xy [2 * vert_cap].  h_need[0..1] receives the contours and
 * vertices needed; PRT_ERR_CAPACITY (nothing copied) when they exceed the
 * caps.  For checking or exporting a few pairs of a result set too large for
 * host memory (no reference counterpart). */
int prt_results_copy_pairs(const prt_results *r, const int64_t *h_pairs, int64_t k, int64_t *h_pair_cont_off,
                           int32_t *h_cont_nverts, int32_t *h_cont_hole, double *h_xy, int64_t cont_cap,
                           int64_t vert_cap, int64_t *h_need);
/* Per-pair intersection area of the results (hole contours negative). */
int prt_results_area(const prt_results *r, double *d_area, void *stream);
int prt_results_free(prt_results *r);

/* Streaming overlay (no reference counterpart; the reference's results live
 * in a 1 GiB device heap, vector_map_overlay_gpc_kernel.cu:72): the pairs of
 * prt_overlay_run are clipped in chunks of at most chunk_pairs, and each
 * chunk's results are copied to host memory in pair order and passed to fn
 * (on the calling thread, in chunk order) once their device memory is
 * released, so device memory holds at most two chunks' results however large
 * the whole result set is.  A chunk's copy-out (a second host thread and
 * stream, through two 256 MiB pinned buffers that the library keeps for the
 * rest of the process, into two pageable buffers reused from chunk to chunk)
 * overlaps the next chunk's clip.  fn receives the chunk's first
 * pair index and pair count and, valid only during the call, the CSR of
 * prt_results_copy (pair_cont_off [n+1] relative to the chunk, cont_nverts /
 * cont_hole per contour, xy as x, y pairs); a non-zero return stops the
 * stream (PRT_ERR_INVALID). */
typedef int (*prt_chunk_fn)(void *user, int64_t first_pair, int64_t n_pairs, const int64_t *pair_cont_off,
                            const int32_t *cont_nverts, const int32_t *cont_hole, const double *xy);
int prt_overlay_stream(const prt_pair *d_pairs, int64_t n_pairs, int32_t offset,
                       const int32_t *d_leaf_to_poly, const prt_layer *base, const prt_layer *overlay,
                       int op, int sched, int64_t chunk_pairs, prt_chunk_fn fn, void *user, void *stream);

/* One pair from host memory (rings as counts + packed xy), clipped on the
 * device; the result is written to host buffers.  Returns PRT_ERR_CAPACITY
 * (with *out_ncont / *out_nv set) when cont_cap / vert_cap are too small. */
int prt_clip_pair_host(int op, int s_ncont, const int32_t *s_nverts, const double *s_xy,
                       int c_ncont, const int32_t *c_nverts, const double *c_xy,
                       int32_t *out_ncont, int32_t cont_cap, int32_t *out_nverts,
                       int32_t *out_hole, int64_t *out_nv, int64_t vert_cap, double *out_xy);

/* ---------------------------------------------------------------- graph pipeline */

/* The whole overlay (the caller the reference leaves out around
 * vector_map_overlay_gpc_kernel.cu:61-113): polygon MBRs of both layers ->
 * bottom-up Morton R-tree over the base layer -> breadth-first join of the
 * overlay layer's MBRs -> batched clip of every candidate pair.  All buffers
 * are allocated by prt_pipeline_create for the capacities in the config; the
 * first prt_pipeline_run captures the launches into a CUDA graph and every run
 * replays it (one cudaGraphLaunch, no host synchronisation).  The layers are
 * referenced, not copied: their vertex coordinates may change between runs
 * (the counts may not).  No reference counterpart (a new entry point). */
/* ---------------------------------------------------------------- batched schedule */

/* How the batched schedule (PRT_SCHED_BATCHED and the graph pipeline) cuts
 * the size-sorted pairs into bins and clips them (no reference counterpart;
 * the reference runs one pair per thread in input order).  Bin b holds the
 * pairs whose vertex count n_subject + n_clip lies in
 * (bin_thresholds[b+1], bin_thresholds[b]]; bins are clipped largest first
 * in one persistent launch.  bin_warp_mode[b] = 1 clips each pair of the bin
 * with a whole warp (an active edge table of up to 32 edges in registers, a
 * larger one in shared memory, aet_slots slots per warp, a larger one still
 * in the pair's arena), 0 with one thread per pair.  The launch starts
 * warps_per_sm persistent warps per SM (at most 12, the resident limit);
 * every warp takes the next pair (warp mode) or the next 32 pairs (thread
 * mode) of the largest bin that still has pairs, so the largest pairs are
 * clipped first by all warps.  A launch whose thread-mode pairs would fill
 * less than half a wave of warps one pair per thread clips every pair in warp
 * mode instead (same output, more warps in flight). */
#define PRT_MAX_BINS 8
typedef struct {
  int32_t nbins;
  int32_t aet_slots;
  int64_t bin_thresholds[PRT_MAX_BINS];
  int32_t bin_warp_mode[PRT_MAX_BINS];
  int32_t warps_per_sm;
  int32_t reserved;
} prt_schedule;

/* Sets the schedule used by later calls of this process (NULL restores the
 * built-in default); returns PRT_ERR_INVALID for an inconsistent one. */
int prt_schedule_set(const prt_schedule *sched);
int prt_schedule_get(prt_schedule *sched);

typedef struct {
  int32_t fanout;             /* tree fanout (default 16) */
  int32_t op;                 /* PRT_GPC_* (default PRT_GPC_INT when cfg is NULL) */
  int64_t max_pairs;          /* candidate pairs kept (default 8 x max layer size) */
  int64_t max_frontier;       /* join frontier items per level (default 64 x overlay + 1 Mi) */
  int64_t max_out_contours;   /* result pool sizes (defaults from the pair and vertex counts) */
  int64_t max_out_vertices;
  int64_t arena_budget_bytes; /* clip scratch (default a third of free memory, at most 48 GB) */
  const prt_schedule *sched;  /* NULL: the schedule set by prt_schedule_set */
} prt_pipeline_config;

typedef struct prt_pipeline prt_pipeline;

int prt_pipeline_create(const prt_layer *base, const prt_layer *overlay, const prt_pipeline_config *cfg,
                        prt_pipeline **out);
/* Enqueues one run on `stream` (a non-default stream). */
int prt_pipeline_run(prt_pipeline *p, void *stream);
/* Synchronises, then: sizes[0] candidate pairs found, [1] contours,
 * [2] vertices, [3] non-empty results, [4] pairs that did not fit their
 * arena or the result pools (their results are empty; rerun with larger
 * capacities), [5] largest join frontier, [6] 1 when pairs or frontier
 * exceeded their capacity, [7] 1 when a bounded wait timed out. */
int prt_pipeline_sizes(prt_pipeline *p, int64_t *sizes);
/* Copies the first min(cap, pairs found) candidate pairs {nodeid, queryid}
 * and the leaf order (record id per leaf entry, one per base polygon) of the
 * last run into caller buffers, host or device (either may be NULL). */
int prt_pipeline_pairs(prt_pipeline *p, prt_pair *pairs, int64_t cap, int32_t *leaf_to_poly);
/* Results of the last run in pair order, as prt_results_copy. */
int prt_pipeline_results(prt_pipeline *p, int64_t *h_pair_cont_off, int32_t *h_cont_nverts,
                         int32_t *h_cont_hole, double *h_xy);
int prt_pipeline_free(prt_pipeline *p);

/* ---------------------------------------------------------------- autotuner */

/* Bounding box (x1, y1, x2, y2) of every polygon of a layer over all its
 * rings, n_poly x 4 doubles into device memory (the MBRs the reference's
 * readData quantises, vector_map_overlay_gpc_kernel.cu:752-888). */
int prt_layer_mbr(const prt_layer *layer, double *d_out, void *stream);

/* The same boxes quantised as readData does before the reference builds its
 * tree: (int)(v * scale) truncated toward zero, scale 1e5 in the reference
 * (vector_map_overlay_gpc_kernel.cu:805-808, 845-848); n_poly x 4 int32 into
 * device memory (values outside the int32 range saturate).  A tree built on
 * them with PRT_COORD_I32, joined with the other layer's quantised boxes,
 * gives the reference's candidate set. */
int prt_layer_mbr_i32(const prt_layer *layer, double scale, int32_t *d_out, void *stream);

/* Autotuner (no reference counterpart): times the build + join for fanouts
 * 8..32 and the batched clip for candidate schedules (warp-mode threshold,
 * shared-memory slots, warps per SM) on an evenly strided sample of at most
 * max_sample_pairs candidate pairs (<= 0: 200,000), within about
 * time_budget_s seconds (<= 0: 30).  Installs the best schedule with
 * prt_schedule_set and returns the choice. */
typedef struct {
  int32_t fanout;
  int32_t candidates;      /* configurations timed */
  int64_t sample_pairs;
  double build_join_ms;    /* best build + join time (ms) */
  double clip_ms;          /* best batched clip time on the sample (ms) */
  double seconds;          /* tuning wall time */
  prt_schedule sched;
} prt_tuning;

int prt_autotune(const prt_layer *base, const prt_layer *overlay, int op, int64_t max_sample_pairs,
                 double time_budget_s, void *stream, prt_tuning *out);

/* ---------------------------------------------------------------- area + adjoint */

/* Intersection area of each pair (subject = base polygon pair_a[i], clip =
 * overlay polygon pair_b[i]) and its gradient with respect to every vertex:
 *   prt_area_fwd: d_area[i] = area(A_i ∩ B_i), the area of GPC's intersection
 *                 within 1e-9 relative: the boundary integral over the pieces
 *                 of each polygon's edges inside the other when every crossing
 *                 of the pair is clean (the rings of a polygon must not cross
 *                 each other or themselves; hole rings flagged), else the GPC
 *                 clip + shoelace of the pair
 *   prt_area_bwd: d_grad_base / d_grad_overlay (V x 2 doubles, accumulated
 *                 with += over pairs; zero them first) += d_upstream[i] *
 *                 d area_i / d vertex, recomputing the boundary pieces. */
int prt_area_fwd(const int32_t *d_pair_a, const int32_t *d_pair_b, int64_t n_pairs,
                 const prt_layer *base, const prt_layer *overlay, double *d_area, void *stream);
int prt_area_bwd(const int32_t *d_pair_a, const int32_t *d_pair_b, int64_t n_pairs,
                 const prt_layer *base, const prt_layer *overlay, const double *d_upstream,
                 double *d_grad_base, double *d_grad_overlay, void *stream);
/* Pairs the last prt_area_fwd call of the process clipped with GPC. */
int prt_area_fwd_fallbacks(int64_t *h_count);

/* ---------------------------------------------------------------- profiling */

/* Kernel launch profiler (no reference counterpart).  Mode 1: every library
 * kernel launch is bracketed by CUDA events on its stream; mode 2: launches
 * are only counted, except those of the kernel named by prt_profile_focus,
 * which are timed; 0: off.  prt_profile_read returns the number of kernel
 * names (up to cap) and writes newline-separated names, summed device
 * milliseconds (0 for counted-only kernels) and launch counts. */
int prt_profile_enable(int mode);
int prt_profile_focus(const char *kernel_name);
int prt_profile_reset(void);
int prt_profile_read(char *names, int names_cap, double *ms_total, int64_t *launches, int cap);

/* ---------------------------------------------------------------- text files */

/* The reference's input files (host code; no device needed).
 * Rect file, data/Rect1024.txt of the R-tree programs (BotomUp-rtree.cu:669-698,
 * TopDown-rtree.cu:487-497): the record count, then per record "x1 x2",
 * "y1 y2" (integers) and an integer key.  Boxes are returned / taken as
 * n x 4 int64 (x1, y1, x2, y2); keys as int32 (NULL when writing: 0..n-1).
 * A count above cap returns PRT_ERR_CAPACITY with *n_read set. */
int prt_rect_file_count(const char *path, int64_t *n);
int prt_read_rect_file(const char *path, int64_t *h_boxes, int32_t *h_keys, int64_t cap, int64_t *n_read);
int prt_write_rect_file(const char *path, const int64_t *h_boxes, const int32_t *h_keys, int64_t n);

/* Polygon file, the base / overlay files of readData
 * (vector_map_overlay_gpc_kernel.cu:752-888): the polygon count, then per
 * polygon its vertex count, hole flag, bounding box (four doubles x1 y1 x2 y2)
 * and vertices ("x y" pairs).  prt_read_polygon_file fills readData's arrays:
 * num[], prefix[] (int64, prefix[i] = prefix[i-1] + num[i-1]), hole[], the box
 * as read (h_mbr, n x 4, optional), the box quantised as readData does
 * ((int)(v * 100000), h_rect, n x 4, optional) and the vertices (x, y pairs,
 * optional).  prt_polygon_file_size gives the counts to size them; caps that
 * are too small return PRT_ERR_CAPACITY.  prt_write_polygon_file writes the
 * exact vertex bounds as the box, every double in a form that reads back to
 * the same value (%.17g). */
int prt_polygon_file_size(const char *path, int64_t *n_poly, int64_t *n_vert);
int prt_read_polygon_file(const char *path, int32_t *h_num, int64_t *h_prefix, int32_t *h_hole, double *h_mbr,
                          int32_t *h_rect, double *h_vertex, int64_t poly_cap, int64_t vert_cap);
int prt_write_polygon_file(const char *path, const int32_t *h_num, const int32_t *h_hole, const double *h_vertex,
                           int64_t n_poly);

/* ---------------------------------------------------------------- bounded waits */

/* Test hook for the bounded device-side waits (no reference counterpart).
 * Every decoupled look-back of the radix sort polls its predecessors at most
 * `polls` times (<= 0: the built-in limit of 4,194,304) before it gives up,
 * records a timeout and returns; the call that launched it then returns
 * PRT_ERR_TIMEOUT.  With never_published != 0 every look-back sees no
 * predecessor published, so each wait runs to its limit: this exercises the
 * timeout path on a device without a hang or a fault.  Applies to the sorts
 * launched after the call, process-wide; prt_debug_wait_limit(0, 0) restores
 * the default. */
int prt_debug_wait_limit(int polls, int never_published);

#ifdef __cplusplus
}
#endif
#endif
