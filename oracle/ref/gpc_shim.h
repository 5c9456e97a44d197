/* Project-written stand-in for the two headers the reference's clip core
 * includes but does not ship ("gpc.h", "common.h";
 * vector_map_overlay_gpc_kernel.cu:7-8).
 *
 * Test infrastructure only.  Every name below is one the reference's clip core
 * uses; each definition is written from that usage and from the published
 * description of the General Polygon Clipper (A. Murta, University of
 * Manchester, 2.3x series; no version is pinned by the reference):
 *   - vertex classes: class = tr + 2 tl + 4 br + 8 bl (GPC:322, GPC:527), each
 *     named for which quadrants around the vertex lie inside the result;
 *   - horizontal states NH/BH/TH index the 3 x 6 table of GPC:62;
 *   - CLIP/SUBJ, LEFT/RIGHT, ABOVE/BELOW index two-element arrays;
 *   - the vertex-filter and bound-extremum macros test the y order of a
 *     vertex's neighbours;
 *   - EQ compares within DBL_EPSILON.
 */
#ifndef PRT_GPC_SHIM_H
#define PRT_GPC_SHIM_H
#include "cuda_host_shim.h"

/* allocation macros of the missing common.h: zero-byte requests give NULL */
#define MALLOC(p, b, s, t) \
  do { if ((b) > 0) { (p) = (t *)malloc(b); if (!(p)) abort(); } else (p) = NULL; } while (0)
#define FREE(p) do { if (p) { free(p); (p) = NULL; } } while (0)

#define LEFT 0
#define RIGHT 1
#define ABOVE 0
#define BELOW 1
#define CLIP 0
#define SUBJ 1
#define TRUE 1
#define FALSE 0

#define GPC_EPSILON (DBL_EPSILON)
#define EQ(a, b) (fabs((a) - (b)) <= GPC_EPSILON)

#define PREV_INDEX(i, n) (((i) + (n) - 1) % (n))
#define NEXT_INDEX(i, n) (((i) + 1) % (n))
/* a vertex is kept unless both neighbours share its y */
#define OPTIMAL(v, i, n) \
  (((v)[PREV_INDEX(i, n)].y != (v)[i].y) || ((v)[NEXT_INDEX(i, n)].y != (v)[i].y))
/* forward (index-increasing) bound starts at a local minimum ... */
#define FWD_MIN(v, i, n) \
  (((v)[PREV_INDEX(i, n)].vertex.y >= (v)[i].vertex.y) && ((v)[NEXT_INDEX(i, n)].vertex.y > (v)[i].vertex.y))
/* ... and continues while the next vertex is strictly higher */
#define NOT_FMAX(v, i, n) ((v)[NEXT_INDEX(i, n)].vertex.y > (v)[i].vertex.y)
#define REV_MIN(v, i, n) \
  (((v)[PREV_INDEX(i, n)].vertex.y > (v)[i].vertex.y) && ((v)[NEXT_INDEX(i, n)].vertex.y >= (v)[i].vertex.y))
#define NOT_RMAX(v, i, n) ((v)[PREV_INDEX(i, n)].vertex.y > (v)[i].vertex.y)

typedef enum { GPC_DIFF, GPC_INT, GPC_XOR, GPC_UNION } gpc_op;

typedef struct { double x, y; } gpc_vertex;
typedef struct { int num_vertices; gpc_vertex *vertex; } gpc_vertex_list;
typedef struct { int num_contours; int *hole; gpc_vertex_list *contour; } gpc_polygon;

/* quadrant classes: bit 0 tr, bit 1 tl, bit 2 br, bit 3 bl */
typedef enum {
  NUL = 0,  /* no quadrant inside */
  EMX = 1,  /* external maximum */
  ELI = 2,  /* external left intermediate */
  TED = 3,  /* top edge */
  ERI = 4,  /* external right intermediate */
  RED = 5,  /* right edge */
  IMM = 6,  /* internal maximum and minimum */
  IMN = 7,  /* internal minimum */
  EMN = 8,  /* external minimum */
  EMM = 9,  /* external maximum and minimum */
  LED = 10, /* left edge */
  ILI = 11, /* internal left intermediate */
  BED = 12, /* bottom edge */
  IRI = 13, /* internal right intermediate */
  IMX = 14, /* internal maximum */
  FUL = 15  /* all quadrants inside */
} vertex_type;

typedef enum { NH = 0, BH = 1, TH = 2 } h_state;
typedef enum { UNBUNDLED = 0, BUNDLE_HEAD = 1, BUNDLE_TAIL = 2 } bundle_state;

typedef struct prt_vtx_node { double x, y; struct prt_vtx_node *next; } vertex_node;

typedef struct prt_poly_node {
  int active;
  int hole;
  vertex_node *v[2];
  struct prt_poly_node *next;
  struct prt_poly_node *proxy;
} polygon_node;

typedef struct prt_edge_node {
  gpc_vertex vertex;
  gpc_vertex bot;
  gpc_vertex top;
  double xb, xt, dx;
  int type;
  int bundle[2][2];
  int bside[2];
  bundle_state bstate[2];
  polygon_node *outp[2];
  struct prt_edge_node *prev, *next, *pred, *succ, *next_bound;
} edge_node;

typedef struct prt_lmt_node { double y; edge_node *first_bound; struct prt_lmt_node *next; } lmt_node;
typedef struct prt_sb_tree { double y; int visited; struct prt_sb_tree *less, *more; } sb_tree;
typedef struct prt_it_node { edge_node *ie[2]; gpc_vertex point; struct prt_it_node *next; } it_node;
typedef struct prt_st_node { edge_node *edge; double xb, xt, dx; struct prt_st_node *prev; } st_node;
typedef struct { double xmin, ymin, xmax, ymax; } bbox;

/* the table uploaded by run() (GPC:62-63); defined by the harness */
extern h_state next_h_state[3][6];

void gpc_polygon_clip(gpc_op op, gpc_polygon *subj, gpc_polygon *clip, gpc_polygon *result);
void gpc_free_polygon(gpc_polygon *p);
void reset_it(it_node **it);
void reset_lmt(lmt_node **lmt);
void insert_bound(edge_node **b, edge_node *e);
edge_node **bound_list(lmt_node **lmt, double y);
void add_to_sbtree(int *entries, sb_tree **sbtree, double y);
void build_sbt(int *entries, double *sbt, sb_tree *sbtree);
void free_sbtree(sb_tree **sbtree);
int count_optimal_vertices(gpc_vertex_list c);
edge_node *build_lmt(lmt_node **lmt, sb_tree **sbtree, int *sbt_entries,
                     gpc_polygon *p, int type, gpc_op op);
void add_edge_to_aet(edge_node **aet, edge_node *edge, edge_node *prev);
void add_intersection(it_node **it, edge_node *edge0, edge_node *edge1, double x, double y);
void add_st_edge(st_node **st, it_node **it, edge_node *edge, double dy);
void build_intersection_table(it_node **it, edge_node *aet, double dy);
int count_contours(polygon_node *polygon);
void add_left(polygon_node *p, double x, double y);
void merge_left(polygon_node *p, polygon_node *q, polygon_node *list);
void add_right(polygon_node *p, double x, double y);
void merge_right(polygon_node *p, polygon_node *q, polygon_node *list);
void add_local_min(polygon_node **p, edge_node *edge, double x, double y);
bbox *create_contour_bboxes(gpc_polygon *p);
void minimax_test(gpc_polygon *subj, gpc_polygon *clip, gpc_op op);
#endif
