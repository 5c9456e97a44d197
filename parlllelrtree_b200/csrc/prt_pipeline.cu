// The whole filter-and-refine overlay as one CUDA graph: polygon MBRs of both
// layers -> bottom-up R-tree over the base layer -> breadth-first join of the
// overlay layer -> batched GPC clip of every candidate pair -> result totals.
// Every buffer is allocated when the pipeline is created, for the capacities
// it is given; the first run captures the launches into a graph and every run
// replays it, so a run is one cudaGraphLaunch.  Sizes that depend on the data
// (pairs found, frontier items, results) stay in device words; an overflow of
// a capacity is reported by prt_pipeline_sizes, never by a host round trip
// inside the run.  The layers are referenced, not copied: a caller may change
// the vertex coordinates between runs (e.g. an alignment loop) and replay.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "prt_gpc.cuh"
#include "prt_internal.cuh"
#include "prt_overlay.cuh"

namespace prt {
namespace {

// Bounding box (x1, y1, x2, y2) of every polygon over all its rings, one warp
// per polygon: the lanes read the vertex array in coalesced 16-byte (x, y)
// loads and reduce by shuffles.  A polygon without vertices gets the empty box
// (DBL_MAX, DBL_MAX, -DBL_MAX, -DBL_MAX).  With Out = int32_t the box is
// quantised as the reference's readData does, (int)(v * scale) truncated
// toward zero (vector_map_overlay_gpc_kernel.cu:805-808, 845-848); values
// outside the int32 range saturate.
template <typename Out>
__global__ void poly_mbr_kernel(LayerDev L, double scale, Out *__restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t p = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; p < L.n_poly; p += nw) {
    const int64_t v0 = L.ring_vert[L.poly_ring[p]], v1 = L.ring_vert[L.poly_ring[p + 1]];
    double x1 = 1.7976931348623157e308, y1 = x1, x2 = -x1, y2 = -x1;
    const bool aligned = (reinterpret_cast<uintptr_t>(L.xy) & 15) == 0;
    const double2 *xy = reinterpret_cast<const double2 *>(L.xy);
    for (int64_t v = v0 + lane; v < v1; v += 32) {
      const double2 q = aligned ? __ldg(&xy[v]) : make_double2(__ldg(&L.xy[2 * v]), __ldg(&L.xy[2 * v + 1]));
      x1 = fmin(x1, q.x);
      y1 = fmin(y1, q.y);
      x2 = fmax(x2, q.x);
      y2 = fmax(y2, q.y);
    }
    for (int o = 16; o; o >>= 1) {
      x1 = fmin(x1, __shfl_xor_sync(0xffffffffu, x1, o));
      y1 = fmin(y1, __shfl_xor_sync(0xffffffffu, y1, o));
      x2 = fmax(x2, __shfl_xor_sync(0xffffffffu, x2, o));
      y2 = fmax(y2, __shfl_xor_sync(0xffffffffu, y2, o));
    }
    if (lane < 4) {
      const double v = lane == 0 ? x1 : lane == 1 ? y1 : lane == 2 ? x2 : y2;
      if constexpr (sizeof(Out) == 8) out[4 * p + lane] = (Out)v;
      else out[4 * p + lane] = (Out)__double2int_rz(v * scale);
    }
  }
}

inline int poly_mbr_grid(int64_t n_poly) { return grid_for(n_poly * 32, 256, 8); }

// Largest vertex count of a polygon of the layer (sizes the biggest arenas).
__global__ void max_poly_vertices_kernel(LayerDev L, unsigned long long *out) {
  unsigned long long m = 0;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < L.n_poly;
       p += (int64_t)gridDim.x * blockDim.x) {
    unsigned long long v = (unsigned long long)(L.ring_vert[L.poly_ring[p + 1]] - L.ring_vert[L.poly_ring[p]]);
    m = v > m ? v : m;
  }
  for (int o = 16; o; o >>= 1) {
    unsigned long long t = __shfl_xor_sync(0xffffffffu, m, o);
    m = t > m ? t : m;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

}  // namespace
}  // namespace prt

struct prt_pipeline {
  prt::LayerDev base, over;
  prt_pipeline_config cfg;
  double *base_mbr = nullptr, *over_mbr = nullptr;
  prt_tree *tree = nullptr;
  unsigned *build_err = nullptr;
  uint2 *frontier[2] = {nullptr, nullptr};
  uint2 *pairs = nullptr;
  unsigned long long *counters = nullptr;  // PRT_MAX_LEVELS + 2
  prt::GraphOverlay G;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int device = 0;
};

namespace prt {
namespace {

void free_pipeline(prt_pipeline *p) {
  if (!p) return;
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  cudaDeviceSynchronize();
  if (p->tree) prt_tree_free(p->tree);
  void *ptrs[] = {p->base_mbr, p->over_mbr, p->build_err, p->frontier[0], p->frontier[1], p->pairs, p->counters,
                  p->G.k0, p->G.k1, p->G.v0, p->G.v1, p->G.order, p->G.sel, p->G.err, p->G.ranges,
                  p->G.thresholds, p->G.tickets, p->G.totals, p->G.arena, p->G.status, p->G.pair_cstart,
                  p->G.pair_ncont, p->G.cont_vstart, p->G.cont_nverts, p->G.cont_hole, p->G.xy, p->G.pool};
  for (void *q : ptrs)
    if (q) cudaFree(q);
  cudaGetLastError();
  delete p;
}

template <typename T>
int alloc(T **p, size_t count) {
  cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), std::max<size_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    return cuda_status(e, "cudaMalloc (pipeline)");
  }
  return PRT_OK;
}

int enqueue_run(prt_pipeline *p, cudaStream_t s) {
  PRT_CUDA(cudaMemsetAsync(p->build_err, 0, 4, s));
  PRT_CUDA(cudaMemsetAsync(p->counters, 0, sizeof(unsigned long long) * (PRT_MAX_LEVELS + 2), s));
  {
    PRT_PROF("poly_mbr", s);
    poly_mbr_kernel<double><<<poly_mbr_grid(p->base.n_poly), 256, 0, s>>>(p->base, 1.0, p->base_mbr);
    poly_mbr_kernel<double><<<poly_mbr_grid(p->over.n_poly), 256, 0, s>>>(p->over, 1.0, p->over_mbr);
  }
  int rc = bu_enqueue(p->tree, p->base_mbr, nullptr, p->build_err, s);
  if (!rc)
    rc = join_enqueue(p->tree, p->over_mbr, p->over.n_poly, p->pairs, p->cfg.max_pairs, p->frontier[0],
                      p->frontier[1], p->cfg.max_frontier, p->counters, s);
  if (rc) return rc;
  PairSrc S;
  memset(&S, 0, sizeof S);
  S.pairs = p->pairs;
  S.offset = 0;
  S.leaf_to_poly = p->tree->d_leaf_id;
  S.base = p->base;
  S.over = p->over;
  S.op = p->cfg.op;
  return overlay_graph_enqueue(S, &p->counters[PRT_MAX_LEVELS], p->G, s);
}

}  // namespace
}  // namespace prt

using namespace prt;

extern "C" {

int prt_pipeline_create(const prt_layer *base, const prt_layer *overlay, const prt_pipeline_config *cfg_in,
                        prt_pipeline **out) {
  PRT_CHECK(base && overlay && out, PRT_ERR_INVALID, "NULL argument");
  PRT_CHECK(base->n_poly >= 1 && overlay->n_poly >= 1, PRT_ERR_INVALID, "empty layer");
  *out = nullptr;
  prt_pipeline_config cfg;
  memset(&cfg, 0, sizeof cfg);
  if (cfg_in) cfg = *cfg_in;
  if (cfg.fanout == 0) cfg.fanout = 16;
  cfg.op = cfg_in ? cfg_in->op : PRT_GPC_INT;
  if (cfg.max_pairs <= 0) cfg.max_pairs = 8 * std::max(base->n_poly, overlay->n_poly);
  if (cfg.max_frontier <= 0) cfg.max_frontier = 64 * overlay->n_poly + (1 << 20);
  PRT_CHECK(cfg.fanout >= 2 && cfg.fanout <= 32, PRT_ERR_INVALID, "fanout %d", cfg.fanout);
  PRT_CHECK(cfg.op >= 0 && cfg.op <= 3, PRT_ERR_INVALID, "op %d", cfg.op);
  const prt_schedule sched = cfg.sched ? *cfg.sched : current_schedule();
  {
    const int rs = schedule_valid(sched);
    if (rs) return rs;
  }
  cfg.sched = nullptr;  // the pipeline keeps its own copy in the plan
  {
    // memory cached by the stream-ordered pool goes back to the device first
    cudaMemPool_t pool;
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceSynchronize() == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess)
      cudaMemPoolTrimTo(pool, 0);
    cudaGetLastError();
  }
  prt_pipeline *p = new prt_pipeline();
  p->cfg = cfg;
  p->base = layer_dev(base);
  p->over = layer_dev(overlay);
  cudaGetDevice(&p->device);
  const int64_t nb = base->n_poly, no = overlay->n_poly, cap = cfg.max_pairs;
  int rc = alloc(&p->base_mbr, 4 * nb);
  if (!rc) rc = alloc(&p->over_mbr, 4 * no);
  if (!rc) rc = alloc(&p->build_err, 2);
  if (!rc) rc = alloc(&p->frontier[0], cfg.max_frontier);
  if (!rc) rc = alloc(&p->frontier[1], cfg.max_frontier);
  if (!rc) rc = alloc(&p->pairs, cap);
  if (!rc) rc = alloc(&p->counters, PRT_MAX_LEVELS + 2);
  if (!rc) rc = tree_alloc(p->base_mbr, PRT_COORD_F64, nb, cfg.fanout, PRT_BOTTOM_UP, PRT_KEY_MORTON32, 0, &p->tree);
  // overlay buffers
  GraphOverlay &G = p->G;
  G.cap_pairs = cap;
  if (!rc) rc = alloc(&G.k0, cap);
  if (!rc) rc = alloc(&G.k1, cap);
  if (!rc) rc = alloc(&G.v0, cap);
  if (!rc) rc = alloc(&G.v1, cap);
  if (!rc) rc = alloc(&G.order, cap);
  if (!rc) rc = alloc(&G.sel, 2);
  if (!rc) rc = alloc(&G.err, 2);
  if (!rc) rc = alloc(&G.ranges, 2 * PRT_MAX_BINS);
  if (!rc) rc = alloc(&G.thresholds, PRT_MAX_BINS);
  if (!rc) rc = alloc(&G.tickets, PRT_MAX_BINS + 1);
  if (!rc) rc = alloc(&G.totals, 4);
  if (!rc) rc = alloc(&G.status, cap);
  if (!rc) rc = alloc(&G.pair_cstart, cap);
  if (!rc) rc = alloc(&G.pair_ncont, cap);
  // the largest pair bounds the first bin's arena slices
  unsigned long long maxv[2] = {0, 0};
  if (!rc) {
    unsigned long long *d = nullptr;
    rc = alloc(&d, 2);
    if (!rc) {
      cudaMemset(d, 0, 16);
      max_poly_vertices_kernel<<<grid_for(nb, 256, 4), 256>>>(p->base, d);
      max_poly_vertices_kernel<<<grid_for(no, 256, 4), 256>>>(p->over, d + 1);
      cudaMemcpy(maxv, d, 16, cudaMemcpyDeviceToHost);
      cudaFree(d);
    }
  }
  // input vertices bound the result pools' first sizes
  int64_t vert_total = 0;
  if (!rc) {
    int64_t rv_b = 0, rv_o = 0, r_b = 0, r_o = 0;
    cudaMemcpy(&r_b, base->poly_ring + nb, 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(&r_o, overlay->poly_ring + no, 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(&rv_b, base->ring_vert + r_b, 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(&rv_o, overlay->ring_vert + r_o, 8, cudaMemcpyDeviceToHost);
    vert_total = rv_b + rv_o;
  }
  G.cap_v = cfg.max_out_vertices > 0 ? cfg.max_out_vertices : std::max<int64_t>(vert_total, 1 << 20);
  G.cap_c = cfg.max_out_contours > 0 ? cfg.max_out_contours : std::max<int64_t>(cap, 1 << 16);
  if (!rc) rc = alloc(&G.cont_vstart, G.cap_c);
  if (!rc) rc = alloc(&G.cont_nverts, G.cap_c);
  if (!rc) rc = alloc(&G.cont_hole, G.cap_c);
  if (!rc) rc = alloc(&G.xy, 2 * G.cap_v);
  if (!rc) rc = alloc(&G.pool, 2);
  // persistent workers per bin, sized for the largest pair each bin can hold
  if (!rc) {
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    const size_t budget = cfg.arena_budget_bytes > 0 ? (size_t)cfg.arena_budget_bytes
                                                     : std::min<size_t>(fr / 3, (size_t)48 << 30);
    const int64_t max_pair = (int64_t)(maxv[0] + maxv[1]);
    int64_t counts[PRT_MAX_BINS], mx[PRT_MAX_BINS];
    for (int b = 0; b < sched.nbins; b++) {
      counts[b] = cap;
      mx[b] = std::min<int64_t>(sched.bin_thresholds[b], max_pair);
    }
    G.arena_bytes = plan_bins(sched, counts, mx, budget, G.plan, &G.smem);
    G.plan.n_pairs = G.cap_pairs;
    rc = prepare_lpt_launch(G.smem);
    if (!rc) rc = alloc(&G.arena, G.arena_bytes);
  }
  if (!rc) {
    cudaError_t e = cudaMemcpy(G.thresholds, sched.bin_thresholds, sizeof(int64_t) * sched.nbins,
                               cudaMemcpyHostToDevice);
    if (e != cudaSuccess) rc = cuda_status(e, "pipeline thresholds");
  }
  if (rc) {
    free_pipeline(p);
    return rc;
  }
  *out = p;
  return PRT_OK;
}

int prt_layer_mbr(const prt_layer *layer, double *d_out, void *stream) {
  PRT_CHECK(layer && d_out, PRT_ERR_INVALID, "NULL argument");
  PRT_CHECK(layer->n_poly >= 0, PRT_ERR_INVALID, "n_poly %lld", (long long)layer->n_poly);
  if (layer->n_poly == 0) return PRT_OK;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  {
    PRT_PROF("poly_mbr", s);
    poly_mbr_kernel<double><<<poly_mbr_grid(layer->n_poly), 256, 0, s>>>(layer_dev(layer), 1.0, d_out);
  }
  PRT_CUDA(cudaGetLastError());
  return PRT_OK;
}

int prt_layer_mbr_i32(const prt_layer *layer, double scale, int32_t *d_out, void *stream) {
  PRT_CHECK(layer && d_out, PRT_ERR_INVALID, "NULL argument");
  PRT_CHECK(layer->n_poly >= 0, PRT_ERR_INVALID, "n_poly %lld", (long long)layer->n_poly);
  PRT_CHECK(scale > 0.0, PRT_ERR_INVALID, "scale %g", scale);
  if (layer->n_poly == 0) return PRT_OK;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  {
    PRT_PROF("poly_mbr", s);
    poly_mbr_kernel<int32_t><<<poly_mbr_grid(layer->n_poly), 256, 0, s>>>(layer_dev(layer), scale, d_out);
  }
  PRT_CUDA(cudaGetLastError());
  return PRT_OK;
}

int prt_pipeline_run(prt_pipeline *p, void *stream) {
  PRT_CHECK(p != nullptr, PRT_ERR_INVALID, "pipeline is NULL");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  PRT_CHECK(s != nullptr, PRT_ERR_INVALID, "a graph is captured on a non-default stream: pass one");
  if (!p->exec) {
    // one uncaptured pass first: it sets up the allocator pool and the
    // kernels' attributes outside of any capture
    int rc = enqueue_run(p, s);
    if (rc) return rc;
    PRT_CUDA(cudaStreamSynchronize(s));
    const bool prof = g_prof_on;
    g_prof_on = false;  // no profiler events inside the graph
    PRT_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    rc = enqueue_run(p, s);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(s, &graph);
    g_prof_on = prof;
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    if (e != cudaSuccess) return cuda_status(e, "cudaStreamEndCapture");
    p->graph = graph;
    e = cudaGraphInstantiate(&p->exec, graph, 0);
    if (e != cudaSuccess) return cuda_status(e, "cudaGraphInstantiate");
  }
  PRT_CUDA(cudaGraphLaunch(p->exec, s));
  return PRT_OK;
}

int prt_pipeline_sizes(prt_pipeline *p, int64_t *sizes) {
  PRT_CHECK(p && sizes, PRT_ERR_INVALID, "NULL argument");
  PRT_CUDA(cudaDeviceSynchronize());
  unsigned long long cnt[PRT_MAX_LEVELS + 2], tot[4];
  unsigned errs[2] = {0, 0};
  PRT_CUDA(cudaMemcpy(cnt, p->counters, sizeof cnt, cudaMemcpyDeviceToHost));
  PRT_CUDA(cudaMemcpy(tot, p->G.totals, sizeof tot, cudaMemcpyDeviceToHost));
  PRT_CUDA(cudaMemcpy(&errs[0], p->build_err, 4, cudaMemcpyDeviceToHost));
  PRT_CUDA(cudaMemcpy(&errs[1], p->G.err, 4, cudaMemcpyDeviceToHost));
  unsigned long long fmax = 0;
  for (int l = 1; l < p->tree->lv.levels; l++) fmax = std::max(fmax, cnt[l]);
  sizes[0] = (int64_t)cnt[PRT_MAX_LEVELS];
  sizes[1] = (int64_t)tot[0];
  sizes[2] = (int64_t)tot[1];
  sizes[3] = (int64_t)tot[2];
  sizes[4] = (int64_t)tot[3];
  sizes[5] = (int64_t)fmax;
  sizes[6] = (int64_t)(cnt[PRT_MAX_LEVELS] > (unsigned long long)p->cfg.max_pairs ||
                       fmax > (unsigned long long)p->cfg.max_frontier);
  sizes[7] = (int64_t)((errs[0] | errs[1]) & kErrTimeout ? 1 : 0);
  return PRT_OK;
}

int prt_pipeline_pairs(prt_pipeline *p, prt_pair *pairs, int64_t cap, int32_t *leaf_to_poly) {
  PRT_CHECK(p != nullptr, PRT_ERR_INVALID, "pipeline is NULL");
  PRT_CUDA(cudaDeviceSynchronize());
  if (pairs && cap > 0) {
    unsigned long long found = 0;
    PRT_CUDA(cudaMemcpy(&found, &p->counters[PRT_MAX_LEVELS], 8, cudaMemcpyDeviceToHost));
    const int64_t n = std::min<int64_t>(std::min<int64_t>((int64_t)found, p->cfg.max_pairs), cap);
    if (n) PRT_CUDA(cudaMemcpy(pairs, p->pairs, 8 * n, cudaMemcpyDefault));
  }
  if (leaf_to_poly) PRT_CUDA(cudaMemcpy(leaf_to_poly, p->tree->d_leaf_id, 4 * p->tree->n, cudaMemcpyDefault));
  return PRT_OK;
}

int prt_pipeline_results(prt_pipeline *p, int64_t *h_pair_cont_off, int32_t *h_cont_nverts, int32_t *h_cont_hole,
                         double *h_xy) {
  PRT_CHECK(p && h_pair_cont_off && h_cont_nverts && h_cont_hole && h_xy, PRT_ERR_INVALID, "NULL argument");
  int64_t sz[8];
  int rc = prt_pipeline_sizes(p, sz);
  if (rc) return rc;
  const int64_t n = std::min<int64_t>(sz[0], p->cfg.max_pairs);
  unsigned long long used[2];
  PRT_CUDA(cudaMemcpy(used, p->G.pool, sizeof used, cudaMemcpyDeviceToHost));
  used[0] = std::min<unsigned long long>(used[0], (unsigned long long)p->G.cap_c);
  used[1] = std::min<unsigned long long>(used[1], (unsigned long long)p->G.cap_v);
  std::vector<int64_t> cs(std::max<int64_t>(n, 1)), cvs(used[0] + 1);
  std::vector<int32_t> nc(std::max<int64_t>(n, 1)), st(std::max<int64_t>(n, 1)), cnv(used[0] + 1), ch(used[0] + 1);
  std::vector<double> xy(2 * used[1] + 2);
  if (n) {
    PRT_CUDA(cudaMemcpy(cs.data(), p->G.pair_cstart, 8 * n, cudaMemcpyDeviceToHost));
    PRT_CUDA(cudaMemcpy(nc.data(), p->G.pair_ncont, 4 * n, cudaMemcpyDeviceToHost));
    PRT_CUDA(cudaMemcpy(st.data(), p->G.status, 4 * n, cudaMemcpyDeviceToHost));
  }
  if (used[0]) {
    PRT_CUDA(cudaMemcpy(cvs.data(), p->G.cont_vstart, 8 * used[0], cudaMemcpyDeviceToHost));
    PRT_CUDA(cudaMemcpy(cnv.data(), p->G.cont_nverts, 4 * used[0], cudaMemcpyDeviceToHost));
    PRT_CUDA(cudaMemcpy(ch.data(), p->G.cont_hole, 4 * used[0], cudaMemcpyDeviceToHost));
  }
  if (used[1]) PRT_CUDA(cudaMemcpy(xy.data(), p->G.xy, 16 * used[1], cudaMemcpyDeviceToHost));
  int64_t c = 0, v = 0;
  h_pair_cont_off[0] = 0;
  for (int64_t i = 0; i < n; i++) {
    if (st[i] == 0) {
      for (int k = 0; k < nc[i]; k++) {
        int64_t cc = cs[i] + k;
        h_cont_nverts[c] = cnv[cc];
        h_cont_hole[c] = ch[cc];
        memcpy(h_xy + 2 * v, xy.data() + 2 * cvs[cc], 16 * (size_t)cnv[cc]);
        v += cnv[cc];
        c++;
      }
    }
    h_pair_cont_off[i + 1] = c;
  }
  return PRT_OK;
}

int prt_pipeline_free(prt_pipeline *p) {
  free_pipeline(p);
  return PRT_OK;
}

}  // extern "C"
