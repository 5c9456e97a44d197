// Streaming overlay: the candidate pairs are clipped in chunks of a bounded
// number of pairs, and each chunk's results are compacted into pair order on
// the device, copied into pinned host memory and handed to a caller callback
// before the chunk's device memory is released.  Device memory then holds one
// chunk's results (plus the one being copied out), not the whole result set,
// so layers whose results exceed HBM can be overlaid; the reference has no
// such path (its only bound is the 1 GiB device malloc heap,
// vector_map_overlay_gpc_kernel.cu:72).
//
// Chunk c's copy-out runs on a second stream while chunk c+1 is clipped on
// the caller's stream; the callback for chunk c runs on the calling thread
// once its copy has landed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "prt_internal.cuh"
#include "prt_overlay.cuh"

namespace prt {
namespace {

// Contour headers in pair order: output contour pair_off[i] + k is pool
// contour pair_cstart[i] + k.
__global__ void compact_headers_kernel(const int64_t *__restrict__ pair_cstart, const int32_t *__restrict__ pair_ncont,
                                       const int64_t *__restrict__ pair_off, int64_t n,
                                       const int32_t *__restrict__ cont_nverts, const int32_t *__restrict__ cont_hole,
                                       const int64_t *__restrict__ cont_vstart, int32_t *__restrict__ out_nverts,
                                       int32_t *__restrict__ out_hole, int64_t *__restrict__ out_src) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int k = pair_ncont[i];
    const int64_t o = pair_off[i], c0 = pair_cstart[i];
    for (int j = 0; j < k; j++) {
      out_nverts[o + j] = cont_nverts[c0 + j];
      out_hole[o + j] = cont_hole[c0 + j];
      out_src[o + j] = cont_vstart[c0 + j];
    }
  }
}

// Vertices in pair order: one warp per output contour, 16-byte (x, y) moves.
__global__ void compact_vertices_kernel(const int64_t *__restrict__ src, const int32_t *__restrict__ nverts,
                                        const int64_t *__restrict__ vert_off, int64_t n_cont,
                                        const double2 *__restrict__ xy, double2 *__restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; c < n_cont; c += nw) {
    const int64_t s0 = src[c], d0 = vert_off[c];
    const int m = nverts[c];
    for (int j = lane; j < m; j += 32) out[d0 + j] = xy[s0 + j];
  }
}

}  // namespace

// Compacts a result set into pair order in device buffers allocated on s:
// pair_off [n+1], nverts / hole [n_cont], xy [2 n_vert] (all in one block
// returned in *block, to be released with dfree).
int results_compact(const prt_results *r, cudaStream_t s, void **block, int64_t **pair_off, int32_t **nverts,
                    int32_t **hole, double **xy) {
  const int64_t n = r->n_pairs, nc = r->n_cont, nv = r->n_vert;
  // layout: pair_off (n+1) | src (nc) | vert_off (nc+1) | xy (2 nv) | nverts (nc) | hole (nc),
  // each part starting on a 256-byte boundary (xy is moved as 16-byte pairs)
  auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t b_off = up(8 * (size_t)(n + 1)), b_src = up(8 * (size_t)nc), b_voff = up(8 * (size_t)(nc + 1));
  const size_t b_xy = up(16 * (size_t)nv), b_nv = up(4 * (size_t)nc);
  unsigned char *p = nullptr;
  int rc = dmalloc(reinterpret_cast<void **>(&p), b_off + b_src + b_voff + b_xy + 2 * b_nv, s);
  if (rc) return rc;
  int64_t *off = reinterpret_cast<int64_t *>(p);
  int64_t *src = reinterpret_cast<int64_t *>(p + b_off);
  int64_t *voff = reinterpret_cast<int64_t *>(p + b_off + b_src);
  double *oxy = reinterpret_cast<double *>(p + b_off + b_src + b_voff);
  int32_t *onv = reinterpret_cast<int32_t *>(p + b_off + b_src + b_voff + b_xy);
  int32_t *oh = reinterpret_cast<int32_t *>(p + b_off + b_src + b_voff + b_xy + b_nv);
  if (n > 0) {
    rc = exclusive_scan<int32_t>(r->pair_ncont, n, off, off + n, s);
  } else {
    cudaError_t e = cudaMemsetAsync(off, 0, 8, s);
    if (e != cudaSuccess) rc = cuda_status(e, "memset");
  }
  if (!rc && nc > 0) {
    {
      PRT_PROF("compact_headers", s);
      compact_headers_kernel<<<grid_for(n, 256, 8), 256, 0, s>>>(r->pair_cstart, r->pair_ncont, off, n, r->cont_nverts,
                                                                 r->cont_hole, r->cont_vstart, onv, oh, src);
    }
    rc = exclusive_scan<int32_t>(onv, nc, voff, voff + nc, s);
    if (!rc) {
      PRT_PROF("compact_vertices", s);
      compact_vertices_kernel<<<grid_for(nc * 32, 256, 8), 256, 0, s>>>(
        src, onv, voff, nc, reinterpret_cast<const double2 *>(r->xy), reinterpret_cast<double2 *>(oxy));
    }
  }
  if (!rc) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) rc = cuda_status(e, "results compact");
  }
  if (rc) {
    dfree(p, s);
    return rc;
  }
  *block = p;
  *pair_off = off;
  *nverts = onv;
  *hole = oh;
  *xy = oxy;
  return PRT_OK;
}

}  // namespace prt

using namespace prt;

namespace {

// One chunk in flight: its results, their compacted device copy and the host
// staging they are copied into.
struct Staging {
  void *host = nullptr;
  size_t cap = 0;
};

struct Chunk {
  int64_t first = 0, n = 0, nc = 0, nv = 0;
  prt_results *res = nullptr;
  void *block = nullptr;
  cudaEvent_t done = nullptr;
  int64_t *h_off = nullptr;
  int32_t *h_nv = nullptr, *h_hole = nullptr;
  double *h_xy = nullptr;
};

int ensure_host(Staging &st, size_t bytes) {
  if (bytes <= st.cap) return PRT_OK;
  const size_t want = std::max(bytes, st.cap + st.cap / 2);
  if (st.host) cudaFreeHost(st.host);
  st.host = nullptr;
  st.cap = 0;
  PRT_CUDA(cudaMallocHost(&st.host, want));
  st.cap = want;
  return PRT_OK;
}

void release(Chunk &c, cudaStream_t s2) {
  if (c.block) dfree(c.block, s2);
  c.block = nullptr;
  if (c.res) prt_results_free(c.res);
  c.res = nullptr;
}

}  // namespace

extern "C" int prt_overlay_stream(const prt_pair *d_pairs, int64_t n_pairs, int32_t offset,
                                  const int32_t *d_leaf_to_poly, const prt_layer *base, const prt_layer *overlay,
                                  int op, int sched, int64_t chunk_pairs, prt_chunk_fn fn, void *user,
                                  void *stream) {
  PRT_CHECK(base && overlay && fn, PRT_ERR_INVALID, "NULL argument");
  PRT_CHECK(d_pairs || n_pairs == 0, PRT_ERR_INVALID, "d_pairs is NULL");
  PRT_CHECK(n_pairs >= 0 && n_pairs < (1ll << 31), PRT_ERR_INVALID, "n_pairs=%lld", (long long)n_pairs);
  PRT_CHECK(chunk_pairs >= 1, PRT_ERR_INVALID, "chunk_pairs %lld", (long long)chunk_pairs);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  cudaStream_t s2 = nullptr;
  PRT_CUDA(cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking));
  Staging stage[2];
  Chunk ch[2];
  int rc = PRT_OK;
  for (int k = 0; k < 2 && !rc; k++) {
    cudaError_t e = cudaEventCreateWithFlags(&ch[k].done, cudaEventDisableTiming);
    if (e != cudaSuccess) rc = cuda_status(e, "cudaEventCreate");
  }
  // hands chunk c (copy enqueued on s2) to the callback once it has landed
  auto deliver = [&](Chunk &c) -> int {
    cudaError_t e = cudaEventSynchronize(c.done);
    if (e != cudaSuccess) return cuda_status(e, "stream copy-out");
    release(c, s2);
    int u = fn(user, c.first, c.n, c.h_off, c.h_nv, c.h_hole, c.h_xy);
    if (u != 0) {
      set_error("overlay_stream: the chunk callback returned %d", u);
      return PRT_ERR_INVALID;
    }
    return PRT_OK;
  };
  int64_t first = 0;
  int cur = 0;
  bool pending = false;  // ch[1 - cur] holds a chunk whose copy is in flight
  while (!rc && first < n_pairs) {
    Chunk &c = ch[cur];
    c.first = first;
    c.n = std::min<int64_t>(chunk_pairs, n_pairs - first);
    PairSrc S;
    memset(&S, 0, sizeof S);
    S.pairs = reinterpret_cast<const uint2 *>(d_pairs + first);
    S.offset = offset;
    S.leaf_to_poly = d_leaf_to_poly;
    S.base = layer_dev(base);
    S.over = layer_dev(overlay);
    S.op = op;
    rc = overlay_impl(S, c.n, sched, nullptr, s, &c.res);
    int64_t *off = nullptr;
    int32_t *nv = nullptr, *hole = nullptr;
    double *xy = nullptr;
    if (!rc) rc = results_compact(c.res, s, &c.block, &off, &nv, &hole, &xy);
    if (!rc) {
      c.nc = c.res->n_cont;
      c.nv = c.res->n_vert;
      // the previous chunk's staging may still be read by its callback only
      // after deliver(); this chunk uses the other staging buffer
      const size_t bytes = 8 * (size_t)(c.n + 1) + 8 * (size_t)c.nc + 16 * (size_t)c.nv + 64;
      rc = ensure_host(stage[cur], bytes);
    }
    if (!rc) {
      unsigned char *h = reinterpret_cast<unsigned char *>(stage[cur].host);
      c.h_off = reinterpret_cast<int64_t *>(h);
      c.h_xy = reinterpret_cast<double *>(h + 8 * (c.n + 1));
      c.h_nv = reinterpret_cast<int32_t *>(h + 8 * (c.n + 1) + 16 * c.nv);
      c.h_hole = c.h_nv + c.nc;
      cudaEvent_t ready = nullptr;
      cudaError_t e = cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventRecord(ready, s);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(s2, ready, 0);
      if (ready) cudaEventDestroy(ready);
      if (e == cudaSuccess) e = cudaMemcpyAsync(c.h_off, off, 8 * (c.n + 1), cudaMemcpyDeviceToHost, s2);
      if (e == cudaSuccess && c.nv) e = cudaMemcpyAsync(c.h_xy, xy, 16 * c.nv, cudaMemcpyDeviceToHost, s2);
      if (e == cudaSuccess && c.nc) e = cudaMemcpyAsync(c.h_nv, nv, 4 * c.nc, cudaMemcpyDeviceToHost, s2);
      if (e == cudaSuccess && c.nc) e = cudaMemcpyAsync(c.h_hole, hole, 4 * c.nc, cudaMemcpyDeviceToHost, s2);
      if (e == cudaSuccess) e = cudaEventRecord(c.done, s2);
      if (e != cudaSuccess) rc = cuda_status(e, "stream copy-out");
    }
    // the previous chunk's copy overlapped this chunk's clip: deliver it
    if (!rc && pending) rc = deliver(ch[1 - cur]);
    pending = !rc;
    first += c.n;
    cur = 1 - cur;
  }
  if (!rc && pending) rc = deliver(ch[1 - cur]);
  cudaStreamSynchronize(s2);
  for (int k = 0; k < 2; k++) {
    release(ch[k], s2);
    if (ch[k].done) cudaEventDestroy(ch[k].done);
  }
  cudaStreamSynchronize(s2);
  cudaStreamDestroy(s2);
  for (int k = 0; k < 2; k++)
    if (stage[k].host) cudaFreeHost(stage[k].host);
  cudaGetLastError();
  return rc;
}
