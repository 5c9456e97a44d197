// Streaming overlay: the candidate pairs are clipped in chunks of a bounded
// number of pairs, and each chunk's results are compacted into pair order on
// the device, copied into host memory and handed to a caller callback before
// the chunk's device memory is released.  Device memory then holds one
// chunk's results (plus the one being copied out), not the whole result set,
// so layers whose results exceed HBM can be overlaid; the reference has no
// such path (its only bound is the 1 GiB device malloc heap,
// vector_map_overlay_gpc_kernel.cu:72).
//
// Chunk c's copy-out runs on a second host thread and a second
// (non-blocking) stream while chunk c+1 is clipped on the caller's stream;
// the callback for chunk c runs on the calling thread once its copy has
// landed.  The host buffers are ordinary (pageable) memory, two of them
// reused from chunk to chunk: pinning a buffer of a chunk's size (gigabytes)
// costs about a second per GB.  The copy thread moves a chunk through two
// small pinned bounce buffers (allocated once per process): asynchronous
// device-to-pinned copies, each followed by a host copy into the pageable
// buffer while the next piece is in flight.  (A device-to-pageable copy
// from the second thread would hold up the calling thread's CUDA calls, and
// so the next clip, for as long as it runs.)
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>

#include <sys/mman.h>

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
// buffer they are copied into.
struct HostBuf {
  void *host = nullptr;
  size_t cap = 0;
};

struct Chunk {
  int64_t first = 0, n = 0, nc = 0, nv = 0;
  prt_results *res = nullptr;
  void *block = nullptr;
  // compacted device arrays of the chunk
  const int64_t *d_off = nullptr;
  const int32_t *d_nv = nullptr, *d_hole = nullptr;
  const double *d_xy = nullptr;
  cudaEvent_t ready = nullptr;  // the compaction has finished (caller's stream)
  int64_t *h_off = nullptr;
  int32_t *h_nv = nullptr, *h_hole = nullptr;
  double *h_xy = nullptr;
};

// Host buffers are anonymous mappings advised for transparent huge pages:
// a chunk's buffer is gigabytes, and the first touch of 4 KiB pages (over a
// million faults per buffer) stalled the calling thread's CUDA calls, and so
// the clip running meanwhile, for seconds.
void free_host(HostBuf &b) {
  if (b.host) munmap(b.host, b.cap);
  b.host = nullptr;
  b.cap = 0;
}

int ensure_host(HostBuf &b, size_t bytes) {
  if (bytes <= b.cap) return PRT_OK;
  const size_t huge = 2ull << 20;
  const size_t want = (std::max(bytes, b.cap + b.cap / 2) + huge - 1) & ~(huge - 1);
  free_host(b);
  void *p = mmap(nullptr, want, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
  PRT_CHECK(p != MAP_FAILED, PRT_ERR_NOMEM, "overlay_stream: %zu bytes of host memory", want);
  madvise(p, want, MADV_HUGEPAGE);  // advisory: without huge pages the buffer still works
  b.host = p;
  b.cap = want;
  return PRT_OK;
}

void release(Chunk &c, cudaStream_t s) {
  if (c.block) dfree(c.block, s);
  c.block = nullptr;
  if (c.res) prt_results_free(c.res);
  c.res = nullptr;
}

// Two pinned bounce buffers of kBounce bytes, shared by the calls of the
// process (one stream copy-out at a time uses them: g_bounce_use).
constexpr size_t kBounce = 256ull << 20;
std::mutex g_bounce_mu, g_bounce_use;
void *g_bounce[2] = {nullptr, nullptr};

cudaError_t bounce_buffers() {
  std::lock_guard<std::mutex> lk(g_bounce_mu);
  for (int k = 0; k < 2; k++)
    if (!g_bounce[k]) {
      cudaError_t e = cudaMallocHost(&g_bounce[k], kBounce);
      if (e != cudaSuccess) {
        g_bounce[k] = nullptr;
        return e;
      }
    }
  return cudaSuccess;
}

// The copy thread's work: wait for the chunk's compaction, then move its four
// arrays into the host buffer piece by piece through the bounce buffers:
// piece k goes device -> bounce[k % 2] on the copy stream while piece k - 1
// is copied bounce -> host buffer.
cudaError_t copy_out(int dev, cudaStream_t s2, cudaEvent_t *ev, const Chunk &c) {
  cudaError_t e = cudaSetDevice(dev);
  if (e == cudaSuccess) e = bounce_buffers();
  if (e == cudaSuccess) e = cudaStreamWaitEvent(s2, c.ready, 0);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> use(g_bounce_use);
  struct Part {
    const void *src;
    void *dst;
    size_t bytes;
  };
  const Part parts[4] = {{c.d_off, c.h_off, 8 * (size_t)(c.n + 1)},
                         {c.d_xy, c.h_xy, 16 * (size_t)c.nv},
                         {c.d_nv, c.h_nv, 4 * (size_t)c.nc},
                         {c.d_hole, c.h_hole, 4 * (size_t)c.nc}};
  unsigned char *pend_dst = nullptr;  // the piece in bounce[pb] waiting for its host copy
  size_t pend_bytes = 0;
  int pb = 0, k = 0;
  for (const Part &pt : parts) {
    for (size_t o = 0; o < pt.bytes && e == cudaSuccess; o += kBounce, k++) {
      const size_t len = std::min(kBounce, pt.bytes - o);
      const int b = k & 1;
      e = cudaMemcpyAsync(g_bounce[b], static_cast<const unsigned char *>(pt.src) + o, len, cudaMemcpyDeviceToHost,
                          s2);
      if (e == cudaSuccess) e = cudaEventRecord(ev[b], s2);
      if (e == cudaSuccess && pend_dst) {  // the previous piece, while this one is in flight
        e = cudaEventSynchronize(ev[pb]);
        if (e == cudaSuccess) memcpy(pend_dst, g_bounce[pb], pend_bytes);
      }
      pend_dst = static_cast<unsigned char *>(pt.dst) + o;
      pend_bytes = len;
      pb = b;
    }
  }
  if (e == cudaSuccess && pend_dst) {
    e = cudaEventSynchronize(ev[pb]);
    if (e == cudaSuccess) memcpy(pend_dst, g_bounce[pb], pend_bytes);
  }
  return e;
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
  int dev = 0;
  PRT_CUDA(cudaGetDevice(&dev));
  cudaStream_t s2 = nullptr;
  PRT_CUDA(cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking));
  HostBuf buf[2];
  Chunk ch[2];
  int rc = PRT_OK;
  cudaEvent_t bev[2] = {nullptr, nullptr};  // the bounce buffers' copies
  for (int k = 0; k < 2 && !rc; k++) {
    cudaError_t e = cudaEventCreateWithFlags(&ch[k].ready, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&bev[k], cudaEventDisableTiming);
    if (e != cudaSuccess) rc = cuda_status(e, "cudaEventCreate");
  }
  std::thread copier;  // copies the newest chunk (at most one at a time)
  cudaError_t copy_err = cudaSuccess;
  auto wait_copy = [&]() -> int {
    copier.join();
    return copy_err == cudaSuccess ? PRT_OK : cuda_status(copy_err, "stream copy-out");
  };
  // hands a landed chunk to the callback, after releasing its device memory
  auto deliver = [&](Chunk &c) -> int {
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
  bool pending = false;  // the copy thread runs for ch[1 - cur]
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
    // the previous chunk's copy overlapped this chunk's clip
    bool landed = false;
    if (pending) {
      pending = false;
      const int rw = wait_copy();
      if (!rc) rc = rw;
      landed = !rc;
    }
    if (!rc) {
      c.nc = c.res->n_cont;
      c.nv = c.res->n_vert;
      c.d_off = off;
      c.d_nv = nv;
      c.d_hole = hole;
      c.d_xy = xy;
      // buf[cur] held the chunk before the previous one, delivered already
      const size_t bytes = 8 * (size_t)(c.n + 1) + 8 * (size_t)c.nc + 16 * (size_t)c.nv + 64;
      rc = ensure_host(buf[cur], bytes);
    }
    if (!rc) {
      unsigned char *h = reinterpret_cast<unsigned char *>(buf[cur].host);
      c.h_off = reinterpret_cast<int64_t *>(h);
      c.h_xy = reinterpret_cast<double *>(h + 8 * (c.n + 1));
      c.h_nv = reinterpret_cast<int32_t *>(h + 8 * (c.n + 1) + 16 * c.nv);
      c.h_hole = c.h_nv + c.nc;
      cudaError_t e = cudaEventRecord(c.ready, s);
      if (e != cudaSuccess) rc = cuda_status(e, "cudaEventRecord");
    }
    if (!rc) {
      Chunk *cc = &c;
      copier = std::thread([&copy_err, dev, s2, cc, &bev]() { copy_err = copy_out(dev, s2, bev, *cc); });
      pending = true;
    }
    // the previous chunk's callback runs while this chunk is copied out
    if (!rc && landed) rc = deliver(ch[1 - cur]);
    first += c.n;
    cur = 1 - cur;
  }
  if (pending) {
    const int rw = wait_copy();
    if (!rc) rc = rw;
    if (!rc) rc = deliver(ch[1 - cur]);
  }
  cudaStreamSynchronize(s2);
  for (int k = 0; k < 2; k++) {
    release(ch[k], s2);
    if (ch[k].ready) cudaEventDestroy(ch[k].ready);
    if (bev[k]) cudaEventDestroy(bev[k]);
  }
  cudaStreamSynchronize(s2);
  cudaStreamDestroy(s2);
  for (int k = 0; k < 2; k++) free_host(buf[k]);
  cudaGetLastError();
  return rc;
}
