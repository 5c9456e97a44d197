// Exclusive prefix sums over int64 arrays (reduce -> scan of tile sums ->
// downsweep), used to turn per-pair sizes into arena and output offsets.
#include <cuda_runtime.h>

#include "prt_internal.cuh"

namespace prt {
namespace {

constexpr int kScanBlock = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanBlock * kScanItems;

template <typename InT>
__global__ void tile_sum_kernel(const InT *__restrict__ in, int64_t n, int64_t *__restrict__ sums) {
  __shared__ int64_t red[kScanBlock / 32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  int64_t s = 0;
  for (int i = 0; i < kScanItems; i++) {
    int64_t idx = base + (int64_t)i * kScanBlock + threadIdx.x;
    if (idx < n) s += (int64_t)in[idx];
  }
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int64_t t = 0;
    for (int w = 0; w < kScanBlock / 32; w++) t += red[w];
    sums[blockIdx.x] = t;
  }
}

// Exclusive scan of one tile with a carried-in offset.
template <typename InT>
__global__ void tile_scan_kernel(const InT *__restrict__ in, int64_t n, const int64_t *__restrict__ tile_off,
                                 int64_t *__restrict__ out) {
  __shared__ int64_t warp_tot[kScanBlock / 32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int64_t v[kScanItems];
  int64_t run = 0;
  for (int i = 0; i < kScanItems; i++) {
    int64_t idx = base + i;
    v[i] = idx < n ? (int64_t)in[idx] : 0;
    int64_t t = v[i];
    v[i] = run;
    run += t;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int64_t incl = run;
  for (int o = 1; o < 32; o <<= 1) {
    int64_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  int64_t woff = 0;
  for (int w = 0; w < warp; w++) woff += warp_tot[w];
  const int64_t off = tile_off[blockIdx.x] + woff + incl - run;
  for (int i = 0; i < kScanItems; i++) {
    int64_t idx = base + i;
    if (idx < n) out[idx] = off + v[i];
  }
}

}  // namespace

template <typename InT>
int exclusive_scan(const InT *d_in, int64_t n, int64_t *d_out, int64_t *d_total, cudaStream_t s) {
  if (n <= 0) {
    if (d_total) PRT_CUDA(cudaMemsetAsync(d_total, 0, sizeof(int64_t), s));
    return PRT_OK;
  }
  const int64_t tiles = (n + kScanTile - 1) / kScanTile;
  int64_t *sums = nullptr, *offs = nullptr;
  int rc = dalloc(&sums, tiles + 1, s);
  if (!rc) rc = dalloc(&offs, tiles + 1, s);
  if (rc) {
    dfree(sums, s);
    return rc;
  }
  {
    PRT_PROF("tile_sum", s);
    tile_sum_kernel<InT><<<(unsigned)tiles, kScanBlock, 0, s>>>(d_in, n, sums);
  }
  if (tiles == 1) {
    cudaMemsetAsync(offs, 0, sizeof(int64_t), s);
    cudaMemcpyAsync(offs + 1, sums, sizeof(int64_t), cudaMemcpyDeviceToDevice, s);
  } else {
    rc = exclusive_scan<int64_t>(sums, tiles, offs, offs + tiles, s);
  }
  if (!rc) {
    {
      PRT_PROF("tile_scan", s);
      tile_scan_kernel<InT><<<(unsigned)tiles, kScanBlock, 0, s>>>(d_in, n, offs, d_out);
    }
    if (d_total) cudaMemcpyAsync(d_total, offs + tiles, sizeof(int64_t), cudaMemcpyDeviceToDevice, s);
  }
  dfree(sums, s);
  dfree(offs, s);
  if (rc) return rc;
  PRT_CUDA(cudaGetLastError());
  return PRT_OK;
}

template int exclusive_scan<int64_t>(const int64_t *, int64_t, int64_t *, int64_t *, cudaStream_t);
template int exclusive_scan<int32_t>(const int32_t *, int64_t, int64_t *, int64_t *, cudaStream_t);

}  // namespace prt
