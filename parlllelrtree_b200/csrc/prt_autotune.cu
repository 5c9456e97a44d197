// Autotuner of the filter-and-refine overlay (no reference counterpart; the
// reference hard-codes a fanout and runs one pair per thread).
//
// 1. Fanout: the bottom-up build over the base layer's polygon MBRs plus the
//    breadth-first join of the overlay layer's MBRs, timed for each candidate
//    fanout; the candidate set is the same for every fanout, only the time
//    differs.
// 2. Batched schedule: coordinate descent over (a) the vertex count above
//    which a pair is clipped by a whole warp, (b) the warp clipper's
//    shared-memory slots per warp, (c) the persistent warps per SM, each
//    candidate timed on an evenly strided sample of the candidate pairs with
//    CUDA events on the caller's stream.
// The best schedule is installed with prt_schedule_set and returned.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <functional>
#include <vector>

#include "prt_internal.cuh"
#include "prt_overlay.cuh"

namespace prt {
namespace {

struct Timer {
  cudaEvent_t a = nullptr, b = nullptr;
  Timer() {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
  }
  ~Timer() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

// Schedule with pairs above warp_above vertices in warp mode.
prt_schedule make_schedule(int64_t warp_above, int slots, int warps) {
  std::vector<int64_t> thr = {1ll << 40, 4096, 1024, 256, 128, 64};
  if (warp_above > 64 && warp_above < 4096) thr.push_back(warp_above);
  std::sort(thr.begin(), thr.end(), std::greater<int64_t>());
  thr.erase(std::unique(thr.begin(), thr.end()), thr.end());
  prt_schedule s;
  memset(&s, 0, sizeof s);
  s.nbins = (int)std::min<size_t>(thr.size(), PRT_MAX_BINS);
  s.aet_slots = slots;
  s.warps_per_sm = warps;
  for (int b = 0; b < s.nbins; b++) {
    const int64_t lower = b + 1 < s.nbins ? thr[b + 1] : 0;  // bin b: (lower, thr[b]]
    s.bin_thresholds[b] = thr[b];
    s.bin_warp_mode[b] = lower >= warp_above ? 1 : 0;
  }
  return s;
}

double secs_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace
}  // namespace prt

using namespace prt;

extern "C" {

int prt_autotune(const prt_layer *base, const prt_layer *overlay, int op, int64_t max_sample_pairs,
                 double time_budget_s, void *stream, prt_tuning *out) {
  PRT_CHECK(base && overlay && out, PRT_ERR_INVALID, "NULL argument");
  PRT_CHECK(base->n_poly >= 1 && overlay->n_poly >= 1, PRT_ERR_INVALID, "empty layer");
  PRT_CHECK(op >= 0 && op <= 3, PRT_ERR_INVALID, "op %d", op);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (max_sample_pairs <= 0) max_sample_pairs = 200000;
  if (time_budget_s <= 0) time_budget_s = 30.0;
  const auto t0 = std::chrono::steady_clock::now();
  memset(out, 0, sizeof *out);
  Timer tm;
  double *mb = nullptr, *mo = nullptr;
  PRT_CUDA(cudaMalloc(&mb, sizeof(double) * 4 * base->n_poly));
  cudaError_t e = cudaMalloc(&mo, sizeof(double) * 4 * overlay->n_poly);
  if (e != cudaSuccess) {
    cudaFree(mb);
    return cuda_status(e, "cudaMalloc (autotune)");
  }
  int rc = prt_layer_mbr(base, mb, stream);
  if (!rc) rc = prt_layer_mbr(overlay, mo, stream);

  // ---- 1. fanout of the build + join
  const int fanouts[] = {8, 12, 16, 24, 32};
  int best_f = 16;
  double best_bj = 1e30;
  int64_t npairs = 0;
  for (int F : fanouts) {
    if (rc) break;
    double t_best = 1e30;
    for (int rep = 0; rep < 2 && !rc; rep++) {
      prt_tree *t = nullptr;
      int64_t cnt = 0;
      cudaEventRecord(tm.a, s);
      rc = prt_build_bottomup(mb, PRT_COORD_F64, nullptr, base->n_poly, F, PRT_KEY_MORTON32, stream, &t);
      if (!rc) rc = prt_join(t, mo, PRT_COORD_F64, overlay->n_poly, nullptr, 0, &cnt, stream);
      cudaEventRecord(tm.b, s);
      cudaEventSynchronize(tm.b);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, tm.a, tm.b);
      if (t) prt_tree_free(t);
      t_best = std::min(t_best, (double)ms);
      npairs = cnt;
    }
    out->candidates++;
    if (t_best < best_bj) {
      best_bj = t_best;
      best_f = F;
    }
  }
  out->fanout = best_f;
  out->build_join_ms = best_bj;

  // ---- 2. the sample of candidate pairs
  prt_tree *t = nullptr;
  prt_pair *all = nullptr, *sample = nullptr;
  int32_t *l2p = nullptr;
  int64_t m = 0;
  if (!rc) rc = prt_build_bottomup(mb, PRT_COORD_F64, nullptr, base->n_poly, best_f, PRT_KEY_MORTON32, stream, &t);
  if (!rc && npairs > 0) {
    e = cudaMalloc(&all, sizeof(prt_pair) * npairs);
    if (e != cudaSuccess) rc = cuda_status(e, "cudaMalloc (autotune pairs)");
    int64_t cnt = 0;
    if (!rc) rc = prt_join(t, mo, PRT_COORD_F64, overlay->n_poly, all, npairs, &cnt, stream);
    const int64_t stride = std::max<int64_t>(1, (npairs + max_sample_pairs - 1) / max_sample_pairs);
    m = (npairs + stride - 1) / stride;
    if (!rc) {
      e = cudaMalloc(&sample, sizeof(prt_pair) * m);
      if (e == cudaSuccess) e = cudaMalloc(&l2p, sizeof(int32_t) * base->n_poly);
      if (e == cudaSuccess)
        e = cudaMemcpy2DAsync(sample, sizeof(prt_pair), all, sizeof(prt_pair) * stride, sizeof(prt_pair), m,
                              cudaMemcpyDeviceToDevice, s);
      if (e != cudaSuccess) rc = cuda_status(e, "autotune sample");
    }
    if (!rc) rc = prt_tree_leaf_order(t, l2p, stream);
  }
  out->sample_pairs = m;

  // ---- 3. schedule: coordinate descent
  prt_schedule saved;
  prt_schedule_get(&saved);
  auto time_sched = [&](const prt_schedule &sc, double *ms_out) -> int {
    int r = prt_schedule_set(&sc);
    if (r) return r;
    double best = 1e30;
    for (int rep = 0; rep < 2; rep++) {
      prt_results *res = nullptr;
      cudaEventRecord(tm.a, s);
      r = prt_overlay_run(sample, m, 0, l2p, base, overlay, op, PRT_SCHED_BATCHED, stream, &res);
      cudaEventRecord(tm.b, s);
      cudaEventSynchronize(tm.b);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, tm.a, tm.b);
      if (res) prt_results_free(res);
      if (r) return r;
      best = std::min(best, (double)ms);
    }
    *ms_out = best;
    out->candidates++;
    return PRT_OK;
  };
  int64_t warp_above = 128;
  int slots = 64, wps = kLptWarpsPerSM;
  prt_schedule best = make_schedule(warp_above, slots, wps);
  double best_ms = 1e30;
  if (!rc && m > 0) {
    rc = time_sched(best, &best_ms);
    const int64_t cands_w[] = {0, 64, 256, 1024, 1ll << 41};
    for (int64_t wa : cands_w) {
      if (rc || secs_since(t0) > time_budget_s) break;
      prt_schedule c = make_schedule(wa, slots, wps);
      double ms = 0;
      rc = time_sched(c, &ms);
      if (!rc && ms < best_ms) {
        best_ms = ms;
        best = c;
        warp_above = wa;
      }
    }
    const int cands_s[] = {32, 128};
    for (int sl : cands_s) {
      if (rc || secs_since(t0) > time_budget_s) break;
      prt_schedule c = make_schedule(warp_above, sl, wps);
      double ms = 0;
      rc = time_sched(c, &ms);
      if (!rc && ms < best_ms) {
        best_ms = ms;
        best = c;
        slots = sl;
      }
    }
    const int cands_wp[] = {4, 6, 8, 10};
    for (int wp : cands_wp) {
      if (rc || secs_since(t0) > time_budget_s) break;
      prt_schedule c = make_schedule(warp_above, slots, wp);
      double ms = 0;
      rc = time_sched(c, &ms);
      if (!rc && ms < best_ms) {
        best_ms = ms;
        best = c;
        wps = wp;
      }
    }
  }
  if (!rc && m > 0) {
    rc = prt_schedule_set(&best);
    out->sched = best;
    out->clip_ms = best_ms;
  } else {
    prt_schedule_set(&saved);
    out->sched = saved;
  }
  out->seconds = secs_since(t0);
  if (t) prt_tree_free(t);
  cudaFree(all);
  cudaFree(sample);
  cudaFree(l2p);
  cudaFree(mb);
  cudaFree(mo);
  return rc;
}

}  // extern "C"
