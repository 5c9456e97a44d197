// Launch profiler: CUDA events around the library's kernel launches, summed
// per kernel name (see PRT_PROF in prt_internal.cuh).
#include <cuda_runtime.h>

#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "prt_internal.cuh"

namespace prt {

bool g_prof_on = false;
static int g_prof_mode = 0;           // 1: time every launch, 2: count all, time the focus kernel only
static std::string g_prof_focus;

namespace {

struct Rec {
  std::string name;
  cudaEvent_t a, b;
};

struct Acc {
  double ms = 0.0;
  int64_t n = 0;
};

std::mutex g_mu;
std::vector<Rec *> g_pending;
std::vector<cudaEvent_t> g_pool;
std::map<std::string, Acc> g_acc;

cudaEvent_t take_event() {
  if (!g_pool.empty()) {
    cudaEvent_t e = g_pool.back();
    g_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return e;
}

void drain_locked() {
  for (Rec *r : g_pending) {
    float ms = 0.f;
    if (r->a && r->b && cudaEventSynchronize(r->b) == cudaSuccess &&
        cudaEventElapsedTime(&ms, r->a, r->b) == cudaSuccess) {
      Acc &x = g_acc[r->name];
      x.ms += ms;
      x.n += 1;
    } else {
      cudaGetLastError();
    }
    if (r->a) g_pool.push_back(r->a);
    if (r->b) g_pool.push_back(r->b);
    delete r;
  }
  g_pending.clear();
}

}  // namespace

void prof_begin(const char *name, cudaStream_t s, void **token) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_prof_mode == 2 && g_prof_focus != name) {
    g_acc[name].n += 1;  // counted, not timed
    *token = nullptr;
    return;
  }
  Rec *r = new Rec();
  r->name = name;
  r->a = take_event();
  r->b = take_event();
  if (r->a) cudaEventRecord(r->a, s);
  *token = r;
}

void prof_end(void *token, cudaStream_t s) {
  std::lock_guard<std::mutex> lk(g_mu);
  Rec *r = reinterpret_cast<Rec *>(token);
  if (r->b) cudaEventRecord(r->b, s);
  g_pending.push_back(r);
  if (g_pending.size() > 8192) drain_locked();
}

}  // namespace prt

using namespace prt;

extern "C" {

int prt_profile_enable(int on) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_prof_on = on != 0;
  g_prof_mode = on;
  return PRT_OK;
}

int prt_profile_focus(const char *name) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_prof_focus = name ? name : "";
  return PRT_OK;
}

int prt_profile_reset(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  drain_locked();
  g_acc.clear();
  return PRT_OK;
}

int prt_profile_read(char *names, int names_cap, double *ms_total, int64_t *launches, int cap) {
  std::lock_guard<std::mutex> lk(g_mu);
  drain_locked();
  int k = 0;
  size_t used = 0;
  if (names && names_cap > 0) names[0] = '\0';
  for (auto &kv : g_acc) {
    if (k >= cap) break;
    size_t len = kv.first.size();
    if (names && used + len + 2 <= (size_t)names_cap) {
      memcpy(names + used, kv.first.data(), len);
      names[used + len] = '\n';
      names[used + len + 1] = '\0';
      used += len + 1;
    }
    if (ms_total) ms_total[k] = kv.second.ms;
    if (launches) launches[k] = kv.second.n;
    k++;
  }
  return k;
}

}  // extern "C"
