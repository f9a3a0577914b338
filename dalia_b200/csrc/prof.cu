// Launch counter and optional per-category CUDA-event timing (prof.cuh).
#include <atomic>
#include <map>
#include <mutex>
#include <set>
#include <tuple>
#include <vector>

#include "../../include/dalia_bta.h"
#include "prof.cuh"

namespace bta {
namespace {

struct Pending {
  int cat;
  cudaEvent_t a, b;
};

std::atomic<long long> g_launches{0};
std::atomic<bool> g_on{false};
std::atomic<int> g_mask{0xFF};  // categories that get events
std::mutex g_mu;
std::vector<Pending> g_pending;
std::vector<cudaEvent_t> g_pool;
double g_ms[PROF_NCAT] = {0};
long long g_cnt[PROF_NCAT] = {0};

cudaEvent_t take_event() {
  if (!g_pool.empty()) {
    cudaEvent_t e = g_pool.back();
    g_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

std::mutex g_attr_mu;
std::set<std::tuple<const void*, int, int>> g_attr_done;  // (kernel, device, bytes)
std::map<int, int> g_sms;

}  // namespace

int ensure_smem_attr(const void* kernel, int bytes) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_attr_mu);
  const auto key = std::make_tuple(kernel, dev, bytes);
  if (g_attr_done.count(key)) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return e;
  g_attr_done.insert(key);
  return cudaSuccess;
}

int device_sm_count() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  std::lock_guard<std::mutex> lk(g_attr_mu);
  auto it = g_sms.find(dev);
  if (it == g_sms.end()) {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    it = g_sms.emplace(dev, sms).first;
  }
  return it->second;
}

namespace {
thread_local int t_retarget = -1;
}  // namespace

int prof_retarget(int cat) {
  const int prev = t_retarget;
  t_retarget = cat;
  return prev;
}

int prof_category(int cat) {
  return (t_retarget >= 0 && (cat == PROF_GEMM || cat == PROF_SLICE)) ? t_retarget : cat;
}

void prof_begin(int cat, cudaStream_t s, cudaEvent_t* ev) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  *ev = nullptr;
  if (!g_on.load(std::memory_order_relaxed) || !((g_mask.load(std::memory_order_relaxed) >> cat) & 1)) return;
  std::lock_guard<std::mutex> lk(g_mu);
  *ev = take_event();
  cudaEventRecord(*ev, s);
}

void prof_end(int cat, cudaStream_t s, cudaEvent_t ev) {
  if (ev == nullptr) return;
  std::lock_guard<std::mutex> lk(g_mu);
  cudaEvent_t e2 = take_event();
  cudaEventRecord(e2, s);
  g_pending.push_back({cat, ev, e2});
}

}  // namespace bta

extern "C" {

long long bta_launch_count(void) { return bta::g_launches.load(); }

int bta_prof_enable(int on) {
  if (on) {
    // events for ~8000 launches made now, so that timing a region costs no
    // event creation inside it (events return to the pool on bta_prof_read)
    std::lock_guard<std::mutex> lk(bta::g_mu);
    while (bta::g_pool.size() < 16384) {
      cudaEvent_t e = nullptr;
      if (cudaEventCreate(&e) != cudaSuccess) return BTA_ERR_CUDA;
      bta::g_pool.push_back(e);
    }
  }
  bta::g_on.store(on != 0);
  return BTA_OK;
}

int bta_prof_mask(int mask) {
  bta::g_mask.store(mask);
  return BTA_OK;
}

int bta_prof_read(double* ms, long long* counts) {
  using namespace bta;
  std::lock_guard<std::mutex> lk(g_mu);
  for (auto& p : g_pending) {
    if (cudaEventSynchronize(p.b) != cudaSuccess) return BTA_ERR_CUDA;
    float t = 0.f;
    cudaEventElapsedTime(&t, p.a, p.b);
    g_ms[p.cat] += t;
    g_cnt[p.cat] += 1;
    g_pool.push_back(p.a);
    g_pool.push_back(p.b);
  }
  g_pending.clear();
  for (int i = 0; i < PROF_NCAT; ++i) {
    if (ms) ms[i] = g_ms[i];
    if (counts) counts[i] = g_cnt[i];
    g_ms[i] = 0;
    g_cnt[i] = 0;
  }
  return BTA_OK;
}

}  // extern "C"
