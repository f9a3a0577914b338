// Online autotuner of launch configurations (tune.cuh).
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/dalia_bta.h"
#include "tune.cuh"

namespace bta {
namespace {

struct Trial {
  int cand;
  cudaEvent_t e0, e1;
};

struct Entry {
  int ncand = 0;
  int best = -1;
  std::vector<Trial> trials;
  std::vector<float> ms;  // best time per candidate once decided
};

std::mutex g_mu;
std::map<std::string, Entry> g_table;
bool g_loaded = false;

const char* cache_path() {
  const char* p = std::getenv("DALIA_B200_TUNE_CACHE");
  return (p && *p) ? p : nullptr;
}

bool tuning_on() {
  const char* p = std::getenv("DALIA_B200_TUNE");
  return !(p && std::strcmp(p, "0") == 0);
}

// DALIA_B200_TUNE_FORCE="family=candidate,..." pins a family's candidate
// (tests use it to run every variant); -1 when the family is not named.
int forced(const char* family) {
  const char* p = std::getenv("DALIA_B200_TUNE_FORCE");
  if (!p || !*p) return -1;
  const size_t fl = std::strlen(family);
  for (const char* q = p; *q;) {
    if (std::strncmp(q, family, fl) == 0 && q[fl] == '=') return std::atoi(q + fl + 1);
    const char* c = std::strchr(q, ',');
    if (!c) break;
    q = c + 1;
  }
  return -1;
}

// "<device name>/<SM count>" of the current device (cached per device; call
// with g_mu held)
std::string device_tag() {
  static std::map<int, std::string> tags;
  int dev = 0;
  cudaGetDevice(&dev);
  auto it = tags.find(dev);
  if (it != tags.end()) return it->second;
  cudaDeviceProp prop;
  std::string s = "unknown";
  if (cudaGetDeviceProperties(&prop, dev) == cudaSuccess) {
    std::ostringstream o;
    o << prop.name << "/" << prop.multiProcessorCount;
    s = o.str();
    for (char& c : s)
      if (c == ' ' || c == '|') c = '_';
  }
  tags[dev] = s;
  return s;
}

// Cache file lines: "<family>|<device>|<key> <best> <ms of every candidate>".
void load_file() {
  g_loaded = true;
  const char* path = cache_path();
  if (!path) return;
  FILE* f = std::fopen(path, "r");
  if (!f) return;
  char line[1024];
  while (std::fgets(line, sizeof(line), f)) {
    std::istringstream in(line);
    std::string key;
    int best = -1;
    if (!(in >> key >> best) || best < 0) continue;
    Entry& e = g_table[key];
    e.best = best;
    e.ms.clear();
    float v;
    while (in >> v) e.ms.push_back(v);
    e.ncand = (int)e.ms.size();
  }
  std::fclose(f);
}

void save_line(const std::string& key, const Entry& e) {
  const char* path = cache_path();
  if (!path) return;
  FILE* f = std::fopen(path, "a");
  if (!f) return;
  std::fprintf(f, "%s %d", key.c_str(), e.best);
  for (float v : e.ms) std::fprintf(f, " %.6g", v);
  std::fprintf(f, "\n");
  std::fclose(f);
}

}  // namespace

TuneLaunch::TuneLaunch(const char* family, const std::vector<long long>& key, int ncand, cudaStream_t s, int reps)
    : stream_(s) {
  const int f = forced(family);
  if (f >= 0) {
    choice_ = f < ncand ? f : 0;
    return;
  }
  if (ncand <= 1 || !tuning_on()) return;
  std::lock_guard<std::mutex> lk(g_mu);
  std::ostringstream o;
  o << family << "|" << device_tag() << "|";
  for (size_t i = 0; i < key.size(); ++i) o << (i ? "," : "") << key[i];
  const std::string k = o.str();
  if (!g_loaded) load_file();
  Entry& e = g_table[k];
  if (e.best >= 0 && e.best < ncand) {
    choice_ = e.best;
    return;
  }
  e.ncand = ncand;
  if ((int)e.trials.size() < ncand * std::max(1, reps)) {
    Trial t{(int)e.trials.size() % ncand, nullptr, nullptr};
    if (cudaEventCreate(&t.e0) != cudaSuccess || cudaEventCreate(&t.e1) != cudaSuccess ||
        cudaEventRecord(t.e0, s) != cudaSuccess) {
      cudaGetLastError();
      return;  // untimed: candidate 0
    }
    e.trials.push_back(t);
    choice_ = t.cand;
    entry_ = &e;
    trial_ = (int)e.trials.size() - 1;
    return;
  }
  // every candidate tried: keep the fastest
  e.ms.assign(ncand, std::numeric_limits<float>::infinity());
  for (Trial& t : e.trials) {
    float ms = 0.f;
    if (cudaEventSynchronize(t.e1) == cudaSuccess && cudaEventElapsedTime(&ms, t.e0, t.e1) == cudaSuccess)
      e.ms[t.cand] = std::min(e.ms[t.cand], ms);
    cudaEventDestroy(t.e0);
    cudaEventDestroy(t.e1);
  }
  cudaGetLastError();
  e.trials.clear();
  int best = 0;
  for (int c = 1; c < ncand; ++c)
    if (e.ms[c] < e.ms[best]) best = c;
  e.best = best;
  choice_ = best;
  save_line(k, e);
}

TuneLaunch::~TuneLaunch() {
  if (!entry_) return;
  std::lock_guard<std::mutex> lk(g_mu);
  Entry* e = static_cast<Entry*>(entry_);
  if (trial_ < (int)e->trials.size()) cudaEventRecord(e->trials[trial_].e1, stream_);
}

}  // namespace bta

extern "C" {

int bta_tune_pending(void) {
  std::lock_guard<std::mutex> lk(bta::g_mu);
  int n = 0;
  for (const auto& kv : bta::g_table)
    if (kv.second.best < 0 && !kv.second.trials.empty()) ++n;
  return n;
}

int bta_tune_report(char* buf, size_t cap, size_t* len) {
  std::ostringstream o;
  {
    std::lock_guard<std::mutex> lk(bta::g_mu);
    for (const auto& kv : bta::g_table) {
      if (kv.second.best < 0) continue;
      o << kv.first << " best=" << kv.second.best << " ms=";
      for (size_t i = 0; i < kv.second.ms.size(); ++i) o << (i ? "," : "") << kv.second.ms[i];
      o << "\n";
    }
  }
  const std::string s = o.str();
  if (len) *len = s.size();
  if (!buf || cap == 0) return BTA_OK;
  const size_t n = std::min(cap - 1, s.size());
  std::memcpy(buf, s.data(), n);
  buf[n] = 0;
  return s.size() < cap ? BTA_OK : BTA_ERR_INVALID;
}

}  // extern "C"
