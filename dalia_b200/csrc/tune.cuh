// Online autotuner of launch configurations.
//
// A tuned launch site names a family ("panel", "sweep", ...), a key (the
// launch shape: block sizes, instance count, ...) and its number of
// candidate configurations.  The first launches of a new (family, key) try
// the candidates in turn -- each `reps` times (default TUNE_REPS), timed by CUDA events on
// the launch's stream -- on the caller's real work (the block columns of a
// factorisation all have one shape, so trying a candidate costs nothing but
// its own speed).  The launch after the last trial reads the event times
// (one host synchronisation per key) and keeps the fastest candidate from
// then on.  Decisions are keyed by device (name and SM count), kept for the
// process and, when the environment variable DALIA_B200_TUNE_CACHE names a
// file, read from and appended to that file, so a later process starts with
// them.  DALIA_B200_TUNE=0 turns tuning off (candidate 0 everywhere).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

namespace bta {

constexpr int TUNE_REPS = 2;

class TuneLaunch {
 public:
  TuneLaunch(const char* family, const std::vector<long long>& key, int ncand, cudaStream_t s,
             int reps = TUNE_REPS);
  ~TuneLaunch();
  int choice() const { return choice_; }

 private:
  int choice_ = 0;
  void* entry_ = nullptr;  // trial bookkeeping of this launch (nullptr: not a trial)
  int trial_ = -1;
  cudaStream_t stream_ = nullptr;
};

}  // namespace bta
