// Launch accounting: every kernel launch of the library is counted, and, when
// enabled, bracketed by CUDA events on its stream so callers can read the
// device time per kernel category (bta_prof_read in include/dalia_bta.h).
#pragma once

#include <cuda_runtime.h>

namespace bta {

// PROF_SLICE: the digit pre-pass of the 8-bit-slice GEMM; PROF_FACTOR_GEMM:
// the GEMMs (and their pre-pass) that apply the factorisation's
// previous-column Schur updates when those run outside the panel kernel.
enum ProfCat : int {
  PROF_PANEL = 0,
  PROF_GEMM = 1,
  PROF_SWEEP = 2,
  PROF_TRTRI = 3,
  PROF_OTHER = 4,
  PROF_SLICE = 5,
  PROF_FACTOR_GEMM = 6,
  PROF_NCAT = 8
};

// While a ProfRetarget lives on this thread, GEMM and pre-pass launches
// count under the given category.
int prof_retarget(int cat);  // returns the previous target (-1: none)
struct ProfRetarget {
  int prev;
  explicit ProfRetarget(int cat) : prev(prof_retarget(cat)) {}
  ~ProfRetarget() { prof_retarget(prev); }
};
int prof_category(int cat);

void prof_begin(int cat, cudaStream_t s, cudaEvent_t* ev);
void prof_end(int cat, cudaStream_t s, cudaEvent_t ev);

// Per-device launch set-up.  A kernel attribute such as its dynamic
// shared-memory limit belongs to the kernel on one device, so the helpers
// below remember what they did per (kernel, device), under a mutex: a process
// may drive several GPUs from several host threads.
// ensure_smem_attr: raise the kernel's dynamic shared-memory limit on the
// current device (once per device); returns a cudaError_t.
int ensure_smem_attr(const void* kernel, int bytes);
// Number of SMs of the current device (cached per device).
int device_sm_count();

struct ProfScope {
  int cat;
  cudaStream_t s;
  cudaEvent_t ev = nullptr;
  ProfScope(int c, cudaStream_t st) : cat(prof_category(c)), s(st) { prof_begin(cat, s, &ev); }
  ~ProfScope() { prof_end(cat, s, ev); }
};

}  // namespace bta
