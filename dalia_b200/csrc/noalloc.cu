// BTA Cholesky for callers that cannot allocate device memory.
//
// Some callers of this library are not allowed to call cudaMalloc/cudaFree:
// code that runs inside a host framework whose pool allocator owns all of the
// GPU's memory (a raw cudaMalloc beside it can fail or fragment that pool),
// and latency-critical loops where cudaFree's implicit device-wide
// synchronisation is unacceptable.  bta_pobtaf needs a handle whose scratch is
// allocated on demand; bta_pobtaf_noalloc below runs the same kernels with all
// of its scratch -- status words, launch task lists, inverses of the 64x64
// diagonal tiles and per-tile dependency counters -- carved out of one
// file-scope device array of fixed size (kScratchBytes, 2 MiB).  Every GPU
// that loads this library holds that array until the process exits.  The
// task lists are written by a small kernel, so a call reads no host memory
// once it has returned.
//
// The array is shared by every call: it keeps the previous call's contents, so
// each call clears what must start at zero, and calls whose work overlaps on
// the GPU (different streams, or different host threads) race on it.
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "../../include/dalia_bta.h"
#include "gemm.cuh"
#include "panel.cuh"

namespace {

constexpr size_t kScratchBytes = size_t(2) << 20;  // 2 MiB
constexpr size_t kAlign = 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// In host code g_noalloc_scratch names a host-side shadow, not device memory:
// the device address comes from cudaGetSymbolAddress, once per device, with
// that device current.
std::mutex g_mu;
std::map<int, char*> g_addr;

int scratch_address(char** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return BTA_ERR_CUDA;
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_addr.find(dev);
  if (it == g_addr.end()) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return BTA_ERR_CUDA;
    }
    it = g_addr.emplace(dev, static_cast<char*>(p)).first;
  }
  *out = it->second;
  return BTA_OK;
}

inline size_t align_up(size_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

struct Layout {
  size_t ws_bytes = 0;  // tile inverses + counters of one panel (reused per step)
  size_t off_ws = 0, off_tasksL = 0, off_tasks0 = 0, off_tasksT = 0, total = 0;
};

size_t panel_ws(int b, int a, bool hasL) {
  const int nq = (b + 63) / 64;
  const int nr = bta::panel_rows(b, a, hasL);
  return align_up((size_t)nq * 4096 * sizeof(double)) + align_up(((size_t)2 * nr * nq + 4) * sizeof(int));
}

// Task list of one panel with no previous-column or tip tasks (the shape this
// entry point launches): tile column r holds nr - r tasks, the diagonal tile
// (r, r) first, then tiles p = r+1 .. nr-1 in order -- the tile just below
// the diagonal tile (p = r+1 < nq) is handed to the chain CTA, every other
// tile gets its triangular solve.  This is the order bta::panel_tasks
// produces for such a panel (checked on the CPU against bta_panel_task_list).
int task_count(int nq, int nr) { return nq * nr - nq * (nq - 1) / 2; }

__global__ void write_tasks_kernel(int4* out, int nq, int nr) {
  const int r = blockIdx.x;
  if (r >= nq) return;
  const int off = r * nr - r * (r - 1) / 2;
  for (int j = threadIdx.x; j < nr - r; j += blockDim.x) {
    const int p = r + j;
    const int kind = j == 0 ? bta::TASK_AGG_DIAG : (p == r + 1 && p < nq ? bta::TASK_AGG_SUB : bta::TASK_AGG_TRSM);
    out[off + j] = make_int4(0, kind, p, r);
  }
}

int write_tasks(int4* out, int b, int a, bool hasL, cudaStream_t s) {
  const int nq = (b + 63) / 64, nr = bta::panel_rows(b, a, hasL);
  write_tasks_kernel<<<nq, 128, 0, s>>>(out, nq, nr);
  return cudaGetLastError() == cudaSuccess ? BTA_OK : BTA_ERR_CUDA;
}

// Status words: [0] abort flag (int), [8] first failing pivot (u64).
int run_panel(char* base, const Layout& lay, const int4* tasks, int ntasks, double* D, double* L, double* Ab, int b,
              int a, long long pivot_base, cudaStream_t s) {
  const bool hasL = L != nullptr;
  const int aa = Ab != nullptr ? a : 0;
  const int nq = (b + 63) / 64;
  const int nr = bta::panel_rows(b, aa, hasL);
  char* ws = base + lay.off_ws;
  double* linv = reinterpret_cast<double*>(ws);
  int* cnt = reinterpret_cast<int*>(ws + align_up((size_t)nq * 4096 * sizeof(double)));
  if (cudaMemsetAsync(cnt, 0, ((size_t)2 * nr * nq + 4) * sizeof(int), s) != cudaSuccess) return BTA_ERR_CUDA;
  bta::PanelBatch B;
  std::memset(&B, 0, sizeof(B));
  B.ninst = 1;
  B.ntasks = ntasks;
  B.tasks = tasks;
  B.counter = cnt + 2 * nr * nq;
  B.abort_flag = reinterpret_cast<int*>(base);
  bta::PanelInst& I = B.inst[0];
  I.D = D;
  I.L = L;
  I.Ab = aa ? Ab : nullptr;
  I.Linv = linv;
  I.upd = cnt;
  I.flag = cnt + nr * nq;
  I.info = reinterpret_cast<unsigned long long*>(base + 8);
  I.pivot_base = pivot_base;
  I.b = b;
  I.a = aa;
  I.nq = nq;
  I.nrows_t = nr;
  return bta::panel_launch(B, 0, s) == cudaSuccess ? BTA_OK : BTA_ERR_CUDA;
}

}  // namespace

extern "C" {

size_t bta_noalloc_scratch_bytes(void) { return kScratchBytes; }

int bta_pobtaf_noalloc(int64_t n, int64_t b, int64_t a, double* D, double* L, double* Ab, double* T, int64_t* info,
                       void* stream) {
  if (n < 1 || b < 1 || a < 0 || !D || (n > 1 && !L) || (a > 0 && (!Ab || !T))) return BTA_ERR_INVALID;
  if (b > BTA_NOALLOC_MAX_B || a > BTA_NOALLOC_MAX_A) return BTA_ERR_INVALID;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int B_ = (int)b, A_ = (int)a;
  const int nqb = (B_ + 63) / 64, nqa = (A_ + 63) / 64;
  const int nL = n > 1 ? task_count(nqb, bta::panel_rows(B_, A_, true)) : 0;
  const int n0 = task_count(nqb, bta::panel_rows(B_, A_, false));
  const int nT = a > 0 ? task_count(nqa, bta::panel_rows(A_, 0, false)) : 0;
  Layout lay;
  lay.ws_bytes = std::max(panel_ws(B_, A_, true), a > 0 ? panel_ws(A_, 0, false) : size_t(0));
  lay.off_ws = kAlign;
  lay.off_tasksL = lay.off_ws + align_up(lay.ws_bytes);
  lay.off_tasks0 = lay.off_tasksL + align_up((size_t)nL * sizeof(int4));
  lay.off_tasksT = lay.off_tasks0 + align_up((size_t)n0 * sizeof(int4));
  lay.total = lay.off_tasksT + align_up((size_t)nT * sizeof(int4));
  if (lay.total > kScratchBytes) return BTA_ERR_INVALID;  // cannot happen within the limits above

  char* base = nullptr;
  int rc = scratch_address(&base);
  if (rc) return rc;
  // clear the status words; write this call's task lists
  if (cudaMemsetAsync(base, 0, 8, s) != cudaSuccess) return BTA_ERR_CUDA;
  if (cudaMemsetAsync(base + 8, 0xff, 8, s) != cudaSuccess) return BTA_ERR_CUDA;
  int4* dL = reinterpret_cast<int4*>(base + lay.off_tasksL);
  int4* d0 = reinterpret_cast<int4*>(base + lay.off_tasks0);
  int4* dT = reinterpret_cast<int4*>(base + lay.off_tasksT);
  if (nL > 0 && (rc = write_tasks(dL, B_, A_, true, s))) return rc;
  if ((rc = write_tasks(d0, B_, A_, false, s))) return rc;
  if (nT > 0 && (rc = write_tasks(dT, A_, 0, false, s))) return rc;

  const size_t bb = (size_t)b * b, ab = (size_t)a * b;
  for (int64_t i = 0; i < n; ++i) {
    const bool hasL = i < n - 1;
    double* Di = D + i * bb;
    double* Li = hasL ? L + i * bb : nullptr;
    double* Abi = a > 0 ? Ab + i * ab : nullptr;
    rc = run_panel(base, lay, hasL ? dL : d0, hasL ? nL : n0, Di, Li, Abi, B_, A_, (long long)(i * b), s);
    if (rc) return rc;
    std::vector<bta::GemmProb> probs;
    if (hasL) {
      bta::GemmProb p = bta::gemm_prob(D + (i + 1) * bb, B_, B_, B_, 1.0, bta::GC_LOWER);
      bta::gemm_add(p, Li, B_, Li, B_, B_, -1.0, 0);
      probs.push_back(p);
    }
    if (a > 0) {
      if (hasL) {
        bta::GemmProb p = bta::gemm_prob(Ab + (i + 1) * ab, B_, A_, B_, 1.0);
        bta::gemm_add(p, Abi, B_, Li, B_, B_, -1.0, 0);
        probs.push_back(p);
      }
      bta::GemmProb p = bta::gemm_prob(T, A_, A_, A_, 1.0);
      bta::gemm_add(p, Abi, B_, Abi, B_, B_, -1.0, 0);
      probs.push_back(p);
    }
    if (!probs.empty() && bta::gemm_launch(probs, s) != cudaSuccess) return BTA_ERR_CUDA;
  }
  if (a > 0) {
    rc = run_panel(base, lay, dT, nT, T, nullptr, nullptr, A_, 0, (long long)(n * b), s);
    if (rc) return rc;
  }
  if (cudaGetLastError() != cudaSuccess) return BTA_ERR_CUDA;
  if (info) return bta_noalloc_get_status(info, stream);
  return BTA_OK;
}

int bta_noalloc_get_status(int64_t* info, void* stream) {
  char* base = nullptr;
  int rc = scratch_address(&base);
  if (rc) return rc;
  unsigned long long hinfo = 0;
  int habort = 0;
  if (cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream)) != cudaSuccess) return BTA_ERR_CUDA;
  if (cudaMemcpy(&habort, base, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return BTA_ERR_CUDA;
  if (cudaMemcpy(&hinfo, base + 8, sizeof(hinfo), cudaMemcpyDeviceToHost) != cudaSuccess) return BTA_ERR_CUDA;
  const bool fail = hinfo != ~0ULL;
  if (info) *info = fail ? (int64_t)hinfo : 0;
  if (habort) return BTA_ERR_TIMEOUT;
  return fail ? BTA_ERR_NOT_SPD : BTA_OK;
}

}  // extern "C"
