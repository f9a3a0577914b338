// Host orchestration of the BTA factorisation, solve, selected inversion and
// log-determinant, exported through the C ABI declared in include/dalia_bta.h.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "../../include/dalia_bta.h"
#include "bta_internal.cuh"
#include "gemm.cuh"
#include "panel.cuh"
#include "prof.cuh"
#include "tune.cuh"

using namespace bta;

struct bta_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  char* ws = nullptr;
  size_t ws_bytes = 0;
  char* ws2 = nullptr;  // digit images of the 8-bit-slice GEMM
  size_t ws2_bytes = 0;
  int* ctl = nullptr;  // [0] abort flag, [1] scratch; ctl+2 (8-aligned): info (u64)
  double* scal = nullptr;
  std::map<std::vector<int>, std::pair<int4*, int>> tasks;
};

namespace {

constexpr size_t kAlign = 256;
inline size_t align_up(size_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

struct Carve {
  char* base;
  size_t off = 0;
  template <class T_>
  T_* take(size_t count) {
    T_* p = reinterpret_cast<T_*>(base + off);
    off = align_up(off + count * sizeof(T_));
    return p;
  }
};

int ensure_ws2(bta_context* h, size_t bytes) {
  if (bytes <= h->ws2_bytes) return BTA_OK;
  if (h->ws2) {
    cudaStreamSynchronize(h->stream);
    cudaFree(h->ws2);
    h->ws2 = nullptr;
    h->ws2_bytes = 0;
  }
  size_t want = align_up(bytes + (bytes >> 3));
  if (cudaMalloc(&h->ws2, want) != cudaSuccess) {
    cudaGetLastError();
    return BTA_ERR_ALLOC;
  }
  h->ws2_bytes = want;
  return BTA_OK;
}

// Grouped GEMM in the requested arithmetic on the handle's stream.
int run_gemm(bta_context* h, const std::vector<GemmProb>& pr, int precision) {
  if (precision == BTA_PREC_TF32X3) return gemm_launch_tc(pr, h->stream, h->ctl) ? BTA_ERR_CUDA : BTA_OK;
  if (precision == BTA_PREC_I8SLICE) {
    size_t need = 0;
    if (gemm_launch_i8(pr, h->stream, h->ctl, nullptr, 0, &need)) return BTA_ERR_INVALID;
    int rc = ensure_ws2(h, need);
    if (rc) return rc;
    return gemm_launch_i8(pr, h->stream, h->ctl, h->ws2, h->ws2_bytes, nullptr) ? BTA_ERR_CUDA : BTA_OK;
  }
  return gemm_launch(pr, h->stream) ? BTA_ERR_CUDA : BTA_OK;
}

int ensure_ws(bta_context* h, size_t bytes) {
  if (bytes <= h->ws_bytes) return BTA_OK;
  if (h->ws) {
    cudaStreamSynchronize(h->stream);
    cudaFree(h->ws);
    h->ws = nullptr;
    h->ws_bytes = 0;
  }
  size_t want = align_up(bytes + (bytes >> 4));
  if (cudaMalloc(&h->ws, want) != cudaSuccess) {
    cudaGetLastError();
    return BTA_ERR_ALLOC;
  }
  h->ws_bytes = want;
  return BTA_OK;
}

inline unsigned long long* info_ptr(bta_context* h) { return reinterpret_cast<unsigned long long*>(h->ctl + 2); }

// Makes the handle's device current for one call and restores the caller's
// device afterwards: a handle's scratch and launches belong to its device.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(const bta_context* h) {
    if (!h) return;
    if (cudaGetDevice(&prev) != cudaSuccess || prev == h->device) {
      prev = -1;
      return;
    }
    cudaSetDevice(h->device);
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

int cuda_rc(cudaError_t e) { return e == cudaSuccess ? BTA_OK : BTA_ERR_CUDA; }
int cuda_rc(int e) { return e == 0 ? BTA_OK : BTA_ERR_CUDA; }

// One instance of a batched panel launch.
struct PanelSpec {
  double* D;
  double* L;
  double* Ab;
  int b, a;
  long long base;
  const double* Lprev = nullptr;
  const double* Abprev = nullptr;
  double* Ttip = nullptr;
};

// Cached device task list of a panel batch with the given instance shapes
// and queue lookahead.
int get_tasks(bta_context* h, const std::vector<PanelInst>& insts, int lookahead, int order, const int4** out,
              int* count) {
  std::vector<int> key{lookahead, order};
  for (const auto& I : insts) {
    key.push_back(I.b);
    key.push_back(I.a);
    key.push_back((I.L != nullptr ? 1 : 0) | (I.Ttip != nullptr ? 2 : 0) | (I.Lprev != nullptr ? 4 : 0) |
                  (I.Abprev != nullptr ? 8 : 0));
  }
  auto it = h->tasks.find(key);
  if (it == h->tasks.end()) {
    std::vector<int4> t;
    panel_tasks(insts, t, lookahead, order);
    int4* d = nullptr;
    if (!t.empty()) {
      if (cudaMalloc(&d, t.size() * sizeof(int4)) != cudaSuccess) return BTA_ERR_ALLOC;
      if (cudaMemcpy(d, t.data(), t.size() * sizeof(int4), cudaMemcpyHostToDevice) != cudaSuccess)
        return BTA_ERR_CUDA;
    }
    it = h->tasks.emplace(key, std::make_pair(d, (int)t.size())).first;
  }
  *out = it->second.first;
  *count = it->second.second;
  return BTA_OK;
}

// Factor one block column of every instance in one launch (chunks of
// PANEL_MAXI instances).
int run_panels(bta_context* h, const std::vector<PanelSpec>& specs, Carve& cv) {
  for (size_t c0 = 0; c0 < specs.size(); c0 += PANEL_MAXI) {
    const size_t c1 = std::min(specs.size(), c0 + (size_t)PANEL_MAXI);
    PanelBatch B;
    std::memset(&B, 0, sizeof(B));
    std::vector<PanelInst> insts;
    size_t cnt_total = 0;
    for (size_t k = c0; k < c1; ++k) {
      const PanelSpec& sp = specs[k];
      const bool hasL = sp.L != nullptr;
      const int aa = sp.Ab != nullptr ? sp.a : 0;
      PanelInst I{};
      I.D = sp.D;
      I.L = sp.L;
      I.Ab = aa ? sp.Ab : nullptr;
      I.b = sp.b;
      I.a = aa;
      I.nq = (sp.b + 63) / 64;
      I.nrows_t = panel_rows(sp.b, aa, hasL);
      I.pivot_base = sp.base;
      I.info = info_ptr(h);
      I.Lprev = sp.Lprev;
      I.Abprev = aa ? sp.Abprev : nullptr;
      I.Ttip = (aa > 0 && aa <= 64) ? sp.Ttip : nullptr;
      I.Linv = cv.take<double>((size_t)I.nq * 64 * 64);
      cnt_total += (size_t)3 * I.nrows_t * I.nq;
      insts.push_back(I);
    }
    int* cnt = cv.take<int>(cnt_total + 4);
    size_t off = 0;
    for (auto& I : insts) {
      I.upd = cnt + off;
      I.flag = cnt + off + (size_t)I.nrows_t * I.nq;
      I.prv = cnt + off + (size_t)2 * I.nrows_t * I.nq;
      off += (size_t)3 * I.nrows_t * I.nq;
    }
    // launch shape: instances, their block and arrow sizes, which terms the
    // launch applies; candidates: resident CTAs per SM x queue order x
    // lookahead of the previous-column terms (when the launch has them)
    std::vector<long long> tkey{(long long)insts.size()};
    for (const auto& I : insts)
      tkey.push_back(((long long)I.b << 20) | ((long long)I.a << 4) | (I.L ? 1 : 0) | (I.Lprev ? 2 : 0) |
                     (I.Abprev ? 4 : 0) | (I.Ttip ? 8 : 0));
    const int occ = panel_ctas_per_sm();
    if (occ < 0) return BTA_ERR_CUDA;
    static const int kLook[3] = {PREV_LOOKAHEAD, 1, 4};
    static const int kOrder[2] = {PANEL_ORDER_CHAIN_AHEAD, PANEL_ORDER_COLUMN};
    // only the launches that repeat within one factorisation (block columns
    // with a block below) are tuned
    bool bulk = true, prev = false;
    for (const auto& I : insts) {
      bulk = bulk && I.L != nullptr;
      prev = prev || I.Lprev != nullptr;
    }
    const int nocc = std::min(occ, 2), nlook = prev ? 3 : 1;
    const int ncand = bulk ? nocc * 2 * nlook : 1;
    TuneLaunch tl("panel", tkey, ncand, h->stream);
    const int c = tl.choice();
    const int grid = device_sm_count() * (occ - c % nocc);
    const int order = kOrder[(c / nocc) % 2];
    const int lookahead = kLook[c / (2 * nocc)];
    const int4* tasks;
    int ntasks;
    int rc = get_tasks(h, insts, lookahead, order, &tasks, &ntasks);
    if (rc) return rc;
    if (cudaMemsetAsync(cnt, 0, (cnt_total + 4) * sizeof(int), h->stream) != cudaSuccess) return BTA_ERR_CUDA;
    B.ninst = (int)insts.size();
    B.ntasks = ntasks;
    B.tasks = tasks;
    B.counter = cnt + cnt_total;
    B.abort_flag = h->ctl;
    for (size_t k = 0; k < insts.size(); ++k) B.inst[k] = insts[k];
    rc = cuda_rc(panel_launch(B, grid, h->stream));
    if (rc) return rc;
  }
  return BTA_OK;
}

// Whether an FP64 factorisation runs as one launch (DALIA_B200_PANEL_PERSIST=1).
// Off by default: measured on B200 it is as fast as one launch per block
// column on the mixed b = 1200 / 600 batch and 7 % slower on the Poisson
// b = 2500 workload (a column launch starts with its dependency-free
// previous-column tasks; in one launch they wait for the previous column).
bool persist_enabled() {
  const char* e = std::getenv("DALIA_B200_PANEL_PERSIST");
  return e && std::strcmp(e, "1") == 0;
}

// A whole FP64 factorisation -- every block column of every instance, the
// previous column's Schur term inside the launch -- in one launch: the
// one-column queues of columns 0, 1, ... one after the other, each column's
// previous-column tasks waiting on the previous column's tiles, one chain CTA
// per instance running its columns in order.  Every column keeps its own
// tile inverses and flags.  BTA_ERR_ALLOC when that workspace cannot be had
// (the caller then launches column by column).
int run_factor_persist(bta_context* h, int count, const int64_t* n, const int64_t* b, const int64_t* a,
                       double* const* D, double* const* L, double* const* Ab, double* const* T) {
  std::vector<int> col_start(count + 1, 0), nn(count);
  std::vector<PanelInst> shapes(count);
  size_t cnt_ints = (size_t)count + 4, linv_bytes = 0;
  for (int k = 0; k < count; ++k) {
    nn[k] = (int)n[k];
    col_start[k + 1] = col_start[k] + nn[k];
    PanelInst S{};
    S.b = (int)b[k];
    S.a = (int)a[k];
    S.nq = (S.b + 63) / 64;
    S.Ttip = a[k] > 0 ? T[k] : nullptr;
    shapes[k] = S;
    for (int c = 0; c < nn[k]; ++c) {
      cnt_ints += (size_t)3 * panel_rows(S.b, S.a, c < nn[k] - 1) * S.nq;
      linv_bytes += align_up((size_t)S.nq * 4096 * sizeof(double));
    }
  }
  const int ncols = col_start[count];
  const size_t need = align_up((size_t)ncols * sizeof(PanelInst)) + align_up(cnt_ints * sizeof(int)) + linv_bytes +
                      4 * kAlign;
  int rc = ensure_ws(h, need);
  if (rc) return rc;
  cudaStream_t s = h->stream;
  Carve cv{h->ws};
  PanelInst* dcols = cv.take<PanelInst>(ncols);
  int* cnt = cv.take<int>(cnt_ints);
  int* tip_seq = cnt;
  int* batch_counter = cnt + count;
  size_t off = (size_t)count + 4;
  std::vector<PanelInst> cols(ncols);
  for (int k = 0; k < count; ++k) {
    const size_t bb = (size_t)b[k] * b[k], ab = (size_t)a[k] * b[k];
    const int B_ = (int)b[k], A_ = (int)a[k], nq = (B_ + 63) / 64;
    for (int c = 0; c < nn[k]; ++c) {
      const int g = col_start[k] + c;
      const bool hasL = c < nn[k] - 1;
      PanelInst& I = cols[g];
      I = PanelInst{};
      I.D = D[k] + c * bb;
      I.L = hasL ? L[k] + c * bb : nullptr;
      I.Ab = A_ > 0 ? Ab[k] + c * ab : nullptr;
      I.b = B_;
      I.a = A_;
      I.nq = nq;
      I.nrows_t = panel_rows(B_, A_, hasL);
      I.info = info_ptr(h);
      I.pivot_base = ((long long)k << 40) + (long long)c * B_;
      I.Lprev = c > 0 ? L[k] + (c - 1) * bb : nullptr;
      I.Abprev = (c > 0 && A_ > 0) ? Ab[k] + (c - 1) * ab : nullptr;
      I.Ttip = A_ > 0 ? T[k] : nullptr;
      I.Linv = cv.take<double>((size_t)nq * 4096);
      I.upd = cnt + off;
      I.flag = I.upd + (size_t)I.nrows_t * nq;
      I.prv = I.flag + (size_t)I.nrows_t * nq;
      off += (size_t)3 * I.nrows_t * nq;
      I.prev_flag = c > 0 ? cols[g - 1].flag : nullptr;
      I.tip_seq = I.Ttip != nullptr ? tip_seq + k : nullptr;
      I.col = c;
    }
  }
  if (cudaMemcpyAsync(dcols, cols.data(), (size_t)ncols * sizeof(PanelInst), cudaMemcpyHostToDevice, s) !=
          cudaSuccess ||
      cudaMemsetAsync(cnt, 0, cnt_ints * sizeof(int), s) != cudaSuccess)
    return BTA_ERR_CUDA;
  // launch shape and candidates as for one column: CTAs per SM x queue order x lookahead
  std::vector<long long> tkey{(long long)count};
  for (int k = 0; k < count; ++k) tkey.push_back(((long long)b[k] << 40) | ((long long)a[k] << 24) | n[k]);
  const int occ = panel_ctas_per_sm();
  if (occ < 0) return BTA_ERR_CUDA;
  static const int kLook[3] = {PREV_LOOKAHEAD, 1, 4};
  static const int kOrder[2] = {PANEL_ORDER_CHAIN_AHEAD, PANEL_ORDER_COLUMN};
  const int nocc = std::min(occ, 2);
  TuneLaunch tl("panel_all", tkey, nocc * 6, s);
  const int ch = tl.choice();
  const int grid = device_sm_count() * (occ - ch % nocc);
  const int order = kOrder[(ch / nocc) % 2], lookahead = kLook[ch / (2 * nocc)];
  std::vector<int> key{-1, lookahead, order};
  for (int k = 0; k < count; ++k) {
    key.push_back((int)b[k]);
    key.push_back((int)a[k]);
    key.push_back(nn[k]);
  }
  auto it = h->tasks.find(key);
  if (it == h->tasks.end()) {
    std::vector<int4> t;
    panel_tasks_persist(shapes, nn, col_start, t, lookahead, order);
    int4* d = nullptr;
    if (cudaMalloc(&d, t.size() * sizeof(int4)) != cudaSuccess) return BTA_ERR_ALLOC;
    if (cudaMemcpy(d, t.data(), t.size() * sizeof(int4), cudaMemcpyHostToDevice) != cudaSuccess) return BTA_ERR_CUDA;
    it = h->tasks.emplace(key, std::make_pair(d, (int)t.size())).first;
  }
  PanelBatch B;
  std::memset(&B, 0, sizeof(B));
  B.ninst = count;
  B.ntasks = it->second.second;
  B.tasks = it->second.first;
  B.counter = batch_counter;
  B.abort_flag = h->ctl;
  B.cols = dcols;
  for (int k = 0; k <= count; ++k) B.col_start[k] = col_start[k];
  return cuda_rc(panel_launch(B, grid, s));
}

size_t panel_ws_bytes(int b, int a) {
  const int nq = (b + 63) / 64;
  const int nr = panel_rows(b, a, true);
  return align_up((size_t)nq * 4096 * 8) + align_up(((size_t)3 * nr * nq + 4) * 4) + 2 * kAlign;
}

int reset_status(bta_context* h) {
  if (cudaMemsetAsync(h->ctl, 0, 8, h->stream) != cudaSuccess) return BTA_ERR_CUDA;
  if (cudaMemsetAsync(info_ptr(h), 0xff, 8, h->stream) != cudaSuccess) return BTA_ERR_CUDA;
  return BTA_OK;
}

int check_status(bta_context* h, int64_t* info) {
  unsigned long long hinfo = 0;
  int habort = 0;
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return BTA_ERR_CUDA;
  if (cudaMemcpy(&hinfo, info_ptr(h), sizeof(hinfo), cudaMemcpyDeviceToHost) != cudaSuccess) return BTA_ERR_CUDA;
  if (cudaMemcpy(&habort, h->ctl, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return BTA_ERR_CUDA;
  const bool fail = hinfo != ~0ULL;
  if (info) *info = fail ? (int64_t)hinfo : 0;
  if (habort) return BTA_ERR_TIMEOUT;
  return fail ? BTA_ERR_NOT_SPD : BTA_OK;
}

__global__ void scatter_coo_kernel(const int64_t* row, const int64_t* col, const double* val, int64_t nnz,
                                   int64_t n, int64_t b, int64_t a, int bt, double* D, double* L, double* Ab,
                                   double* T) {
  const int64_t nb = n * b;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = row[e], c = col[e];
    const double v = val[e];
    if (r < nb && c < nb) {
      const int64_t bi = r / b, bj = c / b;
      if (bi == bj) D[(bi * b + r % b) * b + c % b] = v;
      else if (bi == bj + 1) L[(bj * b + r % b) * b + c % b] = v;
    } else if (!bt && a > 0 && r >= nb && r < nb + a) {
      if (c < nb) Ab[((c / b) * a + (r - nb)) * b + c % b] = v;
      else if (c < nb + a) T[(r - nb) * a + (c - nb)] = v;
    }
  }
}

__global__ void gather_coo_kernel(const int64_t* row, const int64_t* col, int64_t nnz, int64_t n, int64_t b,
                                  int64_t a, int bt, const double* D, const double* L, const double* Ab,
                                  const double* T, double* out) {
  const int64_t nb = n * b;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = row[e], c = col[e];
    double v = 0.0;
    if (r < nb && c < nb) {
      const int64_t bi = r / b, bj = c / b;
      if (bi == bj) v = D[(bi * b + r % b) * b + c % b];
      else if (bi == bj + 1) v = L[(bj * b + r % b) * b + c % b];
    } else if (!bt && a > 0 && r >= nb && r < nb + a) {
      if (c < nb) v = Ab[((c / b) * a + (r - nb)) * b + c % b];
      else if (c < nb + a) v = T[(r - nb) * a + (c - nb)];
    }
    out[e] = v;
  }
}

}  // namespace

extern "C" {

const char* bta_error_string(int code) {
  switch (code) {
    case BTA_OK: return "success";
    case BTA_ERR_INVALID: return "invalid argument";
    case BTA_ERR_CUDA: return "CUDA error";
    case BTA_ERR_NOT_SPD: return "matrix is not positive definite";
    case BTA_ERR_TIMEOUT: return "device-side wait timed out";
    case BTA_ERR_ALLOC: return "scratch allocation failed";
    default: return "unknown error";
  }
}

int bta_create(bta_handle_t* handle) {
  if (!handle) return BTA_ERR_INVALID;
  auto* h = new bta_context();
  cudaGetDevice(&h->device);
  if (cudaMalloc(&h->ctl, 64) != cudaSuccess || cudaMalloc(&h->scal, 64) != cudaSuccess) {
    delete h;
    return BTA_ERR_ALLOC;
  }
  cudaMemset(h->ctl, 0, 64);
  cudaMemset(info_ptr(h), 0xff, 8);
  *handle = h;
  return BTA_OK;
}

int bta_destroy(bta_handle_t h) {
  DeviceGuard dg_(h);
  if (!h) return BTA_ERR_INVALID;
  cudaStreamSynchronize(h->stream);
  for (auto& kv : h->tasks) cudaFree(kv.second.first);
  if (h->ws) cudaFree(h->ws);
  if (h->ws2) cudaFree(h->ws2);
  cudaFree(h->ctl);
  cudaFree(h->scal);
  delete h;
  return BTA_OK;
}

int bta_set_stream(bta_handle_t h, void* stream) {
  if (!h) return BTA_ERR_INVALID;
  h->stream = reinterpret_cast<cudaStream_t>(stream);
  return BTA_OK;
}

size_t bta_workspace_bytes(bta_handle_t h) { return h ? h->ws_bytes : 0; }

int bta_pobtaf_batched(bta_handle_t h, int count, const int64_t* n, const int64_t* b, const int64_t* a,
                       double* const* D, double* const* L, double* const* Ab, double* const* T, int64_t* info) {
  return bta_pobtaf_batched_ex(h, count, n, b, a, D, L, Ab, T, info, BTA_PREC_FP64);
}

int bta_pobtaf_batched_ex(bta_handle_t h, int count, const int64_t* n, const int64_t* b, const int64_t* a,
                          double* const* D, double* const* L, double* const* Ab, double* const* T, int64_t* info,
                          int precision) {
  DeviceGuard dg_(h);
  if (!h || count < 1 || !n || !b || !a || !D) return BTA_ERR_INVALID;
  if (precision != BTA_PREC_FP64 && precision != BTA_PREC_TF32X3 && precision != BTA_PREC_I8SLICE)
    return BTA_ERR_INVALID;
  // FP64: the previous block column's Schur term runs inside the panel launch
  // (dependency-free tile tasks); otherwise it is one grouped GEMM per block
  // column in the requested arithmetic between the panel launches.
  const bool split = precision != BTA_PREC_FP64;
  int64_t maxn = 0;
  size_t need = 0, need_tip = 0;
  for (int k = 0; k < count; ++k) {
    if (n[k] < 1 || b[k] < 1 || a[k] < 0 || !D[k] || (n[k] > 1 && (!L || !L[k])) ||
        (a[k] > 0 && (!Ab || !T || !Ab[k] || !T[k])))
      return BTA_ERR_INVALID;
    if (b[k] > 65535 || a[k] > 4096) return BTA_ERR_INVALID;
    maxn = std::max(maxn, n[k]);
    need += panel_ws_bytes((int)b[k], (int)a[k]);
    if (a[k] > 0) need_tip += panel_ws_bytes((int)a[k], 0);
  }
  int rc = ensure_ws(h, std::max(need, need_tip) + 4 * kAlign);
  if (rc) return rc;
  cudaStream_t s = h->stream;
  if (info) {
    rc = reset_status(h);
    if (rc) return rc;
  }
  // FP64 with every arrow tip inside the panel, when enabled: the whole
  // factorisation in one launch, unless its workspace cannot be had
  bool persist = !split && count <= PANEL_MAXI && persist_enabled();
  for (int k = 0; k < count; ++k) persist = persist && a[k] <= 64;
  if (persist) {
    rc = run_factor_persist(h, count, n, b, a, D, L, Ab, T);
    if (rc == BTA_ERR_ALLOC) {
      persist = false;
      if ((rc = ensure_ws(h, std::max(need, need_tip) + 4 * kAlign))) return rc;
    } else if (rc) {
      return rc;
    }
  }
  // pivot index of instance k: k * 2^40 + global row (1-based).  Each launch
  // factors block column i and applies block column i-1's Schur update to it.
  for (int64_t i = 0; i < (persist ? 0 : maxn); ++i) {
    std::vector<PanelSpec> specs;
    std::vector<GemmProb> probs;
    for (int k = 0; k < count; ++k) {
      if (i >= n[k]) continue;
      const size_t bb = (size_t)b[k] * b[k], ab = (size_t)a[k] * b[k];
      const bool hasL = i < n[k] - 1;
      double* Di = D[k] + i * bb;
      double* Li = hasL ? L[k] + i * bb : nullptr;
      double* Abi = a[k] > 0 ? Ab[k] + i * ab : nullptr;
      PanelSpec sp{Di, Li, Abi, (int)b[k], (int)a[k], ((long long)k << 40) + (long long)(i * b[k])};
      if (i > 0 && !split) {
        sp.Lprev = L[k] + (i - 1) * bb;
        sp.Abprev = a[k] > 0 ? Ab[k] + (i - 1) * ab : nullptr;
      }
      sp.Ttip = a[k] > 0 ? T[k] : nullptr;
      specs.push_back(sp);
      if (a[k] > 64) {  // the in-panel tip task covers one arrow tile row
        const int B_ = (int)b[k], A_ = (int)a[k];
        GemmProb p = gemm_prob(T[k], A_, A_, A_, 1.0);
        gemm_add(p, Abi, B_, Abi, B_, B_, -1.0, 0);
        probs.push_back(p);
      }
    }
    Carve cv{h->ws};
    rc = run_panels(h, specs, cv);
    if (rc) return rc;
    if (!probs.empty() && gemm_launch(probs, s) != cudaSuccess) return BTA_ERR_CUDA;
    if (split) {
      // Schur term of block column i+1: D_{i+1} -= L_i L_i^T (lower half),
      // Ab_{i+1} -= Ab_i L_i^T
      std::vector<GemmProb> sch;
      for (int k = 0; k < count; ++k) {
        if (i >= n[k] - 1) continue;
        const size_t bb = (size_t)b[k] * b[k], ab = (size_t)a[k] * b[k];
        const int B_ = (int)b[k], A_ = (int)a[k];
        double* Li = L[k] + i * bb;
        GemmProb p = gemm_prob(D[k] + (i + 1) * bb, B_, B_, B_, 1.0, GC_LOWER);
        gemm_add(p, Li, B_, Li, B_, B_, -1.0, 0);
        sch.push_back(p);
        if (a[k] > 0) {
          GemmProb q = gemm_prob(Ab[k] + (i + 1) * ab, B_, A_, B_, 1.0);
          gemm_add(q, Ab[k] + i * ab, B_, Li, B_, B_, -1.0, 0);
          sch.push_back(q);
        }
      }
      if (!sch.empty()) {
        ProfRetarget rt(PROF_FACTOR_GEMM);
        if ((rc = run_gemm(h, sch, precision))) return rc;
      }
    }
  }
  std::vector<PanelSpec> tips;
  for (int k = 0; k < count; ++k)
    if (a[k] > 0) tips.push_back({T[k], nullptr, nullptr, (int)a[k], 0, ((long long)k << 40) + (long long)(n[k] * b[k])});
  if (!tips.empty()) {
    Carve cv{h->ws};
    rc = run_panels(h, tips, cv);
    if (rc) return rc;
  }
  if (info) return check_status(h, info);
  return cuda_rc(cudaGetLastError());
}

int bta_pobtaf(bta_handle_t h, int64_t n, int64_t b, int64_t a, double* D, double* L, double* Ab, double* T,
               int64_t* info) {
  if (!h || n < 1 || b < 1 || a < 0 || !D || (n > 1 && !L) || (a > 0 && (!Ab || !T))) return BTA_ERR_INVALID;
  return bta_pobtaf_batched(h, 1, &n, &b, &a, &D, &L, &Ab, &T, info);
}

// Whether a sweep of these instances is faster through block inverses made
// here chunk by chunk (b^3/3 flops per block on the tensor cores, then n
// bandwidth-bound steps of the persistent sweep) than through the tile-task
// sweep (n ceil(b/64) dependent 64-row links per instance, instances in
// parallel).  Model: ~10 us per link, ~2 TB/s for the tile sweep's reads;
// ~20 TF/s for the block inverses, ~15 us per persistent step.
bool sweep_by_inverses(int count, const int64_t* n, const int64_t* b, const int64_t* a) {
  double chain = 0, tile_bytes = 0, inv_flops = 0, inv_bytes = 0;
  int64_t maxn = 0;
  for (int k = 0; k < count; ++k) {
    const double bb = (double)b[k] * b[k];
    chain = std::max(chain, (double)n[k] * ((b[k] + 63) / 64) * 10e-6);
    tile_bytes += 8.0 * (1.5 * n[k] * bb + (double)n[k] * a[k] * b[k]);
    inv_flops += (double)n[k] * bb * b[k] / 3.0;
    inv_bytes += 8.0 * (2.0 * n[k] * bb);
    maxn = std::max(maxn, n[k]);
  }
  const double t_tile = std::max(chain, tile_bytes / 2e12);
  const double t_inv = inv_flops / 20e12 + inv_bytes / 5e12 + maxn * 15e-6;
  return t_inv < t_tile;
}

int bta_pobtas_batched(bta_handle_t h, int count, const int64_t* n, const int64_t* b, const int64_t* a,
                       const double* const* D, const double* const* L, const double* const* Ab,
                       const double* const* T, double* const* rhs, int trans) {
  DeviceGuard dg_(h);
  if (!h || count < 1 || count > SWEEP_MAXI || !n || !b || !a || !D || !rhs) return BTA_ERR_INVALID;
  if (trans != 0 && trans != 1) return BTA_ERR_INVALID;
  for (int k = 0; k < count; ++k) {
    if (n[k] < 1 || b[k] < 1 || a[k] < 0 || !D[k] || !rhs[k] || (n[k] > 1 && (!L || !L[k])) ||
        (a[k] > 0 && (!Ab || !T || !Ab[k] || !T[k])) || b[k] > INT32_MAX / 2)
      return BTA_ERR_INVALID;
  }
  if (sweep_by_inverses(count, n, b, a)) {
    // block inverses of C steps at a time (about 1 GiB for all instances),
    // each chunk then swept by one persistent launch
    std::vector<int> ni(count), bi(count), ai(count), vlo(count, 0);
    std::vector<const double*> Lk(count), Abk(count), Vk(count);
    std::vector<double*> tinv(count), vbuf(count);
    int64_t maxn = 0;
    double per_step = 0;
    size_t apart = 1;
    for (int k = 0; k < count; ++k) {
      ni[k] = (int)n[k];
      bi[k] = (int)b[k];
      ai[k] = (int)a[k];
      Lk[k] = n[k] > 1 ? L[k] : nullptr;
      Abk[k] = a[k] > 0 ? Ab[k] : nullptr;
      maxn = std::max(maxn, n[k]);
      per_step += 8.0 * b[k] * b[k];
      apart = std::max<size_t>(apart, (size_t)n[k] * a[k]);
    }
    const int64_t C = std::max<int64_t>(1, std::min<int64_t>(maxn, (int64_t)((double)(1 << 30) / per_step)));
    size_t need = 4 * kAlign + align_up((sweep_inv_work_total(count, ni.data(), bi.data(), ai.data()) + apart) * 8);
    for (int k = 0; k < count; ++k) {
      const size_t nq = (b[k] + 63) / 64;
      need += align_up(C * nq * 4096 * 8) + align_up(C * (size_t)b[k] * b[k] * 8);
    }
    int rc = ensure_ws(h, need);
    if (rc) return rc;
    cudaStream_t s = h->stream;
    Carve cv{h->ws};
    double* work = cv.take<double>(sweep_inv_work_total(count, ni.data(), bi.data(), ai.data()) + apart);
    for (int k = 0; k < count; ++k) {
      const size_t nq = (b[k] + 63) / 64;
      tinv[k] = cv.take<double>(C * nq * 4096);
      vbuf[k] = cv.take<double>(C * (size_t)b[k] * b[k]);
      Vk[k] = vbuf[k];
    }
    if (trans == 1)
      for (int k = 0; k < count; ++k)
        if (a[k] > 0 && arrow_backward(T[k], rhs[k], ni[k], bi[k], ai[k], s)) return BTA_ERR_CUDA;
    for (int64_t s0 = 0; s0 < maxn; s0 += C) {
      const int64_t s1 = std::min(maxn, s0 + C);
      for (int k = 0; k < count; ++k) {
        const int64_t e = std::min(s1, n[k]), cnt = e - s0;
        if (cnt <= 0) continue;
        const int64_t lo = trans == 0 ? s0 : n[k] - e;
        const size_t bb = (size_t)b[k] * b[k];
        if (diag_tile_inverses(D[k] + lo * bb, (int)cnt, bi[k], tinv[k], s)) return BTA_ERR_CUDA;
        if (block_trtri(D[k] + lo * bb, tinv[k], 0, (int)cnt, bi[k], vbuf[k], s)) return BTA_ERR_CUDA;
        vlo[k] = (int)lo;
      }
      if (sweep_inv_steps(count, ni.data(), bi.data(), ai.data(), Lk.data(), Abk.data(), Vk.data(), vlo.data(), rhs,
                          trans, (int)s0, (int)s1, work, h->ctl, s))
        return BTA_ERR_CUDA;
    }
    if (trans == 0)
      for (int k = 0; k < count; ++k) {
        double* part = work + sweep_inv_work_total(count, ni.data(), bi.data(), ai.data());
        if (a[k] > 0 && arrow_forward(Ab[k], T[k], rhs[k], ni[k], bi[k], ai[k], part, s)) return BTA_ERR_CUDA;
      }
    return cuda_rc(cudaGetLastError());
  }
  size_t need = 4 * kAlign;
  for (int k = 0; k < count; ++k) {
    const size_t nq = (b[k] + 63) / 64;
    need += align_up(n[k] * nq * 4096 * 8) + align_up((n[k] * nq + 4) * 4) + align_up((n[k] * a[k] + 1) * 8) +
            3 * kAlign;
  }
  int rc = ensure_ws(h, need);
  if (rc) return rc;
  cudaStream_t s = h->stream;
  Carve cv{h->ws};
  int* counter = cv.take<int>(4);
  if (cudaMemsetAsync(counter, 0, 4 * sizeof(int), s) != cudaSuccess) return BTA_ERR_CUDA;
  SweepBatch B;
  std::memset(&B, 0, sizeof(B));
  B.count = count;
  B.counter = counter;
  for (int k = 0; k < count; ++k) {
    const int nq = (int)((b[k] + 63) / 64);
    double* tinv = cv.take<double>((size_t)n[k] * nq * 4096);
    int* flags = cv.take<int>((size_t)n[k] * nq + 4);
    if (cudaMemsetAsync(flags, 0, ((size_t)n[k] * nq + 4) * sizeof(int), s) != cudaSuccess) return BTA_ERR_CUDA;
    if (diag_tile_inverses(D[k], (int)n[k], (int)b[k], tinv, s)) return BTA_ERR_CUDA;
    SweepArgs& A = B.inst[k];
    A.D = D[k];
    A.L = L ? L[k] : nullptr;
    A.Ab = Ab ? Ab[k] : nullptr;
    A.Linv = tinv;
    A.x = rhs[k];
    A.flags = flags;
    A.counter = counter;
    A.abort_flag = h->ctl;
    A.n = (int)n[k];
    A.b = (int)b[k];
    A.a = (int)a[k];
    A.nq = nq;
    A.trans = trans;
    if (trans == 1 && arrow_backward(T[k], rhs[k], (int)n[k], (int)b[k], (int)a[k], s)) return BTA_ERR_CUDA;
  }
  if (sweep_launch_batched(B, s)) return BTA_ERR_CUDA;
  if (trans == 0)
    for (int k = 0; k < count; ++k) {
      double* part = cv.take<double>((size_t)n[k] * a[k] + 1);
      if (arrow_forward(Ab ? Ab[k] : nullptr, T ? T[k] : nullptr, rhs[k], (int)n[k], (int)b[k], (int)a[k], part,
                        s))
        return BTA_ERR_CUDA;
    }
  return cuda_rc(cudaGetLastError());
}

int bta_pobtas(bta_handle_t h, int64_t n, int64_t b, int64_t a, const double* D, const double* L,
               const double* Ab, const double* T, double* rhs, int trans) {
  if (!h || n < 1 || b < 1 || a < 0 || !D || !rhs || (n > 1 && !L) || (a > 0 && (!Ab || !T))) return BTA_ERR_INVALID;
  return bta_pobtas_batched(h, 1, &n, &b, &a, &D, &L, &Ab, &T, &rhs, trans);
}

int bta_pobtasi_batched(bta_handle_t h, int count, const int64_t* n, const int64_t* b, const int64_t* a,
                        double* const* D, double* const* L, double* const* Ab, double* const* T) {
  return bta_pobtasi_batched_ex(h, count, n, b, a, D, L, Ab, T, BTA_PREC_FP64);
}

int bta_pobtasi_batched_ex(bta_handle_t h, int count, const int64_t* n, const int64_t* b, const int64_t* a,
                           double* const* D, double* const* L, double* const* Ab, double* const* T,
                           int precision) {
  return bta_pobtasi_batched_v(h, count, n, b, a, D, L, Ab, T, nullptr, precision);
}

// Blocks whose inverses one instance computes at a time when the caller does
// not supply them: the inverses are made chunk by chunk as the backward
// recurrence reaches them, so the workspace holds C blocks (at most 2 GiB)
// instead of n.
inline int64_t inverse_chunk(int64_t n, int64_t b) {
  const int64_t per = b * b * 8;
  return std::max<int64_t>(1, std::min<int64_t>(n, (int64_t(2048) << 20) / per));
}

int bta_pobtasi_batched_v(bta_handle_t h, int count, const int64_t* n, const int64_t* b, const int64_t* a,
                          double* const* D, double* const* L, double* const* Ab, double* const* T,
                          const double* const* V, int precision) {
  DeviceGuard dg_(h);
  if (!h || count < 1 || !n || !b || !a || !D) return BTA_ERR_INVALID;
  if (precision != BTA_PREC_FP64 && precision != BTA_PREC_TF32X3 && precision != BTA_PREC_I8SLICE)
    return BTA_ERR_INVALID;
  // the block products go to the grouped GEMM of the requested arithmetic
  auto launch = [&](const std::vector<GemmProb>& pr) { return run_gemm(h, pr, precision); };
  size_t need = 8 * kAlign;
  int64_t maxn = 0;
  std::vector<int64_t> chunk(count, 0);  // > 0: inverses computed here, chunk blocks at a time
  for (int k = 0; k < count; ++k) {
    if (n[k] < 1 || b[k] < 1 || a[k] < 0 || !D[k] || (n[k] > 1 && (!L || !L[k])) ||
        (a[k] > 0 && (!Ab || !T || !Ab[k] || !T[k])))
      return BTA_ERR_INVALID;
    const size_t nq = (b[k] + 63) / 64, nqa = (a[k] + 63) / 64;
    const size_t bb = (size_t)b[k] * b[k], ab = (size_t)a[k] * b[k];
    if (!V || !V[k]) chunk[k] = inverse_chunk(n[k], b[k]);
    // block inverses (tile inverses + full inverses of a chunk) only when not supplied
    need += (chunk[k] ? align_up(chunk[k] * nq * 4096 * 8) + align_up(chunk[k] * bb * 8) : 0) + align_up(bb * 8) +
            align_up(ab * 8 + 8) + align_up(nqa * 4096 * 8 + 8) + align_up((size_t)a[k] * a[k] * 8 + 8) + 6 * kAlign;
    maxn = std::max(maxn, n[k]);
  }
  int rc = ensure_ws(h, need);
  if (rc) return rc;
  cudaStream_t s = h->stream;
  Carve cv{h->ws};
  struct W {
    double *tinv, *Linv, *G, *Ga, *tinv_t, *Wt;
    int64_t lo;  // first block of the chunk held in Linv (own inverses)
  };
  std::vector<W> w(count);
  for (int k = 0; k < count; ++k) {
    const size_t nq = (b[k] + 63) / 64, nqa = (a[k] + 63) / 64;
    const size_t bb = (size_t)b[k] * b[k], ab = (size_t)a[k] * b[k];
    w[k].tinv = chunk[k] ? cv.take<double>(chunk[k] * nq * 4096) : nullptr;
    w[k].Linv = chunk[k] ? cv.take<double>(chunk[k] * bb) : const_cast<double*>(V[k]);
    w[k].lo = chunk[k] ? n[k] : 0;
    w[k].G = cv.take<double>(bb);
    w[k].Ga = cv.take<double>(ab + 1);
    w[k].tinv_t = cv.take<double>(nqa * 4096 + 1);
    w[k].Wt = cv.take<double>((size_t)a[k] * a[k] + 1);
  }
  std::vector<GemmProb> ptip;
  for (int k = 0; k < count; ++k) {
    if (a[k] > 0) {
      const int A_ = (int)a[k];
      if (diag_tile_inverses(T[k], 1, A_, w[k].tinv_t, s)) return BTA_ERR_CUDA;
      if (block_trtri(T[k], w[k].tinv_t, 0, 1, A_, w[k].Wt, s)) return BTA_ERR_CUDA;
      GemmProb p = gemm_prob(T[k], A_, A_, A_, 0.0, GC_LOWER | GC_MIRROR);
      gemm_add(p, w[k].Wt, A_, w[k].Wt, A_, A_, 1.0, GF_A_T | GF_B_KN | GF_K_GE_M | GF_K_GE_N);
      ptip.push_back(p);
    }
  }
  if (!ptip.empty() && gemm_launch(ptip, s)) return BTA_ERR_CUDA;
  // step st processes block j = n_k - 1 - st of every instance
  for (int64_t st = 0; st < maxn; ++st) {
    std::vector<GemmProb> pa, pb, pc;
    for (int k = 0; k < count; ++k) {
      const int64_t i = n[k] - 1 - st;
      if (i < 0) continue;
      const size_t bb = (size_t)b[k] * b[k], ab = (size_t)a[k] * b[k];
      if (chunk[k] && i < w[k].lo) {
        // inverses of blocks [lo, i] (the factor blocks there are not yet
        // overwritten: the recurrence runs from the last block down)
        const int64_t lo = std::max<int64_t>(0, i + 1 - chunk[k]), cnt = i + 1 - lo;
        if (diag_tile_inverses(D[k] + lo * bb, (int)cnt, (int)b[k], w[k].tinv, s)) return BTA_ERR_CUDA;
        if (block_trtri(D[k] + lo * bb, w[k].tinv, 0, (int)cnt, (int)b[k], w[k].Linv, s)) return BTA_ERR_CUDA;
        w[k].lo = lo;
      }
      const bool hasL = i < n[k] - 1;
      double* Li = hasL ? L[k] + i * bb : nullptr;
      double* Abi = a[k] > 0 ? Ab[k] + i * ab : nullptr;
      const double* Vi = w[k].Linv + (i - w[k].lo) * bb;
      const int B_ = (int)b[k], A_ = (int)a[k];
      if (hasL) {
        GemmProb p = gemm_prob(w[k].G, B_, B_, B_, 0.0);
        gemm_add(p, Li, B_, Vi, B_, B_, 1.0, GF_B_KN | GF_K_GE_N);
        pa.push_back(p);
        GemmProb q = gemm_prob(Li, B_, B_, B_, 0.0);
        gemm_add(q, D[k] + (i + 1) * bb, B_, w[k].G, B_, B_, -1.0, GF_B_KN);
        if (a[k] > 0) gemm_add(q, Ab[k] + (i + 1) * ab, B_, w[k].Ga, B_, A_, -1.0, GF_A_T | GF_B_KN);
        pb.push_back(q);
      }
      if (a[k] > 0) {
        GemmProb p = gemm_prob(w[k].Ga, B_, A_, B_, 0.0);
        gemm_add(p, Abi, B_, Vi, B_, B_, 1.0, GF_B_KN | GF_K_GE_N);
        pa.push_back(p);
        GemmProb q = gemm_prob(Abi, B_, A_, B_, 0.0);
        if (hasL) gemm_add(q, Ab[k] + (i + 1) * ab, B_, w[k].G, B_, B_, -1.0, GF_B_KN);
        gemm_add(q, T[k], A_, w[k].Ga, B_, A_, -1.0, GF_B_KN);
        pb.push_back(q);
      }
      // Sigma_ii replaces the factor block D_i in place: nothing in this
      // step reads D_i (its inverse V_i is held apart), later steps read
      // only blocks above it
      GemmProb r = gemm_prob(D[k] + i * bb, B_, B_, B_, 0.0, GC_LOWER | GC_MIRROR);
      gemm_add(r, Vi, B_, Vi, B_, B_, 1.0, GF_A_T | GF_B_KN | GF_K_GE_M | GF_K_GE_N);
      if (hasL) gemm_add(r, w[k].G, B_, Li, B_, B_, -1.0, GF_A_T | GF_B_KN);
      if (a[k] > 0) gemm_add(r, w[k].Ga, B_, Abi, B_, A_, -1.0, GF_A_T | GF_B_KN);
      pc.push_back(r);
    }
    if (!pa.empty() && (rc = launch(pa))) return rc;
    if (!pb.empty() && (rc = launch(pb))) return rc;
    if (!pc.empty() && (rc = launch(pc))) return rc;
  }
  return cuda_rc(cudaGetLastError());
}

int bta_pobtasi(bta_handle_t h, int64_t n, int64_t b, int64_t a, double* D, double* L, double* Ab, double* T) {
  if (!h || n < 1 || b < 1 || a < 0 || !D || (n > 1 && !L) || (a > 0 && (!Ab || !T))) return BTA_ERR_INVALID;
  return bta_pobtasi_batched(h, 1, &n, &b, &a, &D, &L, &Ab, &T);
}

int bta_panel_task_list_all(int count, const int* b, const int* a, const int* flags, const int* n, int lookahead,
                            int order, int* out, int cap, int* n_out) {
  if (count < 1 || count > PANEL_MAXI || !b || !a || !flags || !n || !n_out || cap < 0 || (cap > 0 && !out) ||
      lookahead < 1 || (order != PANEL_ORDER_COLUMN && order != PANEL_ORDER_CHAIN_AHEAD))
    return BTA_ERR_INVALID;
  static double present;  // stands for the tip: only null / non-null matters here
  std::vector<PanelInst> shapes(count);
  std::vector<int> nn(count), col_start(count + 1, 0);
  for (int k = 0; k < count; ++k) {
    if (b[k] < 1 || a[k] < 0 || a[k] > 64 || n[k] < 1) return BTA_ERR_INVALID;
    PanelInst S{};
    S.b = b[k];
    S.a = a[k];
    S.nq = (b[k] + 63) / 64;
    S.Ttip = ((flags[k] & 8) && a[k] > 0) ? &present : nullptr;
    shapes[k] = S;
    nn[k] = n[k];
    col_start[k + 1] = col_start[k] + n[k];
  }
  std::vector<int4> t;
  panel_tasks_persist(shapes, nn, col_start, t, lookahead, order);
  *n_out = (int)t.size();
  if ((int)t.size() > cap) return BTA_ERR_INVALID;
  for (size_t i = 0; i < t.size(); ++i) {
    out[4 * i] = t[i].x;
    out[4 * i + 1] = t[i].y;
    out[4 * i + 2] = t[i].z;
    out[4 * i + 3] = t[i].w;
  }
  return BTA_OK;
}

int bta_panel_task_list(int count, const int* b, const int* a, const int* flags, int* out, int cap, int* n_out) {
  return bta_panel_task_list_ex(count, b, a, flags, PREV_LOOKAHEAD, PANEL_ORDER_COLUMN, out, cap, n_out);
}

int bta_panel_task_list_ex(int count, const int* b, const int* a, const int* flags, int lookahead, int order,
                           int* out, int cap, int* n_out) {
  if (count < 1 || count > PANEL_MAXI || !b || !a || !flags || !n_out || cap < 0 || (cap > 0 && !out) ||
      lookahead < 1 || (order != PANEL_ORDER_COLUMN && order != PANEL_ORDER_CHAIN_AHEAD))
    return BTA_ERR_INVALID;
  static double present;  // stands for a matrix block: only null / non-null matters here
  std::vector<PanelInst> insts;
  for (int k = 0; k < count; ++k) {
    if (b[k] < 1 || a[k] < 0) return BTA_ERR_INVALID;
    const bool hasL = flags[k] & 1;
    PanelInst I{};
    I.b = b[k];
    I.a = a[k];
    I.nq = (b[k] + 63) / 64;
    I.L = hasL ? &present : nullptr;
    I.Ab = a[k] > 0 ? &present : nullptr;
    I.Lprev = (flags[k] & 2) ? &present : nullptr;
    I.Abprev = ((flags[k] & 4) && a[k] > 0) ? &present : nullptr;
    I.Ttip = ((flags[k] & 8) && a[k] > 0 && a[k] <= 64) ? &present : nullptr;
    I.nrows_t = panel_rows(b[k], a[k], hasL);
    insts.push_back(I);
  }
  std::vector<int4> t;
  panel_tasks(insts, t, lookahead, order);
  *n_out = (int)t.size();
  if ((int)t.size() > cap) return BTA_ERR_INVALID;
  for (size_t i = 0; i < t.size(); ++i) {
    out[4 * i] = t[i].x;
    out[4 * i + 1] = t[i].y;
    out[4 * i + 2] = t[i].z;
    out[4 * i + 3] = t[i].w;
  }
  return BTA_OK;
}

int bta_block_inverses(bta_handle_t h, int count, const int64_t* n, const int64_t* b, const double* const* D,
                       double* const* V) {
  DeviceGuard dg_(h);
  if (!h || count < 1 || !n || !b || !D || !V) return BTA_ERR_INVALID;
  size_t need = kAlign;
  for (int k = 0; k < count; ++k) {
    if (n[k] < 1 || b[k] < 1 || !D[k] || !V[k]) return BTA_ERR_INVALID;
    need = std::max(need, align_up((size_t)n[k] * ((b[k] + 63) / 64) * 4096 * 8));
  }
  int rc = ensure_ws(h, need);
  if (rc) return rc;
  double* tinv = reinterpret_cast<double*>(h->ws);
  for (int k = 0; k < count; ++k) {
    if (diag_tile_inverses(D[k], (int)n[k], (int)b[k], tinv, h->stream)) return BTA_ERR_CUDA;
    if (block_trtri(D[k], tinv, 0, (int)n[k], (int)b[k], V[k], h->stream)) return BTA_ERR_CUDA;
  }
  return cuda_rc(cudaGetLastError());
}

int bta_pobtas_inv_batched(bta_handle_t h, int count, const int64_t* n, const int64_t* b, const int64_t* a,
                           const double* const* L, const double* const* Ab, const double* const* T,
                           const double* const* V, double* const* rhs, int trans) {
  DeviceGuard dg_(h);
  if (!h || count < 1 || !n || !b || !a || !V || !rhs || (trans != 0 && trans != 1)) return BTA_ERR_INVALID;
  std::vector<int> ni(count), bi(count), ai(count);
  std::vector<const double*> Lk(count), Abk(count), Tk(count);
  size_t need = kAlign, apart = 1;
  for (int k = 0; k < count; ++k) {
    if (n[k] < 1 || b[k] < 1 || a[k] < 0 || !V[k] || !rhs[k] || (n[k] > 1 && (!L || !L[k])) ||
        (a[k] > 0 && (!Ab || !T || !Ab[k] || !T[k])) || b[k] > INT32_MAX / 2)
      return BTA_ERR_INVALID;
    ni[k] = (int)n[k];
    bi[k] = (int)b[k];
    ai[k] = (int)a[k];
    Lk[k] = n[k] > 1 ? L[k] : nullptr;
    Abk[k] = a[k] > 0 ? Ab[k] : nullptr;
    Tk[k] = a[k] > 0 ? T[k] : nullptr;
    apart = std::max<size_t>(apart, (size_t)n[k] * a[k]);
  }
  need += (sweep_inv_work_total(count, ni.data(), bi.data(), ai.data()) + apart) * sizeof(double);
  int rc = ensure_ws(h, align_up(need));
  if (rc) return rc;
  return sweep_inv_batched(count, ni.data(), bi.data(), ai.data(), Lk.data(), Abk.data(), Tk.data(), V, rhs, trans,
                           reinterpret_cast<double*>(h->ws), h->ctl, h->stream)
             ? BTA_ERR_CUDA
             : BTA_OK;
}

int bta_gemm(bta_handle_t h, int precision, int64_t M, int64_t N, int64_t K, double alpha, const double* A,
             int64_t lda, int a_trans, const double* B, int64_t ldb, int b_kn, double beta, double* C, int64_t ldc,
             int lower_only, int mirror) {
  DeviceGuard dg_(h);
  if (!h || M < 0 || N < 0 || K < 0 || M > INT32_MAX || N > INT32_MAX || K > INT32_MAX) return BTA_ERR_INVALID;
  if (precision != BTA_PREC_FP64 && precision != BTA_PREC_TF32X3 && precision != BTA_PREC_I8SLICE)
    return BTA_ERR_INVALID;
  if (M == 0 || N == 0) return BTA_OK;
  if (!C || ldc < N || (lower_only && M != N) || (mirror && !lower_only)) return BTA_ERR_INVALID;
  if (K > 0 && (!A || !B || lda < (a_trans ? M : K) || ldb < (b_kn ? N : K))) return BTA_ERR_INVALID;
  GemmProb p = gemm_prob(C, (int)ldc, (int)M, (int)N, beta, (lower_only ? GC_LOWER : 0) | (mirror ? GC_MIRROR : 0));
  if (K > 0) gemm_add(p, A, (int)lda, B, (int)ldb, (int)K, alpha, (a_trans ? GF_A_T : 0) | (b_kn ? GF_B_KN : 0));
  std::vector<GemmProb> v{p};
  return run_gemm(h, v, precision);
}

int bta_logdet(bta_handle_t h, int64_t n, int64_t b, int64_t a, const double* D, const double* T, int include_tip,
               double* out_device, double* out_host) {
  DeviceGuard dg_(h);
  if (!h || n < 1 || b < 1 || a < 0 || !D || (include_tip && a > 0 && !T)) return BTA_ERR_INVALID;
  int rc = ensure_ws(h, align_up((size_t)(n + 2) * 8));
  if (rc) return rc;
  double* part = reinterpret_cast<double*>(h->ws);
  double* out = out_device ? out_device : h->scal;
  const int at = include_tip ? (int)a : 0;
  if (logdet_launch(D, (int)n, (int)b, T, at, part, out, h->stream)) return BTA_ERR_CUDA;
  if (out_host) {
    if (cudaMemcpyAsync(out_host, out, sizeof(double), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess)
      return BTA_ERR_CUDA;
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return BTA_ERR_CUDA;
  }
  return cuda_rc(cudaGetLastError());
}

int bta_get_status(bta_handle_t h, int64_t* info) {
  DeviceGuard dg_(h);
  if (!h) return BTA_ERR_INVALID;
  return check_status(h, info);
}

int bta_reset_status(bta_handle_t h) {
  DeviceGuard dg_(h);
  if (!h) return BTA_ERR_INVALID;
  return reset_status(h);
}

int bta_gather_coo(bta_handle_t h, int64_t n, int64_t b, int64_t a, const int64_t* row, const int64_t* col,
                   int64_t nnz, int sparsity_bt, const double* D, const double* L, const double* Ab, const double* T,
                   double* out) {
  DeviceGuard dg_(h);
  if (!h || n < 1 || b < 1 || a < 0 || !D || (n > 1 && !L) || nnz < 0 || (nnz > 0 && !out)) return BTA_ERR_INVALID;
  if (!sparsity_bt && a > 0 && (!Ab || !T)) return BTA_ERR_INVALID;
  if (nnz > 0) {
    const int grid = (int)std::min<int64_t>((nnz + 255) / 256, 148 * 32);
    {
      bta::ProfScope _ps(bta::PROF_OTHER, h->stream);
      gather_coo_kernel<<<grid, 256, 0, h->stream>>>(row, col, nnz, n, b, a, sparsity_bt, D, L, Ab, T, out);
    }
  }
  return cuda_rc(cudaGetLastError());
}

int bta_scatter_coo(bta_handle_t h, int64_t n, int64_t b, int64_t a, const int64_t* row, const int64_t* col,
                    const double* val, int64_t nnz, int sparsity_bt, double* D, double* L, double* Ab, double* T) {
  DeviceGuard dg_(h);
  if (!h || n < 1 || b < 1 || a < 0 || !D || (n > 1 && !L) || nnz < 0) return BTA_ERR_INVALID;
  if (!sparsity_bt && a > 0 && (!Ab || !T)) return BTA_ERR_INVALID;
  cudaStream_t s = h->stream;
  const size_t bb = (size_t)b * b;
  if (cudaMemsetAsync(D, 0, n * bb * 8, s)) return BTA_ERR_CUDA;
  if (n > 1 && cudaMemsetAsync(L, 0, (n - 1) * bb * 8, s)) return BTA_ERR_CUDA;
  if (!sparsity_bt && a > 0) {
    if (cudaMemsetAsync(Ab, 0, (size_t)n * a * b * 8, s)) return BTA_ERR_CUDA;
    if (cudaMemsetAsync(T, 0, (size_t)a * a * 8, s)) return BTA_ERR_CUDA;
  }
  if (nnz > 0) {
    const int grid = (int)std::min<int64_t>((nnz + 255) / 256, 148 * 32);
    {
      bta::ProfScope _ps(bta::PROF_OTHER, s);
      scatter_coo_kernel<<<grid, 256, 0, s>>>(row, col, val, nnz, n, b, a, sparsity_bt, D, L, Ab, T);
    }
  }
  return cuda_rc(cudaGetLastError());
}

}  // extern "C"
