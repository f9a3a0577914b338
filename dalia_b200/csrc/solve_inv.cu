// Triangular sweeps with precomputed inverses of the diagonal factor blocks.
//
// With V_i = L_ii^-1 available (the selected inversion needs them anyway),
// a sweep over n blocks is n dependent steps of two dense matrix-vector
// products each,
//   forward   y_i = V_i (b_i - L_{i,i-1} y_{i-1}),
//   backward  x_i = V_i^T (y_i - L_{i+1,i}^T x_{i+1} - Ab_i^T x_a),
// instead of ceil(b/64) dependent tile solves per block: every step reads
// its two b x b blocks once, spread over all SMs (HBM bound), and the
// dependency chain is n steps long.  The arrowhead tip is solved by the
// tile sweep's arrow kernels.  Instances of a batch advance together, one
// launch per step and kind of product.
#include <algorithm>
#include <cstring>
#include <vector>

#include "bta_internal.cuh"
#include "common.cuh"
#include "prof.cuh"

namespace bta {
namespace {

constexpr int GV_MAXJ = 64;

// out[r] = beta c[r] + alpha sum_k M[r][k] x[k] for r < rows, k < cols
// (k <= r when lower); M == nullptr gives out = beta c.  out may be c, not x.
struct RowJob {
  const double* M;
  const double* x;
  const double* c;
  double* out;
  double alpha, beta;
  int rows, cols, ld, lower, row_start;
};

struct RowBatch {
  int count, rows;
  RowJob job[GV_MAXJ];
};

// One warp per output row; lanes read the row in 16-byte pieces.
__global__ void __launch_bounds__(256) gemv_rows_kernel(const __grid_constant__ RowBatch B) {
  const int lane = threadIdx.x & 31;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= B.rows) return;
  int j = 0;
  while (j + 1 < B.count && w >= B.job[j + 1].row_start) ++j;
  const RowJob& J = B.job[j];
  const int r = w - J.row_start;
  double s = 0.0;
  if (J.M != nullptr) {
    const int kend = J.lower ? min(J.cols, r + 1) : J.cols;
    const double* row = J.M + (size_t)r * J.ld;
    const bool vec = ((J.ld & 1) == 0) && ((reinterpret_cast<uintptr_t>(J.M) & 15) == 0) &&
                     ((reinterpret_cast<uintptr_t>(J.x) & 15) == 0);
    if (vec) {
      const int kp = kend >> 1;
      for (int q = lane; q < kp; q += 32) {
        const double2 m = *reinterpret_cast<const double2*>(row + 2 * q);
        const double2 xv = *reinterpret_cast<const double2*>(J.x + 2 * q);
        s = fma(m.x, xv.x, s);
        s = fma(m.y, xv.y, s);
      }
      if ((kend & 1) && lane == 0) s = fma(row[kend - 1], J.x[kend - 1], s);
    } else {
      for (int k = lane; k < kend; k += 32) s = fma(row[k], J.x[k], s);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  }
  if (lane == 0) J.out[r] = (J.beta != 0.0 ? J.beta * J.c[r] : 0.0) + J.alpha * s;
}

// Transposed product in two phases: partial[chunk][c] = sum over the chunk's
// rows of M[r][c] x[r] (r >= c when upper), then
// out[c] = beta y[c] + alpha (sum_chunk partial + sum_{q < a} Ab[q][c] xa[q]).
constexpr int CT_COLS = 128;
constexpr int CT_ROWS = 64;

struct ColJob {
  const double* M;   // rows x cols, or nullptr
  const double* x;   // rows
  const double* y;   // cols (read when beta != 0)
  const double* Ab;  // a x cols (row stride cols), or nullptr
  const double* xa;  // a
  double* out;       // cols; may be y, not x
  double* part;      // nchunk x cols
  double alpha, beta;
  int rows, cols, ld, upper, a, nchunk, cta_start, col_start;
};

struct ColBatch {
  int count, ctas, cols;
  ColJob job[GV_MAXJ];
};

__global__ void __launch_bounds__(CT_COLS) gemv_cols_part_kernel(const __grid_constant__ ColBatch B) {
  const int bid = blockIdx.x;
  int j = 0;
  while (j + 1 < B.count && bid >= B.job[j + 1].cta_start) ++j;
  const ColJob& J = B.job[j];
  if (J.M == nullptr || J.nchunk == 0) return;
  const int local = bid - J.cta_start;
  const int cb = local / J.nchunk, ch = local - cb * J.nchunk;
  const int c = cb * CT_COLS + threadIdx.x;
  const int r0 = ch * CT_ROWS, r1 = min(J.rows, r0 + CT_ROWS);
  double s = 0.0;
  if (c < J.cols) {
    const int rs = J.upper ? max(r0, c) : r0;
    for (int r = rs; r < r1; ++r) s = fma(J.M[(size_t)r * J.ld + c], J.x[r], s);
    J.part[(size_t)ch * J.cols + c] = s;
  }
}

__global__ void __launch_bounds__(256) gemv_cols_final_kernel(const __grid_constant__ ColBatch B) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= B.cols) return;
  int j = 0;
  while (j + 1 < B.count && t >= B.job[j + 1].col_start) ++j;
  const ColJob& J = B.job[j];
  const int c = t - J.col_start;
  double s = 0.0;
  if (J.M != nullptr)
    for (int ch = 0; ch < J.nchunk; ++ch) s += J.part[(size_t)ch * J.cols + c];
  if (J.Ab != nullptr)
    for (int q = 0; q < J.a; ++q) s = fma(J.Ab[(size_t)q * J.cols + c], J.xa[q], s);
  J.out[c] = (J.beta != 0.0 ? J.beta * J.y[c] : 0.0) + J.alpha * s;
}

int launch_rows(std::vector<RowJob>& jobs, cudaStream_t s) {
  size_t i = 0;
  while (i < jobs.size()) {
    RowBatch B;
    std::memset(&B, 0, sizeof(B));
    for (; i < jobs.size() && B.count < GV_MAXJ; ++i) {
      jobs[i].row_start = B.rows;
      B.job[B.count++] = jobs[i];
      B.rows += jobs[i].rows;
    }
    if (B.rows == 0) continue;
    bta::ProfScope _ps(bta::PROF_SWEEP, s);
    gemv_rows_kernel<<<(B.rows * 32 + 255) / 256, 256, 0, s>>>(B);
    if (cudaGetLastError() != cudaSuccess) return 1;
  }
  return 0;
}

int launch_cols(std::vector<ColJob>& jobs, cudaStream_t s) {
  size_t i = 0;
  while (i < jobs.size()) {
    ColBatch B;
    std::memset(&B, 0, sizeof(B));
    for (; i < jobs.size() && B.count < GV_MAXJ; ++i) {
      ColJob& J = jobs[i];
      J.nchunk = J.M != nullptr ? (J.rows + CT_ROWS - 1) / CT_ROWS : 0;
      J.cta_start = B.ctas;
      J.col_start = B.cols;
      B.job[B.count++] = J;
      B.ctas += J.nchunk * ((J.cols + CT_COLS - 1) / CT_COLS);
      B.cols += J.cols;
    }
    if (B.cols == 0) continue;
    if (B.ctas > 0) {
      bta::ProfScope _ps(bta::PROF_SWEEP, s);
      gemv_cols_part_kernel<<<B.ctas, CT_COLS, 0, s>>>(B);
    }
    {
      bta::ProfScope _ps(bta::PROF_SWEEP, s);
      gemv_cols_final_kernel<<<(B.cols + 255) / 256, 256, 0, s>>>(B);
    }
    if (cudaGetLastError() != cudaSuccess) return 1;
  }
  return 0;
}

}  // namespace

size_t sweep_inv_work(int n, int b, int a) {
  return (size_t)b * (1 + (b + CT_ROWS - 1) / CT_ROWS) + (size_t)n * a;
}

int sweep_inv_batched(int count, const int* n, const int* b, const int* a, const double* const* L,
                      const double* const* Ab, const double* const* T, const double* const* V, double* const* x,
                      int trans, double* work, cudaStream_t s) {
  std::vector<double*> tmp(count), part(count), apart(count);
  size_t off = 0;
  int maxn = 0;
  for (int k = 0; k < count; ++k) {
    tmp[k] = work + off;
    part[k] = work + off + b[k];
    apart[k] = work + off + (size_t)b[k] * (1 + (b[k] + CT_ROWS - 1) / CT_ROWS);
    off += sweep_inv_work(n[k], b[k], a[k]);
    maxn = std::max(maxn, n[k]);
  }
  if (trans == 0) {
    for (int i = 0; i < maxn; ++i) {
      std::vector<RowJob> ja, jb;
      for (int k = 0; k < count; ++k) {
        if (i >= n[k]) continue;
        const size_t bb = (size_t)b[k] * b[k];
        RowJob r{};
        r.M = i > 0 ? L[k] + (i - 1) * bb : nullptr;
        r.x = i > 0 ? x[k] + (size_t)(i - 1) * b[k] : nullptr;
        r.c = x[k] + (size_t)i * b[k];
        r.out = tmp[k];
        r.alpha = -1.0;
        r.beta = 1.0;
        r.rows = r.cols = r.ld = b[k];
        ja.push_back(r);
        RowJob v{};
        v.M = V[k] + i * bb;
        v.x = tmp[k];
        v.out = x[k] + (size_t)i * b[k];
        v.alpha = 1.0;
        v.rows = v.cols = v.ld = b[k];
        v.lower = 1;
        jb.push_back(v);
      }
      if (launch_rows(ja, s) || launch_rows(jb, s)) return cudaErrorUnknown;
    }
    for (int k = 0; k < count; ++k)
      if (a[k] > 0 && arrow_forward(Ab[k], T[k], x[k], n[k], b[k], a[k], apart[k], s)) return cudaErrorUnknown;
    return cudaGetLastError();
  }
  for (int k = 0; k < count; ++k)
    if (a[k] > 0 && arrow_backward(T[k], x[k], n[k], b[k], a[k], s)) return cudaErrorUnknown;
  for (int st = 0; st < maxn; ++st) {
    std::vector<ColJob> ja, jb;
    for (int k = 0; k < count; ++k) {
      const int i = n[k] - 1 - st;
      if (i < 0) continue;
      const size_t bb = (size_t)b[k] * b[k];
      ColJob c{};
      c.M = i < n[k] - 1 ? L[k] + i * bb : nullptr;
      c.x = i < n[k] - 1 ? x[k] + (size_t)(i + 1) * b[k] : nullptr;
      c.y = x[k] + (size_t)i * b[k];
      c.Ab = a[k] > 0 ? Ab[k] + (size_t)i * a[k] * b[k] : nullptr;
      c.xa = a[k] > 0 ? x[k] + (size_t)n[k] * b[k] : nullptr;
      c.out = tmp[k];
      c.part = part[k];
      c.alpha = -1.0;
      c.beta = 1.0;
      c.rows = c.cols = c.ld = b[k];
      c.a = a[k];
      ja.push_back(c);
      ColJob v{};
      v.M = V[k] + i * bb;
      v.x = tmp[k];
      v.out = x[k] + (size_t)i * b[k];
      v.part = part[k];
      v.alpha = 1.0;
      v.rows = v.cols = v.ld = b[k];
      v.upper = 1;
      jb.push_back(v);
    }
    if (launch_cols(ja, s) || launch_cols(jb, s)) return cudaErrorUnknown;
  }
  return cudaGetLastError();
}

}  // namespace bta
