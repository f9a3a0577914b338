// BTA triangular solves (one sweep per call, like Serinv's pobtas) and the
// batched inverses of the 64x64 diagonal tiles they use.
//
// A sweep is one persistent launch over tile rows (block i, tile p) claimed in
// topological order; each task accumulates its GEMV contributions as the tiles
// it depends on are published (release/acquire flags, bounded waits) and then
// applies the inverse of its diagonal tile.
#include <algorithm>
#include <cstring>

#include "bta_internal.cuh"
#include "common.cuh"
#include "tile_ops.cuh"
#include "prof.cuh"

namespace bta {
namespace {

using namespace tile;
constexpr long long SPIN_LIMIT = 1LL << 24;

__device__ bool wait_flag(const int* p, int* abort_flag) {
  long long it = 0;
  while (ld_acquire(p) < 1) {
    if (ld_acquire(abort_flag)) return false;
    if (++it > SPIN_LIMIT) {
      atomicExch(abort_flag, 1);
      return false;
    }
    __nanosleep(64);
  }
  return true;
}

// Inverse of every 64x64 diagonal tile of the n diagonal factor blocks.
__global__ void __launch_bounds__(THREADS) diag_tile_inverse_kernel(const double* D, int n, int b, int nq,
                                                                     double* out) {
  extern __shared__ __align__(16) double sm[];
  __shared__ double rd[T];
  double* S = sm;
  double* Li = sm + T * SG;
  const int tid = threadIdx.x;
  const int i = blockIdx.x / nq, p = blockIdx.x % nq;
  const int w = min(T, b - p * T);
  const double* src = D + (size_t)i * b * b + (size_t)(p * T) * b + p * T;
  load<SG>(S, src, b, w, w, tid);
  __syncthreads();
  for (int r = w + tid; r < T; r += THREADS) S[r * SG + r] = 1.0;
  __syncthreads();
  trinv(S, Li, rd, tid);
  double* dst = out + (size_t)blockIdx.x * T * T;
  for (int idx = tid; idx < T * T; idx += THREADS) {
    const int r = idx >> 6, c = idx & 63;
    dst[idx] = (r < w && c < w) ? Li[r * SG + c] : 0.0;
  }
}

// acc[r] -= sum_c M[r][c] v[c]  (rows x cols tile, leading dimension ld).
// The factor is read-only during a sweep: read-only cache path, every load of
// a lane issued before the reductions.
__device__ __forceinline__ void gemv_sub(const double* M, int ld, int rows, int cols, const double* v,
                                         double* acc, int tid) {
  const int lane = tid & 31, warp = tid >> 5;
  const double v0 = lane < cols ? v[lane] : 0.0;
  const double v1 = lane + 32 < cols ? v[lane + 32] : 0.0;
  double s[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const int r = warp + 4 * j;
    double x = 0.0;
    if (r < rows) {
      const double* row = M + (size_t)r * ld;
      if (lane < cols) x += __ldg(row + lane) * v0;
      if (lane + 32 < cols) x += __ldg(row + lane + 32) * v1;
    }
    s[j] = x;
  }
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    double x = s[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    const int r = warp + 4 * j;
    if (lane == 0 && r < rows) acc[r] -= x;
  }
}

// acc[c] -= sum_r M[r][c] v[r]; part is a 128-entry smem scratch.
__device__ __forceinline__ void gemv_t_sub(const double* M, int ld, int rows, int cols, const double* v,
                                           double* acc, double* part, int tid) {
  const int c = tid & 63, half = tid >> 6;
  double s = 0.0;
  if (c < cols) {
    const int r0 = half * 32;
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const int r = r0 + j;
      if (r < rows) s += __ldg(M + (size_t)r * ld + c) * v[r];
    }
  }
  part[tid] = s;
  __syncthreads();
  if (tid < 64) acc[tid] -= part[tid] + part[tid + 64];
  __syncthreads();
}

constexpr int SP = T + 1;  // smem stride of the prefetched tiles

// Prefetch a rows x cols tile (ld) into smem (stride SP), zero-filled.
__device__ __forceinline__ void prefetch_tile(double* s, const double* g, int ld, int rows, int cols, int tid) {
#pragma unroll 4
  for (int idx = tid; idx < T * T; idx += THREADS) {
    const int r = idx >> 6, c = idx & 63;
    s[r * SP + c] = (r < rows && c < cols) ? __ldg(g + (size_t)r * ld + c) : 0.0;
  }
}

// acc[r] -= sum_c S[r][c] v[c] from smem (two threads per row)
__device__ __forceinline__ void smem_gemv_sub(const double* S, const double* v, double* acc, int rows, int tid) {
  const int r = tid >> 1, h = tid & 1;
  double s = 0.0;
#pragma unroll 8
  for (int j = 0; j < 32; ++j) s += S[r * SP + h * 32 + j] * v[h * 32 + j];
  s += __shfl_xor_sync(0xffffffffu, s, 1);
  if (h == 0 && r < rows) acc[r] -= s;
}

// acc[c] -= sum_r S[r][c] v[r] from smem (two threads per column)
__device__ __forceinline__ void smem_gemv_t_sub(const double* S, const double* v, double* acc, double* part,
                                                int cols, int tid) {
  const int c = tid & 63, h = tid >> 6;
  double s = 0.0;
#pragma unroll 8
  for (int j = 0; j < 32; ++j) s += S[(h * 32 + j) * SP + c] * v[h * 32 + j];
  part[tid] = s;
  __syncthreads();
  if (tid < cols) acc[tid] -= part[tid] + part[tid + 64];
  __syncthreads();
}

// One sweep.  Task (i, p) owns tile row p of block i.  It prefetches the tile
// that multiplies its last dependency (forward: the tile left of its diagonal
// tile, or the last tile of the block below's row for p = 0; backward: the
// transposed tile below its diagonal tile, or of the next block for the last
// tile row) and the inverse of its diagonal tile, accumulates every other
// contribution as its inputs are published, and only then waits for the last
// one: the critical path per tile is two small GEMVs from shared memory.
__global__ void __launch_bounds__(THREADS) sweep_kernel(const __grid_constant__ SweepBatch BT) {
  extern __shared__ __align__(16) double sm[];
  double* Sc = sm;           // critical tile
  double* Sl = sm + T * SP;  // inverse of the diagonal tile
  __shared__ double acc[T], v[T], part[2 * T];
  __shared__ int s_task, s_ok;
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) s_task = atomicAdd(BT.counter, 1);
    __syncthreads();
    const int tb = s_task;
    if (tb >= BT.total) break;
    const SweepArgs& A = BT.inst[tb % BT.count];
    const int ti = tb / BT.count;
    if (ti >= A.n * A.nq) continue;
    const size_t bb = (size_t)A.b * A.b;
    int i, p;
    if (A.trans == 0) {
      i = ti / A.nq;
      p = ti % A.nq;
    } else {
      i = A.n - 1 - ti / A.nq;
      p = A.nq - 1 - ti % A.nq;
    }
    const int rows = min(T, A.b - p * T);
    double* xi = A.x + (size_t)i * A.b;
    // --- prefetch the critical tile and the diagonal-tile inverse
    const double* crit = nullptr;
    int crows = 0, ccols = 0, cflag = -1;
    const double* cvec = nullptr;
    if (A.trans == 0) {
      if (p > 0) {
        crit = A.D + (size_t)i * bb + (size_t)(p * T) * A.b + (p - 1) * T;
        crows = rows;
        ccols = T;
        cflag = i * A.nq + p - 1;
        cvec = xi + (p - 1) * T;
      } else if (i > 0) {
        const int kq = A.nq - 1;
        crit = A.L + (size_t)(i - 1) * bb + kq * T;  // row tile 0, column tile nq-1
        crows = rows;
        ccols = min(T, A.b - kq * T);
        cflag = (i - 1) * A.nq + kq;
        cvec = A.x + (size_t)(i - 1) * A.b + kq * T;
      }
    } else {
      if (p < A.nq - 1) {
        crit = A.D + (size_t)i * bb + (size_t)((p + 1) * T) * A.b + p * T;  // tile (p+1, p)
        crows = min(T, A.b - (p + 1) * T);
        ccols = rows;
        cflag = i * A.nq + p + 1;
        cvec = xi + (p + 1) * T;
      } else if (i < A.n - 1) {
        crit = A.L + (size_t)i * bb + p * T;  // tile (0, p) of L_i
        crows = min(T, A.b);
        ccols = rows;
        cflag = (i + 1) * A.nq;
        cvec = A.x + (size_t)(i + 1) * A.b;
      }
    }
    if (crit) prefetch_tile(Sc, crit, A.b, crows, ccols, tid);
    prefetch_tile(Sl, A.Linv + (size_t)(i * A.nq + p) * T * T, T, rows, rows, tid);
    if (tid < T) acc[tid] = (tid < rows) ? xi[p * T + tid] : 0.0;
    __syncthreads();
    bool ok = true;
    // --- every non-critical contribution
    if (A.trans == 0) {
      if (i > 0) {
        const double* Lm = A.L + (size_t)(i - 1) * bb + (size_t)(p * T) * A.b;
        const double* yprev = A.x + (size_t)(i - 1) * A.b;
        const int klast = (p == 0) ? A.nq - 1 : A.nq;
        for (int k = 0; k < klast && ok; ++k) {
          if (tid == 0) s_ok = wait_flag(&A.flags[(i - 1) * A.nq + k], A.abort_flag);
          __syncthreads();
          ok = s_ok;
          const int kc = min(T, A.b - k * T);
          if (ok) {
            if (tid < T) v[tid] = tid < kc ? __ldcg(yprev + k * T + tid) : 0.0;
            __syncthreads();
            gemv_sub(Lm + k * T, A.b, rows, kc, v, acc, tid);
          }
          __syncthreads();
        }
      }
      const double* Dm = A.D + (size_t)i * bb + (size_t)(p * T) * A.b;
      for (int k = 0; k + 1 < p && ok; ++k) {
        if (tid == 0) s_ok = wait_flag(&A.flags[i * A.nq + k], A.abort_flag);
        __syncthreads();
        ok = s_ok;
        if (ok) {
          if (tid < T) v[tid] = __ldcg(xi + k * T + tid);
          __syncthreads();
          gemv_sub(Dm + k * T, A.b, rows, T, v, acc, tid);
        }
        __syncthreads();
      }
    } else {
      if (A.a > 0) {
        for (int a0 = 0; a0 < A.a; a0 += T) {
          const int ar = min(T, A.a - a0);
          if (tid < T) v[tid] = tid < ar ? __ldcg(A.x + (size_t)A.n * A.b + a0 + tid) : 0.0;
          __syncthreads();
          gemv_t_sub(A.Ab + (size_t)i * A.a * A.b + (size_t)a0 * A.b + p * T, A.b, ar, rows, v, acc, part, tid);
        }
      }
      if (i < A.n - 1) {
        const double* Lm = A.L + (size_t)i * bb + p * T;
        const double* xnext = A.x + (size_t)(i + 1) * A.b;
        const int kfirst = (p == A.nq - 1) ? 1 : 0;
        for (int k = A.nq - 1; k >= kfirst && ok; --k) {
          if (tid == 0) s_ok = wait_flag(&A.flags[(i + 1) * A.nq + k], A.abort_flag);
          __syncthreads();
          ok = s_ok;
          const int kr = min(T, A.b - k * T);
          if (ok) {
            if (tid < T) v[tid] = tid < kr ? __ldcg(xnext + k * T + tid) : 0.0;
            __syncthreads();
            gemv_t_sub(Lm + (size_t)(k * T) * A.b, A.b, kr, rows, v, acc, part, tid);
          }
        }
      }
      const double* Dm = A.D + (size_t)i * bb + p * T;
      for (int k = A.nq - 1; k > p + 1 && ok; --k) {
        if (tid == 0) s_ok = wait_flag(&A.flags[i * A.nq + k], A.abort_flag);
        __syncthreads();
        ok = s_ok;
        const int kr = min(T, A.b - k * T);
        if (ok) {
          if (tid < T) v[tid] = tid < kr ? __ldcg(xi + k * T + tid) : 0.0;
          __syncthreads();
          gemv_t_sub(Dm + (size_t)(k * T) * A.b, A.b, kr, rows, v, acc, part, tid);
        }
      }
    }
    // --- the critical dependency, then the diagonal tile
    if (ok && crit) {
      if (tid == 0) s_ok = wait_flag(&A.flags[cflag], A.abort_flag);
      __syncthreads();
      ok = s_ok;
      if (ok) {
        const int vn = (A.trans == 0) ? ccols : crows;
        if (tid < T) v[tid] = tid < vn ? __ldcg(cvec + tid) : 0.0;
        __syncthreads();
        if (A.trans == 0) smem_gemv_sub(Sc, v, acc, rows, tid);
        else smem_gemv_t_sub(Sc, v, acc, part, rows, tid);
      }
      __syncthreads();
    }
    if (ok) {
      if (tid < T) v[tid] = acc[tid];
      if (tid < T) acc[tid] = 0.0;
      __syncthreads();
      if (A.trans == 0) smem_gemv_sub(Sl, v, acc, rows, tid);
      else smem_gemv_t_sub(Sl, v, acc, part, rows, tid);
      __syncthreads();
      if (tid < rows) xi[p * T + tid] = -acc[tid];
    }
    __syncthreads();
    if (tid == 0 && ok) {
      __threadfence();
      st_release(&A.flags[i * A.nq + p], 1);
    }
  }
}

// Forward arrow step, y_a = T^-1 (x_a - sum_i Ab_i y_i), in two kernels:
// one CTA per block i writes part[i a + r] = sum_c Ab_i[r][c] y_i[c] (its
// arrow rows and y_i read once, AF_R rows at a time), then one CTA sums the
// parts in block order (deterministic) and solves with the tip factor.
constexpr int AF_THREADS = 256, AF_R = 8;

__global__ void __launch_bounds__(AF_THREADS) arrow_part_kernel(const double* Ab, const double* x, int b, int a,
                                                               double* part) {
  __shared__ double red[AF_THREADS / 32][AF_R];
  const int i = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double* xi = x + (size_t)i * b;
  const double* Ai = Ab + (size_t)i * a * b;
  for (int r0 = 0; r0 < a; r0 += AF_R) {
    double acc[AF_R];
#pragma unroll
    for (int q = 0; q < AF_R; ++q) acc[q] = 0.0;
    for (int c = tid; c < b; c += AF_THREADS) {
      const double xv = xi[c];
#pragma unroll
      for (int q = 0; q < AF_R; ++q)
        if (r0 + q < a) acc[q] = fma(Ai[(size_t)(r0 + q) * b + c], xv, acc[q]);
    }
#pragma unroll
    for (int q = 0; q < AF_R; ++q)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
    if (lane == 0)
#pragma unroll
      for (int q = 0; q < AF_R; ++q) red[warp][q] = acc[q];
    __syncthreads();
    if (tid < AF_R && r0 + tid < a) {
      double sum = 0.0;
      for (int w = 0; w < AF_THREADS / 32; ++w) sum += red[w][tid];
      part[(size_t)i * a + r0 + tid] = sum;
    }
    __syncthreads();
  }
}

__global__ void arrow_solve_kernel(const double* part, const double* Tt, double* x, int n, int b, int a) {
  extern __shared__ double ya[];
  const long long nb = (long long)n * b;
  for (int r = threadIdx.x; r < a; r += blockDim.x) {
    double sum = 0.0;
    for (int i = 0; i < n; ++i) sum += part[(size_t)i * a + r];
    ya[r] = x[nb + r] - sum;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int r = 0; r < a; ++r) {
      double v = ya[r];
      for (int k = 0; k < r; ++k) v -= Tt[r * a + k] * ya[k];
      ya[r] = v / Tt[r * a + r];
      x[nb + r] = ya[r];
    }
  }
}

// Backward arrow step: x_a = T^-T y_a (one thread).
__global__ void arrow_backward_kernel(const double* Tt, double* x, long long nb, int a) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int r = a - 1; r >= 0; --r) {
    double s = x[nb + r];
    for (int k = r + 1; k < a; ++k) s -= Tt[k * a + r] * x[nb + k];
    x[nb + r] = s / Tt[r * a + r];
  }
}

}  // namespace

int diag_tile_inverses(const double* D, int n, int b, double* out, cudaStream_t s) {
  const int nq = (b + T - 1) / T;
  const size_t smem = size_t(2) * T * SG * sizeof(double);
  {
    const int e = ensure_smem_attr(reinterpret_cast<const void*>(diag_tile_inverse_kernel), (int)smem);
    if (e != cudaSuccess) return e;
  }
  if (n * nq == 0) return cudaSuccess;
  {
    bta::ProfScope _ps(bta::PROF_SWEEP, s);
    diag_tile_inverse_kernel<<<n * nq, THREADS, smem, s>>>(D, n, b, nq, out);
  }
  return cudaGetLastError();
}

int sweep_launch_batched(SweepBatch& B, cudaStream_t s) {
  int maxt = 0;
  for (int k = 0; k < B.count; ++k) maxt = std::max(maxt, B.inst[k].n * B.inst[k].nq);
  B.total = B.count * maxt;
  if (B.total == 0) return cudaSuccess;
  const int sms = device_sm_count();
  {
    const int e = ensure_smem_attr(reinterpret_cast<const void*>(sweep_kernel), (int)(2 * T * SP * sizeof(double)));
    if (e != cudaSuccess) return e;
  }
  const int grid = std::min(B.total, sms * 3);
  {
    bta::ProfScope _ps(bta::PROF_SWEEP, s);
    sweep_kernel<<<grid, THREADS, 2 * T * SP * sizeof(double), s>>>(B);
  }
  return cudaGetLastError();
}

int arrow_forward(const double* Ab, const double* Tt, double* x, int n, int b, int a, double* part,
                  cudaStream_t s) {
  if (a <= 0) return cudaSuccess;
  {
    bta::ProfScope _ps(bta::PROF_SWEEP, s);
    arrow_part_kernel<<<n, AF_THREADS, 0, s>>>(Ab, x, b, a, part);
  }
  {
    bta::ProfScope _ps(bta::PROF_SWEEP, s);
    arrow_solve_kernel<<<1, 128, (size_t)a * sizeof(double), s>>>(part, Tt, x, n, b, a);
  }
  return cudaGetLastError();
}

int arrow_backward(const double* Tt, double* x, int n, int b, int a, cudaStream_t s) {
  if (a <= 0) return cudaSuccess;
  {
    bta::ProfScope _ps(bta::PROF_SWEEP, s);
    arrow_backward_kernel<<<1, 32, 0, s>>>(Tt, x, (long long)n * b, a);
  }
  return cudaGetLastError();
}

}  // namespace bta
