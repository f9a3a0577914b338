// Tile-DAG panel kernel of the BTA Cholesky (see panel.cuh).
#include <algorithm>

#include "common.cuh"
#include "panel.cuh"
#include "tile_ops.cuh"

namespace bta {
namespace {

using namespace tile;
constexpr size_t SMEM_BYTES = size_t(2) * T * SG * sizeof(double) + NPAIR * sizeof(uint16_t) + 64;
constexpr long long SPIN_LIMIT = 1LL << 24;

// Bounded wait until *p >= target.  Returns false when the wait gave up.
__device__ bool wait_ge(const int* p, int target, int* abort_flag) {
  long long it = 0;
  while (ld_acquire(p) < target) {
    if (ld_acquire(abort_flag)) return false;
    if (++it > SPIN_LIMIT) {
      atomicExch(abort_flag, 1);
      return false;
    }
    __nanosleep(64);
  }
  return true;
}

struct TileRef {
  double* ptr;
  int rows, cols;
};

__device__ __forceinline__ TileRef tile_of(const PanelInst& I, int p, int c) {
  TileRef t;
  t.cols = min(T, I.b - c * T);
  if (p < I.nq) {
    t.ptr = I.D + (size_t)(p * T) * I.b + c * T;
    t.rows = min(T, I.b - p * T);
  } else if (I.L != nullptr && p < 2 * I.nq) {
    const int pp = p - I.nq;
    t.ptr = I.L + (size_t)(pp * T) * I.b + c * T;
    t.rows = min(T, I.b - pp * T);
  } else {
    const int ar = p - I.nq - (I.L != nullptr ? I.nq : 0);
    t.ptr = I.Ab + (size_t)(ar * T) * I.b + c * T;
    t.rows = min(T, I.a - ar * T);
  }
  return t;
}

__global__ void __launch_bounds__(THREADS) panel_kernel(const __grid_constant__ PanelBatch B) {
  extern __shared__ __align__(16) double sm[];
  double* buf0 = sm;
  double* buf1 = sm + T * SG;
  uint16_t* pairs = reinterpret_cast<uint16_t*>(sm + 2 * T * SG);
  __shared__ int s_task, s_ok;
  __shared__ double dg[T];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1, g = lane >> 2, t = lane & 3;

  build_pairs(pairs, tid);
  __syncthreads();

  for (;;) {
    if (tid == 0) s_task = atomicAdd(B.counter, 1);
    __syncthreads();
    const int ti = s_task;
    if (ti >= B.ntasks) break;
    const int4 tk = B.tasks[ti];
    const PanelInst& I = B.inst[tk.x];
    const int kind = tk.y, p = tk.z, r = tk.w >> 16, q = tk.w & 0xffff;
    const int nq = I.nq;
    if (tid == 0) {
      bool ok;
      if (kind == TASK_POTRF) {
        ok = wait_ge(&I.upd[q * nq + q], q, B.abort_flag);
      } else if (kind == TASK_TRSM) {
        ok = wait_ge(&I.flag[q * nq + q], 1, B.abort_flag) && wait_ge(&I.upd[p * nq + q], q, B.abort_flag);
      } else {
        ok = wait_ge(&I.flag[p * nq + q], 1, B.abort_flag) && wait_ge(&I.flag[r * nq + q], 1, B.abort_flag) &&
             wait_ge(&I.upd[p * nq + r], q, B.abort_flag);
      }
      s_ok = ok ? 1 : 0;
    }
    __syncthreads();
    if (!s_ok) continue;

    if (kind == TASK_POTRF) {
      TileRef d = tile_of(I, q, q);
      load<SC>(buf0, d.ptr, I.b, d.cols, d.cols, tid);
      __syncthreads();
      potrf(buf0, pairs, dg, d.cols, I.info, I.pivot_base + (long long)q * T, tid);
      trinv(buf0, buf1, tid);
      double* linv = I.Linv + (size_t)q * T * T;
      for (int idx = tid; idx < T * T; idx += THREADS) {
        const int i = idx >> 6, k = idx & 63;
        const bool in = i < d.cols && k < d.cols;
        if (in) d.ptr[(size_t)i * I.b + k] = buf0[i * SC + k];
        linv[idx] = in ? buf1[i * SC + k] : 0.0;
      }
      // strictly-upper tiles of this tile column become zero, as in a
      // LAPACK-style lower factor
      for (int qq = 0; qq < q; ++qq) {
        double* up = I.D + (size_t)(qq * T) * I.b + q * T;
        for (int idx = tid; idx < T * T; idx += THREADS) {
          const int i = idx >> 6, k = idx & 63;
          if (k < d.cols) up[(size_t)i * I.b + k] = 0.0;
        }
      }
    } else if (kind == TASK_TRSM) {
      TileRef x = tile_of(I, p, q);
      load<SG>(buf0, x.ptr, I.b, x.rows, x.cols, tid);
      load<SG>(buf1, I.Linv + (size_t)q * T * T, T, T, T, tid);
      __syncthreads();
      double acc[2][4][4];
      zero_acc(acc);
      mma_nt(buf0, buf1, (x.cols + 3) & ~3, acc, wm, wn, g, t);
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int row = wm * 32 + mi * 16 + g + h * 8;
          if (row >= x.rows) continue;
#pragma unroll
          for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              const int col = wn * 32 + ni * 8 + 2 * t + e;
              if (col < x.cols) x.ptr[(size_t)row * I.b + col] = acc[mi][ni][h * 2 + e];
            }
        }
    } else {
      TileRef xp = tile_of(I, p, q);
      TileRef xr = tile_of(I, r, q);
      TileRef c = tile_of(I, p, r);
      load<SG>(buf0, xp.ptr, I.b, xp.rows, xp.cols, tid);
      load<SG>(buf1, xr.ptr, I.b, xr.rows, xr.cols, tid);
      __syncthreads();
      double acc[2][4][4];
      zero_acc(acc);
      mma_nt(buf0, buf1, (xp.cols + 3) & ~3, acc, wm, wn, g, t);
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int row = wm * 32 + mi * 16 + g + h * 8;
          if (row >= c.rows) continue;
#pragma unroll
          for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              const int col = wn * 32 + ni * 8 + 2 * t + e;
              if (col < c.cols) {
                double* dst = c.ptr + (size_t)row * I.b + col;
                *dst = __ldcg(dst) - acc[mi][ni][h * 2 + e];
              }
            }
        }
    }
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      if (kind == TASK_UPDATE) st_release(&I.upd[p * nq + r], q + 1);
      else st_release(&I.flag[p * nq + q], 1);
    }
  }
}

}  // namespace

void panel_tasks(const std::vector<PanelInst>& insts, std::vector<int4>& tasks) {
  int max_nq = 0;
  for (const auto& I : insts) max_nq = std::max(max_nq, I.nq);
  for (int r = 0; r < max_nq; ++r) {
    for (int ii = 0; ii < (int)insts.size(); ++ii) {
      const PanelInst& I = insts[ii];
      if (r >= I.nq) continue;
      // updates of tile column r from every earlier column k
      for (int k = 0; k < r; ++k)
        for (int p = r; p < I.nrows_t; ++p) tasks.push_back(make_int4(ii, TASK_UPDATE, p, (r << 16) | k));
      tasks.push_back(make_int4(ii, TASK_POTRF, r, (r << 16) | r));
      for (int p = r + 1; p < I.nrows_t; ++p) tasks.push_back(make_int4(ii, TASK_TRSM, p, (r << 16) | r));
    }
  }
}

int panel_grid_size() {
  static int grid = 0;
  if (grid == 0) {
    cudaError_t e = cudaFuncSetAttribute(panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)SMEM_BYTES);
    if (e != cudaSuccess) return -(int)e;
    int dev = 0, sms = 0, occ = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, panel_kernel, THREADS, SMEM_BYTES);
    grid = std::max(1, sms * std::max(1, occ));
  }
  return grid;
}

int panel_launch(const PanelBatch& batch, int grid, cudaStream_t stream) {
  int g = panel_grid_size();
  if (g <= 0) return -g;
  if (grid <= 0 || grid > g) grid = g;
  grid = std::min(grid, batch.ntasks);
  if (grid <= 0) return cudaSuccess;
  panel_kernel<<<grid, THREADS, SMEM_BYTES, stream>>>(batch);
  return cudaGetLastError();
}

}  // namespace bta
