// Full inverses of the diagonal factor blocks (used by the selected inversion)
// and the deterministic log-determinant reduction.
#include <algorithm>

#include "bta_internal.cuh"
#include "common.cuh"
#include "tile_ops.cuh"
#include "prof.cuh"

namespace bta {
namespace {

using namespace tile;
// Slab ring of the column substitution: A = 64 rows x 16 k of a row block of
// the factor (k-contiguous, stride TSK), B = 16 k x 64 columns of the output
// (n-contiguous, stride TSN), two stages; three CTAs per SM hide the rest.
constexpr int TK = 16, TSK = TK + 4, TSN = T + 4, TST = 2;
constexpr int TA_SLAB = T * TSK, TB_SLAB = TK * TSN;
// shared memory: the ring (also the staging of a step's sum, 64 x SG), then
// the diagonal tile inverse (64 x SG)
constexpr int TRTRI_RING = TST * (TA_SLAB + TB_SLAB) > T * SG ? TST * (TA_SLAB + TB_SLAB) : T * SG;
constexpr size_t TRTRI_SMEM = size_t(TRTRI_RING + T * SG) * sizeof(double);

__device__ __forceinline__ void trtri_load(double* As, double* Bs, const double* Arow, int rows, const double* Bcol,
                                           int cols, int k0, int kend, int ld, int tid) {
  const bool va = ((ld & 1) == 0) && ((reinterpret_cast<uintptr_t>(Arow) & 15) == 0);
  const bool vb = ((ld & 1) == 0) && ((reinterpret_cast<uintptr_t>(Bcol) & 15) == 0);
#pragma unroll
  for (int j = 0; j < (T * TK / 2) / THREADS; ++j) {
    const int q = tid + j * THREADS;
    // A: row r, k pair kc
    {
      const int r = q >> 3, kc = (q & 7) * 2, gk = k0 + kc;
      double* d = As + r * TSK + kc;
      const bool v0 = r < rows && gk < kend, v1 = r < rows && gk + 1 < kend;
      const double* src = Arow + (size_t)r * ld + gk;
      if (va && v1) {
        cp_async16(d, src, true);
      } else {
        cp_async8(d, v0 ? src : Arow, v0);
        cp_async8(d + 1, v1 ? src + 1 : Arow, v1);
      }
    }
    // B: k row kr, column pair nc
    {
      const int kr = q >> 5, nc = (q & 31) * 2, gk = k0 + kr;
      double* d = Bs + kr * TSN + nc;
      const bool v0 = gk < kend && nc < cols, v1 = gk < kend && nc + 1 < cols;
      const double* src = Bcol + (size_t)gk * ld + nc;
      if (vb && v1) {
        cp_async16(d, src, true);  // .cg: from L2, where this CTA's earlier rows were written
      } else {
        d[0] = v0 ? __ldcg(src) : 0.0;
        d[1] = v1 ? __ldcg(src + 1) : 0.0;
      }
    }
  }
}

// acc += A[:, k0:kend] B[k0:kend, :] with A = rows x (.) at Arow, B = (.) x cols
// at Bcol (both row stride ld), through a 3-stage cp.async ring.
__device__ void trtri_stream(const double* Arow, int rows, const double* Bcol, int cols, int k0, int kend, int ld,
                             double* smem, double (&acc)[2][4][4], int tid, int wm, int wn, int g, int t) {
  double* As = smem;
  double* Bs = smem + TST * TA_SLAB;
  const int nslab = (kend - k0 + TK - 1) / TK;
  __syncthreads();
#pragma unroll
  for (int st = 0; st < TST - 1; ++st) {
    if (st < nslab) trtri_load(As + st * TA_SLAB, Bs + st * TB_SLAB, Arow, rows, Bcol, cols, k0 + st * TK, kend, ld, tid);
    cp_async_commit();
  }
  for (int s = 0; s < nslab; ++s) {
    cp_async_wait<TST - 2>();
    __syncthreads();
    const int nx = s + TST - 1;
    if (nx < nslab)
      trtri_load(As + (nx % TST) * TA_SLAB, Bs + (nx % TST) * TB_SLAB, Arow, rows, Bcol, cols, k0 + nx * TK, kend,
                 ld, tid);
    cp_async_commit();
    const double* X = As + (s % TST) * TA_SLAB;
    const double* Y = Bs + (s % TST) * TB_SLAB;
#pragma unroll
    for (int kk = 0; kk < TK; kk += 4) {
      double a[2][2], bb[4];
#pragma unroll
      for (int mi = 0; mi < 2; ++mi) {
        const int r = wm * 32 + mi * 16 + g;
        a[mi][0] = X[r * TSK + kk + t];
        a[mi][1] = X[(r + 8) * TSK + kk + t];
      }
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) bb[ni] = Y[(kk + t) * TSN + wn * 32 + ni * 8 + g];
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) dmma16x8x4(acc[mi][ni], a[mi][0], a[mi][1], bb[ni]);
    }
  }
  cp_async_wait<0>();
  __syncthreads();
}

// One CTA per (block, tile column c): forward substitution down the column,
//   X[c] = Linv_cc,  X[p] = -Linv_pp * sum_{k=c}^{p-1} L[p][k] X[k]   (p > c).
// blockIdx.x = c * nblk + block so that the longest columns start first.
__global__ void __launch_bounds__(THREADS, 3) block_trtri_kernel(const double* D, const double* tile_inv, int i0,
                                                               int nblk, int b, int nq, double* out) {
  extern __shared__ __align__(16) double sm[];
  double* As = sm;
  double* Ys = sm + TRTRI_RING;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1, g = lane >> 2, t = lane & 3;
  const int c = blockIdx.x / nblk, bi = blockIdx.x % nblk, i = i0 + bi;
  const size_t bb = (size_t)b * b;
  const double* Di = D + (size_t)i * bb;
  double* Oi = out + (size_t)bi * bb;
  const int wc = min(T, b - c * T);

  // zero tiles above the diagonal in this column
  for (int p = 0; p < c; ++p) {
    for (int idx = tid; idx < T * T; idx += THREADS) {
      const int r = idx >> 6, cc = idx & 63;
      if (cc < wc) Oi[(size_t)(p * T + r) * b + c * T + cc] = 0.0;
    }
  }
  // X[c] = Linv_cc
  {
    const double* Lc = tile_inv + (size_t)(i * nq + c) * T * T;
    for (int idx = tid; idx < T * T; idx += THREADS) {
      const int r = idx >> 6, cc = idx & 63;
      if (r < wc && cc < wc) Oi[(size_t)(c * T + r) * b + c * T + cc] = Lc[idx];
    }
  }
  // the column's tiles are read back only by this CTA: a CTA barrier orders them
  __syncthreads();
  for (int p = c + 1; p < nq; ++p) {
    const int rp = min(T, b - p * T);
    // the inverse of diagonal tile p arrives while the column sum streams
    load_async<SG>(Ys, tile_inv + (size_t)(i * nq + p) * T * T, T, T, T, tid);
    cp_async_commit();
    double acc[2][4][4];
    zero_acc(acc);
    // acc = L[p][c..p-1] X[c..p-1][c], streamed over k in 16-wide slabs
    trtri_stream(Di + (size_t)(p * T) * b, rp, Oi + c * T, wc, c * T, p * T, b, As, acc, tid, wm, wn, g, t);
    // As[n][j] = acc[j][n] (the slab ring is free again)
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int j = wm * 32 + mi * 16 + g + h * 8;
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const int n = wn * 32 + ni * 8 + 2 * t + e;
            As[n * SG + j] = acc[mi][ni][h * 2 + e];
          }
      }
    __syncthreads();
    zero_acc(acc);
    mma_nt(Ys, As, 32 * (wm + 1), acc, wm, wn, g, t);  // Linv_pp lower triangular: row j sums k <= j
    {
      // -acc to rows rp x columns wc of the output tile (column pairs as
      // 16-byte stores when the rows allow)
      double* o = Oi + (size_t)(p * T) * b + c * T;
      const bool vec = ((b & 1) == 0) && ((reinterpret_cast<uintptr_t>(o) & 15) == 0);
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int r = wm * 32 + mi * 16 + g + h * 8;
          if (r >= rp) continue;
#pragma unroll
          for (int ni = 0; ni < 4; ++ni) {
            const int n = wn * 32 + ni * 8 + 2 * t;
            double* dst = o + (size_t)r * b + n;
            if (vec && n + 1 < wc) {
              *reinterpret_cast<double2*>(dst) = make_double2(-acc[mi][ni][h * 2], -acc[mi][ni][h * 2 + 1]);
            } else {
              if (n < wc) dst[0] = -acc[mi][ni][h * 2];
              if (n + 1 < wc) dst[1] = -acc[mi][ni][h * 2 + 1];
            }
          }
        }
    }
    __syncthreads();  // the next step reads this tile and refills Ys
  }
}

__global__ void logdet_part_kernel(const double* D, int n, int b, const double* Tt, int a, double* part) {
  __shared__ double red[256];
  const int blk = blockIdx.x, tid = threadIdx.x;
  const double* M;
  int m;
  if (blk < n) {
    M = D + (size_t)blk * b * b;
    m = b;
  } else {
    M = Tt;
    m = a;
  }
  double s = 0.0;
  for (int k = tid; k < m; k += blockDim.x) s += log(M[(size_t)k * m + k]);
  red[tid] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (tid < o) red[tid] += red[tid + o];
    __syncthreads();
  }
  if (tid == 0) part[blk] = red[0];
}

__global__ void logdet_final_kernel(const double* part, int cnt, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < cnt; ++i) s += part[i];
    *out = 2.0 * s;
  }
}

}  // namespace

int block_trtri(const double* D, const double* tile_inv, int i0, int i1, int b, double* out, cudaStream_t s) {
  {
    const int e = ensure_smem_attr(reinterpret_cast<const void*>(block_trtri_kernel), (int)TRTRI_SMEM);
    if (e != cudaSuccess) return e;
  }
  const int nblk = i1 - i0, nq = (b + T - 1) / T;
  if (nblk <= 0) return cudaSuccess;
  {
    bta::ProfScope _ps(bta::PROF_TRTRI, s);
    block_trtri_kernel<<<nblk * nq, THREADS, TRTRI_SMEM, s>>>(D, tile_inv, i0, nblk, b, nq, out);
  }
  return cudaGetLastError();
}

int logdet_launch(const double* D, int n, int b, const double* Tt, int a, double* part, double* out,
                  cudaStream_t s) {
  const int cnt = n + (a > 0 ? 1 : 0);
  if (cnt > 0) {
    bta::ProfScope _ps(bta::PROF_OTHER, s);
    logdet_part_kernel<<<cnt, 256, 0, s>>>(D, n, b, Tt, a, part);
  }
  {
    bta::ProfScope _ps(bta::PROF_OTHER, s);
    logdet_final_kernel<<<1, 32, 0, s>>>(part, cnt, out);
  }
  return cudaGetLastError();
}

}  // namespace bta
