// 64x64 FP64 tile operations in shared memory, used by several kernels.
#pragma once

#include "common.cuh"

namespace bta {
namespace tile {

constexpr int T = TILE;
constexpr int THREADS = 128;
constexpr int SG = T + 4;  // stride of GEMM operand tiles (k-contiguous, conflict-free)
constexpr int SC = T + 1;  // stride of Cholesky / inverse tiles
constexpr int NPAIR = T * (T + 1) / 2;

__device__ __forceinline__ int pair_off(int k) { return T * k - k * (k - 1) / 2; }

// Lower-triangle (i, k), k <= i, pairs ordered by k: the trailing pairs of
// Cholesky step j (k > j) are the suffix starting at pair_off(j + 1).
__device__ __forceinline__ void build_pairs(uint16_t* pairs, int tid) {
  for (int k = tid; k < T; k += THREADS) {
    const int o = pair_off(k);
    for (int i = k; i < T; ++i) pairs[o + i - k] = (uint16_t)((i << 8) | k);
  }
}

// Load a rows x cols tile (leading dimension ld) into smem with stride S,
// zero-filled to 64 x 64.  L2-only loads (data may come from other CTAs).
template <int S>
__device__ __forceinline__ void load(double* s, const double* g, int ld, int rows, int cols, int tid) {
#pragma unroll 8
  for (int idx = tid; idx < T * T; idx += THREADS) {
    const int r = idx >> 6, c = idx & 63;
    s[r * S + c] = (r < rows && c < cols) ? __ldcg(g + (size_t)r * ld + c) : 0.0;
  }
}

__device__ __forceinline__ void zero_acc(double (&acc)[2][4][4]) {
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[mi][ni][e] = 0.0;
}

// acc += X(64 x kw) * Y(64 x kw)^T; X, Y k-contiguous in smem (stride SG).
// Warp (wm, wn) owns rows wm*32.., cols wn*32.. of the 64x64 product.
__device__ __forceinline__ void mma_nt(const double* X, const double* Y, int kw, double (&acc)[2][4][4],
                                       int wm, int wn, int g, int t) {
  for (int kk = 0; kk < kw; kk += 4) {
    double a[2][2], b[4];
#pragma unroll
    for (int mi = 0; mi < 2; ++mi) {
      const int r = wm * 32 + mi * 16 + g;
      a[mi][0] = X[r * SG + kk + t];
      a[mi][1] = X[(r + 8) * SG + kk + t];
    }
#pragma unroll
    for (int ni = 0; ni < 4; ++ni) b[ni] = Y[(wn * 32 + ni * 8 + g) * SG + kk + t];
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) dmma16x8x4(acc[mi][ni], a[mi][0], a[mi][1], b[ni]);
  }
}

// In-place lower Cholesky of the smem tile S (stride SC).  Entries beyond w
// are treated as the identity.  A non-positive pivot j < w records base+j+1
// in *info (atomicMin) and the factorisation continues (NaNs propagate).
// On exit S holds L with zeros above the diagonal.
__device__ __forceinline__ void potrf(double* S, const uint16_t* pairs, double* dg, int w,
                                      unsigned long long* info, long long base, int tid) {
  for (int i = w + tid; i < T; i += THREADS) S[i * SC + i] = 1.0;
  __syncthreads();
  for (int j = 0; j < T; ++j) {
    const double piv = S[j * SC + j];
    if (tid == 0 && j < w && !(piv > 0.0) && info != nullptr)
      atomicMin(info, (unsigned long long)(base + j + 1));
    const double ipiv = 1.0 / piv;
    for (int idx = pair_off(j + 1) + tid; idx < NPAIR; idx += THREADS) {
      const int pk = pairs[idx];
      const int i = pk >> 8, k = pk & 255;
      S[i * SC + k] -= S[i * SC + j] * S[k * SC + j] * ipiv;
    }
    __syncthreads();
  }
  if (tid < T) dg[tid] = sqrt(S[tid * SC + tid]);
  __syncthreads();
  for (int idx = tid; idx < T * T; idx += THREADS) {
    const int i = idx >> 6, k = idx & 63;
    double v;
    if (k < i) v = S[i * SC + k] / dg[k];
    else if (k == i) v = dg[i];
    else v = 0.0;
    S[i * SC + k] = v;
  }
  __syncthreads();
}

// Li <- inverse of the lower-triangular smem tile S (both stride SC, S has
// a non-zero diagonal over the full 64 x 64).  Recursive doubling:
// 16x16 diagonal inverses, then X21 = -inv(L22) L21 inv(L11) for h = 16, 32.
__device__ __forceinline__ void trinv(const double* S, double* Li, int tid) {
  for (int idx = tid; idx < T * T; idx += THREADS) Li[(idx >> 6) * SC + (idx & 63)] = 0.0;
  __syncthreads();
  if (tid < T) {
    const int c = tid, end = (tid >> 4) * 16 + 16;
    Li[c * SC + c] = 1.0 / S[c * SC + c];
    for (int i = c + 1; i < end; ++i) {
      double s0 = 0.0, s1 = 0.0;
      int k = c;
      for (; k + 1 < i; k += 2) {
        s0 += S[i * SC + k] * Li[k * SC + c];
        s1 += S[i * SC + k + 1] * Li[(k + 1) * SC + c];
      }
      if (k < i) s0 += S[i * SC + k] * Li[k * SC + c];
      Li[i * SC + c] = -(s0 + s1) / S[i * SC + i];
    }
  }
  __syncthreads();
  for (int h = 16; h <= 32; h *= 2) {
    const int nblk = T / (2 * h);
    for (int idx = tid; idx < nblk * h * h; idx += THREADS) {
      const int bb = idx / (h * h), rem = idx % (h * h);
      const int i = rem / h, c = rem % h, o = bb * 2 * h;
      double s = 0.0;
      for (int k = c; k < h; ++k) s += S[(o + h + i) * SC + o + k] * Li[(o + k) * SC + o + c];
      Li[(o + i) * SC + o + h + c] = s;  // scratch in the zero upper block
    }
    __syncthreads();
    for (int idx = tid; idx < nblk * h * h; idx += THREADS) {
      const int bb = idx / (h * h), rem = idx % (h * h);
      const int i = rem / h, c = rem % h, o = bb * 2 * h;
      double s = 0.0;
      for (int k = 0; k <= i; ++k) s += Li[(o + h + i) * SC + o + h + k] * Li[(o + k) * SC + o + h + c];
      Li[(o + h + i) * SC + o + c] = -s;
    }
    __syncthreads();
    for (int idx = tid; idx < nblk * h * h; idx += THREADS) {
      const int bb = idx / (h * h), rem = idx % (h * h);
      const int i = rem / h, c = rem % h, o = bb * 2 * h;
      Li[(o + i) * SC + o + h + c] = 0.0;
    }
    __syncthreads();
  }
}

}  // namespace tile
}  // namespace bta
