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

// Asynchronous version of load() for an even stride S: 16-byte cp.async
// (L2 only, zero-filled) when the tile rows are 16-byte aligned, scalar L2
// loads otherwise.  The caller commits, waits and synchronises.
template <int S>
__device__ __forceinline__ void load_async(double* s, const double* g, int ld, int rows, int cols, int tid) {
  static_assert((S & 1) == 0, "16-byte smem rows");
  const bool vec = ((ld & 1) == 0) && ((reinterpret_cast<uintptr_t>(g) & 15) == 0);
  if (vec) {
#pragma unroll
    for (int j = 0; j < (T * T / 2) / THREADS; ++j) {
      const int c = tid + j * THREADS;
      const int r = c >> 5, col = (c & 31) * 2;
      const int nvalid = (r < rows) ? max(0, min(2, cols - col)) : 0;
      const double* src = nvalid ? g + (size_t)r * ld + col : g;
      const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(s + r * S + col));
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(src), "r"(nvalid * 8));
    }
  } else {
    load<S>(s, g, ld, rows, cols, tid);
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

// 1/sqrt(x) for x > 0: hardware seed (rsqrt.approx) refined by three
// Newton-Raphson steps for x^{-1/2}, y <- y + y (1 - x y^2) / 2.
__device__ __forceinline__ double rsqrt_nr(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
#pragma unroll
  for (int it = 0; it < 3; ++it) {
    const double r = fma(-x * y, y, 1.0);
    y = fma(0.5 * y, r, y);
  }
  return y;
}

// 1/x: hardware seed refined by Newton-Raphson for 1/x, y <- y + y (1 - x y).
__device__ __forceinline__ double rcp_nr(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
#pragma unroll
  for (int it = 0; it < 3; ++it) {
    const double r = fma(-x, y, 1.0);
    y = fma(y, r, y);
  }
  return y;
}

// In-place lower Cholesky of the 64x64 smem tile S (stride SG).  Rows and
// columns beyond w are treated as the identity.  A non-positive pivot j < w
// records base+j+1 in *info (atomicMin); the factorisation continues.
// On exit S holds L with zeros above the diagonal.
//
// Blocked right-looking in four 16-wide steps: warp 0 factors the 16x16
// diagonal block with shuffles (one row per lane), the rows below are solved
// row-parallel, and the trailing matrix is updated on the DMMA pipe.
// rd: 64 doubles of smem scratch.
__device__ __forceinline__ void potrf(double* S, double* rd, int w, unsigned long long* info, long long base,
                                      int tid) {
  const int lane = tid & 31, warp = tid >> 5, g = lane >> 2, t = lane & 3;
  for (int idx = tid; idx < T * T; idx += THREADS) {
    const int i = idx >> 6, k = idx & 63;
    if (i >= w || k >= w) S[i * SG + k] = (i == k) ? 1.0 : 0.0;
  }
  __syncthreads();
  for (int kb = 0; kb < 4; ++kb) {
    const int o = kb * 16;
    if (warp == 0) {
      const int i = lane & 15;
      double d[16];
#pragma unroll
      for (int k = 0; k < 16; ++k) d[k] = S[(o + i) * SG + o + k];
      // dn: lane j+1's next pivot, updated from its own l_{j+1,j} (the same
      // fma as its column update, off the shuffle of that update's operand)
      double dn = d[0];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const double piv = __shfl_sync(0xffffffffu, dn, j, 16);
        if (lane == 0 && o + j < w && !(piv > 0.0) && info != nullptr)
          atomicMin(info, (unsigned long long)(base + o + j + 1));
        const double rs = rsqrt_nr(piv);
        const double lij = d[j] * rs;
        if (j + 1 < 16) dn = fma(-lij, lij, d[j + 1]);
#pragma unroll
        for (int k = j + 1; k < 16; ++k) {
          const double lkj = __shfl_sync(0xffffffffu, lij, k, 16);
          d[k] = fma(-lij, lkj, d[k]);
        }
        d[j] = (i > j) ? lij : ((i == j) ? piv * rs : 0.0);
        if (i == j) rd[o + j] = rs;  // 1 / L[j][j]
      }
      if (lane < 16) {
#pragma unroll
        for (int k = 0; k < 16; ++k) S[(o + i) * SG + o + k] = d[k];
      }
    }
    __syncthreads();
    const int R = T - o - 16;  // trailing rows
    if (R == 0) break;
    // rows below: X = S[o+16.., o..o+15] * L_blk^-T (row-parallel substitution)
    if (tid < R) {
      double* x = S + (o + 16 + tid) * SG + o;
      double v[16];
#pragma unroll
      for (int k = 0; k < 16; ++k) v[k] = x[k];
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        double s = v[k];
#pragma unroll
        for (int m = 0; m < k; ++m) s = fma(-v[m], S[(o + k) * SG + o + m], s);
        v[k] = s * rd[o + k];
      }
#pragma unroll
      for (int k = 0; k < 16; ++k) x[k] = v[k];
    }
    __syncthreads();
    // trailing update S[o+16.., o+16..] -= X X^T on the DMMA pipe
    const double* X = S + (o + 16) * SG + o;
    double* C = S + (o + 16) * SG + o + 16;
    const int mt = R / 16, nt = R / 8;
    for (int tile = warp; tile < mt * nt; tile += 4) {
      const int mi = tile / nt, ni = tile % nt;
      if (ni * 8 > mi * 16 + 15) continue;  // strictly above the diagonal
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int kk = 0; kk < 16; kk += 4) {
        const double a0 = X[(mi * 16 + g) * SG + kk + t];
        const double a1 = X[(mi * 16 + g + 8) * SG + kk + t];
        const double b0 = X[(ni * 8 + g) * SG + kk + t];
        dmma16x8x4(acc, a0, a1, b0);
      }
      const int r0 = mi * 16 + g, c0 = ni * 8 + 2 * t;
      C[r0 * SG + c0] -= acc[0];
      C[r0 * SG + c0 + 1] -= acc[1];
      C[(r0 + 8) * SG + c0] -= acc[2];
      C[(r0 + 8) * SG + c0 + 1] -= acc[3];
    }
    __syncthreads();
  }
  // zero the strictly-upper part (off-diagonal 16-blocks still hold input)
  for (int idx = tid; idx < T * T; idx += THREADS) {
    const int i = idx >> 6, k = idx & 63;
    if (k > i) S[i * SG + k] = 0.0;
  }
  __syncthreads();
}

// Li <- inverse of the lower-triangular 64x64 smem tile S (both stride SG;
// non-zero diagonal over the full tile).  Each warp inverts one 16x16
// diagonal block (one column per lane, substitution in registers), then the
// off-diagonal blocks follow from X21 = -inv(L22) L21 inv(L11) for h = 16, 32
// on the DMMA pipe.  rd: 64 doubles of smem scratch.
__device__ __forceinline__ void trinv(const double* S, double* Li, double* rd, int tid) {
  const int lane = tid & 31, warp = tid >> 5, g = lane >> 2, t = lane & 3;
  for (int idx = tid; idx < T * T; idx += THREADS) Li[(idx >> 6) * SG + (idx & 63)] = 0.0;
  if (tid < T) rd[tid] = rcp_nr(S[tid * SG + tid]);
  __syncthreads();
  {
    const int o = warp * 16, c = lane & 15;
    double wv[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      double s = (i == c) ? 1.0 : 0.0;
#pragma unroll
      for (int k = 0; k < i; ++k) s = fma(-S[(o + i) * SG + o + k], wv[k], s);
      wv[i] = (i >= c) ? s * rd[o + i] : 0.0;
    }
    if (lane < 16) {
#pragma unroll
      for (int i = 0; i < 16; ++i) Li[(o + i) * SG + o + c] = wv[i];
    }
  }
  __syncthreads();
  for (int h = 16; h <= 32; h *= 2) {
    // unit of work: one 16x8 output tile (m16n8) of an h x h product
    const int nblk = T / (2 * h);
    const int units = nblk * (h / 16) * (h / 8);
    // Tmp = L21 * inv(L11) -> scratch in the zero upper block Li[o.., o+h..]
    for (int u = warp; u < units; u += 4) {
      const int bb = u / ((h / 16) * (h / 8)), rem = u % ((h / 16) * (h / 8));
      const int mi = rem / (h / 8), ni = rem % (h / 8), o = bb * 2 * h;
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
      for (int kk = 0; kk < h; kk += 4) {
        const double a0 = S[(o + h + mi * 16 + g) * SG + o + kk + t];
        const double a1 = S[(o + h + mi * 16 + g + 8) * SG + o + kk + t];
        const double b0 = Li[(o + kk + t) * SG + o + ni * 8 + g];
        dmma16x8x4(acc, a0, a1, b0);
      }
      double* dst = Li + (o + mi * 16 + g) * SG + o + h + ni * 8 + 2 * t;
      dst[0] = acc[0];
      dst[1] = acc[1];
      dst[8 * SG] = acc[2];
      dst[8 * SG + 1] = acc[3];
    }
    __syncthreads();
    // X21 = -inv(L22) * Tmp
    for (int u = warp; u < units; u += 4) {
      const int bb = u / ((h / 16) * (h / 8)), rem = u % ((h / 16) * (h / 8));
      const int mi = rem / (h / 8), ni = rem % (h / 8), o = bb * 2 * h;
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
      for (int kk = 0; kk < h; kk += 4) {
        const double a0 = Li[(o + h + mi * 16 + g) * SG + o + h + kk + t];
        const double a1 = Li[(o + h + mi * 16 + g + 8) * SG + o + h + kk + t];
        const double b0 = Li[(o + kk + t) * SG + o + h + ni * 8 + g];
        dmma16x8x4(acc, a0, a1, b0);
      }
      double* dst = Li + (o + h + mi * 16 + g) * SG + o + ni * 8 + 2 * t;
      dst[0] = -acc[0];
      dst[1] = -acc[1];
      dst[8 * SG] = -acc[2];
      dst[8 * SG + 1] = -acc[3];
    }
    __syncthreads();
    for (int idx = tid; idx < nblk * h * h; idx += THREADS) {
      const int bb = idx / (h * h), rem = idx % (h * h);
      const int i = rem / h, c = rem % h, o = bb * 2 * h;
      Li[(o + i) * SG + o + h + c] = 0.0;
    }
    __syncthreads();
  }
}

}  // namespace tile
}  // namespace bta
