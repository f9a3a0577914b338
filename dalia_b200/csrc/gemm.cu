// Grouped FP64 GEMM on the DMMA tensor pipe: 64x64 output tile per CTA,
// 4 warps of 32x32, mma.m16n8k4.f64, 3-stage cp.async pipeline over k-tiles
// of 16.  See gemm.cuh for the operand conventions.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "gemm.cuh"
#include "prof.cuh"

namespace bta {
namespace {

constexpr int BM = 64, BN = 64, BK = 16;
constexpr int SK = BK + 4;  // row stride of a k-contiguous stage (64 rows x 16 k)
constexpr int SM = BM + 4;  // row stride of a row-contiguous stage (16 k x 64 rows)
constexpr int STAGE_OP = BM * SK;
constexpr int STAGES = 3;
constexpr int THREADS = 128;
constexpr size_t SMEM_BYTES = size_t(STAGES) * 2 * STAGE_OP * sizeof(double);
static_assert(STAGE_OP >= BK * SM, "stage buffer too small");

// Stage one 64 x 16 operand slab into shared memory.  Element (r, k) lives at
// P[r*ld + k] when kcontig, else at P[k*ld + r].  Out-of-range elements are
// zero-filled by cp.async (src-size 0).
__device__ __forceinline__ void load_op(double* s, const double* P, int ld, bool kcontig, bool vec,
                                        int r0, int rmax, int k0, int kmax, int tid) {
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int c = tid + j * THREADS;
    if (kcontig) {
      const int r = c >> 3, kc = (c & 7) * 2;
      const int gr = r0 + r, gk = k0 + kc;
      double* d = s + r * SK + kc;
      const bool v0 = gr < rmax && gk < kmax;
      const bool v1 = gr < rmax && gk + 1 < kmax;
      const double* src = P + (size_t)gr * ld + gk;
      if (vec && v1) {
        cp_async16(d, src, true);
      } else {
        cp_async8(d, v0 ? src : P, v0);
        cp_async8(d + 1, v1 ? src + 1 : P, v1);
      }
    } else {
      const int kr = c >> 5, rc = (c & 31) * 2;
      const int gk = k0 + kr, gr = r0 + rc;
      double* d = s + kr * SM + rc;
      const bool v0 = gk < kmax && gr < rmax;
      const bool v1 = gk < kmax && gr + 1 < rmax;
      const double* src = P + (size_t)gk * ld + gr;
      if (vec && v1) {
        cp_async16(d, src, true);
      } else {
        cp_async8(d, v0 ? src : P, v0);
        cp_async8(d + 1, v1 ? src + 1 : P, v1);
      }
    }
  }
}

template <bool AK, bool BKC>
__device__ __forceinline__ void compute_stage(const double* As, const double* Bs, double (&acc)[2][4][4],
                                              int wm, int wn, int g, int t, double alpha) {
#pragma unroll
  for (int kk = 0; kk < BK; kk += 4) {
    double a[2][2], b[4];
#pragma unroll
    for (int mi = 0; mi < 2; ++mi) {
      const int r = wm * 32 + mi * 16 + g;
      if (AK) {
        a[mi][0] = As[r * SK + kk + t];
        a[mi][1] = As[(r + 8) * SK + kk + t];
      } else {
        a[mi][0] = As[(kk + t) * SM + r];
        a[mi][1] = As[(kk + t) * SM + r + 8];
      }
      a[mi][0] *= alpha;
      a[mi][1] *= alpha;
    }
#pragma unroll
    for (int ni = 0; ni < 4; ++ni) {
      const int c = wn * 32 + ni * 8 + g;
      b[ni] = BKC ? Bs[c * SK + kk + t] : Bs[(kk + t) * SM + c];
    }
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) dmma16x8x4(acc[mi][ni], a[mi][0], a[mi][1], b[ni]);
  }
}

template <bool AK, bool BKC>
__device__ __forceinline__ void run_segment(double* smem, const GemmSeg& s, int M, int N, int m0, int n0,
                                            double (&acc)[2][4][4], int tid, int wm, int wn, int g, int t) {
  int kmin = 0, kmax = s.K;
  if (s.flags & GF_K_GE_M) kmin = max(kmin, m0);
  if (s.flags & GF_K_GE_N) kmin = max(kmin, n0);
  if (s.flags & GF_K_LE_M) kmax = min(kmax, m0 + BM);
  if (s.flags & GF_K_LE_N) kmax = min(kmax, n0 + BN);
  const int kb = kmin & ~(BK - 1);
  if (kmax <= kb) return;
  const int nk = (kmax - kb + BK - 1) / BK;
  const bool vecA = ((s.lda & 1) == 0) && ((reinterpret_cast<uintptr_t>(s.A) & 15) == 0);
  const bool vecB = ((s.ldb & 1) == 0) && ((reinterpret_cast<uintptr_t>(s.B) & 15) == 0);
  double* As = smem;
  double* Bs = smem + STAGES * STAGE_OP;
  auto issue = [&](int stage, int kt) {
    const int k0 = kb + kt * BK;
    load_op(As + stage * STAGE_OP, s.A, s.lda, AK, vecA, m0, M, k0, kmax, tid);
    load_op(Bs + stage * STAGE_OP, s.B, s.ldb, BKC, vecB, n0, N, k0, kmax, tid);
  };
#pragma unroll
  for (int st = 0; st < STAGES - 1; ++st) {
    if (st < nk) issue(st, st);
    cp_async_commit();
  }
  for (int kt = 0; kt < nk; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    const int nxt = kt + STAGES - 1;
    if (nxt < nk) issue(nxt % STAGES, nxt);
    cp_async_commit();
    const int cur = kt % STAGES;
    compute_stage<AK, BKC>(As + cur * STAGE_OP, Bs + cur * STAGE_OP, acc, wm, wn, g, t, s.alpha);
  }
  cp_async_wait<0>();
  __syncthreads();
}

__global__ void __launch_bounds__(THREADS) gemm_f64_kernel(const __grid_constant__ GemmBatch batch) {
  extern __shared__ __align__(16) double smem[];
  const int bid = blockIdx.x;
  int pi = 0;
  while (pi + 1 < batch.count && bid >= batch.tile_start[pi + 1]) ++pi;
  const GemmProb& P = batch.p[pi];
  const int local = bid - batch.tile_start[pi];
  int tm, tn;
  if (P.cflags & GC_LOWER) {
    tm = (int)((sqrt(8.0 * local + 1.0) - 1.0) * 0.5);
    while ((tm + 1) * (tm + 2) / 2 <= local) ++tm;
    while (tm * (tm + 1) / 2 > local) --tm;
    tn = local - tm * (tm + 1) / 2;
  } else {
    tm = local / batch.tiles_n[pi];
    tn = local % batch.tiles_n[pi];
  }
  const int m0 = tm * BM, n0 = tn * BN;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1, g = lane >> 2, t = lane & 3;

  double acc[2][4][4];
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[mi][ni][e] = 0.0;

  for (int si = 0; si < P.nseg; ++si) {
    const GemmSeg& s = P.seg[si];
    const bool ak = !(s.flags & GF_A_T);
    const bool bk = !(s.flags & GF_B_KN);
    if (ak && bk) run_segment<true, true>(smem, s, P.M, P.N, m0, n0, acc, tid, wm, wn, g, t);
    else if (ak) run_segment<true, false>(smem, s, P.M, P.N, m0, n0, acc, tid, wm, wn, g, t);
    else if (bk) run_segment<false, true>(smem, s, P.M, P.N, m0, n0, acc, tid, wm, wn, g, t);
    else run_segment<false, false>(smem, s, P.M, P.N, m0, n0, acc, tid, wm, wn, g, t);
  }

  const bool lower = P.cflags & GC_LOWER;
  const bool mirror = P.cflags & GC_MIRROR;
  const double beta = P.beta;
  double* C = P.C;
  const int ldc = P.ldc;
#pragma unroll
  for (int mi = 0; mi < 2; ++mi) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int row = m0 + wm * 32 + mi * 16 + g + h * 8;
      if (row >= P.M) continue;
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int col = n0 + wn * 32 + ni * 8 + 2 * t + e;
          if (col >= P.N) continue;
          if (lower && col > row) continue;
          double v = acc[mi][ni][h * 2 + e];
          double* dst = C + (size_t)row * ldc + col;
          if (beta != 0.0) v += beta * *dst;
          *dst = v;
          if (mirror && col < row) C[(size_t)col * ldc + row] = v;
        }
      }
    }
  }
}

}  // namespace

int gemm_launch(const std::vector<GemmProb>& probs, cudaStream_t stream) {
  {
    const int e = ensure_smem_attr(reinterpret_cast<const void*>(gemm_f64_kernel), (int)SMEM_BYTES);
    if (e != cudaSuccess) return (cudaError_t)e;
  }
  size_t i = 0;
  while (i < probs.size()) {
    GemmBatch b;
    std::memset(&b, 0, sizeof(b));
    int total = 0;
    b.count = 0;
    for (; i < probs.size() && b.count < GEMM_MAXP; ++i) {
      const GemmProb& p = probs[i];
      if (p.M <= 0 || p.N <= 0) continue;
      const int tmn = (p.M + BM - 1) / BM, tnn = (p.N + BN - 1) / BN;
      int tiles;
      if (p.cflags & GC_LOWER) {
        if (p.M != p.N) return cudaErrorInvalidValue;
        tiles = tmn * (tmn + 1) / 2;
      } else {
        tiles = tmn * tnn;
      }
      b.p[b.count] = p;
      b.tiles_n[b.count] = tnn;
      b.tile_start[b.count] = total;
      total += tiles;
      b.count++;
    }
    if (b.count == 0) continue;
    b.tile_start[b.count] = total;
    {
      bta::ProfScope _ps(bta::PROF_GEMM, stream);
      gemm_f64_kernel<<<total, THREADS, SMEM_BYTES, stream>>>(b);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace bta
