// Grouped FP64 GEMM on the DMMA tensor pipe (sm_100a).
//
//   C = beta * C + sum_s alpha_s * opA_s * opB_s      (up to 3 segments)
//
// Row-major operands.  opA_s[m][k] = A[m*lda+k], or A[k*lda+m] with GF_A_T.
// opB_s[k][n] = B[n*ldb+k] (the "A B^T" form used by every Schur update), or
// B[k*ldb+n] with GF_B_KN.  The K_* flags restrict the summed k-range of an
// output tile to where a triangular operand is non-zero; the skipped region
// must hold zeros.  GC_LOWER computes only tiles on or below the diagonal and
// writes only elements with m >= n; GC_MIRROR also writes C[n][m].
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <vector>

namespace bta {

enum : int {
  GF_A_T = 1,
  GF_B_KN = 2,
  GF_K_GE_M = 4,
  GF_K_LE_M = 8,
  GF_K_GE_N = 16,
  GF_K_LE_N = 32,
};

enum : int {
  GC_LOWER = 1,
  GC_MIRROR = 2,
};

struct GemmSeg {
  const double* A;
  const double* B;
  int lda, ldb, K, flags;
  double alpha;
};

struct GemmProb {
  double* C;
  int ldc, M, N, nseg, cflags, pad_;
  double beta;
  GemmSeg seg[3];
};

constexpr int GEMM_MAXP = 48;

struct GemmBatch {
  int count;
  int tile_start[GEMM_MAXP + 1];
  int tiles_n[GEMM_MAXP];
  GemmProb p[GEMM_MAXP];
};

// Host helper: builds a batch and launches it (splitting into several launches
// when there are more than GEMM_MAXP problems).  Problems in one call must not
// write overlapping C regions.  Returns a cudaError_t.
int gemm_launch(const std::vector<GemmProb>& probs, cudaStream_t stream);

// The same problems with FP32-class arithmetic on the tcgen05 tensor cores
// (split TF32 x3, gemm_tc.cu).  abort_flag (device int) is raised when a
// bounded wait inside the kernel gives up.
int gemm_launch_tc(const std::vector<GemmProb>& probs, cudaStream_t stream, int* abort_flag);

// The same problems with 8-bit digit products accumulated exactly in INT32
// (gemm_i8.cu).  With ws == nullptr only *ws_needed (bytes of workspace for
// the exponents and digit images) is set; otherwise ws must hold that many.
int gemm_launch_i8(const std::vector<GemmProb>& probs, cudaStream_t stream, int* abort_flag, void* ws,
                   size_t ws_bytes, size_t* ws_needed);

inline GemmProb gemm_prob(double* C, int ldc, int M, int N, double beta, int cflags = 0) {
  GemmProb p{};
  p.C = C;
  p.ldc = ldc;
  p.M = M;
  p.N = N;
  p.beta = beta;
  p.cflags = cflags;
  p.nseg = 0;
  return p;
}

inline void gemm_add(GemmProb& p, const double* A, int lda, const double* B, int ldb, int K,
                     double alpha, int flags) {
  GemmSeg& s = p.seg[p.nseg++];
  s.A = A;
  s.B = B;
  s.lda = lda;
  s.ldb = ldb;
  s.K = K;
  s.flags = flags;
  s.alpha = alpha;
}

}  // namespace bta
