// Internal host-side interfaces between the kernel translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace bta {

struct SweepArgs {
  const double* D;     // n x b x b factor diagonal blocks
  const double* L;     // (n-1) x b x b factor sub-diagonal blocks
  const double* Ab;    // n x a x b factor arrow blocks
  const double* Linv;  // n*nq inverses of the 64x64 diagonal tiles
  double* x;           // right-hand side in, solution out (n*b + a)
  int* flags;          // n*nq, zeroed before the launch
  int* counter;        // zeroed before the launch
  int* abort_flag;
  int n, b, a, nq;
  int trans;  // 0: L y = x,  1: L^T x = y
};

constexpr int SWEEP_MAXI = 32;

// Several independent sweeps in one launch; tasks of the instances interleave
// (task t belongs to instance t % count), each instance keeps its own order.
struct SweepBatch {
  int count;
  int total;  // count * max_tasks
  int* counter;
  SweepArgs inst[SWEEP_MAXI];
};

int diag_tile_inverses(const double* D, int n, int b, double* out, cudaStream_t s);
int sweep_launch_batched(SweepBatch& B, cudaStream_t s);
// part: n * a doubles of scratch.
int arrow_forward(const double* Ab, const double* T, double* x, int n, int b, int a, double* part, cudaStream_t s);
int arrow_backward(const double* T, double* x, int n, int b, int a, cudaStream_t s);

// Sweeps with precomputed block inverses V (solve_inv.cu): count instances,
// x[k] of length n[k] b[k] + a[k].  sweep_inv_steps runs steps [s0, s1) in
// processing order (forward: block i = s; backward: block i = n - 1 - s) as
// one persistent cooperative launch per PS chunk of instances, with V[k]
// holding the inverse of block vlo[k] (vlo == nullptr: 0) and those after
// it; work holds sweep_inv_work_total(...) doubles.  The arrowhead steps are
// not included.  sweep_inv_batched is a whole sweep with every block inverse
// supplied, arrowhead included; its work also holds max_k n[k] a[k] more
// doubles.  abort_flag is raised when a grid barrier's bounded wait runs out.
size_t sweep_inv_work(int n, int b, int a);
size_t sweep_inv_work_total(int count, const int* n, const int* b, const int* a);
int sweep_inv_steps(int count, const int* n, const int* b, const int* a, const double* const* L,
                    const double* const* Ab, const double* const* V, const int* vlo, double* const* x, int trans,
                    int s0, int s1, double* work, int* abort_flag, cudaStream_t s);
int sweep_inv_batched(int count, const int* n, const int* b, const int* a, const double* const* L,
                      const double* const* Ab, const double* const* T, const double* const* V, double* const* x,
                      int trans, double* work, int* abort_flag, cudaStream_t s);

// Full inverses of the lower-triangular factor blocks D[i0..i1) -> out
// (i1-i0 blocks of b x b, zeros above the diagonal); tile_inv holds the
// inverses of their diagonal tiles (from diag_tile_inverses, same indexing).
int block_trtri(const double* D, const double* tile_inv, int i0, int i1, int b, double* out, cudaStream_t s);

// 2 * sum log(diag) over the n diagonal factor blocks (+ the tip when a > 0),
// written to out (device).  part: n+1 doubles of scratch.
int logdet_launch(const double* D, int n, int b, const double* T, int a, double* part, double* out,
                  cudaStream_t s);

}  // namespace bta
