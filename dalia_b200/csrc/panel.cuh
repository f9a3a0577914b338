// Tile-DAG kernel for one block column ("panel") of the BTA Cholesky.
//
// The panel of step i is the tall matrix [D_i; L_i; Ab_i] (tile rows of the
// diagonal block, of the block below it, and of the arrow), cut into 64x64
// tiles with nq = ceil(b/64) tile columns.  It is factored in place by
//   POTRF(q)       D_i[q][q] <- chol(D_i[q][q]);  Linv_q <- its inverse
//   TRSM(p, q)     tile(p, q) <- tile(p, q) * Linv_q^T           (p below q)
//   UPDATE(p,r,q)  tile(p, r) <- tile(p, r) - tile(p, q) tile(r, q)^T
// The critical path -- TRSM(q, q-1), UPDATE(q, q, q-1), POTRF(q) for
// q = 0..nq-1 -- runs in one dedicated "chain" CTA per instance that keeps the
// inverse of the previous diagonal tile in shared memory.  Every other task is
// claimed from a queue in a fixed topological order by the remaining
// persistent CTAs.  Dependencies are tracked per tile with release/acquire
// counters; every wait is bounded and sets an abort flag instead of hanging.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <vector>

namespace bta {

struct PanelInst {
  double* D;     // b x b, ld = b (diagonal block; tip block for the arrow tip)
  double* L;     // b x b block below D, or nullptr
  double* Ab;    // a x b arrow rows, or nullptr
  double* Linv;  // workspace: nq tiles of 64x64 (inverses of the diagonal tiles)
  int* upd;      // [nrows_t * nq] number of column updates applied to a tile
  int* flag;     // [nrows_t * nq] tile final (potrf / trsm done)
  unsigned long long* info;  // min failing pivot (1-based global index)
  long long pivot_base;      // global row index of D's first row
  int b, a, nq, nrows_t;
};

constexpr int PANEL_MAXI = 64;

struct PanelBatch {
  int ninst;
  int ntasks;
  const int4* tasks;  // queue tasks {inst, kind, p, (r << 16) | q}
  int* counter;       // [0] next queue task, [1] next chain role
  int* abort_flag;    // set on a timed-out wait (all later waits return)
  PanelInst inst[PANEL_MAXI];
};

enum : int { TASK_POTRF = 0, TASK_TRSM = 1, TASK_UPDATE = 2 };

// Number of tile rows of a panel (diag rows, lower rows, arrow rows).
inline int panel_rows(int b, int a, bool has_L) {
  const int nq = (b + 63) / 64;
  return nq + (has_L ? nq : 0) + (a + 63) / 64;
}

// Queue tasks (everything except the chain) of all instances, stage by stage.
void panel_tasks(const std::vector<PanelInst>& insts, std::vector<int4>& tasks);

// Launch one panel batch.  The counters of every instance, batch.counter[0..1]
// and the abort flag must be zero-initialised by the caller.
int panel_launch(const PanelBatch& batch, int grid, cudaStream_t stream);

int panel_grid_size();

}  // namespace bta
