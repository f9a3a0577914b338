// Tile-DAG kernel for one block column ("panel") of the BTA Cholesky.
//
// The panel of step i is the tall matrix [D_i; L_i; Ab_i] (tile rows of the
// diagonal block, of the block below it, and of the arrow), cut into 64x64
// tiles with nq = ceil(b/64) tile columns, and factored in place:
//   X(p, r) = (A(p, r) - sum_{k<r} X(p, k) X(r, k)^T) Linv_r^T   (p > r)
//   L_rr    = chol(A(r, r) - sum_{k<r} X(r, k) X(r, k)^T),  Linv_r = L_rr^-1
// When Lprev / Abprev are given, the previous block column's Schur update
// (D -= Lprev Lprev^T, Ab -= Abprev Lprev^T) is applied by one dependency-free
// task per tile, queued a few tile columns ahead of the tile's own task, and
// a tip task applies T -= Ab Ab^T, so a whole BTA step is one launch.
// The critical path -- X(q, q-1), the last update of tile (q, q), POTRF(q) and
// Linv_q for q = 0..nq-1 -- runs in one dedicated "chain" CTA per instance that
// keeps Linv_{q-1} in shared memory.  Every other tile is one left-looking task
// claimed from a queue in a fixed topological order by the remaining
// persistent CTAs: it streams its row strips through a shared-memory ring,
// accumulating in registers as the source columns become final, then applies
// its TRSM (or hands the tile to the chain).  Dependencies are release/acquire flags per tile; every wait is
// bounded and sets an abort flag instead of hanging.
// An FP64 factorisation can also run whole in one launch: the queues of all
// block columns one after the other, each column's previous-column tasks
// waiting on the previous column's tiles, the chain CTA of an instance
// running its columns in order (PanelBatch::cols; off unless
// DALIA_B200_PANEL_PERSIST=1, as it measured no faster than column launches).
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
  const double* Lprev;   // factor block below the previous diagonal block (its
                         // rows are this D's rows), or nullptr
  const double* Abprev;  // previous arrow block, or nullptr
  double* Ttip;          // arrow tip (a x a, a <= 64) updated by this panel, or nullptr
  int* upd;      // [nrows_t * nq] chain input tile accumulated (set to 1)
  int* flag;     // [nrows_t * nq] tile final (X computed; diagonal: Linv ready)
  int* prv;      // [nrows_t * nq] previous column's update applied (when Lprev)
  // A factorisation in one launch: the previous column's flags (its block
  // below and arrow rows become Lprev / Abprev while this launch runs, so
  // the previous-column tasks wait for their source tiles), and the
  // instance's count of finished tip tasks (the tip tasks of consecutive
  // columns update T one after the other).  nullptr in a one-column launch.
  const int* prev_flag;
  int* tip_seq;
  unsigned long long* info;  // min failing pivot (1-based global index)
  long long pivot_base;      // global row index of D's first row
  int b, a, nq, nrows_t;
  int col;       // block column index (the tip tasks' order)
};

constexpr int PANEL_MAXI = 64;

struct PanelBatch {
  int ninst;
  int ntasks;
  const int4* tasks;  // queue tasks {inst, kind, p, r}: one per tile (p, r)
  int* counter;       // [0] next queue task, [1] next chain role
  int* abort_flag;    // set on a timed-out wait (all later waits return)
  PanelInst inst[PANEL_MAXI];
  // Whole factorisation in one launch (cols != nullptr): one descriptor per
  // (instance, block column) in device memory, instance k's columns at
  // cols[col_start[k] .. col_start[k + 1]); task x fields index cols, and
  // chain CTA k runs its instance's columns in order.
  const PanelInst* cols;
  int col_start[PANEL_MAXI + 1];
};

// Queue task kinds: the left-looking accumulation into a tile that the chain
// CTA finishes (the diagonal tile, without its last update; the tile below
// the diagonal), or accumulation followed by the TRSM with the inverse of the
// column's diagonal tile.
// TASK_TIP subtracts the panel's arrow rows from the tip: T -= X_a X_a^T.
// TASK_PREV applies the previous block column's term to one tile (no waits).
enum : int { TASK_AGG_DIAG = 3, TASK_AGG_SUB = 4, TASK_AGG_TRSM = 5, TASK_TIP = 6, TASK_PREV = 7 };

// Tile columns by which the previous-column tasks run ahead of the tiles'
// own tasks in the queue (default; the autotuner tries others).
constexpr int PREV_LOOKAHEAD = 2;

// Number of tile rows of a panel (diag rows, lower rows, arrow rows).
inline int panel_rows(int b, int a, bool has_L) {
  const int nq = (b + 63) / 64;
  return nq + (has_L ? nq : 0) + (a + 63) / 64;
}

// Queue orders: column by column (the chain's inputs of column r at its
// head), or the chain's critical tasks two columns ahead of the bulk.
enum : int { PANEL_ORDER_COLUMN = 0, PANEL_ORDER_CHAIN_AHEAD = 1 };

// Queue tasks (every tile except those the chain finishes) of all instances.
void panel_tasks(const std::vector<PanelInst>& insts, std::vector<int4>& tasks, int lookahead = PREV_LOOKAHEAD,
                 int order = PANEL_ORDER_COLUMN);

// Queue of a whole factorisation in one launch: the one-column queues of
// block columns 0, 1, ... one after the other (column c holding the
// instances with more than c columns), task x = the column's index in the
// descriptor array (col_start[k] + c for instance k).  cols[k] describes
// instance k's columns' shape (b, a, tip); n[k] its number of columns.
void panel_tasks_persist(const std::vector<PanelInst>& shapes, const std::vector<int>& n,
                         const std::vector<int>& col_start, std::vector<int4>& tasks, int lookahead, int order);

// Launch one panel batch.  The counters of every instance, batch.counter[0..1]
// and the abort flag must be zero-initialised by the caller.
int panel_launch(const PanelBatch& batch, int grid, cudaStream_t stream);

int panel_grid_size();
// CTAs per SM that fit (the largest grid is panel_grid_size()).
int panel_ctas_per_sm();

}  // namespace bta
