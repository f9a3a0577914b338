/*
 * dalia_bta.h -- C ABI of the B200 block-tridiagonal-arrowhead (BTA) solver.
 *
 * Drop-in for the structured-solver path of DALIA (affifboudaoud/DALIA).  The
 * reference keeps the matrix in four dense FP64 arrays and calls Serinv:
 *
 *   D  [n][b][b]   diagonal blocks          (src/dalia/solvers/structured_solver.py:38-41)
 *   L  [n-1][b][b] sub-diagonal blocks      (structured_solver.py:42-49)
 *   Ab [n][a][b]   arrow bottom blocks      (structured_solver.py:53-56)
 *   T  [a][a]      arrow tip                (structured_solver.py:57-60)
 *
 * All arrays are C-contiguous row-major FP64 in device memory owned by the
 * caller; every routine works in place, stream-ordered on the handle's stream.
 * Return value: BTA_OK or an error code (bta_error_string).  A handle owns only
 * scratch memory and cached launch plans; use one handle per stream.
 */
#ifndef DALIA_BTA_H
#define DALIA_BTA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BTA_OK 0
#define BTA_ERR_INVALID 1   /* invalid argument (sizes, null pointers, sparsity) */
#define BTA_ERR_CUDA 2      /* CUDA runtime error                                 */
#define BTA_ERR_NOT_SPD 3   /* non-positive pivot: matrix not positive definite   */
#define BTA_ERR_TIMEOUT 4   /* a bounded device-side wait gave up                 */
#define BTA_ERR_ALLOC 5     /* scratch allocation failed                          */

typedef struct bta_context* bta_handle_t;

/* Handle life cycle.  The handle binds to the current CUDA device; every call
 * on it makes that device current for its duration (the caller's current
 * device is restored). */
int bta_create(bta_handle_t* handle);
int bta_destroy(bta_handle_t handle);
/* stream: a cudaStream_t (NULL = legacy default stream). */
int bta_set_stream(bta_handle_t handle, void* stream);
const char* bta_error_string(int code);
/* Bytes of scratch currently held by the handle. */
size_t bta_workspace_bytes(bta_handle_t handle);

/*
 * In-place BTA Cholesky Q = L L^T.  Replaces Serinv's
 *   pobtaf(A_diagonal_blocks, A_lower_diagonal_blocks, A_arrow_bottom_blocks, A_arrow_tip_block)
 * called at src/dalia/solvers/structured_solver.py:83-88.
 * On exit D holds the lower factors (zeros above the diagonal), L, Ab and T the
 * factor blocks.  a = 0 gives the BT factorisation (pobtf, :90-93); Ab and T
 * may then be NULL.  If info != NULL the call clears the handle's status,
 * synchronises the stream and writes 0 on success or the 1-based global index
 * of the first non-positive pivot (then returns BTA_ERR_NOT_SPD).  With
 * info == NULL the call is asynchronous and the status accumulates on the
 * handle until bta_get_status / bta_reset_status.
 */
int bta_pobtaf(bta_handle_t h, int64_t n, int64_t b, int64_t a, double* D, double* L, double* Ab, double* T,
               int64_t* info);

/*
 * Batched forms: count independent BTA matrices (instance k has sizes n[k],
 * b[k], a[k] and arrays D[k], L[k], Ab[k], T[k]; L/Ab/T entries may be NULL
 * where unused) factored / selected-inverted together, block column by block
 * column, so that the critical paths of all instances run concurrently in one
 * launch.  This is the batched launch over the theta points of a
 * finite-difference stencil or a line search (the reference evaluates them one
 * after another, src/dalia/core/dalia.py:558-564).  For the batched
 * factorisation, info = k * 2^40 + pivot identifies instance k.  The batched
 * sweep takes up to 32 instances, each with its own right-hand side rhs[k].
 */
int bta_pobtaf_batched(bta_handle_t h, int count, const int64_t* n, const int64_t* b, const int64_t* a,
                       double* const* D, double* const* L, double* const* Ab, double* const* T, int64_t* info);
int bta_pobtas_batched(bta_handle_t h, int count, const int64_t* n, const int64_t* b, const int64_t* a,
                       const double* const* D, const double* const* L, const double* const* Ab,
                       const double* const* T, double* const* rhs, int trans);
int bta_pobtasi_batched(bta_handle_t h, int count, const int64_t* n, const int64_t* b, const int64_t* a,
                        double* const* D, double* const* L, double* const* Ab, double* const* T);

/*
 * Arithmetic of the selected inversion's block products (no counterpart in
 * the reference, which computes in the precision of its arrays):
 * BTA_PREC_FP64 -- FP64 on the DMMA tensor pipe (the default everywhere);
 * BTA_PREC_TF32X3 -- FP32-class: every FP64 operand is split into two TF32
 * values and the products are accumulated in FP32 on the tcgen05 tensor
 * cores (relative error of the selected inverse ~1e-5, growing with b: the
 * tensor cores accumulate FP32 with truncation);
 * BTA_PREC_I8SLICE -- every operand row / column scaled by a power of two and
 * cut into seven signed 7-bit digits; the digit products are accumulated
 * exactly in INT32 on the tcgen05 tensor cores (kind::i8) and recombined in
 * FP64 (relative error ~1e-14 against sum |a||b|; block sizes up to 19000).
 * The factor, the diagonal-block inverses and all storage stay FP64.
 */
#define BTA_PREC_FP64 0
#define BTA_PREC_TF32X3 1
#define BTA_PREC_I8SLICE 2
int bta_pobtasi_batched_ex(bta_handle_t h, int count, const int64_t* n, const int64_t* b, const int64_t* a,
                           double* const* D, double* const* L, double* const* Ab, double* const* T,
                           int precision);

/*
 * The batched factorisation with the previous block column's Schur update
 * (D_i -= L_{i-1} L_{i-1}^T, Ab_i -= Ab_{i-1} L_{i-1}^T) in the given
 * BTA_PREC_* arithmetic: with BTA_PREC_I8SLICE or BTA_PREC_TF32X3 it runs as
 * one grouped tensor-core GEMM per block column between the panel launches,
 * while the diagonal-block POTRF, the triangular solves inside the panel,
 * the arrow tip and every stored block stay FP64.  BTA_PREC_FP64 is
 * bta_pobtaf_batched.  No counterpart in the reference (Serinv computes in
 * the precision of its arrays).
 */
int bta_pobtaf_batched_ex(bta_handle_t h, int count, const int64_t* n, const int64_t* b, const int64_t* a,
                          double* const* D, double* const* L, double* const* Ab, double* const* T, int64_t* info,
                          int precision);

/*
 * Inverses of the diagonal factor blocks, V[k][i] = L_ii^-1 (n[k] blocks of
 * b[k] x b[k], lower triangular, zeros above the diagonal) into caller
 * buffers; with them a triangular sweep is n dependent steps of two
 * bandwidth-bound matrix-vector products (bta_pobtas_inv_batched: same
 * trans and rhs conventions as bta_pobtas_batched; D is not read), and the
 * selected inversion skips its own block inversion
 * (bta_pobtasi_batched_v; V == NULL, or V[k] == NULL for one instance,
 * computes them as bta_pobtasi_batched_ex does: chunk by chunk as the
 * recurrence reaches them, in at most 2 GiB of workspace per instance).
 * No counterpart in the reference: Serinv's pobtas solves with the factor
 * blocks directly.
 */
int bta_block_inverses(bta_handle_t h, int count, const int64_t* n, const int64_t* b, const double* const* D,
                       double* const* V);
int bta_pobtas_inv_batched(bta_handle_t h, int count, const int64_t* n, const int64_t* b, const int64_t* a,
                           const double* const* L, const double* const* Ab, const double* const* T,
                           const double* const* V, double* const* rhs, int trans);
int bta_pobtasi_batched_v(bta_handle_t h, int count, const int64_t* n, const int64_t* b, const int64_t* a,
                          double* const* D, double* const* L, double* const* Ab, double* const* T,
                          const double* const* V, int precision);

/*
 * C = beta C + alpha op(A) op(B) (row-major FP64; op(A)[m][k] = A[m*lda+k], or
 * A[k*lda+m] with a_trans; op(B)[k][n] = B[n*ldb+k], or B[k*ldb+n] with b_kn)
 * with the library's grouped GEMM in the given BTA_PREC_* arithmetic, on the
 * handle's stream.  lower_only: compute and write only C[m][n] with m >= n
 * (M == N); mirror (with lower_only): also write C[n][m].  The block-product
 * kernel of the factorisation and selected inversion, exported for testing
 * and for callers that need it; no counterpart in the reference.
 */
int bta_gemm(bta_handle_t h, int precision, int64_t M, int64_t N, int64_t K, double alpha, const double* A,
             int64_t lda, int a_trans, const double* B, int64_t ldb, int b_kn, double beta, double* C, int64_t ldc,
             int lower_only, int mirror);

/*
 * One triangular sweep with the factor, in place on rhs (length n*b + a).
 * trans = 0: solve L y = rhs (Serinv trans="N"); trans = 1: solve L^T x = rhs
 * (trans="C").  Replaces pobtas (structured_solver.py:112-127) and, with a = 0,
 * pobts (:129-140).
 */
int bta_pobtas(bta_handle_t h, int64_t n, int64_t b, int64_t a, const double* D, const double* L,
               const double* Ab, const double* T, double* rhs, int trans);

/*
 * In-place selected inversion of the factor: afterwards D, L, Ab, T hold the
 * corresponding blocks of Q^{-1} (D full symmetric).  Replaces pobtasi
 * (structured_solver.py:176-181) and, with a = 0, pobtsi (:183-186).
 */
int bta_pobtasi(bta_handle_t h, int64_t n, int64_t b, int64_t a, double* D, double* L, double* Ab, double* T);

/*
 * log det Q = 2 (sum_i sum_k log D_i[k][k] + [include_tip] sum_k log T[k][k])
 * from the factor (SerinvSolver.logdet, structured_solver.py:151-166; the tip
 * is excluded for sparsity "bt").  out_device (may be NULL) receives the value
 * stream-ordered; out_host (may be NULL) synchronises and receives it.
 */
int bta_logdet(bta_handle_t h, int64_t n, int64_t b, int64_t a, const double* D, const double* T,
               int include_tip, double* out_device, double* out_host);

/*
 * Synchronise the handle's stream and report the status of the last
 * factorisation: info = 0 or the first non-positive pivot (1-based), return
 * BTA_ERR_NOT_SPD / BTA_ERR_TIMEOUT accordingly.
 */
int bta_get_status(bta_handle_t h, int64_t* info);

/* Clear the handle's status (stream-ordered). */
int bta_reset_status(bta_handle_t h);

/*
 * Scatter a COO matrix (row, col, val; nnz entries, symmetric storage as
 * produced by scipy) into zeroed BTA blocks: the device counterpart of
 * SerinvSolver._spmatrix_to_structured (structured_solver.py:192-390).
 * Entries outside the BTA pattern are ignored; sparsity_bt != 0 keeps only the
 * diagonal and sub-diagonal blocks ("bt").
 */
int bta_scatter_coo(bta_handle_t h, int64_t n, int64_t b, int64_t a, const int64_t* row, const int64_t* col,
                    const double* val, int64_t nnz, int sparsity_bt, double* D, double* L, double* Ab,
                    double* T);

/*
 * Gather the BTA entries at the COO positions (row, col) into out[nnz]
 * (zero outside the pattern): the device counterpart of
 * SerinvSolver._structured_to_spmatrix (structured_solver.py:470-538), which
 * reads the selected inverse at the lower-triangle pattern of a given matrix.
 */
int bta_gather_coo(bta_handle_t h, int64_t n, int64_t b, int64_t a, const int64_t* row, const int64_t* col,
                   int64_t nnz, int sparsity_bt, const double* D, const double* L, const double* Ab, const double* T,
                   double* out);

/*
 * bta_pobtaf without any device allocation.  No counterpart in the reference:
 * it exists for callers that may not call cudaMalloc/cudaFree themselves or
 * through a library -- code inside a framework whose pool allocator owns the
 * GPU's memory, or latency-critical loops that cannot afford cudaFree's
 * device-wide synchronisation.  Same arguments and results as bta_pobtaf, but
 * no handle: the work runs on `stream` (a cudaStream_t, NULL = legacy default
 * stream) and all scratch lives in one fixed 2 MiB device array inside the
 * library (bta_noalloc_scratch_bytes), which every GPU that loads the library
 * holds until the process exits.  Sizes: b <= BTA_NOALLOC_MAX_B and
 * a <= BTA_NOALLOC_MAX_A (any n); larger problems are rejected with
 * BTA_ERR_INVALID before any GPU work.  The first call on a device looks up
 * the array's device address (cudaGetSymbolAddress).  With info != NULL the call synchronises the
 * stream and reports a non-positive pivot (info, BTA_ERR_NOT_SPD) or a
 * timed-out device wait (BTA_ERR_TIMEOUT).  With info == NULL it returns
 * without waiting; the status stays in the array until the next call clears
 * it, and bta_noalloc_get_status (same stream) synchronises and reads it.
 * All calls share the array and each clears what must start at zero, so calls
 * whose work overlaps on the GPU (other streams, other threads) race.
 */
#define BTA_NOALLOC_MAX_B 2048
#define BTA_NOALLOC_MAX_A 128
int bta_pobtaf_noalloc(int64_t n, int64_t b, int64_t a, double* D, double* L, double* Ab, double* T, int64_t* info,
                       void* stream);
int bta_noalloc_get_status(int64_t* info, void* stream);
size_t bta_noalloc_scratch_bytes(void);

/*
 * Launch accounting (no counterpart in the reference, which has no native
 * kernels): total kernel launches of this library in the process, and
 * optional per-category device time from CUDA events recorded around every
 * launch on its stream.  Categories: 0 panel factorisation, 1 GEMM, 2 solve
 * sweeps, 3 block inverses, 4 other, 5 digit pre-pass of the 8-bit-slice
 * GEMM, 6 the factorisation's Schur-update GEMMs (with their pre-pass) when
 * they run outside the panel kernel (bta_pobtaf_batched_ex).  bta_prof_enable(1) creates the
 * events beforehand (for about 8000 launches), so a timed region pays no
 * event creation; bta_prof_mask limits the events to the categories whose
 * bits are set (default: all), since events around every launch slow a step
 * of many small launches measurably.  bta_prof_read synchronises on the
 * recorded events, returns the accumulated milliseconds and launch counts
 * (8 entries each) and clears them.
 */
long long bta_launch_count(void);
int bta_prof_enable(int on);
int bta_prof_mask(int mask);
int bta_prof_read(double* ms, long long* counts);

/*
 * Task queue of one block-column launch of the factorisation, for tests of
 * its order (no counterpart in the reference).  For count matrices (at most
 * 64) with block size b[k], arrow size a[k] and flags[k] (bit 0: a block
 * below the diagonal block, bit 1: the previous block column's Schur term,
 * bit 2: the previous arrow block, bit 3: the arrow tip), writes up to cap
 * tasks {matrix, kind, tile row, tile column} as four ints each to out and
 * their number to *n_out (kinds: 3 diagonal tile, 4 tile below it, 5 tile with
 * its triangular solve, 6 arrow tip, 7 previous-column term).  Host code only:
 * needs no device.  BTA_ERR_INVALID when cap is too small.
 */
int bta_panel_task_list(int count, const int* b, const int* a, const int* flags, int* out, int cap, int* n_out);
/* The same with the queue lookahead and order the autotuner chooses from:
 * lookahead = tile columns by which the previous-column terms run ahead
 * (bta_panel_task_list uses 2); order 0 = column by column with the chain
 * CTA's inputs of column r at its head (bta_panel_task_list), order 1 = the
 * solve of tile (r+2, r) and the chain's inputs of step r+2 ahead of the
 * rest of column r. */
int bta_panel_task_list_ex(int count, const int* b, const int* a, const int* flags, int lookahead, int order,
                           int* out, int cap, int* n_out);
/* The queue of a whole FP64 factorisation in one launch (what
 * bta_pobtaf_batched runs when every arrow is at most 64 rows and the
 * environment variable DALIA_B200_PANEL_PERSIST is 1): the
 * one-column queues of block columns 0, 1, ... one after the other, matrix k
 * having n[k] block columns (flags[k] bit 3: arrow tip); task field 0 is the
 * column's global index (matrix k's column c is sum_{j<k} n[j] + c).  In it
 * a previous-column task waits for its source tiles of the previous column,
 * and the tip tasks of a matrix's columns run in column order. */
int bta_panel_task_list_all(int count, const int* b, const int* a, const int* flags, const int* n, int lookahead,
                            int order, int* out, int cap, int* n_out);

/*
 * Autotuner (no counterpart in the reference).  Launch configurations of the
 * factorisation's block-column kernel (queue lookahead, resident CTAs per SM)
 * and of the persistent sweep (CTAs per SM, row segments) are tuned online:
 * the first launches of a new launch shape try every candidate (twice for
 * the factorisation's block columns, once for a sweep) on the real work,
 * timed by CUDA events, and the fastest is kept for that shape on that
 * device; the 8-bit-slice GEMM's output tile width (64, or 32 with two
 * tensor-memory accumulator sets) is chosen the same way per launch shape.
 * DALIA_B200_TUNE=0 turns it off; DALIA_B200_TUNE_CACHE=<file> reads earlier
 * decisions from, and appends new ones to, that file;
 * DALIA_B200_TUNE_FORCE="family=candidate,..." pins candidates (families
 * "panel", "sweep", "gemm_i8").
 * bta_tune_report writes one line per decision ("family|device|shape
 * best=<candidate> ms=<time of each candidate>") into buf (cap bytes, NUL
 * terminated) and its full length to *len; BTA_ERR_INVALID when truncated.
 */
int bta_tune_report(char* buf, size_t cap, size_t* len);
/* Launch shapes whose candidates are still being tried. */
int bta_tune_pending(void);

#ifdef __cplusplus
}
#endif

#endif /* DALIA_BTA_H */
