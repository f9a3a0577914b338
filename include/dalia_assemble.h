/*
 * dalia_assemble.h -- device assembly of the spatio-temporal precision in BTA
 * storage and the sparse/vector kernels of the INLA objective (C ABI).
 *
 * These replace the reference's host-side scipy.sparse construction and
 * block scatter of Q_prior(theta) and Q_conditional(theta) = Q_prior - A^T D A:
 *   SpatioTemporalSubModel.construct_Q_prior   src/dalia/submodels/spatio_temporal.py:114-149
 *   Model.construct_Q_prior / construct_Q_conditional   src/dalia/core/model.py:306-423
 *   SerinvSolver._spmatrix_to_bta             src/dalia/solvers/structured_solver.py:252-390
 *   Model.construct_information_vector        src/dalia/core/model.py:425-449
 * All pointers are device pointers; stream is a cudaStream_t; return values
 * are the BTA_* codes of dalia_bta.h.
 */
#ifndef DALIA_ASSEMBLE_H
#define DALIA_ASSEMBLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Dense write of the 2n-1 lower BTA blocks of sum_K coef[blk][K] * K, K in
 * {c0, g1, g2, g3} given on their union CSR pattern (rowptr[b+1], colidx,
 * vals4[nnz][4]).  coef[blk][4]: blk < n diagonal block t, blk >= n the
 * sub-diagonal block (blk-n+1, blk-n).  Every element of D and L is written. */
int bta_assemble_prior(void* stream, int64_t n, int64_t b, const double* coef, const int* rowptr,
                       const int* colidx, const double* vals4, double* D, double* L);

/* base[dst[e]] += dscale * sum_{j in [off[e], off[e+1])} d[obs[j]] * fac[j]
 * (d == NULL means 1): the row-parallel A^T D A contribution per BTA entry. */
int bta_add_entries(void* stream, int64_t nent, const int64_t* dst, const int64_t* off, const int* obs,
                    const double* fac, const double* d, double dscale, double* base);

/* T = prec I + dscale * X^T diag(d) X for the fixed-effect tip (X: nobs x a). */
int bta_arrow_tip(void* stream, int64_t nobs, int64_t a, const double* X, const double* d, double prec,
                  double dscale, double* part, int nparts, double* T);

/* out[blk][K] = <block blk of S, K> over the union pattern (trace terms of the
 * adjoint gradient, tr(S dQ/dtheta) for Kronecker-structured dQ). */
int bta_block_inner(void* stream, int64_t n, int64_t b, const int* rowptr, const int* colidx,
                    const double* vals4, const double* D, const double* L, double* out);

/* out[blk][K] = x_r^T K x_c: block quadratic forms of a vector x (length n*b)
 * with the Kronecker blocks, (r, c) = (t, t) or (t+1, t). */
int bta_block_quad(void* stream, int64_t n, int64_t b, const int* rowptr, const int* colidx,
                   const double* vals4, const double* x, double* out);

/* *out = sum_e w[e] * base[idx[e]] */
int bta_gather_dot(void* stream, int64_t nent, const int64_t* idx, const double* w, const double* base,
                   double* part, int nparts, double* out);

/* y = alpha A x + beta y, CSR A with m rows */
int bta_csr_spmv(void* stream, int64_t m, const int64_t* rowptr, const int* col, const double* val,
                 const double* x, double alpha, double beta, double* y);

/* y = Q x for a symmetric BTA matrix given by its lower blocks */
int bta_symv(void* stream, int64_t n, int64_t b, int64_t a, const double* D, const double* L, const double* Ab,
             const double* T, const double* x, double* y);

/* *out = x . y */
int bta_dot(void* stream, int64_t n, const double* x, const double* y, double* part, int nparts, double* out);

/* y = alpha x + beta y */
int bta_axpby(void* stream, int64_t n, double alpha, const double* x, double beta, double* y);

#ifdef __cplusplus
}
#endif

#endif /* DALIA_ASSEMBLE_H */
