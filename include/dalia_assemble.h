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

/* y[0 : n*b] = alpha * Q_st x + beta * y[0 : n*b]: the spatio-temporal block
 * applied through its Kronecker structure (coef and the union pattern as in
 * bta_assemble_prior); the product -Q_prior x of the reference's information
 * vector (src/dalia/core/model.py:425-449) without forming Q_prior. */
int bta_kron_symv(void* stream, int64_t n, int64_t b, const double* coef, const int* rowptr, const int* colidx,
                  const double* vals4, const double* x, double alpha, double beta, double* y);

/* Multivariate forms (nv variates interleaved per time step, block size
 * b = nv ns; the reference's CoregionalModel permutation,
 * src/dalia/models/coregional_model.py:770-797): coef[blk][v][w][K] gives
 * sub-block (v, w) = sum_K coef K of block blk; block_inner_mv and
 * block_quad_mv return out[blk][v][w][K] (sub-block inner products with K, and
 * x_{r,v}^T K x_{c,w}).  nv = 1 is the univariate form above. */
int bta_assemble_prior_mv(void* stream, int64_t n, int64_t ns, int64_t nv, const double* coef, const int* rowptr,
                          const int* colidx, const double* vals4, double* D, double* L);
int bta_block_inner_mv(void* stream, int64_t n, int64_t ns, int64_t nv, const int* rowptr, const int* colidx,
                       const double* vals4, const double* D, const double* L, double* out);
int bta_block_quad_mv(void* stream, int64_t n, int64_t ns, int64_t nv, const int* rowptr, const int* colidx,
                      const double* vals4, const double* x, double* out);

/* Poisson likelihood at eta (src/dalia/likelihoods/poisson.py:35-63):
 * d = e exp(eta) (minus the Hessian diagonal), g = y - d (gradient),
 * *lik = eta . y - sum(e exp(eta)). */
int bta_poisson_terms(void* stream, int64_t nobs, const double* eta, const double* y, const double* e, double* d,
                      double* g, double* part, int nparts, double* lik);

/* out[blk][K] = u_t^T K x_t (blk = t < n) or u_{t+1}^T K x_t + u_t^T K x_{t+1}
 * (blk = n + t): u^T dQ_st x for Kronecker-structured dQ_st. */
int bta_block_bilinear(void* stream, int64_t n, int64_t b, const int* rowptr, const int* colidx, const double* vals4,
                       const double* u, const double* x, double* out);

/* out[i] = scale[i] * a_i^T S a_i (scale NULL means 1) for every row a_i of
 * A = [A_st | X], with S on the BTA pattern given by per-observation entry
 * lists (off[nobs+1], dst = element offsets into base, w = weight products,
 * doubled for L and Ab entries) and the tip T (a x a) with the dense rows of
 * X: diag(A S A^T), the observation marginal variances of
 * src/dalia/core/dalia.py:964-1021 when S = Q_c^{-1}. */
int bta_obs_quad(void* stream, int64_t nobs, const int64_t* off, const int64_t* dst, const double* w,
                 const double* base, int64_t a, const double* X, const double* T, const double* scale, double* out);

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
