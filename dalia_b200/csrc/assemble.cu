// Direct assembly of the spatio-temporal precision into BTA storage, plus the
// sparse gathers the objective and its gradient need.
//
// Every block of Q_st(theta) = e^{2g_st}[M0 (x) q3 + e^{g_t} M1 (x) q2 + e^{2g_t} M2 (x) q1]
// (src/dalia/submodels/spatio_temporal.py:114-149) is a linear combination of
// the four spatial matrices c0, g1, g2, g3; with their union sparsity pattern
// in CSR and the four values per entry, block (t, t') = sum_K coef[t,t',K] K.
// The dense writer emits every element of a block exactly once (zeros and
// values in one coalesced row pass), so no separate memset is needed.
// A^T D A (src/dalia/core/model.py:421) is added entry-wise: each BTA entry it
// touches has a precomputed list of (observation, weight product) pairs.
#include <algorithm>

#include "../../include/dalia_assemble.h"
#include "../../include/dalia_bta.h"
#include "prof.cuh"

namespace {

// one CTA per (block, 8-row slab): write rows of D_t (blk < n) or L_t (blk >= n)
__global__ void __launch_bounds__(256) assemble_prior_kernel(int n, int b, const double* coef, const int* rowptr,
                                                             const int* colidx, const double* vals4, double* D,
                                                             double* L) {
  const int rows_per = 8;
  const int slabs = (b + rows_per - 1) / rows_per;
  const int blk = blockIdx.x / slabs, slab = blockIdx.x % slabs;
  const bool lower = blk >= n;
  const int t = lower ? blk - n : blk;
  double* M = lower ? L + (size_t)t * b * b : D + (size_t)t * b * b;
  const double* cf = coef + (size_t)blk * 4;
  const double c0 = cf[0], c1 = cf[1], c2 = cf[2], c3 = cf[3];
  for (int rr = 0; rr < rows_per; ++rr) {
    const int row = slab * rows_per + rr;
    if (row >= b) break;
    double* out = M + (size_t)row * b;
    // zero the row (vectorised when aligned)
    if ((b & 1) == 0 && ((reinterpret_cast<uintptr_t>(out) & 15) == 0)) {
      double2* o2 = reinterpret_cast<double2*>(out);
      for (int c = threadIdx.x; c < b / 2; c += blockDim.x) o2[c] = make_double2(0.0, 0.0);
    } else {
      for (int c = threadIdx.x; c < b; c += blockDim.x) out[c] = 0.0;
    }
    __syncthreads();
    for (int e = rowptr[row] + threadIdx.x; e < rowptr[row + 1]; e += blockDim.x) {
      const double* v = vals4 + (size_t)e * 4;
      out[colidx[e]] = c0 * v[0] + c1 * v[1] + c2 * v[2] + c3 * v[3];
    }
    __syncthreads();
  }
}

// value of entry e = scale * sum_{j in [off[e], off[e+1])} d[obs[j]] * fac[j]
// added to the BTA array element dst[e] (precomputed flat index per entry).
__global__ void add_entries_kernel(int64_t nent, const int64_t* dst, const int64_t* off, const int* obs,
                                   const double* fac, const double* d, double dscale, double* base) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nent; e += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int64_t j = off[e]; j < off[e + 1]; ++j) s += (d ? d[obs[j]] : 1.0) * fac[j];
    base[dst[e]] += dscale * s;
  }
}

// T = prec I + dscale * X^T diag(d) X  (X: nobs x a row-major); partials per CTA.
__global__ void __launch_bounds__(256) tip_partial_kernel(int64_t nobs, int a, const double* X, const double* d,
                                                          double* part) {
  extern __shared__ double red[];
  const int npair = a * (a + 1) / 2;
  for (int pq = 0; pq < npair; ++pq) {
    int p = 0, q = pq;
    while (q >= a - p) {
      q -= a - p;
      ++p;
    }
    q += p;
    double s = 0.0;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nobs; r += (int64_t)gridDim.x * blockDim.x)
      s += (d ? d[r] : 1.0) * X[r * a + p] * X[r * a + q];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
      if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0) part[(size_t)blockIdx.x * npair + pq] = red[0];
    __syncthreads();
  }
}

__global__ void tip_final_kernel(int nparts, int a, const double* part, double prec, double dscale, double* T) {
  const int npair = a * (a + 1) / 2;
  for (int pq = threadIdx.x; pq < npair; pq += blockDim.x) {
    int p = 0, q = pq;
    while (q >= a - p) {
      q -= a - p;
      ++p;
    }
    q += p;
    double s = 0.0;
    for (int i = 0; i < nparts; ++i) s += part[(size_t)i * npair + pq];
    const double v = dscale * s + (p == q ? prec : 0.0);
    T[p * a + q] = v;
    T[q * a + p] = v;
  }
}

// out[blk][K] = sum over the union pattern of block blk of S_blk[row][col] * K_e
// (blk < n: diagonal block D_t; else sub-diagonal block L_{blk-n}).
__global__ void __launch_bounds__(256) block_inner_kernel(int n, int b, const int* rowptr, const int* colidx,
                                                          const double* vals4, const double* D, const double* L,
                                                          double* out) {
  __shared__ double red[4][256];
  const int blk = blockIdx.x;
  const bool lower = blk >= n;
  const int t = lower ? blk - n : blk;
  const double* M = lower ? L + (size_t)t * b * b : D + (size_t)t * b * b;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  const int nnz = rowptr[b];
  // row of entry e by binary search is avoided: walk rows with a strided loop
  for (int row = threadIdx.x; row < b; row += blockDim.x) {
    for (int e = rowptr[row]; e < rowptr[row + 1]; ++e) {
      const double m = M[(size_t)row * b + colidx[e]];
      const double* v = vals4 + (size_t)e * 4;
      s[0] += m * v[0];
      s[1] += m * v[1];
      s[2] += m * v[2];
      s[3] += m * v[3];
    }
  }
  (void)nnz;
  for (int k = 0; k < 4; ++k) red[k][threadIdx.x] = s[k];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int k = 0; k < 4; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x < 4) out[(size_t)blk * 4 + threadIdx.x] = red[threadIdx.x][0];
}

// out[blk][K] = x_r^T K x_c over the union pattern, (r, c) = (t, t) for the
// diagonal block t = blk < n, (t+1, t) for the sub-diagonal block t = blk-n.
__global__ void __launch_bounds__(256) block_quad_kernel(int n, int b, const int* rowptr, const int* colidx,
                                                         const double* vals4, const double* x, double* out) {
  __shared__ double red[4][256];
  const int blk = blockIdx.x;
  const bool lower = blk >= n;
  const int t = lower ? blk - n : blk;
  const double* xr = x + (size_t)(lower ? t + 1 : t) * b;
  const double* xc = x + (size_t)t * b;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (int row = threadIdx.x; row < b; row += blockDim.x) {
    const double xv = xr[row];
    for (int e = rowptr[row]; e < rowptr[row + 1]; ++e) {
      const double m = xv * xc[colidx[e]];
      const double* v = vals4 + (size_t)e * 4;
      s[0] += m * v[0];
      s[1] += m * v[1];
      s[2] += m * v[2];
      s[3] += m * v[3];
    }
  }
  for (int k = 0; k < 4; ++k) red[k][threadIdx.x] = s[k];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int k = 0; k < 4; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x < 4) out[(size_t)blk * 4 + threadIdx.x] = red[threadIdx.x][0];
}

// out[blockIdx] partial of sum_e w[e] * base[idx[e]]
__global__ void __launch_bounds__(256) gather_dot_kernel(int64_t nent, const int64_t* idx, const double* w,
                                                         const double* base, double* part) {
  __shared__ double red[256];
  double s = 0.0;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nent; e += (int64_t)gridDim.x * blockDim.x)
    s += w[e] * base[idx[e]];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void sum_kernel(const double* part, int cnt, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < cnt; ++i) s += part[i];
    *out = s;
  }
}

// y = alpha * A x + beta * y for CSR A (m rows); one warp per row.
__global__ void csr_spmv_kernel(int64_t m, const int64_t* rowptr, const int* col, const double* val, const double* x,
                                double alpha, double beta, double* y) {
  const int lane = threadIdx.x & 31;
  for (int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; r < m;
       r += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    double s = 0.0;
    for (int64_t e = rowptr[r] + lane; e < rowptr[r + 1]; e += 32) s += val[e] * x[col[e]];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) y[r] = alpha * s + (beta != 0.0 ? beta * y[r] : 0.0);
  }
}

// y = Q x for a symmetric BTA matrix stored by its lower blocks (one CTA row
// per 8 rows of a block row); includes the arrow rows when a > 0.
__global__ void __launch_bounds__(256) bta_symv_kernel(int n, int b, int a, const double* D, const double* L,
                                                       const double* Ab, const double* T, const double* x,
                                                       double* y) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t nb = (int64_t)n * b;
  const int64_t row = (int64_t)blockIdx.x * 8 + warp;
  if (row >= nb + a) return;
  double s = 0.0;
  if (row < nb) {
    const int i = (int)(row / b), r = (int)(row % b);
    const size_t bb = (size_t)b * b;
    // diagonal block: lower part row r, upper via column r of the lower part
    const double* Di = D + i * bb;
    for (int c = lane; c < b; c += 32) {
      const double m = (c <= r) ? Di[(size_t)r * b + c] : Di[(size_t)c * b + r];
      s += m * x[(size_t)i * b + c];
    }
    if (i > 0) {
      const double* Lm = L + (i - 1) * bb;
      for (int c = lane; c < b; c += 32) s += Lm[(size_t)r * b + c] * x[(size_t)(i - 1) * b + c];
    }
    if (i < n - 1) {
      const double* Lm = L + i * bb;
      for (int c = lane; c < b; c += 32) s += Lm[(size_t)c * b + r] * x[(size_t)(i + 1) * b + c];
    }
    for (int c = lane; c < a; c += 32) s += Ab[((size_t)i * a + c) * b + r] * x[nb + c];
  } else {
    const int j = (int)(row - nb);
    for (int64_t c = lane; c < nb; c += 32) {
      const int64_t i = c / b;
      s += Ab[((size_t)i * a + j) * b + c % b] * x[c];
    }
    for (int c = lane; c < a; c += 32) s += T[(size_t)j * a + c] * x[nb + c];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) y[row] = s;
}

__global__ void __launch_bounds__(256) dot_kernel(int64_t n, const double* x, const double* y, double* part) {
  __shared__ double red[256];
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s += x[i] * y[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void axpby_kernel(int64_t n, double alpha, const double* x, double beta, double* y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = alpha * x[i] + (beta != 0.0 ? beta * y[i] : 0.0);
}

}  // namespace

extern "C" {

int bta_dot(void* stream, int64_t n, const double* x, const double* y, double* part, int nparts, double* out) {
  if (n < 0 || nparts < 1 || !part || !out) return BTA_ERR_INVALID;
  {
    bta::ProfScope _ps(bta::PROF_OTHER, (cudaStream_t)stream);
    dot_kernel<<<nparts, 256, 0, (cudaStream_t)stream>>>(n, x, y, part);
  }
  {
    bta::ProfScope _ps(bta::PROF_OTHER, (cudaStream_t)stream);
    sum_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(part, nparts, out);
  }
  return cudaGetLastError() == cudaSuccess ? BTA_OK : BTA_ERR_CUDA;
}

int bta_axpby(void* stream, int64_t n, double alpha, const double* x, double beta, double* y) {
  if (n < 0 || (n > 0 && (!x || !y))) return BTA_ERR_INVALID;
  if (n == 0) return BTA_OK;
  const int grid = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
  {
    bta::ProfScope _ps(bta::PROF_OTHER, (cudaStream_t)stream);
    axpby_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(n, alpha, x, beta, y);
  }
  return cudaGetLastError() == cudaSuccess ? BTA_OK : BTA_ERR_CUDA;
}


int bta_assemble_prior(void* stream, int64_t n, int64_t b, const double* coef, const int* rowptr, const int* colidx,
                       const double* vals4, double* D, double* L) {
  if (n < 1 || b < 1 || !coef || !rowptr || !colidx || !vals4 || !D || (n > 1 && !L)) return BTA_ERR_INVALID;
  const int slabs = (int)((b + 7) / 8);
  const int nblk = (int)(2 * n - 1);
  {
    bta::ProfScope _ps(bta::PROF_OTHER, (cudaStream_t)stream);
    assemble_prior_kernel<<<nblk * slabs, 256, 0, (cudaStream_t)stream>>>((int)n, (int)b, coef, rowptr, colidx, vals4,
                                                                         D, L);
  }
  return cudaGetLastError() == cudaSuccess ? BTA_OK : BTA_ERR_CUDA;
}

int bta_add_entries(void* stream, int64_t nent, const int64_t* dst, const int64_t* off, const int* obs,
                    const double* fac, const double* d, double dscale, double* base) {
  if (nent < 0 || (nent > 0 && (!dst || !off || !base))) return BTA_ERR_INVALID;
  if (nent == 0) return BTA_OK;
  const int grid = (int)std::min<int64_t>((nent + 255) / 256, 148 * 16);
  {
    bta::ProfScope _ps(bta::PROF_OTHER, (cudaStream_t)stream);
    add_entries_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(nent, dst, off, obs, fac, d, dscale, base);
  }
  return cudaGetLastError() == cudaSuccess ? BTA_OK : BTA_ERR_CUDA;
}

int bta_arrow_tip(void* stream, int64_t nobs, int64_t a, const double* X, const double* d, double prec,
                  double dscale, double* part, int nparts, double* T) {
  if (a < 1 || nobs < 0 || !X || !T || !part || nparts < 1) return BTA_ERR_INVALID;
  {
    bta::ProfScope _ps(bta::PROF_OTHER, (cudaStream_t)stream);
    tip_partial_kernel<<<nparts, 256, 256 * sizeof(double), (cudaStream_t)stream>>>(nobs, (int)a, X, d, part);
  }
  {
    bta::ProfScope _ps(bta::PROF_OTHER, (cudaStream_t)stream);
    tip_final_kernel<<<1, 128, 0, (cudaStream_t)stream>>>(nparts, (int)a, part, prec, dscale, T);
  }
  return cudaGetLastError() == cudaSuccess ? BTA_OK : BTA_ERR_CUDA;
}

int bta_block_inner(void* stream, int64_t n, int64_t b, const int* rowptr, const int* colidx, const double* vals4,
                    const double* D, const double* L, double* out) {
  if (n < 1 || b < 1 || !out) return BTA_ERR_INVALID;
  {
    bta::ProfScope _ps(bta::PROF_OTHER, (cudaStream_t)stream);
    block_inner_kernel<<<(int)(2 * n - 1), 256, 0, (cudaStream_t)stream>>>((int)n, (int)b, rowptr, colidx, vals4, D, L,
                                                                         out);
  }
  return cudaGetLastError() == cudaSuccess ? BTA_OK : BTA_ERR_CUDA;
}

int bta_block_quad(void* stream, int64_t n, int64_t b, const int* rowptr, const int* colidx, const double* vals4,
                   const double* x, double* out) {
  if (n < 1 || b < 1 || !out || !x) return BTA_ERR_INVALID;
  {
    bta::ProfScope _ps(bta::PROF_OTHER, (cudaStream_t)stream);
    block_quad_kernel<<<(int)(2 * n - 1), 256, 0, (cudaStream_t)stream>>>((int)n, (int)b, rowptr, colidx, vals4, x, out);
  }
  return cudaGetLastError() == cudaSuccess ? BTA_OK : BTA_ERR_CUDA;
}

int bta_gather_dot(void* stream, int64_t nent, const int64_t* idx, const double* w, const double* base, double* part,
                   int nparts, double* out) {
  if (nent < 0 || nparts < 1 || !part || !out) return BTA_ERR_INVALID;
  {
    bta::ProfScope _ps(bta::PROF_OTHER, (cudaStream_t)stream);
    gather_dot_kernel<<<nparts, 256, 0, (cudaStream_t)stream>>>(nent, idx, w, base, part);
  }
  {
    bta::ProfScope _ps(bta::PROF_OTHER, (cudaStream_t)stream);
    sum_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(part, nparts, out);
  }
  return cudaGetLastError() == cudaSuccess ? BTA_OK : BTA_ERR_CUDA;
}

int bta_csr_spmv(void* stream, int64_t m, const int64_t* rowptr, const int* col, const double* val, const double* x,
                 double alpha, double beta, double* y) {
  if (m < 0 || (m > 0 && (!rowptr || !x || !y))) return BTA_ERR_INVALID;
  if (m == 0) return BTA_OK;
  const int grid = (int)std::min<int64_t>((m * 32 + 255) / 256, 148 * 32);
  {
    bta::ProfScope _ps(bta::PROF_OTHER, (cudaStream_t)stream);
    csr_spmv_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(m, rowptr, col, val, x, alpha, beta, y);
  }
  return cudaGetLastError() == cudaSuccess ? BTA_OK : BTA_ERR_CUDA;
}

int bta_symv(void* stream, int64_t n, int64_t b, int64_t a, const double* D, const double* L, const double* Ab,
             const double* T, const double* x, double* y) {
  if (n < 1 || b < 1 || a < 0 || !D || !x || !y) return BTA_ERR_INVALID;
  const int64_t rows = n * b + a;
  {
    bta::ProfScope _ps(bta::PROF_OTHER, (cudaStream_t)stream);
    bta_symv_kernel<<<(int)((rows + 7) / 8), 256, 0, (cudaStream_t)stream>>>((int)n, (int)b, (int)a, D, L, Ab, T, x,
                                                                            y);
  }
  return cudaGetLastError() == cudaSuccess ? BTA_OK : BTA_ERR_CUDA;
}

}  // extern "C"
