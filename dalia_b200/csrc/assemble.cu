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

// One CTA per (block, 8-row slab): write rows of D_t (blk < n) or L_t
// (blk >= n).  With nv variates interleaved per time step the block is
// (nv ns) x (nv ns); row r = v ns + s holds, for every variate w, the spatial
// row s of sub-block (v, w) = sum_K coef[blk][v][w][K] K at columns w ns + c.
__global__ void __launch_bounds__(256) assemble_prior_kernel(int n, int ns, int nv, const double* coef,
                                                             const int* rowptr, const int* colidx,
                                                             const double* vals4, double* D, double* L) {
  const int rows_per = 8;
  const int b = nv * ns;
  const int slabs = (b + rows_per - 1) / rows_per;
  const int blk = blockIdx.x / slabs, slab = blockIdx.x % slabs;
  const bool lower = blk >= n;
  const int t = lower ? blk - n : blk;
  double* M = lower ? L + (size_t)t * b * b : D + (size_t)t * b * b;
  for (int rr = 0; rr < rows_per; ++rr) {
    const int row = slab * rows_per + rr;
    if (row >= b) break;
    const int v = row / ns, sr = row - v * ns;
    double* out = M + (size_t)row * b;
    // zero the row (vectorised when aligned)
    if ((b & 1) == 0 && ((reinterpret_cast<uintptr_t>(out) & 15) == 0)) {
      double2* o2 = reinterpret_cast<double2*>(out);
      for (int c = threadIdx.x; c < b / 2; c += blockDim.x) o2[c] = make_double2(0.0, 0.0);
    } else {
      for (int c = threadIdx.x; c < b; c += blockDim.x) out[c] = 0.0;
    }
    __syncthreads();
    const int e0 = rowptr[sr], e1 = rowptr[sr + 1], len = e1 - e0;
    for (int q = threadIdx.x; q < nv * len; q += blockDim.x) {
      const int w = q / len, e = e0 + (q - w * len);
      const double* cf = coef + (((size_t)blk * nv + v) * nv + w) * 4;
      const double* vv = vals4 + (size_t)e * 4;
      out[w * ns + colidx[e]] = cf[0] * vv[0] + cf[1] * vv[1] + cf[2] * vv[2] + cf[3] * vv[3];
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

// out[blk][v][w][K] = sum over the union pattern of sub-block (v, w) of block
// blk of S[v ns + s][w ns + c] * K[s][c] (blk < n: diagonal block D_t; else
// sub-diagonal block L_{blk-n}).  One CTA per (blk, v, w).
__global__ void __launch_bounds__(256) block_inner_kernel(int n, int ns, int nv, const int* rowptr,
                                                          const int* colidx, const double* vals4, const double* D,
                                                          const double* L, double* out) {
  __shared__ double red[4][256];
  const int blk = blockIdx.x / (nv * nv), vw = blockIdx.x % (nv * nv), v = vw / nv, w = vw % nv;
  const int b = nv * ns;
  const bool lower = blk >= n;
  const int t = lower ? blk - n : blk;
  const double* M = (lower ? L + (size_t)t * b * b : D + (size_t)t * b * b) + (size_t)v * ns * b + w * ns;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (int row = threadIdx.x; row < ns; row += blockDim.x) {
    for (int e = rowptr[row]; e < rowptr[row + 1]; ++e) {
      const double m = M[(size_t)row * b + colidx[e]];
      const double* vv = vals4 + (size_t)e * 4;
      s[0] += m * vv[0];
      s[1] += m * vv[1];
      s[2] += m * vv[2];
      s[3] += m * vv[3];
    }
  }
  for (int k = 0; k < 4; ++k) red[k][threadIdx.x] = s[k];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int k = 0; k < 4; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x < 4) out[(size_t)blockIdx.x * 4 + threadIdx.x] = red[threadIdx.x][0];
}

// out[blk][v][w][K] = x_{r,v}^T K x_{c,w} over the union pattern, where x_{t,v}
// is variate v's segment of time step t, (r, c) = (t, t) for the diagonal
// block t = blk < n and (t+1, t) for the sub-diagonal block t = blk - n.
__global__ void __launch_bounds__(256) block_quad_kernel(int n, int ns, int nv, const int* rowptr,
                                                         const int* colidx, const double* vals4, const double* x,
                                                         double* out) {
  __shared__ double red[4][256];
  const int blk = blockIdx.x / (nv * nv), vw = blockIdx.x % (nv * nv), v = vw / nv, w = vw % nv;
  const int b = nv * ns;
  const bool lower = blk >= n;
  const int t = lower ? blk - n : blk;
  const double* xr = x + (size_t)(lower ? t + 1 : t) * b + v * ns;
  const double* xc = x + (size_t)t * b + w * ns;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (int row = threadIdx.x; row < ns; row += blockDim.x) {
    const double xv = xr[row];
    for (int e = rowptr[row]; e < rowptr[row + 1]; ++e) {
      const double m = xv * xc[colidx[e]];
      const double* vv = vals4 + (size_t)e * 4;
      s[0] += m * vv[0];
      s[1] += m * vv[1];
      s[2] += m * vv[2];
      s[3] += m * vv[3];
    }
  }
  for (int k = 0; k < 4; ++k) red[k][threadIdx.x] = s[k];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int k = 0; k < 4; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x < 4) out[(size_t)blockIdx.x * 4 + threadIdx.x] = red[threadIdx.x][0];
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

// y_r = alpha * (Q_st x)_r + beta * y_r for every row r = t*b + s of the
// spatio-temporal block: the row meets the blocks (t, t-1), (t, t) and
// (t, t+1) = (t+1, t)^T, each sum_K coef[blk][K] K (K symmetric).  One warp
// per row; lanes stride the union pattern of the spatial row s.
__global__ void __launch_bounds__(256) kron_symv_kernel(int n, int b, const double* coef, const int* rowptr,
                                                        const int* colidx, const double* vals4, const double* x,
                                                        double alpha, double beta, double* y) {
  const int lane = threadIdx.x & 31;
  const int64_t rows = (int64_t)n * b;
  for (int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; r < rows;
       r += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    const int t = (int)(r / b), s = (int)(r - (int64_t)t * b);
    const double* cd = coef + (size_t)t * 4;
    const double* cl = t > 0 ? coef + (size_t)(n + t - 1) * 4 : nullptr;
    const double* cu = t < n - 1 ? coef + (size_t)(n + t) * 4 : nullptr;
    const double* x0 = x + (size_t)t * b;
    double acc = 0.0;
    for (int e = rowptr[s] + lane; e < rowptr[s + 1]; e += 32) {
      const int c = colidx[e];
      const double* v = vals4 + (size_t)e * 4;
      const double v0 = v[0], v1 = v[1], v2 = v[2], v3 = v[3];
      acc += (cd[0] * v0 + cd[1] * v1 + cd[2] * v2 + cd[3] * v3) * x0[c];
      if (cl) acc += (cl[0] * v0 + cl[1] * v1 + cl[2] * v2 + cl[3] * v3) * x0[c - b];
      if (cu) acc += (cu[0] * v0 + cu[1] * v1 + cu[2] * v2 + cu[3] * v3) * x0[c + b];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) y[r] = alpha * acc + (beta != 0.0 ? beta * y[r] : 0.0);
  }
}

// Poisson terms at eta: d = e exp(eta) (minus the likelihood Hessian diagonal),
// g = y - d (likelihood gradient), part[blockIdx] = partial sum of eta y - d.
__global__ void __launch_bounds__(256) poisson_terms_kernel(int64_t m, const double* eta, const double* y,
                                                            const double* e, double* d, double* g, double* part) {
  __shared__ double red[256];
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
    const double et = eta[i];
    const double di = e[i] * exp(et);
    d[i] = di;
    g[i] = y[i] - di;
    s += et * y[i] - di;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// out[blk][K] = u_t^T K x_t (diagonal block t = blk < n) or
// u_{t+1}^T K x_t + u_t^T K x_{t+1} (sub-diagonal block t = blk - n): the
// bilinear form u^T (E (x) K) x of the symmetric Kronecker block pair.
__global__ void __launch_bounds__(256) block_bilinear_kernel(int n, int b, const int* rowptr, const int* colidx,
                                                             const double* vals4, const double* u, const double* x,
                                                             double* out) {
  __shared__ double red[4][256];
  const int blk = blockIdx.x;
  const bool lower = blk >= n;
  const int t = lower ? blk - n : blk;
  const double* ur = u + (size_t)(lower ? t + 1 : t) * b;
  const double* xc = x + (size_t)t * b;
  const double* ur2 = u + (size_t)t * b;
  const double* xc2 = x + (size_t)(t + 1) * b;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (int row = threadIdx.x; row < b; row += blockDim.x) {
    const double uv = ur[row];
    const double uv2 = lower ? ur2[row] : 0.0;
    for (int e = rowptr[row]; e < rowptr[row + 1]; ++e) {
      const int c = colidx[e];
      const double m = uv * xc[c] + (lower ? uv2 * xc2[c] : 0.0);
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

// out[i] = scale[i] * (a_i^T S a_i) for every observation row a_i of A, with
// S on the BTA pattern: the (entry, weight) pairs of row i (off/dst/w, weights
// already doubled for entries of L and Ab blocks) plus the fixed-effect part
// x_i^T T x_i (X: nobs x a, row-major).  One warp per observation.
__global__ void __launch_bounds__(256) obs_quad_kernel(int64_t nobs, const int64_t* off, const int64_t* dst,
                                                       const double* w, const double* base, int a, const double* X,
                                                       const double* T, const double* scale, double* out) {
  const int lane = threadIdx.x & 31;
  for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < nobs;
       i += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    double s = 0.0;
    for (int64_t j = off[i] + lane; j < off[i + 1]; j += 32) s += w[j] * base[dst[j]];
    if (a > 0) {
      const double* xi = X + (size_t)i * a;
      for (int pq = lane; pq < a * a; pq += 32) {
        const int p = pq / a, q = pq - p * a;
        s += xi[p] * xi[q] * T[pq];
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) out[i] = scale ? scale[i] * s : s;
  }
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


int bta_assemble_prior_mv(void* stream, int64_t n, int64_t ns, int64_t nv, const double* coef, const int* rowptr,
                          const int* colidx, const double* vals4, double* D, double* L) {
  if (n < 1 || ns < 1 || nv < 1 || !coef || !rowptr || !colidx || !vals4 || !D || (n > 1 && !L))
    return BTA_ERR_INVALID;
  const int64_t b = nv * ns;
  const int slabs = (int)((b + 7) / 8);
  const int nblk = (int)(2 * n - 1);
  {
    bta::ProfScope _ps(bta::PROF_OTHER, (cudaStream_t)stream);
    assemble_prior_kernel<<<nblk * slabs, 256, 0, (cudaStream_t)stream>>>((int)n, (int)ns, (int)nv, coef, rowptr,
                                                                         colidx, vals4, D, L);
  }
  return cudaGetLastError() == cudaSuccess ? BTA_OK : BTA_ERR_CUDA;
}

int bta_assemble_prior(void* stream, int64_t n, int64_t b, const double* coef, const int* rowptr, const int* colidx,
                       const double* vals4, double* D, double* L) {
  return bta_assemble_prior_mv(stream, n, b, 1, coef, rowptr, colidx, vals4, D, L);
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

int bta_block_inner_mv(void* stream, int64_t n, int64_t ns, int64_t nv, const int* rowptr, const int* colidx,
                       const double* vals4, const double* D, const double* L, double* out) {
  if (n < 1 || ns < 1 || nv < 1 || !out || !D || (n > 1 && !L)) return BTA_ERR_INVALID;
  {
    bta::ProfScope _ps(bta::PROF_OTHER, (cudaStream_t)stream);
    block_inner_kernel<<<(int)((2 * n - 1) * nv * nv), 256, 0, (cudaStream_t)stream>>>(
        (int)n, (int)ns, (int)nv, rowptr, colidx, vals4, D, L, out);
  }
  return cudaGetLastError() == cudaSuccess ? BTA_OK : BTA_ERR_CUDA;
}

int bta_block_inner(void* stream, int64_t n, int64_t b, const int* rowptr, const int* colidx, const double* vals4,
                    const double* D, const double* L, double* out) {
  return bta_block_inner_mv(stream, n, b, 1, rowptr, colidx, vals4, D, L, out);
}

int bta_block_quad_mv(void* stream, int64_t n, int64_t ns, int64_t nv, const int* rowptr, const int* colidx,
                      const double* vals4, const double* x, double* out) {
  if (n < 1 || ns < 1 || nv < 1 || !out || !x) return BTA_ERR_INVALID;
  {
    bta::ProfScope _ps(bta::PROF_OTHER, (cudaStream_t)stream);
    block_quad_kernel<<<(int)((2 * n - 1) * nv * nv), 256, 0, (cudaStream_t)stream>>>(
        (int)n, (int)ns, (int)nv, rowptr, colidx, vals4, x, out);
  }
  return cudaGetLastError() == cudaSuccess ? BTA_OK : BTA_ERR_CUDA;
}

int bta_block_quad(void* stream, int64_t n, int64_t b, const int* rowptr, const int* colidx, const double* vals4,
                   const double* x, double* out) {
  return bta_block_quad_mv(stream, n, b, 1, rowptr, colidx, vals4, x, out);
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

int bta_kron_symv(void* stream, int64_t n, int64_t b, const double* coef, const int* rowptr, const int* colidx,
                  const double* vals4, const double* x, double alpha, double beta, double* y) {
  if (n < 1 || b < 1 || !coef || !rowptr || !colidx || !vals4 || !x || !y) return BTA_ERR_INVALID;
  const int64_t rows = n * b;
  const int grid = (int)std::min<int64_t>((rows * 32 + 255) / 256, 148 * 32);
  {
    bta::ProfScope _ps(bta::PROF_OTHER, (cudaStream_t)stream);
    kron_symv_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>((int)n, (int)b, coef, rowptr, colidx, vals4, x, alpha,
                                                             beta, y);
  }
  return cudaGetLastError() == cudaSuccess ? BTA_OK : BTA_ERR_CUDA;
}

int bta_poisson_terms(void* stream, int64_t nobs, const double* eta, const double* y, const double* e, double* d,
                      double* g, double* part, int nparts, double* lik) {
  if (nobs < 0 || nparts < 1 || !part || !lik || (nobs > 0 && (!eta || !y || !e || !d || !g)))
    return BTA_ERR_INVALID;
  {
    bta::ProfScope _ps(bta::PROF_OTHER, (cudaStream_t)stream);
    poisson_terms_kernel<<<nparts, 256, 0, (cudaStream_t)stream>>>(nobs, eta, y, e, d, g, part);
  }
  {
    bta::ProfScope _ps(bta::PROF_OTHER, (cudaStream_t)stream);
    sum_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(part, nparts, lik);
  }
  return cudaGetLastError() == cudaSuccess ? BTA_OK : BTA_ERR_CUDA;
}

int bta_block_bilinear(void* stream, int64_t n, int64_t b, const int* rowptr, const int* colidx, const double* vals4,
                       const double* u, const double* x, double* out) {
  if (n < 1 || b < 1 || !rowptr || !colidx || !vals4 || !u || !x || !out) return BTA_ERR_INVALID;
  {
    bta::ProfScope _ps(bta::PROF_OTHER, (cudaStream_t)stream);
    block_bilinear_kernel<<<(int)(2 * n - 1), 256, 0, (cudaStream_t)stream>>>((int)n, (int)b, rowptr, colidx, vals4,
                                                                            u, x, out);
  }
  return cudaGetLastError() == cudaSuccess ? BTA_OK : BTA_ERR_CUDA;
}

int bta_obs_quad(void* stream, int64_t nobs, const int64_t* off, const int64_t* dst, const double* w,
                 const double* base, int64_t a, const double* X, const double* T, const double* scale, double* out) {
  if (nobs < 0 || a < 0 || (nobs > 0 && (!off || !out || !base)) || (a > 0 && (!X || !T))) return BTA_ERR_INVALID;
  if (nobs == 0) return BTA_OK;
  const int grid = (int)std::min<int64_t>((nobs * 32 + 255) / 256, 148 * 32);
  {
    bta::ProfScope _ps(bta::PROF_OTHER, (cudaStream_t)stream);
    obs_quad_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(nobs, off, dst, w, base, (int)a, X, T, scale, out);
  }
  return cudaGetLastError() == cudaSuccess ? BTA_OK : BTA_ERR_CUDA;
}

}  // extern "C"
