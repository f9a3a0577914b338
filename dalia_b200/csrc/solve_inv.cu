// Triangular sweeps with precomputed inverses of the diagonal factor blocks.
//
// With V_i = L_ii^-1 available, a sweep over n blocks is n dependent steps of
// two dense matrix-vector products each,
//   forward   y_i = V_i (b_i - L_{i,i-1} y_{i-1}),
//   backward  x_i = V_i^T (y_i - L_{i+1,i}^T x_{i+1} - Ab_i^T x_a),
// instead of ceil(b/64) dependent tile solves per block.  Every step reads
// its two b x b blocks once, so a sweep is bound by HBM bandwidth as long as
// the step-to-step hand-over is short.  One persistent cooperative launch
// covers a range of steps of every instance of a batch: all CTAs take part in
// every product and meet at a grid barrier between the two products of a
// step, so a step costs its bytes at full bandwidth plus two barriers (no
// kernel launch per product).
//
// Forward products are row dot products (one warp per row, 16-byte loads).
// Backward products are column sums of row-major blocks: a warp owns 32
// columns and one of S row segments and writes a partial sum per column;
// the next phase sums the S partials of the rows it needs in a fixed order,
// so the results do not depend on scheduling.  The arrowhead tip is solved by
// the tile sweep's arrow kernels before (backward) or after (forward).
#include <algorithm>
#include <cstring>
#include <vector>

#include "bta_internal.cuh"
#include "common.cuh"
#include "prof.cuh"
#include "tune.cuh"

namespace bta {
namespace {

constexpr int PS_THREADS = 256;
constexpr int PS_WARPS = PS_THREADS / 32;
constexpr int PS_MAXI = 64;
constexpr int PS_MAXS = 32;  // row segments of the column sums (one lane each when summed)
constexpr long long PS_SPIN_LIMIT = 1LL << 24;

struct PInst {
  const double* L;   // (n-1) b x b sub-diagonal factor blocks, or nullptr (n = 1)
  const double* Ab;  // n a x b arrow blocks, or nullptr
  const double* V;   // inverse of block vlo at V, block i at V + (i - vlo) b^2
  double* x;         // n b + a, in place
  double* t;         // b (forward: b_i - L y_{i-1})
  double* pa;        // S b partial column sums (backward, first product)
  double* pb;        // S b partial column sums (backward, second product)
  int n, b, a, vlo;
  int S, seg;        // row segments and rows per segment (backward)
  int ncc;           // 32-column chunks (backward)
  int row0;          // first forward unit of this instance
  int unit0;         // first backward unit of this instance
};

struct PSweep {
  int count, trans, s0, s1;
  int rows_total;   // forward units (rows of all instances)
  int units_total;  // backward units (S * ncc summed over instances)
  unsigned* bar;    // [0] arrivals, [1] generation
  int* abort_flag;
  PInst inst[PS_MAXI];
};

__device__ __forceinline__ unsigned ld_acquire_u(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release_u(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

// Grid-wide barrier of a cooperative launch (every CTA resident).  Bounded:
// a wait that runs out sets the abort flag, and every later barrier returns
// at once, so the launch always ends.  Returns false once aborted.
__device__ bool grid_barrier(const PSweep& P, unsigned& gen) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = ld_acquire(P.abort_flag) == 0;
    if (ok) {
      __threadfence();
      if (atomicAdd(&P.bar[0], 1u) == gridDim.x - 1) {
        P.bar[0] = 0;
        __threadfence();
        st_release_u(&P.bar[1], gen + 1);
      } else {
        long long it = 0;
        while (ld_acquire_u(&P.bar[1]) == gen) {
          if (ld_acquire(P.abort_flag)) {
            ok = 0;
            break;
          }
          if (++it > PS_SPIN_LIMIT) {
            atomicExch(P.abort_flag, 1);
            ok = 0;
            break;
          }
          __nanosleep(20);
        }
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  ++gen;
  return s_ok != 0;
}

// dot of one row (cnt entries at M) with v, by one warp (16-byte loads when aligned)
__device__ __forceinline__ double warp_dot(const double* M, const double* v, int cnt, int lane) {
  double s = 0.0;
  const bool vec = ((reinterpret_cast<uintptr_t>(M) | reinterpret_cast<uintptr_t>(v)) & 15) == 0;
  if (vec) {
    const int kp = cnt >> 1;
#pragma unroll 4
    for (int q = lane; q < kp; q += 32) {
      const double2 m = __ldg(reinterpret_cast<const double2*>(M) + q);
      const double2 xv = __ldcg(reinterpret_cast<const double2*>(v) + q);
      s = fma(m.x, xv.x, s);
      s = fma(m.y, xv.y, s);
    }
    if ((cnt & 1) && lane == 0) s = fma(__ldg(M + cnt - 1), __ldcg(v + cnt - 1), s);
  } else {
    for (int k = lane; k < cnt; k += 32) s = fma(__ldg(M + k), __ldcg(v + k), s);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

// instance of forward unit u (rows concatenated)
__device__ __forceinline__ int inst_of_row(const PSweep& P, int u) {
  int k = 0;
  while (k + 1 < P.count && u >= P.inst[k + 1].row0) ++k;
  return k;
}

__device__ __forceinline__ int inst_of_unit(const PSweep& P, int u) {
  int k = 0;
  while (k + 1 < P.count && u >= P.inst[k + 1].unit0) ++k;
  return k;
}

// sum of the S partial column sums of column c, in segment order
__device__ __forceinline__ double sum_parts(const double* part, int S, int b, int c) {
  double s = 0.0;
  for (int q = 0; q < S; ++q) s += __ldcg(part + (size_t)q * b + c);
  return s;
}

__global__ void __launch_bounds__(PS_THREADS) sweep_persist_kernel(const __grid_constant__ PSweep P) {
  extern __shared__ double seg_vec[];  // PS_WARPS x (max rows per segment)
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int gw = blockIdx.x * PS_WARPS + wib, nw = gridDim.x * PS_WARPS;
  unsigned gen = ld_acquire_u(&P.bar[1]);
  int maxseg = 1;
  for (int k = 0; k < P.count; ++k) maxseg = max(maxseg, P.inst[k].seg);
  double* sv = seg_vec + (size_t)wib * maxseg;

  if (P.trans == 0) {
    for (int st = P.s0; st < P.s1; ++st) {
      // t = b_i - L_{i,i-1} y_{i-1}
      for (int u = gw; u < P.rows_total; u += nw) {
        const PInst& I = P.inst[inst_of_row(P, u)];
        const int i = st, r = u - I.row0;
        if (i >= I.n) continue;
        double s = 0.0;
        if (i > 0) s = warp_dot(I.L + (size_t)(i - 1) * I.b * I.b + (size_t)r * I.b, I.x + (size_t)(i - 1) * I.b, I.b,
                                lane);
        if (lane == 0) I.t[r] = __ldcg(I.x + (size_t)i * I.b + r) - s;
      }
      if (!grid_barrier(P, gen)) return;
      // y_i = V_i t  (V_i lower triangular: row r has r + 1 entries)
      for (int u = gw; u < P.rows_total; u += nw) {
        const PInst& I = P.inst[inst_of_row(P, u)];
        const int i = st, r = u - I.row0;
        if (i >= I.n) continue;
        const double s = warp_dot(I.V + (size_t)(i - I.vlo) * I.b * I.b + (size_t)r * I.b, I.t, r + 1, lane);
        if (lane == 0) I.x[(size_t)i * I.b + r] = s;
      }
      if (!grid_barrier(P, gen)) return;
    }
    return;
  }

  // backward: step st handles block i = n - 1 - st of every instance
  for (int st = P.s0; st < P.s1; ++st) {
    // pa[s][c] = sum over segment s's rows r of L_i[r][c] x_{i+1}[r]
    //            (+ sum_q Ab_i[q][c] x_a[q] in segment 0)
    for (int u = gw; u < P.units_total; u += nw) {
      const PInst& I = P.inst[inst_of_unit(P, u)];
      const int i = I.n - 1 - st;
      if (i < 0) continue;
      const int v = u - I.unit0, sgi = v / I.ncc, j = v - sgi * I.ncc;
      const int c = 32 * j + lane;
      const int r0 = sgi * I.seg, r1 = min(I.b, r0 + I.seg);
      double acc = 0.0;
      if (i < I.n - 1 && r0 < r1) {
        // x_{i+1} of this segment's rows: the sum of the previous step's
        // partials, or the vector itself at the first step of the launch
        const double* xn = I.x + (size_t)(i + 1) * I.b;
        for (int r = r0 + lane; r < r1; r += 32)
          sv[r - r0] = (st == P.s0) ? __ldcg(xn + r) : sum_parts(I.pb, I.S, I.b, r);
        __syncwarp();
        if (j == 0 && st != P.s0)
          for (int r = r0 + lane; r < r1; r += 32) I.x[(size_t)(i + 1) * I.b + r] = sv[r - r0];
        if (c < I.b) {
          const double* Lm = I.L + (size_t)i * I.b * I.b + c;
#pragma unroll 8
          for (int r = r0; r < r1; ++r) acc = fma(__ldg(Lm + (size_t)r * I.b), sv[r - r0], acc);
        }
        __syncwarp();
      }
      if (sgi == 0 && I.a > 0 && c < I.b) {
        const double* Am = I.Ab + (size_t)i * I.a * I.b + c;
        const double* xa = I.x + (size_t)I.n * I.b;
        for (int q = 0; q < I.a; ++q) acc = fma(__ldg(Am + (size_t)q * I.b), __ldcg(xa + q), acc);
      }
      if (c < I.b) I.pa[(size_t)sgi * I.b + c] = acc;
    }
    if (!grid_barrier(P, gen)) return;
    // pb[s][c] = sum over segment s's rows r >= c of V_i[r][c] t[r],
    //            t = y_i - sum_s pa[s]
    for (int u = gw; u < P.units_total; u += nw) {
      const PInst& I = P.inst[inst_of_unit(P, u)];
      const int i = I.n - 1 - st;
      if (i < 0) continue;
      const int v = u - I.unit0, sgi = v / I.ncc, j = v - sgi * I.ncc;
      const int c = 32 * j + lane;
      const int r0 = max(sgi * I.seg, 32 * j), r1 = min(I.b, sgi * I.seg + I.seg);
      double acc = 0.0;
      if (r0 < r1) {
        const double* yi = I.x + (size_t)i * I.b;
        for (int r = r0 + lane; r < r1; r += 32) sv[r - r0] = __ldcg(yi + r) - sum_parts(I.pa, I.S, I.b, r);
        __syncwarp();
        if (c < I.b) {
          const double* Vm = I.V + (size_t)(i - I.vlo) * I.b * I.b + c;
#pragma unroll 8
          for (int r = r0; r < r1; ++r) acc = fma(__ldg(Vm + (size_t)r * I.b), sv[r - r0], acc);
        }
        __syncwarp();
      }
      if (c < I.b) I.pb[(size_t)sgi * I.b + c] = acc;
    }
    if (!grid_barrier(P, gen)) return;
  }
  // x of the last block each instance processed in this launch
  for (int k = 0; k < P.count; ++k) {
    const PInst& I = P.inst[k];
    const int st_last = min(P.s1, I.n) - 1;
    if (st_last < P.s0) continue;
    const int i = I.n - 1 - st_last;
    for (int c = blockIdx.x * PS_THREADS + threadIdx.x; c < I.b; c += gridDim.x * PS_THREADS)
      I.x[(size_t)i * I.b + c] = sum_parts(I.pb, I.S, I.b, c);
  }
}

// resident CTAs per SM of the persistent sweep (at most 4)
int persist_occupancy(size_t smem) {
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, sweep_persist_kernel, PS_THREADS, smem) != cudaSuccess)
    return -1;
  return std::min(occ, 4);
}

int max_segments(int b) { return std::min(PS_MAXS, std::max(1, (b + 47) / 48)); }

}  // namespace

size_t sweep_inv_work(int n, int b, int a) { return (size_t)b * (1 + 2 * max_segments(b)) + (size_t)n * a + 64; }

int sweep_inv_steps(int count, const int* n, const int* b, const int* a, const double* const* L,
                    const double* const* Ab, const double* const* V, const int* vlo, double* const* x, int trans,
                    int s0, int s1, double* work, int* abort_flag, cudaStream_t s) {
  if (count < 1 || count > PS_MAXI || s1 <= s0) return count < 1 || count > PS_MAXI ? cudaErrorInvalidValue : 0;
  // candidates: (CTAs per SM, row segments) = (all, most), (2, most), (all, half)
  int bsum = 0, bmax = 0, nmax = 0;
  for (int k = 0; k < count; ++k) {
    bsum += b[k];
    bmax = std::max(bmax, b[k]);
    nmax = std::max(nmax, n[k]);
  }
  TuneLaunch tl("sweep", {count, trans, bsum, bmax, s1 - s0}, 3, s, 1);
  const int cand = tl.choice();
  PSweep P;
  std::memset(&P, 0, sizeof(P));
  P.count = count;
  P.trans = trans;
  P.s0 = s0;
  P.s1 = s1;
  P.abort_flag = abort_flag;
  size_t off = 0;
  int maxseg = 1;
  for (int k = 0; k < count; ++k) {
    PInst& I = P.inst[k];
    I.L = n[k] > 1 ? L[k] : nullptr;
    I.Ab = a[k] > 0 ? Ab[k] : nullptr;
    I.V = V[k];
    I.vlo = vlo ? vlo[k] : 0;
    I.x = x[k];
    I.n = n[k];
    I.b = b[k];
    I.a = a[k];
    I.S = cand == 2 ? std::max(1, max_segments(b[k]) / 2) : max_segments(b[k]);
    I.seg = (b[k] + I.S - 1) / I.S;
    I.ncc = (b[k] + 31) / 32;
    I.t = work + off;
    I.pa = work + off + b[k];
    I.pb = work + off + (size_t)b[k] * (1 + max_segments(b[k]));
    off += sweep_inv_work(n[k], b[k], a[k]);
    I.row0 = P.rows_total;
    P.rows_total += b[k];
    I.unit0 = P.units_total;
    P.units_total += I.S * I.ncc;
    maxseg = std::max(maxseg, I.seg);
  }
  // barrier words after the instances' scratch
  P.bar = reinterpret_cast<unsigned*>(work + off);
  if (cudaMemsetAsync(P.bar, 0, 2 * sizeof(unsigned), s) != cudaSuccess) return cudaErrorUnknown;
  const size_t smem = (size_t)PS_WARPS * maxseg * sizeof(double);
  if (smem > 48 * 1024) {
    const int e = ensure_smem_attr(reinterpret_cast<const void*>(sweep_persist_kernel), (int)smem);
    if (e != cudaSuccess) return e;
  }
  const int occ = persist_occupancy(smem);
  if (occ <= 0) return cudaErrorUnknown;
  const int grid = (cand == 1 ? std::min(occ, 2) : occ) * device_sm_count();
  void* args[] = {&P};
  bta::ProfScope _ps(bta::PROF_SWEEP, s);
  return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(sweep_persist_kernel), dim3(grid),
                                     dim3(PS_THREADS), args, smem, s);
}

size_t sweep_inv_work_total(int count, const int* n, const int* b, const int* a) {
  size_t w = 0;
  for (int k = 0; k < count; ++k) w += sweep_inv_work(n[k], b[k], a[k]);
  return w + 64;
}

int sweep_inv_batched(int count, const int* n, const int* b, const int* a, const double* const* L,
                      const double* const* Ab, const double* const* T, const double* const* V, double* const* x,
                      int trans, double* work, int* abort_flag, cudaStream_t s) {
  int maxn = 0;
  for (int k = 0; k < count; ++k) maxn = std::max(maxn, n[k]);
  // arrow scratch of the forward arrow step after the instances' sweep scratch
  double* apart = work + sweep_inv_work_total(count, n, b, a);
  if (trans == 1)
    for (int k = 0; k < count; ++k)
      if (a[k] > 0 && arrow_backward(T[k], x[k], n[k], b[k], a[k], s)) return cudaErrorUnknown;
  for (int c0 = 0; c0 < count; c0 += PS_MAXI) {
    const int c1 = std::min(count, c0 + PS_MAXI);
    int cn = 0;
    for (int k = c0; k < c1; ++k) cn = std::max(cn, n[k]);
    const int e = sweep_inv_steps(c1 - c0, n + c0, b + c0, a + c0, L + c0, Ab + c0, V + c0, nullptr, x + c0, trans,
                                  0, cn, work, abort_flag, s);
    if (e) return e;
  }
  if (trans == 0)
    for (int k = 0; k < count; ++k) {
      if (a[k] <= 0) continue;
      if (arrow_forward(Ab[k], T[k], x[k], n[k], b[k], a[k], apart, s)) return cudaErrorUnknown;
    }
  return cudaGetLastError();
}

}  // namespace bta
