// Tile-DAG panel kernel of the BTA Cholesky (see panel.cuh).
#include <algorithm>

#include "common.cuh"
#include "panel.cuh"
#include "tile_ops.cuh"
#include "prof.cuh"

namespace bta {
namespace {

using namespace tile;

#ifdef BTA_TRACE
// Compile-time task tracer: per event {kind, instance, p, r|q, smid, t_claim, t_ready, t_done}.
__device__ unsigned long long* g_trace = nullptr;
__device__ int g_trace_n = 0;
__device__ __forceinline__ unsigned long long gtime() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void trace(int kind, int inst, int p, int rq, unsigned long long t0,
                                      unsigned long long t1) {
  if (threadIdx.x != 0 || g_trace == nullptr) return;
  const int i = atomicAdd(&g_trace_n, 1);
  if (i >= (1 << 20)) return;
  unsigned smid;
  asm volatile("mov.u32 %0, %smid;" : "=r"(smid));
  unsigned long long* e = g_trace + (size_t)i * 4;
  e[0] = ((unsigned long long)kind << 56) | ((unsigned long long)(inst & 0xff) << 48) |
         ((unsigned long long)(p & 0xff) << 40) | ((unsigned long long)(rq & 0xffffff) << 16) | smid;
  e[1] = t0;
  e[2] = t1;
  e[3] = gtime();
}
#define TRACE_T0() unsigned long long _t0 = gtime()
#define TRACE_T1() unsigned long long _t1 = gtime()
#define TRACE(kind, inst, p, rq) trace(kind, inst, p, rq, _t0, _t1)
#else
#define TRACE_T0()
#define TRACE_T1()
#define TRACE(kind, inst, p, rq)
#endif

constexpr size_t SMEM_BYTES = size_t(2) * T * SG * sizeof(double);
constexpr long long SPIN_LIMIT = 1LL << 24;

// Bounded wait until *p >= target.  Returns false when the wait gave up.
__device__ bool wait_ge(const int* p, int target, int* abort_flag) {
  long long it = 0;
  while (ld_acquire(p) < target) {
    if (ld_acquire(abort_flag)) return false;
    if (++it > SPIN_LIMIT) {
      atomicExch(abort_flag, 1);
      return false;
    }
    __nanosleep(32);
  }
  return true;
}

struct TileRef {
  double* ptr;
  int rows, cols;
};

__device__ __forceinline__ TileRef tile_of(const PanelInst& I, int p, int c) {
  TileRef t;
  t.cols = min(T, I.b - c * T);
  if (p < I.nq) {
    t.ptr = I.D + (size_t)(p * T) * I.b + c * T;
    t.rows = min(T, I.b - p * T);
  } else if (I.L != nullptr && p < 2 * I.nq) {
    const int pp = p - I.nq;
    t.ptr = I.L + (size_t)(pp * T) * I.b + c * T;
    t.rows = min(T, I.b - pp * T);
  } else {
    const int ar = p - I.nq - (I.L != nullptr ? I.nq : 0);
    t.ptr = I.Ab + (size_t)(ar * T) * I.b + c * T;
    t.rows = min(T, I.a - ar * T);
  }
  return t;
}


// Tile (p, c) of the previous block column's sub-diagonal and arrow blocks:
// rows of this panel's diagonal block read L_prev, arrow rows read Ab_prev;
// rows of the block below have no previous-step term (returns rows = 0).
__device__ __forceinline__ TileRef prev_tile_of(const PanelInst& I, int p, int c) {
  TileRef t;
  t.cols = min(T, I.b - c * T);
  if (p < I.nq) {
    t.ptr = const_cast<double*>(I.Lprev) + (size_t)(p * T) * I.b + c * T;
    t.rows = min(T, I.b - p * T);
  } else if (I.L != nullptr && p < 2 * I.nq) {
    t.ptr = nullptr;
    t.rows = 0;
  } else if (I.Abprev != nullptr) {
    const int ar = p - I.nq - (I.L != nullptr ? I.nq : 0);
    t.ptr = const_cast<double*>(I.Abprev) + (size_t)(ar * T) * I.b + c * T;
    t.rows = min(T, I.a - ar * T);
  } else {
    t.ptr = nullptr;
    t.rows = 0;
  }
  return t;
}

// Tile row of the previous block column holding row p's previous-column
// source: the block below it for rows of the diagonal block, its arrow rows
// for arrow rows (the previous column always has a block below).
__device__ __forceinline__ int prev_row(const PanelInst& I, int p) {
  if (p < I.nq) return I.nq + p;
  return 2 * I.nq + (p - I.nq - (I.L != nullptr ? I.nq : 0));
}

// Whether tile (p, r) receives a previous-column term (its own TASK_PREV).
__device__ __forceinline__ bool has_prev(const PanelInst& I, int p) {
  return I.Lprev != nullptr && prev_tile_of(I, p, 0).rows > 0;
}

// Accumulations stream whole 64-row strips through a ring of 16-wide k-slabs,
// so loading slab s+2 overlaps the DMMA work on slab s.
constexpr int PK = 16;
constexpr int PSK = PK + 4;  // slab row stride: conflict-light DMMA fragment loads
constexpr int PST = 3;
constexpr int PSLAB = T * PSK;
static_assert(2 * PST * PSLAB <= 2 * T * SG, "slab ring exceeds the two tile buffers");

// 64 x 16 slab of a row block at g (row stride ld): rows < rows and columns
// k0 .. k0+15 < kmax, zero-filled elsewhere.  Reads bypass L1: the strips of
// this panel are written by other CTAs during the launch.
__device__ __forceinline__ void load_slab(double* s, const double* g, int ld, int rows, int k0, int kmax, bool vec,
                                          int tid) {
#pragma unroll
  for (int j = 0; j < (T * PK / 2) / THREADS; ++j) {
    const int c = tid + j * THREADS;
    const int r = c >> 3, kc = (c & 7) * 2;
    const int gk = k0 + kc;
    double* d = s + r * PSK + kc;
    const bool v0 = r < rows && gk < kmax;
    const bool v1 = r < rows && gk + 1 < kmax;
    const double* src = g + (size_t)r * ld + gk;
    if (vec) {
      if (v1) {
        cp_async16(d, src, true);
      } else {
        d[0] = v0 ? __ldcg(src) : 0.0;
        d[1] = 0.0;
      }
    } else {
      d[0] = v0 ? __ldcg(src) : 0.0;
      d[1] = v1 ? __ldcg(src + 1) : 0.0;
    }
  }
}

__device__ __forceinline__ void mma_slab(const double* X, const double* Y, double (&acc)[2][4][4], int wm, int wn,
                                         int g, int t) {
#pragma unroll
  for (int kk = 0; kk < PK; kk += 4) {
    double a[2][2], b[4];
#pragma unroll
    for (int mi = 0; mi < 2; ++mi) {
      const int r = wm * 32 + mi * 16 + g;
      a[mi][0] = X[r * PSK + kk + t];
      a[mi][1] = X[(r + 8) * PSK + kk + t];
    }
#pragma unroll
    for (int ni = 0; ni < 4; ++ni) b[ni] = Y[(wn * 32 + ni * 8 + g) * PSK + kk + t];
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) dmma16x8x4(acc[mi][ni], a[mi][0], a[mi][1], b[ni]);
  }
}

// Block-wide wait by thread 0; returns the verdict to every thread.
__device__ __forceinline__ bool block_wait(const int* p, int target, int* abort_flag, int* s_ok) {
  if (threadIdx.x == 0) *s_ok = wait_ge(p, target, abort_flag) ? 1 : 0;
  __syncthreads();
  return *s_ok != 0;
}

// acc += X Y^T over columns [0, kcols) of two 64-row strips x (xrows valid
// rows) and y (yrows valid rows), row stride ld.  With gates, the columns of
// tile k are loaded only once gx[k] and gy[k] are set (their producers
// finished).  Returns false when such a wait gave up.
__device__ bool acc_stream(const double* x, int xrows, const double* y, int yrows, int ld, int kcols, const int* gx,
                           const int* gy, int* abort_flag, int* s_ok, double* smem, double (&acc)[2][4][4], int tid,
                           int wm, int wn, int g, int t) {
  const int nslab = (kcols + PK - 1) / PK;
  if (nslab == 0) return true;
  const bool vec = ((ld & 1) == 0) && ((reinterpret_cast<uintptr_t>(x) & 15) == 0) &&
                   ((reinterpret_cast<uintptr_t>(y) & 15) == 0);
  double* As = smem;
  double* Bs = smem + PST * PSLAB;
  bool ok = true;
  // The leading source tiles whose producers have finished: one scan of
  // their flags (relaxed loads in flight together, then one fence for
  // acquire semantics) instead of a round trip per tile; later tiles are
  // waited for one by one below.
  __shared__ int s_ready;
  if (gx != nullptr && tid == 0) {
    const int nk = (kcols + T - 1) / T;
    int r = 0;
    bool run = true;
    while (run && r < nk) {
      int v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) v[u] = (r + u < nk) ? min(ld_relaxed(gx + r + u), ld_relaxed(gy + r + u)) : 0;
      int cnt = 0;
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        if (run && v[u] >= 1) ++cnt;
        else run = false;
      }
      r += cnt;
    }
    __threadfence();
    s_ready = r;
  }
  // issue slab j (after its gate, at the first slab of every tile)
  auto issue = [&](int j) {
    if (gx != nullptr && ok && (j * PK) % T == 0 && (j * PK) / T >= s_ready) {
      const int k = (j * PK) / T;
      if (tid == 0) *s_ok = (wait_ge(gx + k, 1, abort_flag) && wait_ge(gy + k, 1, abort_flag)) ? 1 : 0;
      __syncthreads();
      ok = *s_ok != 0;
    }
    if (ok) {
      load_slab(As + (j % PST) * PSLAB, x, ld, xrows, j * PK, kcols, vec, tid);
      load_slab(Bs + (j % PST) * PSLAB, y, ld, yrows, j * PK, kcols, vec, tid);
    }
  };
  __syncthreads();  // the tile buffers may still be read by the previous step
#pragma unroll
  for (int st = 0; st < PST - 1; ++st) {
    if (st < nslab) issue(st);
    cp_async_commit();
  }
  for (int s = 0; s < nslab && ok; ++s) {
    cp_async_wait<PST - 2>();
    __syncthreads();
    const int nx = s + PST - 1;
    if (nx < nslab) issue(nx);
    cp_async_commit();
    if (ok) mma_slab(As + (s % PST) * PSLAB, Bs + (s % PST) * PSLAB, acc, wm, wn, g, t);
  }
  cp_async_wait<0>();
  __syncthreads();
  return ok;
}

__device__ __forceinline__ void release(int* p, int v) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    st_release(p, v);
  }
}

// acc -= the tile at p (rows x cols valid, zero elsewhere), element for
// element in the accumulator layout: acc becomes acc - A, i.e. the caller
// negates.  All loads are issued before any use, so a read-modify-write of
// the tile costs one L2 round trip instead of one per element (a store
// between two loads would otherwise keep them in order).
__device__ __forceinline__ void frag_rsub(const double* p, int ld, int rows, int cols, double (&acc)[2][4][4], int wm,
                                          int wn, int g, int t) {
  const bool vec = ((ld & 1) == 0) && ((reinterpret_cast<uintptr_t>(p) & 15) == 0);
  double v[2][2][4][2];
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int row = wm * 32 + mi * 16 + g + h * 8;
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) {
        const int col = wn * 32 + ni * 8 + 2 * t;  // even: a column pair
        const double* src = p + (size_t)row * ld + col;
        if (vec && row < rows && col + 1 < cols) {
          const double2 x = __ldcg(reinterpret_cast<const double2*>(src));
          v[mi][h][ni][0] = x.x;
          v[mi][h][ni][1] = x.y;
        } else {
          v[mi][h][ni][0] = (row < rows && col < cols) ? __ldcg(src) : 0.0;
          v[mi][h][ni][1] = (row < rows && col + 1 < cols) ? __ldcg(src + 1) : 0.0;
        }
      }
    }
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int ni = 0; ni < 4; ++ni)
#pragma unroll
        for (int e = 0; e < 2; ++e) acc[mi][ni][h * 2 + e] = v[mi][h][ni][e] - acc[mi][ni][h * 2 + e];
}

// Writes the accumulator tile to rows x cols of p (column pairs as 16-byte
// stores when the rows allow).
__device__ __forceinline__ void store_frag(double* p, int ld, int rows, int cols, const double (&acc)[2][4][4],
                                           int wm, int wn, int g, int t) {
  const bool vec = ((ld & 1) == 0) && ((reinterpret_cast<uintptr_t>(p) & 15) == 0);
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int row = wm * 32 + mi * 16 + g + h * 8;
      if (row >= rows) continue;
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) {
        const int col = wn * 32 + ni * 8 + 2 * t;
        double* dst = p + (size_t)row * ld + col;
        if (vec && col + 1 < cols) {
          *reinterpret_cast<double2*>(dst) = make_double2(acc[mi][ni][h * 2], acc[mi][ni][h * 2 + 1]);
        } else {
          if (col < cols) dst[0] = acc[mi][ni][h * 2];
          if (col + 1 < cols) dst[1] = acc[mi][ni][h * 2 + 1];
        }
      }
    }
}

// The critical path of one instance: for q = 0..nq-1,
//   X = A(q, q-1) Linv_{q-1}^T;  A(q, q) -= X X^T;  POTRF(q);  Linv_q.
// The two smem buffers swap roles every step: Lv holds Linv_{q-1}, Wk is work.
__device__ void run_chain(const PanelInst& I, int inst, double* bufA, double* bufL, double* rd, int* abort_flag,
                          int* s_ok) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1, g = lane >> 2, t = lane & 3;
  (void)inst;  // read by the compile-time tracer only
  const int nq = I.nq, ld = I.b;
  double* Lv = bufL;
  double* Wk = bufA;
  for (int q = 0; q < nq; ++q) {
    const TileRef d = tile_of(I, q, q);
    const int w = d.cols;
    TRACE_T0();
    if (q > 0) {
      if (!block_wait(&I.upd[q * nq + q - 1], 1, abort_flag, s_ok)) return;
      const TileRef x = tile_of(I, q, q - 1);
      load_async<SG>(Wk, x.ptr, ld, x.rows, x.cols, tid);
      cp_async_commit();
      cp_async_wait<0>();
      __syncthreads();
      double acc[2][4][4];
      zero_acc(acc);
      // Linv_{q-1} is lower triangular: output column n sums k <= n only
      mma_nt(Wk, Lv, 32 * (wn + 1), acc, wm, wn, g, t);
      __syncthreads();
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int row = wm * 32 + mi * 16 + g + h * 8;
#pragma unroll
          for (int ni = 0; ni < 4; ++ni) {
            const int col = wn * 32 + ni * 8 + 2 * t;
            const bool in = row < x.rows;
            *reinterpret_cast<double2*>(Wk + row * SG + col) =
                make_double2(in ? acc[mi][ni][h * 2] : 0.0, in ? acc[mi][ni][h * 2 + 1] : 0.0);
          }
        }
      store_frag(x.ptr, ld, x.rows, x.cols, acc, wm, wn, g, t);
      release(&I.flag[q * nq + q - 1], 1);
      if (!block_wait(&I.upd[q * nq + q], 1, abort_flag, s_ok)) return;
      TRACE_T1();
      TRACE(8, inst, q, 0);
      zero_acc(acc);
      mma_nt(Wk, Wk, T, acc, wm, wn, g, t);
      // Lv (previous inverse) is dead: it becomes the Cholesky buffer
      frag_rsub(d.ptr, ld, w, w, acc, wm, wn, g, t);
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int row = wm * 32 + mi * 16 + g + h * 8;
#pragma unroll
          for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int e = 0; e < 2; ++e) Lv[row * SG + wn * 32 + ni * 8 + 2 * t + e] = acc[mi][ni][h * 2 + e];
        }
      __syncthreads();
    } else {
      if (!block_wait(&I.upd[0], 1, abort_flag, s_ok)) return;
      load<SG>(Lv, d.ptr, ld, w, w, tid);
      __syncthreads();
    }
    {
      TRACE_T0();
      potrf(Lv, rd, w, I.info, I.pivot_base + (long long)q * T, tid);
      TRACE_T1();
      trinv(Lv, Wk, rd, tid);
      TRACE(9, inst, q, 0);
    }
    double* linv = I.Linv + (size_t)q * T * T;
    // two columns per thread (16-byte accesses when the tile's rows allow)
    const bool vec = ((ld & 1) == 0) && ((reinterpret_cast<uintptr_t>(d.ptr) & 15) == 0);
    for (int idx = 2 * tid; idx < T * T; idx += 2 * THREADS) {
      const int i = idx >> 6, k = idx & 63;
      const bool in0 = i < w && k < w, in1 = i < w && k + 1 < w;
      const double2 l = *reinterpret_cast<const double2*>(Lv + i * SG + k);
      const double2 v = *reinterpret_cast<const double2*>(Wk + i * SG + k);
      const double2 li = make_double2(in0 ? v.x : 0.0, in1 ? v.y : 0.0);
      double* dp = d.ptr + (size_t)i * ld + k;
      if (vec && in1) {
        *reinterpret_cast<double2*>(dp) = l;
      } else {
        if (in0) dp[0] = l.x;
        if (in1) dp[1] = l.y;
      }
      *reinterpret_cast<double2*>(linv + idx) = li;
      *reinterpret_cast<double2*>(Wk + i * SG + k) = li;  // zero-padded operand for the next step
    }
    double* tmp = Lv;
    Lv = Wk;
    Wk = tmp;
    release(&I.flag[q * nq + q], 1);
  }
}

// Writes tile -= acc over its valid rows x cols (L2 reads: other CTAs wrote it).
__device__ __forceinline__ void sub_acc(const TileRef& c, int ld, double (&acc)[2][4][4], int wm, int wn, int g,
                                        int t) {
  frag_rsub(c.ptr, ld, c.rows, c.cols, acc, wm, wn, g, t);
  store_frag(c.ptr, ld, c.rows, c.cols, acc, wm, wn, g, t);
}

// ALL: a whole factorisation in one launch (descriptors in B.cols); the
// one-column launch reads its descriptors from the kernel parameters.
template <bool ALL>
__global__ void __launch_bounds__(THREADS, 3) panel_kernel(const __grid_constant__ PanelBatch B) {
  extern __shared__ __align__(16) double sm[];
  double* bufA = sm;
  double* bufL = sm + T * SG;
  __shared__ int s_task, s_ok;
  __shared__ double rd[T];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1, g = lane >> 2, t = lane & 3;

  // the first CTAs to start take the chain roles (one per instance; in a
  // whole-factorisation launch the chain runs the instance's columns in order)
  if (tid == 0) s_task = atomicAdd(&B.counter[1], 1);
  __syncthreads();
  if (s_task < B.ninst) {
    if constexpr (ALL) {
      for (int c = B.col_start[s_task]; c < B.col_start[s_task + 1]; ++c) {
        run_chain(B.cols[c], s_task, bufA, bufL, rd, B.abort_flag, &s_ok);
        if (ld_acquire(B.abort_flag)) break;
      }
    } else {
      run_chain(B.inst[s_task], s_task, bufA, bufL, rd, B.abort_flag, &s_ok);
    }
    return;
  }

  for (;;) {
    __syncthreads();
    if (tid == 0) s_task = atomicAdd(&B.counter[0], 1);
    __syncthreads();
    const int ti = s_task;
    if (ti >= B.ntasks) break;
    const int4 tk = B.tasks[ti];
    const PanelInst& I = ALL ? B.cols[tk.x] : B.inst[tk.x];
    const int kind = tk.y, p = tk.z, r = tk.w;
    const int nq = I.nq, ld = I.b;
    TRACE_T0();
    double acc[2][4][4];
    zero_acc(acc);
    if (kind == TASK_PREV) {
      // tile(p, r) -= Xprev(p) Xprev(r)^T: that column is final before a
      // one-column launch; in a whole-factorisation launch each source tile
      // is waited for on the previous column's flags
      const TileRef xp = prev_tile_of(I, p, 0), yp = prev_tile_of(I, r, 0);
      const int* gx = I.prev_flag != nullptr ? I.prev_flag + prev_row(I, p) * nq : nullptr;
      const int* gy = I.prev_flag != nullptr ? I.prev_flag + prev_row(I, r) * nq : nullptr;
      if (!acc_stream(xp.ptr, xp.rows, yp.ptr, yp.rows, ld, I.b, gx, gy, B.abort_flag, &s_ok, bufA, acc, tid, wm,
                      wn, g, t))
        continue;
      TRACE_T1();
      sub_acc(tile_of(I, p, r), ld, acc, wm, wn, g, t);
      release(&I.prv[p * nq + r], 1);
      TRACE(kind, tk.x, p, r);
      continue;
    }
    if (kind == TASK_TIP) {
      // T -= sum_k X(arrow, k) X(arrow, k)^T as the arrow row becomes final
      // (after the previous columns' tip tasks in a whole-factorisation launch)
      const int pa = I.nrows_t - 1;
      const TileRef xa = tile_of(I, pa, 0);
      const int* gate = I.flag + pa * nq;
      if (!acc_stream(xa.ptr, xa.rows, xa.ptr, xa.rows, ld, I.b, gate, gate, B.abort_flag, &s_ok, bufA, acc, tid,
                      wm, wn, g, t))
        continue;
      if (I.tip_seq != nullptr && !block_wait(I.tip_seq, I.col, B.abort_flag, &s_ok)) continue;
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int row = wm * 32 + mi * 16 + g + h * 8;
          if (row >= I.a) continue;
#pragma unroll
          for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              const int col = wn * 32 + ni * 8 + 2 * t + e;
              if (col < I.a) {
                double* tp = I.Ttip + row * I.a + col;  // L2: an earlier tip task of another CTA wrote it
                __stcg(tp, __ldcg(tp) - acc[mi][ni][h * 2 + e]);
              }
            }
        }
      if (I.tip_seq != nullptr) release(I.tip_seq, I.col + 1);
      continue;
    }
    // zero the mirrored strictly-upper tile (r, p) of the diagonal block
    if (p < nq && p > r) {
      double* up = I.D + (size_t)(r * T) * ld + p * T;
      const int cw = min(T, I.b - p * T);
      for (int idx = tid; idx < T * T; idx += THREADS) {
        const int i = idx >> 6, k = idx & 63;
        if (k < cw) up[(size_t)i * ld + k] = 0.0;
      }
    }
    // left-looking accumulation of tile(p, r) -= sum_{k < kmax} X(p, k) X(r, k)^T
    // as the source columns become final
    const int kmax = (kind == TASK_AGG_DIAG) ? r - 1 : r;
    {
      const TileRef xs = tile_of(I, p, 0), ys = tile_of(I, r, 0);
      if (!acc_stream(xs.ptr, xs.rows, ys.ptr, ys.rows, ld, max(kmax, 0) * T, I.flag + p * nq, I.flag + r * nq,
                      B.abort_flag, &s_ok, bufA, acc, tid, wm, wn, g, t))
        continue;
    }
    // the previous column's term of this tile has been applied
    if (has_prev(I, p) && !block_wait(&I.prv[p * nq + r], 1, B.abort_flag, &s_ok)) continue;
    TRACE_T1();
    const TileRef c = tile_of(I, p, r);
    if (kind != TASK_AGG_TRSM) {
      // chain input: write the accumulated tile, the chain CTA finishes it
      sub_acc(c, ld, acc, wm, wn, g, t);
      release(&I.upd[p * nq + r], 1);
      TRACE(kind, tk.x, p, r);
      continue;
    }
    // X(p, r) = (A(p, r) - acc) Linv_r^T
    if (tid == 0) s_ok = wait_ge(&I.flag[r * nq + r], 1, B.abort_flag) ? 1 : 0;
    __syncthreads();
    if (!s_ok) continue;
    load_async<SG>(bufL, I.Linv + (size_t)r * T * T, T, T, T, tid);
    cp_async_commit();
    frag_rsub(c.ptr, ld, c.rows, c.cols, acc, wm, wn, g, t);
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int row = wm * 32 + mi * 16 + g + h * 8;
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
          for (int e = 0; e < 2; ++e) bufA[row * SG + wn * 32 + ni * 8 + 2 * t + e] = acc[mi][ni][h * 2 + e];
      }
    cp_async_wait<0>();
    __syncthreads();
    zero_acc(acc);
    // Linv_r is lower triangular: output column n sums k <= n only
    mma_nt(bufA, bufL, min((c.cols + 3) & ~3, 32 * (wn + 1)), acc, wm, wn, g, t);
    store_frag(c.ptr, ld, c.rows, c.cols, acc, wm, wn, g, t);
    release(&I.flag[p * nq + r], 1);
    TRACE(kind, tk.x, p, r);
  }
}

}  // namespace

#ifdef BTA_TRACE
extern "C" int bta_trace_setup(unsigned long long* buf) {
  int zero = 0;
  cudaMemcpyToSymbol(g_trace, &buf, sizeof(buf));
  return (int)cudaMemcpyToSymbol(g_trace_n, &zero, sizeof(int));
}
#endif

// Queue order: one task per tile, column by column; within a column the two
// tiles the chain CTA consumes next (the diagonal tile and the one below it)
// come first, then the remaining rows of the diagonal block, then the rows of
// the block below and of the arrow.  Every such task only waits on outputs of
// earlier columns or of the chain, so the order is topological.  The
// previous-column tasks wait on nothing; those of column r + PREV_LOOKAHEAD
// are queued before column r's tasks (diagonal and sub-diagonal tiles first),
// so the term is applied before the chain needs the tile.  Instances are
// interleaved column by column.
namespace {

bool host_has_prev(const PanelInst& I, int p) {
  if (I.Lprev == nullptr) return false;
  if (p < I.nq) return true;
  if (I.L != nullptr && p < 2 * I.nq) return false;
  return I.Abprev != nullptr;
}

void prev_tasks(const std::vector<PanelInst>& insts, int c, std::vector<int4>& tasks) {
  for (int ii = 0; ii < (int)insts.size(); ++ii) {
    const PanelInst& I = insts[ii];
    if (c >= I.nq || I.Lprev == nullptr) continue;
    for (int p = c; p < std::min(c + 2, I.nq); ++p) tasks.push_back(make_int4(ii, TASK_PREV, p, c));
  }
  for (int ii = 0; ii < (int)insts.size(); ++ii) {
    const PanelInst& I = insts[ii];
    if (c >= I.nq || I.Lprev == nullptr) continue;
    for (int p = std::min(c + 2, I.nq); p < I.nrows_t; ++p)
      if (host_has_prev(I, p)) tasks.push_back(make_int4(ii, TASK_PREV, p, c));
  }
}

}  // namespace

void panel_tasks(const std::vector<PanelInst>& insts, std::vector<int4>& tasks, int lookahead, int order) {
  lookahead = std::max(1, lookahead);
  int max_nq = 0;
  for (const auto& I : insts) max_nq = std::max(max_nq, I.nq);
  if (order == PANEL_ORDER_CHAIN_AHEAD) {
    // Critical tasks first: chain step q consumes tiles (q, q-1) and (q, q),
    // whose accumulations read rows q-1 and q of the columns up to q-2; of
    // those, only tile (q, q-2) is a queue task that needs the chain's
    // inverse of column q-2.  So at column r the queue holds, for every
    // instance, the solve of tile (r+2, r) and then the chain inputs of step
    // r+2, ahead of the bulk of column r's solves; the chain runs up to two
    // steps ahead of the bulk instead of waiting behind it.  The
    // previous-column terms of the chain-input tiles come before them, the
    // rest of a column's terms `lookahead` columns ahead of its solves.
    int crit_done = -1, bulk_done = -1;
    auto crit_upto = [&](int c) {
      for (c = std::min(c, max_nq - 1); crit_done < c;) {
        ++crit_done;
        for (int ii = 0; ii < (int)insts.size(); ++ii) {
          const PanelInst& I = insts[ii];
          if (crit_done >= I.nq || I.Lprev == nullptr) continue;
          for (int p = crit_done; p < std::min(crit_done + 2, I.nq); ++p)
            tasks.push_back(make_int4(ii, TASK_PREV, p, crit_done));
        }
      }
    };
    auto bulk_upto = [&](int c) {
      for (c = std::min(c, max_nq - 1); bulk_done < c;) {
        ++bulk_done;
        crit_upto(bulk_done);
        for (int ii = 0; ii < (int)insts.size(); ++ii) {
          const PanelInst& I = insts[ii];
          if (bulk_done >= I.nq || I.Lprev == nullptr) continue;
          for (int p = std::min(bulk_done + 2, I.nq); p < I.nrows_t; ++p)
            if (host_has_prev(I, p)) tasks.push_back(make_int4(ii, TASK_PREV, p, bulk_done));
        }
      }
    };
    crit_upto(1);
    for (int ii = 0; ii < (int)insts.size(); ++ii) {
      const PanelInst& I = insts[ii];
      tasks.push_back(make_int4(ii, TASK_AGG_DIAG, 0, 0));
      if (I.nq > 1) {
        tasks.push_back(make_int4(ii, TASK_AGG_SUB, 1, 0));
        tasks.push_back(make_int4(ii, TASK_AGG_DIAG, 1, 1));
      }
    }
    for (int r = 0; r < max_nq; ++r) {
      bulk_upto(r);
      for (int ii = 0; ii < (int)insts.size(); ++ii)
        if (r + 2 < insts[ii].nq) tasks.push_back(make_int4(ii, TASK_AGG_TRSM, r + 2, r));
      crit_upto(r + 2);
      for (int ii = 0; ii < (int)insts.size(); ++ii) {
        if (r + 2 >= insts[ii].nq) continue;
        tasks.push_back(make_int4(ii, TASK_AGG_SUB, r + 2, r + 1));
        tasks.push_back(make_int4(ii, TASK_AGG_DIAG, r + 2, r + 2));
      }
      bulk_upto(r + lookahead);
      for (int ii = 0; ii < (int)insts.size(); ++ii) {
        const PanelInst& I = insts[ii];
        if (r >= I.nq) continue;
        for (int p = r + 3; p < I.nq; ++p) tasks.push_back(make_int4(ii, TASK_AGG_TRSM, p, r));
      }
      for (int ii = 0; ii < (int)insts.size(); ++ii) {
        const PanelInst& I = insts[ii];
        if (r >= I.nq) continue;
        for (int p = std::max(I.nq, r + 1); p < I.nrows_t; ++p) tasks.push_back(make_int4(ii, TASK_AGG_TRSM, p, r));
      }
    }
  } else {
    int prev_done = -1;  // last column whose previous-column tasks are queued
    for (int r = 0; r < max_nq; ++r) {
      if (prev_done < r) prev_tasks(insts, ++prev_done, tasks);
      for (int ii = 0; ii < (int)insts.size(); ++ii) {
        const PanelInst& I = insts[ii];
        if (r >= I.nq) continue;
        tasks.push_back(make_int4(ii, TASK_AGG_DIAG, r, r));
        if (r + 1 < I.nq) tasks.push_back(make_int4(ii, TASK_AGG_SUB, r + 1, r));
      }
      while (prev_done < std::min(r + lookahead, max_nq - 1)) prev_tasks(insts, ++prev_done, tasks);
      for (int ii = 0; ii < (int)insts.size(); ++ii) {
        const PanelInst& I = insts[ii];
        if (r >= I.nq) continue;
        for (int p = r + 2; p < I.nq; ++p) tasks.push_back(make_int4(ii, TASK_AGG_TRSM, p, r));
      }
      for (int ii = 0; ii < (int)insts.size(); ++ii) {
        const PanelInst& I = insts[ii];
        if (r >= I.nq) continue;
        for (int p = std::max(I.nq, r + 1); p < I.nrows_t; ++p) tasks.push_back(make_int4(ii, TASK_AGG_TRSM, p, r));
      }
    }
  }
  for (int ii = 0; ii < (int)insts.size(); ++ii)
    if (insts[ii].Ttip != nullptr) tasks.push_back(make_int4(ii, TASK_TIP, 0, 0));
}

void panel_tasks_persist(const std::vector<PanelInst>& shapes, const std::vector<int>& n,
                         const std::vector<int>& col_start, std::vector<int4>& tasks, int lookahead, int order) {
  static double present;  // stands for a matrix block: only null / non-null matters to the queue
  int maxn = 0;
  for (int v : n) maxn = std::max(maxn, v);
  std::vector<PanelInst> insts;
  std::vector<int> gidx;
  std::vector<int4> col;
  for (int c = 0; c < maxn; ++c) {
    insts.clear();
    gidx.clear();
    for (size_t k = 0; k < shapes.size(); ++k) {
      if (c >= n[k]) continue;
      PanelInst I = shapes[k];
      const bool hasL = c < n[k] - 1;
      I.L = hasL ? &present : nullptr;
      I.Ab = I.a > 0 ? &present : nullptr;
      I.Lprev = c > 0 ? &present : nullptr;
      I.Abprev = (c > 0 && I.a > 0) ? &present : nullptr;
      I.nq = (I.b + 63) / 64;
      I.nrows_t = panel_rows(I.b, I.a, hasL);
      insts.push_back(I);
      gidx.push_back(col_start[k] + c);
    }
    col.clear();
    panel_tasks(insts, col, lookahead, order);
    for (int4 x : col) {
      x.x = gidx[x.x];
      tasks.push_back(x);
    }
  }
}

int panel_ctas_per_sm() {
  int e = ensure_smem_attr(reinterpret_cast<const void*>(panel_kernel<false>), (int)SMEM_BYTES);
  if (e == cudaSuccess) e = ensure_smem_attr(reinterpret_cast<const void*>(panel_kernel<true>), (int)SMEM_BYTES);
  if (e != cudaSuccess) return -e;
  // resident CTAs per SM at this shared-memory and register use (the
  // occupancy query is cheap next to a panel launch, and answers for the
  // current device)
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, panel_kernel<false>, THREADS, SMEM_BYTES);
  int occ_all = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_all, panel_kernel<true>, THREADS, SMEM_BYTES);
  occ = std::min(occ, occ_all);
  return std::max(1, occ);
}

int panel_grid_size() {
  const int occ = panel_ctas_per_sm();
  if (occ < 0) return occ;
  return std::max(2, device_sm_count() * occ);
}

int panel_launch(const PanelBatch& batch, int grid, cudaStream_t stream) {
  int g = panel_grid_size();
  if (g <= 0) return -g;
  if (grid <= 0 || grid > g) grid = g;
  grid = std::min(grid, batch.ntasks + batch.ninst);
  grid = std::max(grid, batch.ninst + (batch.ntasks > 0 ? 1 : 0));
  {
    bta::ProfScope _ps(bta::PROF_PANEL, stream);
    if (batch.cols != nullptr) panel_kernel<true><<<grid, THREADS, SMEM_BYTES, stream>>>(batch);
    else panel_kernel<false><<<grid, THREADS, SMEM_BYTES, stream>>>(batch);
  }
  return cudaGetLastError();
}

}  // namespace bta
