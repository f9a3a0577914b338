// Grouped GEMM with FP32-class accuracy on the 5th-generation tensor cores
// (tcgen05.mma kind::tf32, accumulator in tensor memory).
//
// Every FP64 operand element x is split into two TF32 values, hi = tf32(x)
// and lo = tf32(x - hi), and C = beta C + sum_s alpha_s opA_s opB_s is
// accumulated in FP32 as A_hi B_hi + A_hi B_lo + A_lo B_hi: each product is
// exact in FP32, the dropped A_lo B_lo term is below 2^-22 |a||b|, so the
// result carries FP32 accumulation error (the "split TF32 x3" scheme).
// Operand conventions and problem batching are those of the FP64 kernel
// (gemm.cuh); only the arithmetic differs.
//
// CTA layout: 8 producer warps + 1 MMA warp.  Producers read FP64 operand
// slabs of 128 rows x 32 k in 4x4 micro-tiles (coalesced along whichever
// dimension is contiguous in memory), split them and store hi / lo into
// 128-byte-swizzled K-major shared memory; one thread of the MMA warp issues
// 12 MMAs (128x128x8 each) per slab into a 128-column TMEM accumulator and
// releases the slab with tcgen05.commit.  A 3-slab ring of full / empty
// mbarriers connects the two sides.  The producers then read the accumulator
// back (tcgen05.ld) and write C in FP64.  Every wait is bounded (about two
// seconds of SM clock) and raises the abort flag instead of hanging.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "gemm.cuh"
#include "prof.cuh"

namespace bta {
namespace {

constexpr int TBM = 128, TBN = 128, TBK = 32;  // output tile; k-slab = one 128-byte row of FP32
constexpr int TSTAGES = 3;
constexpr int PRODUCERS = 256;
constexpr int TTHREADS = PRODUCERS + 32;
constexpr int OP_BYTES = TBM * TBK * 4;   // one split half of one operand slab (16 KB)
constexpr int STAGE_BYTES = 4 * OP_BYTES;  // A_hi, A_lo, B_hi, B_lo
constexpr int BAR_BYTES = 128;
constexpr size_t TSMEM_BYTES = size_t(TSTAGES) * STAGE_BYTES + BAR_BYTES + 1024;
constexpr long long WAIT_CYCLES = 4000000000LL;
static_assert(TBM == TBN, "producer mapping assumes square tiles");

// Instruction descriptor: D FP32 (bits 4-5 = 1), A and B TF32 (bits 7-9,
// 10-12 = 2), both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28.
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TBN >> 3) << 17) |
                           ((uint32_t)(TBM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor of a K-major operand in the 128-byte
// swizzle layout: rows of 128 bytes, 8-row groups 1024 bytes apart (stride
// byte offset), descriptor version 1, layout type 2 (SWIZZLE_128B).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the phase of the given parity; false on timeout or abort.
__device__ bool mbar_wait(uint32_t bar, uint32_t parity, int* abort_flag) {
  if (mbar_try(bar, parity)) return true;
  const long long t0 = clock64();
  for (int it = 1;; ++it) {
    if (mbar_try(bar, parity)) return true;
    if ((it & 63) == 0) {
      if (*reinterpret_cast<volatile int*>(abort_flag)) return false;
      if (clock64() - t0 > WAIT_CYCLES) {
        atomicExch(abort_flag, 1);
        return false;
      }
    }
  }
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(IDESC), "r"(accum), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

// 32 consecutive FP32 accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Round an FP32 value to the nearest TF32 value (10 explicit mantissa bits).
__device__ __forceinline__ float tf32_rn(float f) {
  return __uint_as_float((__float_as_uint(f) + 0x1000u) & 0xFFFFE000u);
}

__device__ __forceinline__ void split2(double x, float& hi, float& lo) {
  hi = tf32_rn(__double2float_rn(x));
  lo = tf32_rn(__double2float_rn(x - (double)hi));
}

// k-range [kb, kmax) of one segment for the output tile at (m0, n0); kb is
// rounded down to the slab size (the skipped region holds zeros).
__device__ __forceinline__ int seg_range(const GemmSeg& s, int m0, int n0, int& kb, int& kmax) {
  int kmin = 0;
  kmax = s.K;
  if (s.flags & GF_K_GE_M) kmin = max(kmin, m0);
  if (s.flags & GF_K_GE_N) kmin = max(kmin, n0);
  if (s.flags & GF_K_LE_M) kmax = min(kmax, m0 + TBM);
  if (s.flags & GF_K_LE_N) kmax = min(kmax, n0 + TBN);
  kb = kmin & ~(TBK - 1);
  return kmax > kb ? (kmax - kb + TBK - 1) / TBK : 0;
}

// Stage one 128 x 32 operand slab: element (r, k) of the operand is
// P[r*ld + k] (kcontig) or P[k*ld + r]; rows >= rmax and k >= kmax read as 0.
// Thread t owns a 4x4 micro-tile and writes one 16-byte chunk per row into
// the hi and lo buffers (chunk index XOR row % 8: the 128-byte swizzle).
__device__ __forceinline__ void stage_operand(uint8_t* hi_base, uint8_t* lo_base, const double* P, int ld,
                                              bool kcontig, bool vec, int r0, int rmax, int k0, int kmax,
                                              double alpha, int t) {
  double v[4][4];
  int ri, ki;
  if (kcontig) {
    ki = t & 7;
    ri = t >> 3;
    const int gk = k0 + 4 * ki;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int gr = r0 + 4 * ri + e;
      const double* src = P + (size_t)gr * ld + gk;
      if (vec && gr < rmax && gk + 3 < kmax) {
        const double2 x0 = *reinterpret_cast<const double2*>(src);
        const double2 x1 = *reinterpret_cast<const double2*>(src + 2);
        v[e][0] = x0.x;
        v[e][1] = x0.y;
        v[e][2] = x1.x;
        v[e][3] = x1.y;
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) v[e][j] = (gr < rmax && gk + j < kmax) ? src[j] : 0.0;
      }
    }
  } else {
    ri = t & 31;
    ki = t >> 5;
    const int gr = r0 + 4 * ri;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gk = k0 + 4 * ki + j;
      const double* src = P + (size_t)gk * ld + gr;
      if (vec && gk < kmax && gr + 3 < rmax) {
        const double2 x0 = *reinterpret_cast<const double2*>(src);
        const double2 x1 = *reinterpret_cast<const double2*>(src + 2);
        v[0][j] = x0.x;
        v[1][j] = x0.y;
        v[2][j] = x1.x;
        v[3][j] = x1.y;
      } else {
#pragma unroll
        for (int e = 0; e < 4; ++e) v[e][j] = (gk < kmax && gr + e < rmax) ? src[e] : 0.0;
      }
    }
  }
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int row = 4 * ri + e;
    const uint32_t off = (uint32_t)row * 128u + ((uint32_t)(ki ^ (row & 7)) << 4);
    float4 h, l;
    split2(alpha * v[e][0], h.x, l.x);
    split2(alpha * v[e][1], h.y, l.y);
    split2(alpha * v[e][2], h.z, l.z);
    split2(alpha * v[e][3], h.w, l.w);
    *reinterpret_cast<float4*>(hi_base + off) = h;
    *reinterpret_cast<float4*>(lo_base + off) = l;
  }
}

__global__ void __launch_bounds__(TTHREADS, 1) gemm_tc_kernel(const __grid_constant__ GemmBatch batch,
                                                               int* abort_flag) {
  extern __shared__ uint8_t smem_raw[];
  // the 128-byte swizzle repeats every 1024 bytes of shared-window address
  uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  uint8_t* bars = smem + TSTAGES * STAGE_BYTES;
  const uint32_t full0 = smem_u32(bars), empty0 = full0 + 8 * TSTAGES, done_bar = empty0 + 8 * TSTAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 8 * (2 * TSTAGES + 1));

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int bid = blockIdx.x;
  int pi = 0;
  while (pi + 1 < batch.count && bid >= batch.tile_start[pi + 1]) ++pi;
  const GemmProb& P = batch.p[pi];
  const int local = bid - batch.tile_start[pi];
  int tm, tn;
  if (P.cflags & GC_LOWER) {
    tm = (int)((sqrt(8.0 * local + 1.0) - 1.0) * 0.5);
    while ((tm + 1) * (tm + 2) / 2 <= local) ++tm;
    while (tm * (tm + 1) / 2 > local) --tm;
    tn = local - tm * (tm + 1) / 2;
  } else {
    tm = local / batch.tiles_n[pi];
    tn = local % batch.tiles_n[pi];
  }
  const int m0 = tm * TBM, n0 = tn * TBN;

  if (warp == PRODUCERS / 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"((uint32_t)TBN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int s = 0; s < TSTAGES; ++s) {
      mbar_init(full0 + 8 * s, PRODUCERS);
      mbar_init(empty0 + 8 * s, 1);
    }
    mbar_init(done_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  int nsteps = 0;
  for (int si = 0; si < P.nseg; ++si) {
    int kb, kmax;
    nsteps += seg_range(P.seg[si], m0, n0, kb, kmax);
  }
  const uint32_t stage0 = smem_u32(smem);

  if (warp < PRODUCERS / 32) {
    // ---------------------------------------------------------- producers
    bool ok = true;
    int step = 0;
    for (int si = 0; si < P.nseg && ok; ++si) {
      const GemmSeg& s = P.seg[si];
      int kb, kmax;
      const int nk = seg_range(s, m0, n0, kb, kmax);
      const bool akc = !(s.flags & GF_A_T);
      const bool bkc = !(s.flags & GF_B_KN);
      const bool vecA = ((s.lda & 1) == 0) && ((reinterpret_cast<uintptr_t>(s.A) & 15) == 0);
      const bool vecB = ((s.ldb & 1) == 0) && ((reinterpret_cast<uintptr_t>(s.B) & 15) == 0);
      for (int kt = 0; kt < nk; ++kt, ++step) {
        const int st = step % TSTAGES;
        if (step >= TSTAGES && !mbar_wait(empty0 + 8 * st, ((step / TSTAGES) - 1) & 1, abort_flag)) {
          ok = false;
          break;
        }
        uint8_t* base = smem + st * STAGE_BYTES;
        const int k0 = kb + kt * TBK;
        stage_operand(base, base + OP_BYTES, s.A, s.lda, akc, vecA, m0, P.M, k0, kmax, s.alpha, tid);
        stage_operand(base + 2 * OP_BYTES, base + 3 * OP_BYTES, s.B, s.ldb, bkc, vecB, n0, P.N, k0, kmax, 1.0,
                      tid);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive(full0 + 8 * st);
      }
    }
    // ---------------------------------------------------------- epilogue
    const bool have = __all_sync(0xffffffffu, nsteps > 0 && mbar_wait(done_bar, 0, abort_flag));
    tc_fence_after();
    const int q = warp & 3, h = warp >> 2;
    const int row = m0 + 32 * q + lane;
    const bool lower = P.cflags & GC_LOWER;
    const bool mirror = P.cflags & GC_MIRROR;
    const double beta = P.beta;
    double* C = P.C;
    const int ldc = P.ldc;
#pragma unroll 1
    for (int c = 0; c < 2; ++c) {
      const int col0 = n0 + 64 * h + 32 * c;
      float acc[32];
      if (have) {
        tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(64 * h + 32 * c), acc);
      } else {
#pragma unroll
        for (int j = 0; j < 32; ++j) acc[j] = 0.0f;
      }
      if (row >= P.M || col0 >= P.N || (lower && col0 > row)) continue;
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const int col = col0 + j;
        if (col >= P.N || (lower && col > row)) continue;
        double v = (double)acc[j];
        double* dst = C + (size_t)row * ldc + col;
        if (beta != 0.0) v += beta * *dst;
        *dst = v;
        if (mirror && col < row) C[(size_t)col * ldc + row] = v;
      }
    }
  } else if (lane == 0) {
    // ---------------------------------------------------------- MMA issuer
    for (int step = 0; step < nsteps; ++step) {
      const int st = step % TSTAGES;
      if (!mbar_wait(full0 + 8 * st, (step / TSTAGES) & 1, abort_flag)) break;
      tc_fence_after();
      const uint32_t a_hi = stage0 + st * STAGE_BYTES, a_lo = a_hi + OP_BYTES;
      const uint32_t b_hi = a_lo + OP_BYTES, b_lo = b_hi + OP_BYTES;
#pragma unroll
      for (int kk = 0; kk < TBK / 8; ++kk) {
        const uint32_t o = kk * 32;
        mma_tf32(tmem, sw128_desc(a_hi + o), sw128_desc(b_hi + o), (step | kk) != 0 ? 1u : 0u);
        mma_tf32(tmem, sw128_desc(a_hi + o), sw128_desc(b_lo + o), 1u);
        mma_tf32(tmem, sw128_desc(a_lo + o), sw128_desc(b_hi + o), 1u);
      }
      tc_commit(empty0 + 8 * st);
    }
    tc_commit(done_bar);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == PRODUCERS / 32) {
    tc_fence_after();
    // every issued MMA has completed: the epilogue waited for done_bar, or
    // (no steps / abort) nothing is outstanding beyond what done_bar tracks
    if (nsteps > 0 && lane == 0) mbar_wait(done_bar, 0, abort_flag);
    __syncwarp();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)TBN)
                 : "memory");
  }
}

}  // namespace

int gemm_launch_tc(const std::vector<GemmProb>& probs, cudaStream_t stream, int* abort_flag) {
  {
    const int e = ensure_smem_attr(reinterpret_cast<const void*>(gemm_tc_kernel), (int)TSMEM_BYTES);
    if (e != cudaSuccess) return (cudaError_t)e;
  }
  if (!abort_flag) return cudaErrorInvalidValue;
  size_t i = 0;
  while (i < probs.size()) {
    GemmBatch b;
    std::memset(&b, 0, sizeof(b));
    int total = 0;
    for (; i < probs.size() && b.count < GEMM_MAXP; ++i) {
      const GemmProb& p = probs[i];
      if (p.M <= 0 || p.N <= 0) continue;
      const int tmn = (p.M + TBM - 1) / TBM, tnn = (p.N + TBN - 1) / TBN;
      int tiles;
      if (p.cflags & GC_LOWER) {
        if (p.M != p.N) return cudaErrorInvalidValue;
        tiles = tmn * (tmn + 1) / 2;
      } else {
        tiles = tmn * tnn;
      }
      b.p[b.count] = p;
      b.tiles_n[b.count] = tnn;
      b.tile_start[b.count] = total;
      total += tiles;
      b.count++;
    }
    if (b.count == 0) continue;
    b.tile_start[b.count] = total;
    {
      bta::ProfScope _ps(bta::PROF_GEMM, stream);
      gemm_tc_kernel<<<total, TTHREADS, TSMEM_BYTES, stream>>>(b, abort_flag);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace bta
