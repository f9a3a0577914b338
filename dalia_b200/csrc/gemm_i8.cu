// Grouped GEMM with near-FP64 accuracy from 8-bit tensor-core products
// (tcgen05.mma kind::i8, exact INT32 accumulation in tensor memory): the
// Ozaki splitting scheme.
//
// Every row m of op(A) (over all segments of a problem) gets one power-of-two
// scale 2^e_m with max_k |alpha A[m][k]| < 2^e_m, every column n of op(B) one
// scale 2^f_n; the scaled entries lie in (-1, 1) and are cut into OZ_S signed
// 7-bit digits (truncation: |x 2^-e - sum_p a_p 2^-7p| < 2^-7 OZ_S).  Then
//   C[m][n] = beta C + 2^(e_m + f_n) sum_{d} 2^-7d sum_{p+q=d} (a_p . b_q)
// where every digit product sum is exact in INT32 (|a_p b_q| <= 127^2, at
// most OZ_S pairs per d, K <= 19000).  Keeping the pairs with p + q <= OZ_S - 1
// (28 of 49, digits counted from 0) drops products below 2^-7(OZ_S+2) 127^2
// per element product: an error of ~1e-14 relative to max_k |a_mk| max_k
// |b_kn| K for OZ_S = 7 (small entries of a row or column with a wide range
// keep fewer bits than their own magnitude would allow).  Seven digits are needed because the
// selected inversion of an ill-conditioned precision (cond ~1e9 per block)
// amplifies the truncation: five digits left gradient errors of 2e-3 at
// b = 1500.
//
// Pipeline: slice_kernel (per 16 rows of a problem side: the maxima over all
// segments -> exponents, then the digits, written as the 32-byte-swizzled
// K-major shared-memory images the MMA reads) and gemm_i8_kernel, persistent
// CTAs over 128 x 64 output tiles: one producer thread bulk-copies the digit
// images of each 32-wide k-slab (A: 128 rows x OZ_S digits, B: 64 rows x OZ_S
// digits, no multicast) into a 3-stage ring; one thread issues the products
// of the slab, one MMA per A digit p against the stacked B digits (N up to
// 256: 10 MMAs for 28 digit pairs), each pair (p, q) landing in the TMEM
// accumulator of d = p + q; eight epilogue warps (two per 32-lane quarter of
// tensor memory, each taking half of the tile's columns) read the OZ_S
// accumulators (tcgen05.ld), combine them exactly, scale, release the tensor
// memory to the next tile and write C in FP64 through a shared-memory stage.  Every
// wait is bounded and raises the abort flag on timeout.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "gemm.cuh"
#include "prof.cuh"
#include "tune.cuh"

namespace bta {
namespace {

constexpr int OZ_S = 7;                        // digits per operand
constexpr int QBM = 128, QBK = 32;             // output tile rows, k-slab (32 int8 = one 32-byte row)
constexpr int IMG = 64 * QBK;                  // one 64-row digit image (2 KB)
constexpr int QSTAGES = 4;
constexpr int A_SLICE = 2 * IMG;               // 128 rows
constexpr int QEPI_WARPS = 8;                  // warps 0-7: epilogue (warp w: lanes 32 (w % 4).., column half w / 4)
constexpr int QPROD_WARP = QEPI_WARPS, QMMA_WARP = QEPI_WARPS + 1;
constexpr int QTHREADS = (QEPI_WARPS + 2) * 32;
constexpr int TMEM_COLS = 512;
constexpr long long QWAIT_CYCLES = 4000000000LL;
constexpr int EXP_NONE = -1100;                // exponent of an all-zero row

// The output tile is QBM x BN, BN = 64 or 32 columns (a template parameter
// of the kernel; the autotuner picks it per launch shape).  The OZ_S level
// accumulators of a tile take OZ_S BN columns of tensor memory: with BN = 64
// one set (448 of 512 columns), so a tile's products wait until the epilogue
// has read the previous tile's; with BN = 32 two sets (224 columns each, at
// columns 0 and 256), so the products of tile t+1 run while the epilogue
// drains tile t -- at the price of half the B operand per A slab.
template <int BN>
struct QTile {
  static constexpr int B_SLICE = BN * QBK;                   // BN rows of a digit image
  static constexpr int STAGE_BYTES = OZ_S * (A_SLICE + B_SLICE);
  static constexpr int NSETS = BN == 32 ? 2 : 1;             // accumulator sets in tensor memory
  static constexpr int SET_COLS = 256;
  static constexpr int CW = BN / 2;                          // columns per epilogue warp
  static constexpr int STAGE_LD = 17;                        // its staging rows (16 columns at a time), padded
  static constexpr int EPI_BYTES = QEPI_WARPS * 32 * STAGE_LD * 8;
  static constexpr size_t SMEM_BYTES = size_t(QSTAGES) * STAGE_BYTES + EPI_BYTES + 256 + 1024;
  static_assert(BN == 32 || BN == 64, "tile width");
  static_assert(OZ_S * BN <= (NSETS == 2 ? SET_COLS : TMEM_COLS), "accumulators exceed tensor memory");
};

// Instruction descriptor: D S32 (bits 4-5 = 2), A and B signed 8-bit (bits
// 7-9, 10-12 = 1), both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28.
__host__ __device__ constexpr uint32_t idesc_i8(int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(QBM >> 4) << 24);
}
constexpr int QMMA_NMAX = 256;  // largest N of one M = 128 MMA

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Exact double of an integer |n| < 2^51: the bits of 1.5 2^52 + n, minus 1.5 2^52.
__device__ __forceinline__ double exact_double(long long n) {
  return __longlong_as_double(0x4338000000000000LL + n) - 6755399441055744.0;
}

// K-major operand in the 32-byte swizzle layout: rows of 32 bytes, 8-row
// groups 256 bytes apart, descriptor version 1, layout type 6 (SWIZZLE_32B).
__device__ __forceinline__ uint64_t sw32_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(256 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)6 << 61);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%1], %0;" ::"r"(bytes), "r"(bar) : "memory");
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
__device__ bool mbar_wait(uint32_t bar, uint32_t parity, int* abort_flag) {
  if (mbar_try(bar, parity)) return true;
  const long long t0 = clock64();
  for (int it = 1;; ++it) {
    if (mbar_try(bar, parity)) return true;
    if ((it & 63) == 0) {
      if (*reinterpret_cast<volatile int*>(abort_flag)) return false;
      if (clock64() - t0 > QWAIT_CYCLES) {
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
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}
// 16 columns of the warp's 32 lanes, asynchronous: the registers are valid
// after tmem_wait16().
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
}
// Waits for the outstanding tensor-memory loads; r (the destination of the
// last one) is an operand so no read of it moves above the wait.
__device__ __forceinline__ void tmem_wait16(uint32_t (&r)[16]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                 "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
               :
               : "memory");
}


// ---------------------------------------------------------------- slicing
// One side of one problem: the op(A) (or op(B)) operands of its segments,
// which share one exponent per image row.  Segment s: element (r, k) at
// P[r*ld + k] (kcontig) or P[k*ld + r], scaled by alpha; its digits go to
// out[(p*KT + kt)*RB + rb] (one 2 KB image per 64 rows x 32 k).
struct SliceSeg {
  const double* P;
  int8_t* out;
  double alpha;
  int ld, K, kcontig, KT;
};

struct SliceGroup {
  int* exps;       // exponent of every image row < rows
  int rows;        // rows with data (M or N); image rows up to 64 RB are zero
  int RB;          // 64-row image blocks
  int nseg;
  int unit_start;  // first SU-row unit of this group
  SliceSeg s[3];
};

constexpr int SLICE_MAXG = 48;
constexpr int SLICE_THREADS = 256;
constexpr int SU = 16;  // image rows per slicing unit

struct SliceBatch {
  int count;
  int units;
  SliceGroup g[SLICE_MAXG];
};

__device__ __forceinline__ int exponent_of(double m) {
  if (!(m > 0.0)) return EXP_NONE;
  int e;
  frexp(m, &e);  // m = f 2^e, f in [0.5, 1): m < 2^e
  return e;
}

// 4 x 4 byte transpose: out[i] byte j = in[j] byte i.
__device__ __forceinline__ void transpose4(const uint32_t (&in)[4], uint32_t (&out)[4]) {
  const uint32_t t0 = __byte_perm(in[0], in[1], 0x5140), t1 = __byte_perm(in[0], in[1], 0x7362);
  const uint32_t t2 = __byte_perm(in[2], in[3], 0x5140), t3 = __byte_perm(in[2], in[3], 0x7362);
  out[0] = __byte_perm(t0, t2, 0x5410);
  out[1] = __byte_perm(t0, t2, 0x7632);
  out[2] = __byte_perm(t1, t3, 0x5410);
  out[3] = __byte_perm(t1, t3, 0x7632);
}

// Digits of one 16-k chunk (image row rg, k = 16 kc ..) of segment S with
// exponent e, written to the swizzled K-major image.  The truncated integer
// U = |alpha x| 2^(7 OZ_S - e) < 2^49 splits into 28 + 21 bits; each half's
// 7-bit digits are spread to bytes (digit 3 and digit 6 in byte 0), negated
// per byte for negative entries, and four consecutive k are transposed into
// the digit planes (byte j of a plane word = k offset j).
static_assert(OZ_S == 7, "the digit spreading below cuts 4 + 3 digits");
__device__ __forceinline__ void cut_chunk(const SliceSeg& S, int RB, int rg, bool rowok, int kc, int e) {
  const int k0 = kc * 16;
  double xs[16];
  if (S.kcontig && rowok && k0 + 15 < S.K && ((S.ld & 1) == 0) && ((reinterpret_cast<uintptr_t>(S.P) & 15) == 0)) {
    const double2* src = reinterpret_cast<const double2*>(S.P + (size_t)rg * S.ld + k0);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const double2 v = src[j];
      xs[2 * j] = v.x;
      xs[2 * j + 1] = v.y;
    }
  } else {
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int k = k0 + j;
      xs[j] = (rowok && k < S.K) ? S.P[S.kcontig ? (size_t)rg * S.ld + k : (size_t)k * S.ld + rg] : 0.0;
    }
  }
  // |alpha| 2^(7 OZ_S - e) is exact; products with it round like alpha x
  // scaled afterwards.  Scales beyond the double range (tiny rows) scale
  // |alpha x| by 2^(sh - 600) and 2^600, both exact; an all-zero row gets 0.
  // Every entry takes the same three products (no per-entry branch).
  const int sh = 7 * OZ_S - e;
  const bool direct = e != EXP_NONE && sh < 1000;
  const double s1 = direct ? ldexp(fabs(S.alpha), sh)
                           : (e == EXP_NONE ? 0.0 : __longlong_as_double((long long)(sh - 600 + 1023) << 52));
  const double s2 = direct ? 1.0 : 0x1p600;
  const double a1 = direct ? 1.0 : S.alpha;
  const bool aneg = S.alpha < 0.0;
  uint32_t w[OZ_S][4];
#pragma unroll
  for (int g4 = 0; g4 < 4; ++g4) {
    uint32_t hw[4], lw[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const double x = xs[4 * g4 + i];
      const unsigned long long U = __double2ull_rz((fabs(x * a1) * s1) * s2);
      const uint32_t hi = (uint32_t)(U >> 21), lo = (uint32_t)U & 0x1FFFFFu;
      uint32_t H = (hi & 0x7Fu) | ((hi << 1) & 0x7F00u) | ((hi << 2) & 0x7F0000u) | ((hi << 3) & 0x7F000000u);
      uint32_t Lw = (lo & 0x7Fu) | ((lo << 1) & 0x7F00u) | ((lo << 2) & 0x7F0000u);
      if ((x < 0.0) != aneg) {
        H = __vneg4(H);
        Lw = __vneg4(Lw);
      }
      hw[i] = H;
      lw[i] = Lw;
    }
    uint32_t th[4], tl[4];
    transpose4(hw, th);
    transpose4(lw, tl);
    // H byte b holds digit 3 - b, Lw byte b digit 6 - b
    w[0][g4] = th[3];
    w[1][g4] = th[2];
    w[2][g4] = th[1];
    w[3][g4] = th[0];
    w[4][g4] = tl[2];
    w[5][g4] = tl[1];
    w[6][g4] = tl[0];
  }
  const int kt = kc >> 1, c = kc & 1, rb = rg >> 6, rr = rg & 63;
  const size_t off = (size_t)rr * 32 + ((size_t)(c ^ ((rr >> 2) & 1)) << 4);
#pragma unroll
  for (int p = 0; p < OZ_S; ++p) {
    int8_t* dst = S.out + (((size_t)p * S.KT + kt) * RB + rb) * IMG + off;
    *reinterpret_cast<uint4*>(dst) = make_uint4(w[p][0], w[p][1], w[p][2], w[p][3]);
  }
}

// A CTA per unit of SU image rows of one group: the rows' maxima over all
// segments, their exponents, then the digits of every segment.
__global__ void __launch_bounds__(SLICE_THREADS, 4) slice_kernel(const __grid_constant__ SliceBatch B) {
  constexpr int NW = SLICE_THREADS / 32;
  __shared__ double red[NW][32];
  __shared__ int ex[SU];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int u = blockIdx.x; u < B.units; u += gridDim.x) {
    int gi = 0;
    while (gi + 1 < B.count && u >= B.g[gi + 1].unit_start) ++gi;
    const SliceGroup& G = B.g[gi];
    const int r0 = (u - G.unit_start) * SU;
    double m = 0.0;  // row max (thread r < SU)
    for (int si = 0; si < G.nseg; ++si) {
      const SliceSeg& S = G.s[si];
      double ms = 0.0;
      if (S.kcontig) {
        // a row per SLICE_THREADS / SU threads (whole warps), 16-byte loads along k
        constexpr int TPR = SLICE_THREADS / SU;
        const int r = tid / TPR, sub = tid % TPR, rg = r0 + r;
        if (rg < G.rows) {
          const double* row = S.P + (size_t)rg * S.ld;
          if (((S.ld & 1) == 0) && ((reinterpret_cast<uintptr_t>(S.P) & 15) == 0)) {
            int k = 2 * sub;
#pragma unroll 4
            for (; k + 1 < S.K; k += 2 * TPR) {
              const double2 v = *reinterpret_cast<const double2*>(row + k);
              ms = fmax(ms, fmax(fabs(v.x), fabs(v.y)));
            }
            if (k < S.K) ms = fmax(ms, fabs(row[k]));
          } else {
            for (int k = sub; k < S.K; k += TPR) ms = fmax(ms, fabs(row[k]));
          }
        }
#pragma unroll
        for (int o = (TPR < 32 ? TPR : 32) / 2; o > 0; o >>= 1) ms = fmax(ms, __shfl_xor_sync(0xffffffffu, ms, o));
        red[warp][lane] = ms;  // every thread of a row (or of a warp of it) holds its maximum
        __syncthreads();
        if (tid < SU) {
          double v = 0.0;
          if (TPR >= 32) {
            for (int w = tid * (TPR / 32); w < (tid + 1) * (TPR / 32); ++w) v = fmax(v, red[w][0]);
          } else {
            v = red[(tid * TPR) / 32][(tid * TPR) % 32];
          }
          m = fmax(m, fabs(S.alpha) * v);
        }
        __syncthreads();
      } else {
        // column c = tid % SU of the unit, k phases tid / SU
        constexpr int KP = SLICE_THREADS / SU;
        const int c = tid % SU, ph = tid / SU, rg = r0 + c;
        if (rg < G.rows) {
          const double* col = S.P + rg;
          int k = ph;
          for (; k + 7 * KP < S.K; k += 8 * KP) {  // eight independent loads in flight
            double v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = col[(size_t)(k + j * KP) * S.ld];
#pragma unroll
            for (int j = 0; j < 8; ++j) ms = fmax(ms, fabs(v[j]));
          }
          for (; k < S.K; k += KP) ms = fmax(ms, fabs(col[(size_t)k * S.ld]));
        }
#pragma unroll
        for (int o = SU; o < 32; o <<= 1) ms = fmax(ms, __shfl_xor_sync(0xffffffffu, ms, o));
        if (lane < SU) red[warp][lane] = ms;
        __syncthreads();
        if (tid < SU) {
          double v = 0.0;
#pragma unroll
          for (int w = 0; w < NW; ++w) v = fmax(v, red[w][tid]);
          m = fmax(m, fabs(S.alpha) * v);
        }
        __syncthreads();
      }
    }
    if (tid < SU) {
      const int e = exponent_of(m);
      ex[tid] = e;
      if (r0 + tid < G.rows) G.exps[r0 + tid] = e;
    }
    __syncthreads();
    // digits: chunk (row r, 16-k chunk kc), consecutive threads along k for
    // kcontig segments, along rows otherwise (coalesced FP64 reads)
    for (int si = 0; si < G.nseg; ++si) {
      const SliceSeg& S = G.s[si];
      const int nkc = 2 * S.KT;
      for (int q = tid; q < SU * nkc; q += SLICE_THREADS) {
        int r, kc;
        if (S.kcontig) {
          r = q / nkc;
          kc = q - r * nkc;
        } else {
          kc = q / SU;
          r = q - kc * SU;
        }
        const int rg = r0 + r;
        const bool rowok = rg < G.rows;
        cut_chunk(S, G.RB, rg, rowok, kc, rowok ? max(ex[r], EXP_NONE) : EXP_NONE);
      }
    }
    __syncthreads();  // ex and red are reused by the next unit
  }
}

// ---------------------------------------------------------------- GEMM
struct QSeg {
  const int8_t* A;  // digit images of op(A): OZ_S x KT x RBa images
  const int8_t* B;  // digit images of op(B): OZ_S x KT x RBb images
  int KT, RBa, RBb, kflags, K;
};

struct QProb {
  double* C;
  const int* eA;  // M row exponents
  const int* fB;  // N column exponents
  double beta;
  double sgn;     // +1, or -1 when a one-segment product's alpha = -1 is applied here
  int ldc, M, N, nseg, cflags, tmn, tnn;
  QSeg seg[3];
};

constexpr int QMAXP = 48;

struct QBatch {
  int count;
  int tile_start[QMAXP + 1];
  QProb p[QMAXP];
};

// lower-only tiles: (tm, tn) with tn * BN <= tm * QBM + QBM - 1
__host__ __device__ __forceinline__ int lower_tiles_row(int tm, int tnn, int bn) {
  return min((tm + 1) * (QBM / bn), tnn);
}

template <int BN>
__device__ __forceinline__ int qseg_range(const QSeg& s, int m0, int n0, int& kt0) {
  int kmin = 0, kmax = s.K;
  if (s.kflags & GF_K_GE_M) kmin = max(kmin, m0);
  if (s.kflags & GF_K_GE_N) kmin = max(kmin, n0);
  if (s.kflags & GF_K_LE_M) kmax = min(kmax, m0 + QBM);
  if (s.kflags & GF_K_LE_N) kmax = min(kmax, n0 + BN);
  kt0 = kmin / QBK;
  const int kt1 = (kmax + QBK - 1) / QBK;
  return kt1 > kt0 ? kt1 - kt0 : 0;
}

// Tile t of a batch: problem, tile row, tile column.
template <int BN>
__device__ __forceinline__ void decode_tile(const QBatch& batch, int t, int& pi, int& tm, int& tn) {
  pi = 0;
  while (pi + 1 < batch.count && t >= batch.tile_start[pi + 1]) ++pi;
  const QProb& P = batch.p[pi];
  int local = t - batch.tile_start[pi];
  tm = 0;
  if (P.cflags & GC_LOWER) {
    while (local >= lower_tiles_row(tm, P.tnn, BN)) local -= lower_tiles_row(tm++, P.tnn, BN);
    tn = local;
  } else {
    tm = local / P.tnn;
    tn = local - tm * P.tnn;
  }
}

template <int BN>
__device__ __forceinline__ int tile_steps(const QProb& P, int m0, int n0) {
  int nsteps = 0;
  for (int si = 0; si < P.nseg; ++si) {
    int kt0;
    nsteps += qseg_range<BN>(P.seg[si], m0, n0, kt0);
  }
  return nsteps;
}

// Persistent: CTA c takes tiles c, c + grid, ...  The producer's ring runs
// across tile boundaries; tile number it (of this CTA) accumulates into set
// it % NSETS, and the MMA warp starts it once the epilogue has read the
// accumulators of tile it - NSETS out of tensor memory (tmem_empty of that
// set), so the epilogue's scaling and stores overlap later tiles' products.
template <int BN>
__global__ void __launch_bounds__(QTHREADS, 1) gemm_i8_kernel(const __grid_constant__ QBatch batch, int total_tiles,
                                                               int* abort_flag) {
  using TT = QTile<BN>;
  constexpr int NSETS = TT::NSETS;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  double* epi_stage = reinterpret_cast<double*>(smem + QSTAGES * TT::STAGE_BYTES);
  uint8_t* bars = smem + QSTAGES * TT::STAGE_BYTES + TT::EPI_BYTES;
  // barriers: full[QSTAGES], empty[QSTAGES], done[2], tmem_empty[2], drain
  const uint32_t full0 = smem_u32(bars), empty0 = full0 + 8 * QSTAGES, done0 = empty0 + 8 * QSTAGES;
  const uint32_t tmem_empty0 = done0 + 16, drain_bar = done0 + 32;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 8 * (2 * QSTAGES + 5));

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (warp == QMMA_WARP) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"((uint32_t)TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int s = 0; s < QSTAGES; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    for (int k = 0; k < 2; ++k) {
      mbar_init(done0 + 8 * k, 1);
      mbar_init(tmem_empty0 + 8 * k, QEPI_WARPS);  // one arrival per epilogue warp
    }
    mbar_init(drain_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t stage0 = smem_u32(smem);

  if (warp == QPROD_WARP) {
    // ------------------------------------------------------ producer
    if (lane == 0) {
      int step = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < total_tiles && ok; t += gridDim.x) {
        int pi, tm, tn;
        decode_tile<BN>(batch, t, pi, tm, tn);
        const QProb& P = batch.p[pi];
        // B rows of this tile: image (tn BN) / 64, from row (tn BN) % 64 (the
        // second 32 rows of an image start 1 KB in: four whole 8-row groups)
        const size_t bimg = (size_t)(tn * BN) / 64, boff = (size_t)((tn * BN) % 64) * QBK;
        for (int si = 0; si < P.nseg && ok; ++si) {
          const QSeg& sg = P.seg[si];
          int kt0;
          const int nk = qseg_range<BN>(sg, tm * QBM, tn * BN, kt0);
          for (int i = 0; i < nk; ++i, ++step) {
            const int st = step % QSTAGES;
            if (step >= QSTAGES && !mbar_wait(empty0 + 8 * st, ((step / QSTAGES) - 1) & 1, abort_flag)) {
              ok = false;
              break;
            }
            const int kt = kt0 + i;
            const uint32_t bar = full0 + 8 * st;
            mbar_expect_tx(bar, TT::STAGE_BYTES);
            const uint32_t dst = stage0 + st * TT::STAGE_BYTES;
#pragma unroll
            for (int p = 0; p < OZ_S; ++p) {
              bulk_g2s(dst + p * A_SLICE, sg.A + (((size_t)p * sg.KT + kt) * sg.RBa + 2 * tm) * IMG, A_SLICE, bar);
              bulk_g2s(dst + OZ_S * A_SLICE + p * TT::B_SLICE,
                       sg.B + (((size_t)p * sg.KT + kt) * sg.RBb + bimg) * IMG + boff, TT::B_SLICE, bar);
            }
          }
        }
      }
    }
  } else if (warp == QMMA_WARP) {
    // ------------------------------------------------------ MMA issuer
    if (lane == 0) {
      int step = 0, it = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < total_tiles && ok; t += gridDim.x, ++it) {
        int pi, tm, tn;
        decode_tile<BN>(batch, t, pi, tm, tn);
        const int nsteps = tile_steps<BN>(batch.p[pi], tm * QBM, tn * BN);
        const int set = it % NSETS, use = it / NSETS;
        const uint32_t tacc = tmem + (uint32_t)(set * TT::SET_COLS);
        // the epilogue has read the accumulators of this set's previous tile
        if (use > 0 && !mbar_wait(tmem_empty0 + 8 * set, (use - 1) & 1, abort_flag)) break;
        tc_fence_after();
        for (int ks = 0; ks < nsteps; ++ks, ++step) {
          const int st = step % QSTAGES;
          if (!mbar_wait(full0 + 8 * st, (step / QSTAGES) & 1, abort_flag)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a0 = stage0 + st * TT::STAGE_BYTES, b0 = a0 + OZ_S * A_SLICE;
#pragma unroll
          for (int p = 0; p < OZ_S; ++p) {
            // digit p of A against the stacked digit slices q = q0 .. q0+nq-1
            // of B (consecutive BN-row slices form one K-major operand of
            // BN nq rows): product (p, q) lands in columns (p + q) BN .. of
            // the set's tensor memory, the accumulator of d = p + q.  The
            // first products of a tile, p = 0 at its first step, overwrite
            // every accumulator.
            const uint32_t acc = (ks > 0 || p > 0) ? 1u : 0u;
#pragma unroll
            for (int q0 = 0; q0 < OZ_S - p; q0 += QMMA_NMAX / BN) {
              const int nq = min(QMMA_NMAX / BN, OZ_S - p - q0);
              mma_i8(tacc + (uint32_t)((p + q0) * BN), sw32_desc(a0 + p * A_SLICE),
                     sw32_desc(b0 + q0 * TT::B_SLICE), idesc_i8(nq * BN), acc);
            }
          }
          tc_commit(empty0 + 8 * st);
        }
        tc_commit(done0 + 8 * set);  // also for a tile without products: the epilogue then writes beta C
      }
      // every product issued has completed before the tensor memory is freed
      tc_commit(drain_bar);
      mbar_wait(drain_bar, 0, abort_flag);
    }
  } else {
    // ------------------------------------------------------ epilogue (warp w: rows 32 (w % 4) ..,
    // columns (w / 4) CW .. of the tile)
    // Per 16 columns: the seven level accumulators combine exactly,
    // hi = sum_{d<4} acc_d 2^(7(3-d)) (< 2^49) and lo = sum_{d>=4} acc_d
    // 2^(7(6-d)); C = (hi + lo 2^-21) 2^(e_m + f_n - 35) goes to the warp's
    // registers.  Then the tensor memory is released and the warp writes
    // whole 16-column row segments through its staging rows while the next
    // tile's products run.
    constexpr int CW = TT::CW, LD = TT::STAGE_LD;
    const int quad = warp & 3, cb = (warp >> 2) * CW;
    double* stage = epi_stage + warp * (32 * LD);
    const uint32_t trow = tmem + ((uint32_t)(32 * quad) << 16);
    int it = 0;
    for (int t = blockIdx.x; t < total_tiles; t += gridDim.x, ++it) {
      int pi, tm, tn;
      decode_tile<BN>(batch, t, pi, tm, tn);
      const QProb& P = batch.p[pi];
      const int m0 = tm * QBM, n0 = tn * BN;
      const int nsteps = tile_steps<BN>(P, m0, n0);
      const int set = it % NSETS, use = it / NSETS;
      if (!__all_sync(0xffffffffu, mbar_wait(done0 + 8 * set, use & 1, abort_flag))) break;
      tc_fence_after();
      const bool have = nsteps > 0;
      const int row = m0 + 32 * quad + lane;
      const bool rowok = row < P.M;
      const int er = rowok ? max(P.eA[row], EXP_NONE) : 0;
      const int col0 = n0 + cb;
      const int fcol = (lane < CW && col0 + lane < P.N) ? max(P.fB[col0 + lane], EXP_NONE) : 0;
      // exponents in the normal range (every tile of ordinary data): two
      // exact power-of-two products; otherwise ldexp on a separate path
      const bool fast = __all_sync(0xffffffffu, er > -900 && er < 900 && fcol > -900 && fcol < 900);
      const double srow = fast ? __longlong_as_double((long long)(er - 35 + 1023) << 52) : 0.0;
      const double scol = fast ? __longlong_as_double((long long)(fcol + 1023) << 52) : 0.0;
      double res[CW / 16][16];  // this lane's row, the warp's CW columns
#pragma unroll
      for (int h = 0; h < CW / 16; ++h) {
        long long hi[16], lo[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) hi[j] = lo[j] = 0;
        if (have) {
          uint32_t ra[16], rb[16];
          const uint32_t tcol = trow + (uint32_t)(set * TT::SET_COLS + cb + 16 * h);
          tmem_ld16(tcol, ra);
#pragma unroll
          for (int d = 0; d < OZ_S; ++d) {
            uint32_t cur[16];
            if (d & 1) {
              tmem_wait16(rb);
#pragma unroll
              for (int j = 0; j < 16; ++j) cur[j] = rb[j];
            } else {
              tmem_wait16(ra);
#pragma unroll
              for (int j = 0; j < 16; ++j) cur[j] = ra[j];
            }
            if (d + 1 < OZ_S) {
              if (d & 1) tmem_ld16(tcol + (uint32_t)((d + 1) * BN), ra);
              else tmem_ld16(tcol + (uint32_t)((d + 1) * BN), rb);
            }
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              if (d < 4) hi[j] = hi[j] * 128 + (int)cur[j];
              else lo[j] = lo[j] * 128 + (int)cur[j];
            }
          }
        }
        if (fast) {
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const double sc = __shfl_sync(0xffffffffu, scol, 16 * h + j);
            const double v = fma(exact_double(lo[j]), 0x1p-21, exact_double(hi[j]));
            res[h][j] = ((v * srow) * sc) * P.sgn;
          }
        } else {
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int fc = __shfl_sync(0xffffffffu, fcol, 16 * h + j);
            const double v = fma(exact_double(lo[j]), 0x1p-21, exact_double(hi[j]));
            res[h][j] = ldexp(v, er + fc - 35) * P.sgn;
          }
        }
      }
      // accumulators read: the next tile's products may start
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(tmem_empty0 + 8 * set);
      const bool lower = P.cflags & GC_LOWER;
      const bool mirror = P.cflags & GC_MIRROR;
      double* C = P.C;
      const int rbase = m0 + 32 * quad;
#pragma unroll
      for (int h = 0; h < CW / 16; ++h) {
        // 16 columns through the staging rows: lane = row to stage them,
        // then lane % 16 = column, two rows at a time, for the stores
#pragma unroll
        for (int j = 0; j < 16; ++j) stage[lane * LD + j] = res[h][j];
        __syncwarp();
        const int c0 = col0 + 16 * h;
        const int cl = lane & 15, ro = lane >> 4;
        const int col = c0 + cl;
#pragma unroll 4
        for (int rr = ro; rr < 32; rr += 2) {
          const int rw = rbase + rr;
          if (rw < P.M && col < P.N && (!lower || col <= rw)) {
            double* dst = C + (size_t)rw * P.ldc + col;
            double x = stage[rr * LD + cl];
            if (P.beta != 0.0) {
              x += P.beta * *dst;
              stage[rr * LD + cl] = x;  // the mirror copies the final value
            }
            *dst = x;
          }
        }
        __syncwarp();
        // mirror: lane = row, so the transposed writes are contiguous too
        if (mirror && rowok) {
#pragma unroll 4
          for (int j = 0; j < 16; ++j) {
            const int cm = c0 + j;
            if (cm < row && cm < P.N) C[(size_t)cm * P.ldc + row] = stage[lane * LD + j];
          }
        }
        __syncwarp();
      }
      __syncwarp();
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == QMMA_WARP) {
    tc_fence_after();
    __syncwarp();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)TMEM_COLS)
                 : "memory");
  }
}

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }


}  // namespace

int gemm_launch_i8(const std::vector<GemmProb>& probs, cudaStream_t stream, int* abort_flag, void* ws,
                   size_t ws_bytes, size_t* ws_needed) {
  // workspace: per problem the exponents of its rows and columns, per segment
  // the digit images of both operands
  size_t need = 0;
  for (const GemmProb& p : probs) {
    if (p.M <= 0 || p.N <= 0) continue;
    need += align256((size_t)p.M * 4) + align256((size_t)p.N * 4);
    for (int s = 0; s < p.nseg; ++s) {
      const size_t KT = (size_t)(p.seg[s].K + QBK - 1) / QBK;
      const size_t RBa = 2 * (size_t)((p.M + QBM - 1) / QBM), RBb = (size_t)(p.N + 63) / 64;
      need += align256(OZ_S * KT * RBa * IMG) + align256(OZ_S * KT * RBb * IMG);
      if (p.seg[s].K > 19000) return cudaErrorInvalidValue;  // INT32 accumulation bound
    }
  }
  if (ws_needed) *ws_needed = need;
  if (!ws) return cudaSuccess;
  if (ws_bytes < need || !abort_flag) return cudaErrorInvalidValue;
  // output tile width: 64 (one accumulator set) or 32 (two sets), chosen by
  // the autotuner per launch shape
  long long work = 0;
  for (const GemmProb& p : probs)
    for (int s = 0; s < p.nseg; ++s) work += (long long)p.M * p.N / 64 * ((p.seg[s].K + 63) / 64);
  TuneLaunch tl("gemm_i8", {(long long)probs.size(), probs.empty() ? 0 : probs[0].M, probs.empty() ? 0 : probs[0].N,
                            probs.empty() ? 0 : (long long)probs[0].cflags, work},
                2, stream);
  const int BN = tl.choice() == 1 ? 32 : 64;
  {
    const int e = BN == 64
                      ? ensure_smem_attr(reinterpret_cast<const void*>(gemm_i8_kernel<64>), (int)QTile<64>::SMEM_BYTES)
                      : ensure_smem_attr(reinterpret_cast<const void*>(gemm_i8_kernel<32>), (int)QTile<32>::SMEM_BYTES);
    if (e != cudaSuccess) return (cudaError_t)e;
  }
  uint8_t* w = static_cast<uint8_t*>(ws);
  std::vector<SliceGroup> groups;
  std::vector<QProb> qp;
  for (const GemmProb& p : probs) {
    if (p.M <= 0 || p.N <= 0) continue;
    QProb q{};
    q.C = p.C;
    q.ldc = p.ldc;
    q.M = p.M;
    q.N = p.N;
    q.beta = p.beta;
    // the digits of -x are those of x negated (|x| is cut, the sign kept
    // apart), so a one-segment product with alpha = -1 cuts A unscaled and
    // negates in the epilogue -- bit for bit the same result -- and A can
    // then share its digit images with an equal B side (D -= L L^T cuts L once)
    const bool neg1 = p.nseg == 1 && p.seg[0].alpha == -1.0;
    q.sgn = neg1 ? -1.0 : 1.0;
    q.cflags = p.cflags;
    q.nseg = p.nseg;
    q.tmn = (p.M + QBM - 1) / QBM;
    q.tnn = (p.N + BN - 1) / BN;
    if ((p.cflags & GC_LOWER) && p.M != p.N) return cudaErrorInvalidValue;
    SliceGroup ga{}, gb{};
    ga.rows = p.M;
    ga.RB = 2 * q.tmn;
    ga.nseg = p.nseg;
    gb.rows = p.N;
    gb.RB = (p.N + 63) / 64;
    gb.nseg = p.nseg;
    for (int s = 0; s < p.nseg; ++s) {
      const GemmSeg& g = p.seg[s];
      const int KT = (g.K + QBK - 1) / QBK;
      ga.s[s] = SliceSeg{g.A, nullptr, neg1 ? 1.0 : g.alpha, g.lda, g.K, (g.flags & GF_A_T) ? 0 : 1, KT};
      gb.s[s] = SliceSeg{g.B, nullptr, 1.0, g.ldb, g.K, (g.flags & GF_B_KN) ? 0 : 1, KT};
    }
    // a side equal to one already planned in this launch (same operands,
    // orientation, scaling and image shape: e.g. the same block multiplied by
    // the main and the arrow rows) shares its exponents and digit images;
    // otherwise it gets its own
    auto plan = [&](SliceGroup& gr) {
      for (const SliceGroup& o : groups) {
        bool eq = o.rows == gr.rows && o.RB == gr.RB && o.nseg == gr.nseg;
        for (int s = 0; eq && s < gr.nseg; ++s)
          eq = o.s[s].P == gr.s[s].P && o.s[s].alpha == gr.s[s].alpha && o.s[s].ld == gr.s[s].ld &&
               o.s[s].K == gr.s[s].K && o.s[s].kcontig == gr.s[s].kcontig && o.s[s].KT == gr.s[s].KT;
        if (eq) {
          gr = o;
          return;
        }
      }
      gr.exps = reinterpret_cast<int*>(w);
      w += align256((size_t)gr.rows * 4);
      for (int s = 0; s < gr.nseg; ++s) {
        gr.s[s].out = reinterpret_cast<int8_t*>(w);
        w += align256((size_t)OZ_S * gr.s[s].KT * gr.RB * IMG);
      }
      groups.push_back(gr);
    };
    plan(ga);
    plan(gb);
    q.eA = ga.exps;
    q.fB = gb.exps;
    for (int s = 0; s < p.nseg; ++s)
      q.seg[s] = QSeg{ga.s[s].out, gb.s[s].out, ga.s[s].KT, ga.RB, gb.RB, p.seg[s].flags, p.seg[s].K};
    qp.push_back(q);
  }
  // exponents and digits, SU image rows of a problem side per unit
  {
    size_t i = 0;
    while (i < groups.size()) {
      SliceBatch sb;
      std::memset(&sb, 0, sizeof(sb));
      int units = 0;
      for (; i < groups.size() && sb.count < SLICE_MAXG; ++i) {
        SliceGroup g = groups[i];
        g.unit_start = units;
        units += g.RB * (64 / SU);
        sb.g[sb.count++] = g;
      }
      sb.units = units;
      if (units == 0) continue;
      bta::ProfScope _ps(bta::PROF_SLICE, stream);
      slice_kernel<<<units, SLICE_THREADS, 0, stream>>>(sb);
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return e;
    }
  }
  size_t i = 0;
  while (i < qp.size()) {
    QBatch b;
    std::memset(&b, 0, sizeof(b));
    int total = 0;
    for (; i < qp.size() && b.count < QMAXP; ++i) {
      const QProb& q = qp[i];
      int tiles = 0;
      if (q.cflags & GC_LOWER) {
        for (int tm = 0; tm < q.tmn; ++tm) tiles += lower_tiles_row(tm, q.tnn, BN);
      } else {
        tiles = q.tmn * q.tnn;
      }
      b.p[b.count] = q;
      b.tile_start[b.count] = total;
      total += tiles;
      b.count++;
    }
    b.tile_start[b.count] = total;
    if (total > 0) {
      const int sms = device_sm_count();
      bta::ProfScope _ps(bta::PROF_GEMM, stream);
      if (BN == 64)
        gemm_i8_kernel<64><<<std::min(total, sms), QTHREADS, QTile<64>::SMEM_BYTES, stream>>>(b, total, abort_flag);
      else
        gemm_i8_kernel<32><<<std::min(total, sms), QTHREADS, QTile<32>::SMEM_BYTES, stream>>>(b, total, abort_flag);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace bta
