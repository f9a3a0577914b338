// Shared device helpers for the BTA kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace bta {

// Tile edge used by every FP64 kernel (64 x 64 doubles = 32 KiB).
constexpr int TILE = 64;

// FP64 tensor-core MMA (DMMA), D[16x8] += A[16x4] * B[4x8].
// Fragment layout (PTX ISA, mma.m16n8k4 .f64): g = lane>>2, t = lane&3;
// a0 = A[g][t], a1 = A[g+8][t]; b0 = B[t][g];
// c0,c1 = C[g][2t..2t+1]; c2,c3 = C[g+8][2t..2t+1].
__device__ __forceinline__ void dmma16x8x4(double (&d)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 "
      "{%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool valid) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  int n = valid ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }

template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Loads that bypass L1 (data produced by other CTAs of the same launch).
__device__ __forceinline__ double ld_cg(const double* p) { return __ldcg(p); }

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Relaxed load: a scan of several flags issues them back to back; a fence
// afterwards gives the ones seen set acquire semantics.
__device__ __forceinline__ int ld_relaxed(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

}  // namespace bta
