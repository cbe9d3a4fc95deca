// Device helpers shared by the BSOF/I kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define BSOFI_DEVINL __device__ __forceinline__

// Column-major element offset.
__host__ __device__ __forceinline__ size_t cm(long long i, long long j, long long ld) {
  return (size_t)(j * ld + i);
}

// ---------------------------------------------------------------- cp.async
// 16-byte copy global->shared; bytes beyond src_bytes (0, 8 or 16) are
// zero-filled, so masked and out-of-range elements cost no extra pass.
BSOFI_DEVINL void cp_async16(void* smem, const void* gmem, int src_bytes) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s),
               "l"(gmem), "r"(src_bytes));
}
// 8-byte copy (for leading dimensions that break 16-byte alignment).
BSOFI_DEVINL void cp_async8(void* smem, const void* gmem, int src_bytes) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s),
               "l"(gmem), "r"(src_bytes));
}
BSOFI_DEVINL void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
BSOFI_DEVINL void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// ---------------------------------------------------------------- DMMA
// D = A(16x4, row) * B(4x8, col) + D, FP64 tensor-core MMA.
// Fragment ownership (g = lane/4, t = lane%4):
//   a0 = A[g][t], a1 = A[g+8][t]; b0 = B[t][g];
//   d0,d1 = D[g][2t], D[g][2t+1]; d2,d3 = D[g+8][2t], D[g+8][2t+1].
BSOFI_DEVINL void dmma_16x8x4(double (&d)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 "
      "{%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

// D = A(16x8, row) * B(8x8, col) + D.  a0 = A[g][t], a1 = A[g+8][t],
// a2 = A[g][t+4], a3 = A[g+8][t+4]; b0 = B[t][g], b1 = B[t+4][g]; D as above.
BSOFI_DEVINL void dmma_16x8x8(double (&d)[4], double a0, double a1, double a2, double a3,
                              double b0, double b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}

// D = A(16x16, row) * B(16x8, col) + D, FP64 (the sm_90+ shape with twice
// the K of m16n8k8): a[2q+h] = A[g+8h][t+4q], b[q] = B[t+4q][g] (q = 0..3),
// d as for m16n8k8.
BSOFI_DEVINL void dmma_16x8x16(double (&d)[4], const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]),
        "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

// D = A(8x4, row) * B(4x8, col) + D, FP64.  a0 = A[g][t]; b0 = B[t][g];
// d0, d1 = D[g][2t], D[g][2t+1].
BSOFI_DEVINL void dmma_8x8x4(double (&d)[2], double a0, double b0) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 "
      "{%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(d[0]), "+d"(d[1])
      : "d"(a0), "d"(b0));
}

// ---------------------------------------------------------------- warp sums
BSOFI_DEVINL double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Error word written by kernels that detect a bad state (never traps).
#define BSOFI_KERR_NONE 0
