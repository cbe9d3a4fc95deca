// BSTRI building blocks: batched inversion of the upper-triangular diagonal
// blocks of R, and small utility kernels.
//
// Reference: lapackXbstri, src/bsofi_cpu.c:146-177 (dtrtri of the 3n corner
// and of each n x n diagonal block).  The diagonal blocks are independent of
// the block recurrence, so all of them are inverted in one launch (one CTA
// per block), in place in the upper triangle; the strict lower part, which
// holds Householder vectors, is never touched (as with LAPACK dtrtri).
#include <climits>
#include "bsofi_common.cuh"
#include "bsofi_kernels.h"

namespace bsofi {

constexpr int TB = 32;

// Inverts the upper-triangular n x n block at A + blockIdx.x * bstride.
// Column blocks of width 32, left to right (LAPACK dtrtri 'U' order):
//   D = U_jj^{-1} (in shared memory),
//   U(0:j, j) <- -X(0:j,0:j) U(0:j, j) D   with X = U(0:j,0:j)^{-1} already
//   in place; row chunks are produced top-down so the in-place update only
//   overwrites rows that later chunks no longer read.
// An exactly zero diagonal entry leaves the block untouched and records the
// smallest 1-based global index (block * n + i + 1) in *info.
__global__ void __launch_bounds__(256) trtri_blocks_kernel(double* A, long long ld, int n,
                                                           long long bstride, int* info) {
  __shared__ double sD[TB][TB + 1];
  __shared__ double sX[TB][TB + 1];
  __shared__ double sY[TB][TB + 1];
  __shared__ double sS[TB][TB + 1];
  __shared__ int sbad;
  const int tid = threadIdx.x;
  double* U = A + (long long)blockIdx.x * bstride;

  if (tid == 0) sbad = INT_MAX;
  __syncthreads();
  for (int i = tid; i < n; i += blockDim.x)
    if (U[cm(i, i, ld)] == 0.0) atomicMin(&sbad, i);
  __syncthreads();
  if (sbad != INT_MAX) {
    if (tid == 0) atomicMin(info, blockIdx.x * n + sbad + 1);
    return;
  }

  const int tr = tid % TB, tc = tid / TB;  // tc in 0..7
  for (int jb = 0; jb < n; jb += TB) {
    const int w = min(TB, n - jb);
    // Diagonal block, upper part.
    for (int e = tid; e < TB * TB; e += blockDim.x) {
      int r = e % TB, c = e / TB;
      sD[r][c] = (r <= c && r < w && c < w) ? U[cm(jb + r, jb + c, ld)] : 0.0;
    }
    __syncthreads();
    // dtrti2 on sD by warp 0: column j: d = 1/D_jj; D(0:j,j) = -d triu(D(0:j,0:j)) D(0:j,j).
    if (tid < 32) {
      for (int j = 0; j < w; j++) {
        double djj = 1.0 / sD[j][j];
        double s = 0.0;
        if (tid < j)
          for (int k = tid; k < j; k++) s = fma(sD[tid][k], sD[k][j], s);
        __syncwarp();
        if (tid < j) sD[tid][j] = -djj * s;
        if (tid == j) sD[j][j] = djj;
        __syncwarp();
      }
    }
    __syncthreads();
    // Off-diagonal column block rows 0..jb.
    for (int r0 = 0; r0 < jb; r0 += TB) {
      const int h = min(TB, jb - r0);
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
      for (int k0 = r0; k0 < jb; k0 += TB) {
        const int kw = min(TB, jb - k0);
        __syncthreads();
        for (int e = tid; e < TB * TB; e += blockDim.x) {
          int r = e % TB, c = e / TB;
          // X(r0+r, k0+c), upper triangular.
          sX[r][c] = (r < h && c < kw && r0 + r <= k0 + c) ? U[cm(r0 + r, k0 + c, ld)] : 0.0;
          // top(k0+r, c) = U(k0+r, jb+c)
          sY[r][c] = (r < kw && c < w) ? U[cm(k0 + r, jb + c, ld)] : 0.0;
        }
        __syncthreads();
#pragma unroll 8
        for (int k = 0; k < TB; k++) {
          double x = sX[tr][k];
#pragma unroll
          for (int q = 0; q < 4; q++) acc[q] = fma(x, sY[k][tc + 8 * q], acc[q]);
        }
      }
      __syncthreads();
#pragma unroll
      for (int q = 0; q < 4; q++) sS[tr][tc + 8 * q] = acc[q];
      __syncthreads();
      // out = -S D
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int c = tc + 8 * q;
        double s = 0.0;
        for (int k = 0; k <= c; k++) s = fma(sS[tr][k], sD[k][c], s);
        if (tr < h && c < w) U[cm(r0 + tr, jb + c, ld)] = -s;
      }
    }
    __syncthreads();
    for (int e = tid; e < TB * TB; e += blockDim.x) {
      int r = e % TB, c = e / TB;
      if (r <= c && c < w) U[cm(jb + r, jb + c, ld)] = sD[r][c];
    }
    __syncthreads();
  }
}

cudaError_t launch_trtri_blocks(double* A, long long ld, int n, long long bstride, int nblk,
                                int* info, cudaStream_t st) {
  if (nblk <= 0) return cudaSuccess;
  trtri_blocks_kernel<<<nblk, 256, 0, st>>>(A, ld, n, bstride, info);
  return cudaGetLastError();
}

// ------------------------------------------------------------------ utilities
__global__ void set_identity_kernel(double* G, long long ld, int m, long long bs) {
  double* g = G + (long long)blockIdx.y * bs;
  long long total = (long long)m * m;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int r = (int)(e % m), c = (int)(e / m);
    g[cm(r, c, ld)] = (r == c) ? 1.0 : 0.0;
  }
}

cudaError_t launch_set_identity(double* G, long long ld, int m, long long bs, int batch,
                                cudaStream_t st) {
  if (batch <= 0 || m <= 0) return cudaSuccess;
  long long total = (long long)m * m;
  int gx = (int)min((total + 255) / 256, (long long)1024);
  set_identity_kernel<<<dim3(gx, batch), 256, 0, st>>>(G, ld, m, bs);
  return cudaGetLastError();
}

__global__ void copy_masked_kernel(double* dst, long long ldd, const double* src, long long lds,
                                   int rows, int cols, int roff, int* fold) {
  // fold (optional): the workspace info words {BSTRI info, BSOF error, BSOI
  // error, BSTRI error}; a bounded wait that gave up turns the info word into
  // an error.
  if (fold != nullptr && blockIdx.x == 0 && threadIdx.x == 0 && (fold[1] | fold[2] | fold[3]) != 0)
    fold[0] = kInfoWaitFailed;
  long long total = (long long)rows * cols;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int r = (int)(e % rows), c = (int)(e / rows);
    double v = ((long long)r - roff > c) ? 0.0 : src[cm(r, c, lds)];
    dst[cm(r, c, ldd)] = v;
  }
}

cudaError_t launch_copy_masked(double* dst, long long ldd, const double* src, long long lds,
                               int rows, int cols, int roff, cudaStream_t st, int* fold) {
  long long total = (long long)rows * cols;
  if (total <= 0) return cudaSuccess;
  int gx = (int)min((total + 255) / 256, (long long)4096);
  copy_masked_kernel<<<gx, 256, 0, st>>>(dst, ldd, src, lds, rows, cols, roff, fold);
  return cudaGetLastError();
}

__global__ void zero_structural_kernel(double* A, long long ld, int n, int L) {
  // blockIdx.y < L-1: superdiagonal block (k, k+1); else last-column block (k, L-1).
  int b = blockIdx.y, bi, bj;
  if (b < L - 1) {
    bi = b;
    bj = b + 1;
  } else {
    bi = b - (L - 1) + 1;
    bj = L - 1;
  }
  long long total = (long long)n * n;
  double* blk = A + cm((long long)bi * n, (long long)bj * n, ld);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x)
    blk[cm(e % n, e / n, ld)] = 0.0;
}

cudaError_t launch_zero_structural(double* A, long long ld, int n, int L, cudaStream_t st) {
  int nb = (L - 1) + (L >= 3 ? L - 2 : 0);
  if (nb <= 0) return cudaSuccess;
  long long total = (long long)n * n;
  int gx = (int)min((total + 255) / 256, (long long)64);
  zero_structural_kernel<<<dim3(gx, nb), 256, 0, st>>>(A, ld, n, L);
  return cudaGetLastError();
}

}  // namespace bsofi
