// Compact-WY application of panel reflectors for the explicit Q_k^T of BSOI
// (reference: the dormqr('R','T') of lapackXbsoi_ormqr, src/bsofi_cpu.c:
// 234-245, here by forming Q_k^T once per panel, as lapackXbsoi_orgqr does at
// :307-329).
#include "bsofi_common.cuh"
#include "bsofi_kernels.h"

namespace bsofi {

// C <- (I - V T V^T)^T C  (trans = 1)  or  C <- (I - V T V^T) C  (trans = 0)
// for the column segments s0|s1|s2 (all with m rows), V the m x nb unit lower
// trapezoidal leaf stored below the diagonal at V (LAPACK layout), T nb x nb
// (ld 16).  blockIdx.x picks a 32-column chunk, blockIdx.y a batch entry.
constexpr int WY_CW = 32, WY_RC = 64, WY_THREADS = 256;

__global__ void __launch_bounds__(WY_THREADS) wy_apply_kernel(WyArgs args) {
  __shared__ double sV[WY_RC][17];
  __shared__ double sC[WY_RC][WY_CW + 1];
  __shared__ double sW[16][WY_CW + 1];
  __shared__ double sT[16][17];
  const int tid = threadIdx.x;
  const int bz = blockIdx.y;
  const int m = args.m, nb = args.nb;
  const double* V = args.V + (long long)bz * args.vbs;
  const double* T = args.T + (long long)bz * args.tbs;

  // Locate this chunk inside the concatenated segments.
  int col0 = blockIdx.x * WY_CW;
  double* C = nullptr;
  long long ldc = 0;
  int ncols = 0;
  {
    int c = col0;
#pragma unroll
    for (int s = 0; s < 3; s++) {
      int chunks = (args.seg[s].ncols + WY_CW - 1) / WY_CW;
      if (C == nullptr && c < chunks * WY_CW) {
        C = args.seg[s].p + (long long)bz * args.seg[s].bs;
        ldc = args.seg[s].ld;
        ncols = min(WY_CW, args.seg[s].ncols - c);
        C += (long long)c * ldc;
      } else if (C == nullptr) {
        c -= chunks * WY_CW;
      }
    }
  }
  if (C == nullptr || ncols <= 0) return;

  for (int e = tid; e < 16 * 16; e += WY_THREADS) sT[e % 16][e / 16] = T[e];

  // Phase 1: W = V^T C  (nb x ncols); each thread owns two entries.
  double w0 = 0.0, w1 = 0.0;
  const int wa = tid % 16, wc = tid / 16;  // entries (wa, wc) and (wa, wc + 16)
  for (int r0 = 0; r0 < m; r0 += WY_RC) {
    __syncthreads();
    for (int e = tid; e < WY_RC * 16; e += WY_THREADS) {
      int rr = e % WY_RC, aa = e / WY_RC, r = r0 + rr;
      double v = 0.0;
      if (r < m && aa < nb) v = (r == aa) ? 1.0 : (r > aa ? V[cm(r, aa, args.ldv)] : 0.0);
      sV[rr][aa] = v;
    }
    for (int e = tid; e < WY_RC * WY_CW; e += WY_THREADS) {
      int rr = e % WY_RC, cc = e / WY_RC, r = r0 + rr;
      sC[rr][cc] = (r < m && cc < ncols) ? C[cm(r, cc, ldc)] : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int rr = 0; rr < WY_RC; rr++) {
      double v = sV[rr][wa];
      w0 = fma(v, sC[rr][wc], w0);
      w1 = fma(v, sC[rr][wc + 16], w1);
    }
  }
  sW[wa][wc] = w0;
  sW[wa][wc + 16] = w1;
  __syncthreads();
  // Phase 2: W <- T^T W (trans) or T W.
  {
    double s0 = 0.0, s1 = 0.0;
    if (args.trans) {
      for (int b = 0; b <= wa; b++) {
        s0 = fma(sT[b][wa], sW[b][wc], s0);
        s1 = fma(sT[b][wa], sW[b][wc + 16], s1);
      }
    } else {
      for (int b = wa; b < 16; b++) {
        s0 = fma(sT[wa][b], sW[b][wc], s0);
        s1 = fma(sT[wa][b], sW[b][wc + 16], s1);
      }
    }
    __syncthreads();
    sW[wa][wc] = s0;
    sW[wa][wc + 16] = s1;
  }
  // Phase 3: C <- C - V W.
  for (int r0 = 0; r0 < m; r0 += WY_RC) {
    __syncthreads();
    for (int e = tid; e < WY_RC * 16; e += WY_THREADS) {
      int rr = e % WY_RC, aa = e / WY_RC, r = r0 + rr;
      double v = 0.0;
      if (r < m && aa < nb) v = (r == aa) ? 1.0 : (r > aa ? V[cm(r, aa, args.ldv)] : 0.0);
      sV[rr][aa] = v;
    }
    __syncthreads();
    for (int e = tid; e < WY_RC * WY_CW; e += WY_THREADS) {
      int rr = e % WY_RC, cc = e / WY_RC, r = r0 + rr;
      if (r < m && cc < ncols) {
        double s = 0.0;
#pragma unroll
        for (int aa = 0; aa < 16; aa++) s = fma(sV[rr][aa], sW[aa][cc], s);
        double* p = C + cm(r, cc, ldc);
        *p -= s;
      }
    }
  }
}

// ------------------------------------------------------------------ launchers
int leaf_width(int n) { return (2 * n <= 1024) ? 16 : 8; }

cudaError_t launch_wy_apply(const WyArgs& a, int batch, cudaStream_t st) {
  int chunks = 0;
  for (int s = 0; s < 3; s++) chunks += (a.seg[s].ncols + WY_CW - 1) / WY_CW;
  if (chunks == 0 || batch == 0) return cudaSuccess;
  dim3 grid(chunks, batch);
  wy_apply_kernel<<<grid, WY_THREADS, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t preload_panel(size_t* local) { return preload_one(wy_apply_kernel, local); }

}  // namespace bsofi
