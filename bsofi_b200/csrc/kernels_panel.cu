// BSOF panel kernels: Householder QR of the stacked 2n x n panels
// [R~_k; B_k] and compact-WY application of the resulting block reflectors.
//
// Reference: lapackXbsof, src/bsofi_cpu.c:86-118 (dgeqrf of each 2n x n panel,
// dormqr('L','T') of A_BLK(k,k+1) and A_BLK(k,L-1)); final 2n x 2n dgeqrf.
// Householder convention of LAPACK dlarfg/dgeqr2 (the reflector scalars tau and
// the signs of diag(R) are part of the observable state after XbsoftriH).
#include "bsofi_common.cuh"
#include "bsofi_kernels.h"

namespace bsofi {

// Sum NB values per lane over a warp with a transpose-reduction: afterwards
// lane l holds the warp sum of value (l >> (5 - log2 NB)) & (NB - 1).
template <int NB>
BSOFI_DEVINL double warp_transpose_sum(double (&v)[NB], int lane) {
  constexpr int LOG = (NB == 16) ? 4 : (NB == 8) ? 3 : 2;
  static_assert(NB == 16 || NB == 8 || NB == 4, "NB");
#pragma unroll
  for (int lev = 0; lev < LOG; lev++) {
    const int off = 16 >> lev;
    const int half = NB >> (lev + 1);
    const bool upper = (lane & off) != 0;
#pragma unroll
    for (int j = 0; j < half; j++) {
      double send = upper ? v[j] : v[j + half];
      double keep = upper ? v[j + half] : v[j];
      v[j] = keep + __shfl_xor_sync(0xffffffffu, send, off);
    }
  }
  double s = v[0];
#pragma unroll
  for (int off = 16 >> LOG; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  return s;
}

// Householder QR of one leaf: the m x nc block at P (nc <= NB), rows held in
// registers (thread t owns rows t + 512 r).  One block-wide reduction per
// column carries, in NB slots, both the dot products needed for the column's
// reflector and its trailing update (d_c = sum_{r>i} a_ri a_rc, c >= i) and
// the dot products of the new reflector with the previous ones
// (e_j = sum_{r>i} v_j[r] a_ri, j < i) that build the compact-WY factor T
// (LAPACK dlarft recurrence T(0:i,i) = -tau_i T(0:i,0:i) V^T v_i).
template <int R, int NB>
__global__ void __launch_bounds__(512) panel_leaf_kernel(
    double* __restrict__ P, long long ldp, int m, int nc, double* __restrict__ tau,
    double* __restrict__ Tout) {
  constexpr int NT = 512, NW = NT / 32;
  constexpr int GROUPS = 32 / NB;  // lane groups in the cross-warp stage
  __shared__ double red[2][NW][NB];
  __shared__ double prow[2][NB];
  __shared__ double wsh[NW][NB];
  __shared__ double sT[NB][NB + 1];
  __shared__ double gsh[NB];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  double a[R][NB];
#pragma unroll
  for (int r = 0; r < R; r++) {
    const int row = tid + NT * r;
#pragma unroll
    for (int c = 0; c < NB; c++)
      a[r][c] = (row < m && c < nc) ? P[cm(row, c, ldp)] : 0.0;
  }
  if (warp == 0) {
    for (int e = lane; e < NB * (NB + 1); e += 32) (&sT[0][0])[e] = 0.0;
  }

#pragma unroll
  for (int i = 0; i < NB; i++) {
    if (i < nc) {
    const int buf = i & 1;
    if (tid == i) {
#pragma unroll
      for (int c = 0; c < NB; c++) prow[buf][c] = a[0][c];
    }
    double part[NB];
#pragma unroll
    for (int c = 0; c < NB; c++) part[c] = 0.0;
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int row = tid + NT * r;
      if (row > i && row < m) {
        const double x = a[r][i];
#pragma unroll
        for (int c = 0; c < NB; c++) part[c] = fma(x, a[r][c], part[c]);
      }
    }
    {
      double s = warp_transpose_sum<NB>(part, lane);
      constexpr int SH = (NB == 16) ? 1 : (NB == 8) ? 2 : 3;
      if ((lane & ((1 << SH) - 1)) == 0) red[buf][warp][(lane >> SH) & (NB - 1)] = s;
    }
    __syncthreads();
    // Every warp re-reduces the NW partial vectors: lane l -> slot l % NB.
    double tot;
    {
      const int slot = lane % NB, grp = lane / NB;
      double s = 0.0;
#pragma unroll
      for (int w = grp; w < NW; w += GROUPS) s += red[buf][w][slot];
#pragma unroll
      for (int off = NB; off < 32; off <<= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
      tot = s;
    }
    const double xnorm2 = __shfl_sync(0xffffffffu, tot, i);
    const double alpha = prow[buf][i];
    double beta, taui, scale;
    if (xnorm2 == 0.0) {
      taui = 0.0;
      beta = alpha;
      scale = 1.0;
    } else {
      beta = -copysign(sqrt(fma(alpha, alpha, xnorm2)), alpha);
      taui = (beta - alpha) / beta;
      scale = 1.0 / (alpha - beta);
    }
    {
      const int slot = lane % NB;
      // w_c = v_i^T a_c for the trailing leaf columns.
      if (lane < NB) wsh[warp][slot] = fma(scale, tot, prow[buf][slot]);
      __syncwarp();
    }
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int row = tid + NT * r;
      if (row > i && row < m) {
        const double v = a[r][i] * scale;
        a[r][i] = v;
        const double tv = taui * v;
#pragma unroll
        for (int c = i + 1; c < NB; c++) a[r][c] = fma(-tv, wsh[warp][c], a[r][c]);
      } else if (row == i) {
        a[r][i] = beta;
#pragma unroll
        for (int c = i + 1; c < NB; c++) a[r][c] = fma(-taui, wsh[warp][c], a[r][c]);
      }
    }
    if (warp == 0) {
      // T(0:i, i) = -tau_i T(0:i,0:i) g, g_j = v_j^T v_i = v_j[i] + scale e_j.
      const int slot = lane % NB;
      if (lane < i) gsh[lane] = fma(scale, tot, prow[buf][slot]);
      __syncwarp();
      if (lane < i) {
        double s = 0.0;
        for (int b = lane; b < i; b++) s = fma(sT[lane][b], gsh[b], s);
        sT[lane][i] = -taui * s;
      }
      if (lane == i) sT[i][i] = taui;
      if (lane == 0) tau[i] = taui;
      __syncwarp();
    }
    }
  }
#pragma unroll
  for (int r = 0; r < R; r++) {
    const int row = tid + NT * r;
    if (row < m) {
#pragma unroll
      for (int c = 0; c < NB; c++)
        if (c < nc) P[cm(row, c, ldp)] = a[r][c];
    }
  }
  __syncthreads();
  for (int e = tid; e < 16 * 16; e += NT) {
    int rr = e % 16, cc = e / 16;
    Tout[e] = (rr < NB && cc < NB && rr < nc && cc < nc) ? sT[rr][cc] : 0.0;
  }
}

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
int leaf_rows_per_thread(int m) { return (m + 511) / 512; }

int leaf_width(int n) { return (2 * n <= 1024) ? 16 : 8; }

cudaError_t launch_panel_leaf(double* P, long long ldp, int m, int nc, double* tau,
                              double* Tout, int nbw, cudaStream_t st) {
  int R = leaf_rows_per_thread(m);
  if (nbw == 16) {
    if (R == 1) panel_leaf_kernel<1, 16><<<1, 512, 0, st>>>(P, ldp, m, nc, tau, Tout);
    else if (R == 2) panel_leaf_kernel<2, 16><<<1, 512, 0, st>>>(P, ldp, m, nc, tau, Tout);
    else return cudaErrorInvalidValue;
  } else {
    if (R == 1) panel_leaf_kernel<1, 8><<<1, 512, 0, st>>>(P, ldp, m, nc, tau, Tout);
    else if (R == 2) panel_leaf_kernel<2, 8><<<1, 512, 0, st>>>(P, ldp, m, nc, tau, Tout);
    else if (R == 3) panel_leaf_kernel<3, 8><<<1, 512, 0, st>>>(P, ldp, m, nc, tau, Tout);
    else if (R == 4) panel_leaf_kernel<4, 8><<<1, 512, 0, st>>>(P, ldp, m, nc, tau, Tout);
    else return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_wy_apply(const WyArgs& a, int batch, cudaStream_t st) {
  int chunks = 0;
  for (int s = 0; s < 3; s++) chunks += (a.seg[s].ncols + WY_CW - 1) / WY_CW;
  if (chunks == 0 || batch == 0) return cudaSuccess;
  dim3 grid(chunks, batch);
  wy_apply_kernel<<<grid, WY_THREADS, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace bsofi
