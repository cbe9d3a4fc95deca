// BSTRI row recurrence as one persistent kernel.
//
// Reference: lapackXbstri, src/bsofi_cpu.c:159-172.  After the diagonal
// blocks are inverted and W_i = -X_ii R_{i,i+1}, Z_i = -X_ii R_{i,L-1}
// X_{L-1,L-1} are formed, row block i of R^{-1} is
//   X_{i, i+1:L} = W_i X_{i+1, i+1:L}  (+ Z_i on block column L-1),
// for i = L-3 down to 0.  An output tile of row block i only reads the same
// columns of row block i+1, so the steps need not wait for each other as a
// whole: tiles are claimed in (step, column tile, row tile) order from a
// global counter, and a tile waits (bounded) only for the tiles of the
// previous step that cover its columns.  Every wait is on a tile claimed
// earlier, whose CTA is already running, so an ordinary launch cannot
// deadlock.
#include <climits>
#include "bsofi_common.cuh"
#include "bsofi_kernels.h"

namespace bsofi {

struct RecArgs {
  double* A;
  long long ld;
  const double* W;  // (L-2) blocks of n x n, leading dimension n
  int n, L, ctmax;
  int* done;  // (L-2) x ctmax: finished row tiles per (step, column tile)
  int* next;  // tile counter
  int* err;
  long long spin_limit;
};

BSOFI_DEVINL int rec_ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

template <class Cfg, bool ALIGNED>
__global__ void __launch_bounds__(Cfg::THREADS) bstri_recurrence_kernel(RecArgs s) {
  extern __shared__ __align__(16) double smem_rec[];
  __shared__ int s_tile, s_ok;
  const int n = s.n, L = s.L;
  const int RT = (n + Cfg::BM - 1) / Cfg::BM;
  // Step st (0 .. L-3) computes row block i = L-3-st over (st+2)*n columns.
  long long total = 0;
  for (int st = 0; st < L - 2; st++) total += (long long)RT * (((st + 2) * n + Cfg::BN - 1) / Cfg::BN);
  for (;;) {
    __syncthreads();  // the previous tile's shared memory is no longer read
    if (threadIdx.x == 0) s_tile = atomicAdd(s.next, 1);
    __syncthreads();
    long long rem = s_tile;
    if (rem >= total) return;
    int st = 0, ct_n = 0;
    for (;; st++) {
      ct_n = ((st + 2) * n + Cfg::BN - 1) / Cfg::BN;
      if (rem < (long long)RT * ct_n) break;
      rem -= (long long)RT * ct_n;
    }
    const int ct = (int)(rem / RT), rt = (int)(rem % RT);
    const int i = L - 3 - st, ncol = (st + 2) * n;
    if (st > 0) {
      // Columns [ct*BN, ct*BN + BN) of this step are columns shifted by n in
      // the previous step; those below n lie in the diagonal block X_{i+1,i+1}.
      if (threadIdx.x == 0) {
        int ok = 1;
        const int lo = ct * Cfg::BN - n, hi = ct * Cfg::BN + Cfg::BN - 1 - n;
        const int prev_cols = (st + 1) * n;
        if (hi >= 0) {
          const int c0 = (lo > 0 ? lo : 0) / Cfg::BN;
          const int c1 = (hi < prev_cols - 1 ? hi : prev_cols - 1) / Cfg::BN;
          for (int c = c0; c <= c1 && ok; c++) {
            const int* flag = s.done + (long long)(st - 1) * s.ctmax + c;
            long long it = 0;
            while (rec_ld_acquire(flag) < RT) {
              if (rec_ld_acquire(s.err) != 0 || ++it > s.spin_limit) {
                atomicExch(s.err, 1);
                ok = 0;
                break;
              }
              __nanosleep(64);
            }
          }
        }
        s_ok = ok;
      }
      __syncthreads();
      if (!s_ok) return;
    }
    GemmDims d = {n, ncol, n};
    GemmA a;
    a.p0 = s.W + (long long)i * n * n;
    a.p1 = nullptr;
    a.ld0 = n;
    a.ld1 = 2;
    a.bs0 = a.bs1 = 0;
    a.ksplit = n;
    a.rlim0 = INT_MAX;
    a.roff0 = kNoMask;
    a.rlim1 = INT_MAX;
    a.roff1 = kNoMask;
    // X_{i+1, i+1:L}; its first block is upper triangular (reflectors below).
    GemmB b = {s.A + cm((long long)(i + 1) * n, (long long)(i + 1) * n, s.ld), s.ld, 0, 0};
    GemmC c;
    c.p0 = s.A + cm((long long)i * n, (long long)(i + 1) * n, s.ld);
    c.p1 = s.A + cm((long long)i * n, (long long)(L - 1) * n, s.ld);
    c.ld0 = c.ld1 = s.ld;
    c.bs0 = c.bs1 = 0;
    c.nsplit = ncol - n;
    c.alpha = 1.0;
    c.beta0 = 0.0;
    c.beta1 = 1.0;
    gemm_tile<Cfg, ALIGNED>(d, a, b, c, rt * Cfg::BM, ct * Cfg::BN, 0, smem_rec);
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      asm volatile("red.release.gpu.global.add.s32 [%0], 1;" ::"l"(s.done + (long long)st * s.ctmax + ct)
                   : "memory");
    }
  }
}

int bstri_recurrence_ctmax(int n, int L) { return ((L - 1) * n + CfgS::BN - 1) / CfgS::BN; }

template <bool AL>
static cudaError_t rec_launch(const RecArgs& s, long long tiles, cudaStream_t st) {
  static PerDevice once;
  const int pend = once.pending();
  if (pend >= 0) {
    cudaError_t e = cudaFuncSetAttribute(bstri_recurrence_kernel<CfgS, AL>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)CfgS::SMEM);
    if (e != cudaSuccess) return e;
    once.mark(pend);
  }
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, bstri_recurrence_kernel<CfgS, AL>,
                                                CfgS::THREADS, CfgS::SMEM);
  long long grid = (long long)sms * (per > 0 ? per : 1);
  if (tiles < grid) grid = tiles;
  bstri_recurrence_kernel<CfgS, AL><<<(int)grid, CfgS::THREADS, CfgS::SMEM, st>>>(s);
  return cudaGetLastError();
}

cudaError_t launch_bstri_recurrence(double* A, long long ld, const double* W, int n, int L,
                                    int* done, int* next, int* err, cudaStream_t st) {
  if (L < 3) return cudaSuccess;
  RecArgs s;
  s.A = A;
  s.ld = ld;
  s.W = W;
  s.n = n;
  s.L = L;
  s.ctmax = bstri_recurrence_ctmax(n, L);
  s.done = done;
  s.next = next;
  s.err = err;
  s.spin_limit = 1ll << 22;
  const int RT = (n + CfgS::BM - 1) / CfgS::BM;
  long long tiles = 0;
  for (int k = 0; k < L - 2; k++) tiles += (long long)RT * (((k + 2) * n + CfgS::BN - 1) / CfgS::BN);
  const bool al = ((uintptr_t)A % 16 == 0) && ((uintptr_t)W % 16 == 0) && ld % 2 == 0 && n % 2 == 0;
  return al ? rec_launch<true>(s, tiles, st) : rec_launch<false>(s, tiles, st);
}

}  // namespace bsofi
