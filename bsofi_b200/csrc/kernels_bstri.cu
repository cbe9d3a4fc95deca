// BSTRI row recurrence as one persistent kernel.
//
// Reference: lapackXbstri, src/bsofi_cpu.c:159-172.  After the diagonal
// blocks are inverted and W_i = -X_ii R_{i,i+1}, Z_i = -X_ii R_{i,L-1}
// X_{L-1,L-1} are formed, row block i of R^{-1} is
//   X_{i, i+1:L} = W_i X_{i+1, i+1:L}  (+ Z_i on block column L-1),
// for i = L-3 down to 0.  The blocked form takes the rows in groups of grp
// from the bottom (group g: rows t..b, b = L-3-g grp) and computes a whole
// group from the row below it with the stacked products P of the group:
//   X_{t:b, b+1:L} = P_g X_{b+1, b+1:L}  (+ Zc on block column L-1);
// grp = 1 is the one-row recurrence with P_g = W_b.  With a column floor h
// > 0 a step only computes block columns from max(b+1, h) on (the columns
// left of h were formed earlier, overlapped with the factorization).  An
// output tile of group g
// only reads the top row block of group g-1 over its own columns, so the steps
// need not wait for each other as a whole: tiles are claimed in (step, column
// tile, row tile) order from a global counter, and a tile waits (bounded) only
// for the top-row tiles of the previous step that cover its columns.  Every
// wait is on a tile claimed earlier, whose CTA is already running, so an
// ordinary launch cannot deadlock.
#include <climits>
#include "bsofi_common.cuh"
#include "bsofi_kernels.h"

namespace bsofi {

struct RecArgs {
  double* A;
  long long ld;
  const double* P;  // step g's left operand: P + g pstep + (grp - m_g) n, leading dimension pld
  long long pstep, pld;
  int n, L, grp, ctmax;
  int hfloor;  // first block column computed (0: every column beyond the step's rows)
  int* done;  // steps x ctmax: finished top-row tiles per (step, column tile)
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
  const int n = s.n, L = s.L, grp = s.grp;
  const int nsteps = (L - 2 + grp - 1) / grp;
  const int top = (n + Cfg::BM - 1) / Cfg::BM;  // row tiles covering a step's top row block
  // Step g computes rows t..b (b = L-3-g grp, m = b-t+1 <= grp) over block
  // columns cs..L-1, cs = max(b+1, hfloor).
  long long total = 0;
  for (int g = 0; g < nsteps; g++) {
    const int b = L - 3 - g * grp, m = b + 1 < grp ? b + 1 : grp;
    const int cs = b + 1 > s.hfloor ? b + 1 : s.hfloor;
    total += (long long)((m * n + Cfg::BM - 1) / Cfg::BM) * (((L - cs) * n + Cfg::BN - 1) / Cfg::BN);
  }
  for (;;) {
    __syncthreads();  // the previous tile's shared memory is no longer read
    if (threadIdx.x == 0) s_tile = atomicAdd(s.next, 1);
    __syncthreads();
    long long rem = s_tile;
    if (rem >= total) return;
    int g = 0, b = 0, m = 0, cs = 0, rt_n = 0, ct_n = 0;
    for (;; g++) {
      b = L - 3 - g * grp;
      m = b + 1 < grp ? b + 1 : grp;
      cs = b + 1 > s.hfloor ? b + 1 : s.hfloor;
      rt_n = (m * n + Cfg::BM - 1) / Cfg::BM;
      ct_n = ((L - cs) * n + Cfg::BN - 1) / Cfg::BN;
      if (rem < (long long)rt_n * ct_n) break;
      rem -= (long long)rt_n * ct_n;
    }
    const int ct = (int)(rem / rt_n), rt = (int)(rem % rt_n);
    const int t = b - m + 1, ncol = (L - cs) * n;
    if (g > 0) {
      // Columns [ct*BN, ct*BN + BN) of this step are columns shifted by
      // (cs_prev - cs) n in the previous step; those left of the previous
      // step's first column lie in the previous group's diagonal and in-group
      // blocks (or left of the floor), final before this kernel.
      if (threadIdx.x == 0) {
        int ok = 1;
        const int pb = b + grp, pm = pb + 1 < grp ? pb + 1 : grp;
        const int pcs = pb + 1 > s.hfloor ? pb + 1 : s.hfloor;
        const int shift = (pcs - cs) * n;
        const int lo = ct * Cfg::BN - shift, hi = ct * Cfg::BN + Cfg::BN - 1 - shift;
        const int prev_cols = (L - pcs) * n;
        const int prt = (pm * n + Cfg::BM - 1) / Cfg::BM;
        const int need = top < prt ? top : prt;
        if (hi >= 0) {
          const int c0 = (lo > 0 ? lo : 0) / Cfg::BN;
          const int c1 = (hi < prev_cols - 1 ? hi : prev_cols - 1) / Cfg::BN;
          for (int c = c0; c <= c1 && ok; c++) {
            const int* flag = s.done + (long long)(g - 1) * s.ctmax + c;
            long long it = 0;
            while (rec_ld_acquire(flag) < need) {
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
    GemmDims d = {m * n, ncol, n};
    GemmA a;
    a.p0 = s.P + (long long)g * s.pstep + (long long)(grp - m) * n;
    a.p1 = nullptr;
    a.ld0 = s.pld;
    a.ld1 = 2;
    a.bs0 = a.bs1 = 0;
    a.ksplit = n;
    a.rlim0 = INT_MAX;
    a.roff0 = kNoMask;
    a.rlim1 = INT_MAX;
    a.roff1 = kNoMask;
    // X_{b+1, cs:L}; when cs = b+1 its first block is upper triangular
    // (reflectors below).
    GemmB bb = {s.A + cm((long long)(b + 1) * n, (long long)cs * n, s.ld), s.ld, 0,
                cs == b + 1 ? 0 : kNoMask};
    GemmC c;
    c.p0 = s.A + cm((long long)t * n, (long long)cs * n, s.ld);
    c.p1 = s.A + cm((long long)t * n, (long long)(L - 1) * n, s.ld);
    c.ld0 = c.ld1 = s.ld;
    c.bs0 = c.bs1 = 0;
    c.nsplit = ncol - n;
    c.alpha = 1.0;
    c.beta0 = 0.0;
    c.beta1 = 1.0;
    gemm_tile<Cfg, ALIGNED>(d, a, bb, c, rt * Cfg::BM, ct * Cfg::BN, 0, smem_rec);
    __syncthreads();
    if (threadIdx.x == 0 && rt < top) {
      __threadfence();
      asm volatile("red.release.gpu.global.add.s32 [%0], 1;" ::"l"(s.done + (long long)g * s.ctmax + ct)
                   : "memory");
    }
  }
}

int bstri_recurrence_ctmax(int n, int L) { return ((L - 1) * n + CfgS::BN - 1) / CfgS::BN; }

template <class Cfg, bool AL>
static cudaError_t rec_launch(const RecArgs& s, cudaStream_t st) {
  static PerDevice once;
  const int pend = once.pending();
  if (pend >= 0) {
    cudaError_t e = cudaFuncSetAttribute(bstri_recurrence_kernel<Cfg, AL>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)Cfg::SMEM);
    if (e != cudaSuccess) return e;
    once.mark(pend);
  }
  long long tiles = 0;
  for (int g = 0, nsteps = (s.L - 2 + s.grp - 1) / s.grp; g < nsteps; g++) {
    const int b = s.L - 3 - g * s.grp, m = b + 1 < s.grp ? b + 1 : s.grp;
    const int cs = b + 1 > s.hfloor ? b + 1 : s.hfloor;
    tiles += (long long)((m * s.n + Cfg::BM - 1) / Cfg::BM) *
             (((s.L - cs) * s.n + Cfg::BN - 1) / Cfg::BN);
  }
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, bstri_recurrence_kernel<Cfg, AL>,
                                                Cfg::THREADS, Cfg::SMEM);
  long long grid = (long long)sms * (per > 0 ? per : 1);
  if (tiles < grid) grid = tiles;
  bstri_recurrence_kernel<Cfg, AL><<<(int)grid, Cfg::THREADS, Cfg::SMEM, st>>>(s);
  return cudaGetLastError();
}

static RecArgs rec_args(double* A, long long ld, int n, int L, int* done, int* next, int* err) {
  RecArgs s;
  s.A = A;
  s.ld = ld;
  s.n = n;
  s.L = L;
  s.ctmax = bstri_recurrence_ctmax(n, L);
  s.done = done;
  s.next = next;
  s.err = err;
  s.spin_limit = 1ll << 22;
  s.hfloor = 0;
  return s;
}

cudaError_t launch_bstri_recurrence(double* A, long long ld, const double* W, int n, int L,
                                    int* done, int* next, int* err, cudaStream_t st) {
  if (L < 3) return cudaSuccess;
  RecArgs s = rec_args(A, ld, n, L, done, next, err);
  // One row per step: step g uses W_{L-3-g}.
  s.grp = 1;
  s.P = W + (long long)(L - 3) * n * n;
  s.pstep = -(long long)n * n;
  s.pld = n;
  const bool al = ((uintptr_t)A % 16 == 0) && ((uintptr_t)W % 16 == 0) && ld % 2 == 0 && n % 2 == 0;
  return al ? rec_launch<CfgS, true>(s, st) : rec_launch<CfgS, false>(s, st);
}

cudaError_t launch_bstri_recurrence_blocked(double* A, long long ld, const double* P,
                                            long long pld, long long pstep, int grp, int n, int L,
                                            int* done, int* next, int* err, cudaStream_t st,
                                            int hfloor) {
  if (L < 3) return cudaSuccess;
  RecArgs s = rec_args(A, ld, n, L, done, next, err);
  s.grp = grp;
  s.hfloor = hfloor;
  s.P = P;
  s.pstep = pstep;
  s.pld = pld;
  const bool al = ((uintptr_t)A % 16 == 0) && ((uintptr_t)P % 16 == 0) && ld % 2 == 0 &&
                  n % 2 == 0 && pld % 2 == 0 && pstep % 2 == 0;
  return al ? rec_launch<CfgM, true>(s, st) : rec_launch<CfgM, false>(s, st);
}

cudaError_t preload_bstri(size_t* local) {
  cudaError_t e;
  if ((e = preload_one(bstri_recurrence_kernel<CfgM, true>, local)) != cudaSuccess) return e;
  if ((e = preload_one(bstri_recurrence_kernel<CfgM, false>, local)) != cudaSuccess) return e;
  if ((e = preload_one(bstri_recurrence_kernel<CfgS, true>, local)) != cudaSuccess) return e;
  return preload_one(bstri_recurrence_kernel<CfgS, false>, local);
}

}  // namespace bsofi
