// BSOI as one persistent kernel: all p-1 steps X(:,k:k+1) <- X(:,k:k+1) Q_k^T.
//
// Reference: lapackXbsoi_ormqr / _orgqr, src/bsofi_cpu.c:211-333 (applied
// from k = L-2 down to 0).  Step k is the product
//   [X(:,k) | carry] (N x 2n) * Q_k^T (2n x 2n)  ->  [carry' | X(:,k+1) final]
// on 128 x 128 output tiles.  Rows are independent across steps, so a tile of
// step k only waits for the tiles of step k+1 in the same row band (they wrote
// the carry it reads and read the buffers it overwrites), not for the whole
// step: there is no per-step wave tail and no launch gap.  Tiles are claimed
// in (step, row band, column) order from a global counter and every wait is
// on a tile claimed earlier, whose CTA is already running: progress needs no
// co-residency, so the launch is an ordinary one (a cooperative launch would
// wait for the whole GPU and serialise batched inversions on other streams).
// Every spin is bounded and reports through an error word.  A launch may be
// restricted to the row bands [rb0, rb1): each of its tiles is then the tile a
// launch over all rows computes (rows of X are independent in BSOI), which is
// how one inversion's BSOI is split across GPUs by rows.
#include <climits>
#include "bsofi_common.cuh"
#include "bsofi_kernels.h"

namespace bsofi {

struct BsoiArgs {
  double* A;
  long long ld;
  double* carry[2];  // ldd x n each; the carry written by step k is carry[(L-1-k) & 1]
  long long ldc;
  const double* G;   // (L-1) x (2n)^2, G_k = Q_k^T
  int n, L, N;
  int* done;         // (L-1) x row bands: finished column tiles
  int* next;         // tile counter
  int* err;
  long long spin_limit;
  int rb0, rb1;      // row bands computed (of the tile height)
  const int* never;  // diagnostics: when set, every step wait polls this word instead
};

BSOFI_DEVINL int ld_acq(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

template <class Cfg, bool ALIGNED>
__global__ void __launch_bounds__(Cfg::THREADS, 1) bsoi_persistent_kernel(BsoiArgs s) {
  extern __shared__ __align__(16) double smem_bsoi[];
  __shared__ int s_tile, s_ok;
  const int n2 = 2 * s.n;
  const int RT = (s.N + Cfg::BM - 1) / Cfg::BM, CT = (n2 + Cfg::BN - 1) / Cfg::BN;
  const int RS = s.rb1 - s.rb0;  // row bands of this launch
  const long long total = (long long)(s.L - 1) * RS * CT;
  for (;;) {
    __syncthreads();  // the previous tile's shared memory is no longer read
    if (threadIdx.x == 0) s_tile = atomicAdd(s.next, 1);
    __syncthreads();
    const long long tile = s_tile;
    if (tile >= total) return;
    const int step = (int)(tile / ((long long)RS * CT));  // 0 = k = L-2
    const int rem = (int)(tile % ((long long)RS * CT));
    const int rb = s.rb0 + rem / CT, cb = rem % CT;
    const int k = s.L - 2 - step;
    if (step > 0) {
      if (threadIdx.x == 0) {
        const int* flag = s.never ? s.never : s.done + (long long)(step - 1) * RT + rb;
        long long it = 0;
        int ok = 1;
        while (ld_acq(flag) < CT) {
          if (ld_acq(s.err) != 0 || ++it > s.spin_limit) {
            atomicExch(s.err, 1);
            ok = 0;
            break;
          }
          __nanosleep(64);
        }
        s_ok = ok;
      }
      __syncthreads();
      if (!s_ok) return;
    }
    GemmDims d = {s.N, n2, n2};
    GemmA a;
    a.p0 = s.A + cm(0, (long long)k * s.n, s.ld);
    a.ld0 = s.ld;
    a.p1 = s.carry[(s.L - 2 - k) & 1];
    a.ld1 = s.ldc;
    a.bs0 = a.bs1 = 0;
    a.ksplit = s.n;
    a.rlim0 = (k + 1) * s.n;
    a.roff0 = k * s.n;
    a.rlim1 = INT_MAX;
    a.roff1 = kNoMask;
    GemmB b = {s.G + (long long)k * n2 * n2, n2, 0, kNoMask};
    GemmC c;
    c.p0 = s.carry[(s.L - 1 - k) & 1];
    c.ld0 = s.ldc;
    c.p1 = s.A + cm(0, (long long)(k + 1) * s.n, s.ld);
    c.ld1 = s.ld;
    c.bs0 = c.bs1 = 0;
    c.nsplit = s.n;
    c.alpha = 1.0;
    c.beta0 = c.beta1 = 0.0;
    gemm_tile<Cfg, ALIGNED>(d, a, b, c, rb * Cfg::BM, cb * Cfg::BN, 0, smem_bsoi);
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      asm volatile("red.release.gpu.global.add.s32 [%0], 1;" ::"l"(s.done + (long long)step * RT + rb)
                   : "memory");
    }
  }
}

// Row bands of the smallest tile height (sizes the done counters for every
// tile configuration).
int bsoi_row_bands(int N) { return (N + CfgS::BM - 1) / CfgS::BM; }

template <class Cfg, bool AL>
static cudaError_t launch_al(const BsoiArgs& s, cudaStream_t st) {
  static PerDevice once;
  const int pend = once.pending();
  if (pend >= 0) {
    cudaError_t e = cudaFuncSetAttribute(bsoi_persistent_kernel<Cfg, AL>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)Cfg::SMEM);
    if (e != cudaSuccess) return e;
    once.mark(pend);
  }
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, bsoi_persistent_kernel<Cfg, AL>,
                                                Cfg::THREADS, Cfg::SMEM);
  BsoiArgs a = s;
  const int RT = (s.N + Cfg::BM - 1) / Cfg::BM, CT = (2 * s.n + Cfg::BN - 1) / Cfg::BN;
  // Rows [row0, row1) in bands of the tile height; row0 must start a band and
  // row1 end one (or be N).
  if (s.rb0 % Cfg::BM != 0 || (s.rb1 % Cfg::BM != 0 && s.rb1 != s.N) || s.rb0 >= s.rb1)
    return cudaErrorInvalidValue;
  a.rb0 = s.rb0 / Cfg::BM;
  a.rb1 = (s.rb1 + Cfg::BM - 1) / Cfg::BM;
  if (a.rb1 > RT) return cudaErrorInvalidValue;
  long long tiles = (long long)(s.L - 1) * (a.rb1 - a.rb0) * CT;
  int grid = sms * (per > 0 ? per : 1);
  if (tiles < grid) grid = (int)tiles;
  bsoi_persistent_kernel<Cfg, AL><<<grid, Cfg::THREADS, Cfg::SMEM, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_bsoi_persistent(double* A, long long ld, double* carry0, double* carry1,
                                   long long ldc, const double* G, int n, int L, int* done,
                                   int* next, int* err, bool small, cudaStream_t st, int row0,
                                   int row1, const int* never) {
  BsoiArgs s;
  s.A = A;
  s.ld = ld;
  s.carry[0] = carry0;
  s.carry[1] = carry1;
  s.ldc = ldc;
  s.G = G;
  s.n = n;
  s.L = L;
  s.N = n * L;
  s.done = done;
  s.next = next;
  s.err = err;
  s.spin_limit = never ? 1ll << 12 : 1ll << 22;
  s.never = never;
  // Row range in rows here; launch_al turns it into row bands of its tiles.
  s.rb0 = row0;
  s.rb1 = row1 < 0 ? s.N : row1;
  const bool al = ((uintptr_t)A % 16 == 0) && ((uintptr_t)carry0 % 16 == 0) &&
                  ((uintptr_t)carry1 % 16 == 0) && ((uintptr_t)G % 16 == 0) && ld % 2 == 0 &&
                  ldc % 2 == 0 && n % 2 == 0;
  if (gemm_k16()) {
    if (small) return al ? launch_al<CfgS16, true>(s, st) : launch_al<CfgS16, false>(s, st);
    return al ? launch_al<CfgM16, true>(s, st) : launch_al<CfgM16, false>(s, st);
  }
  if (small) return al ? launch_al<CfgS, true>(s, st) : launch_al<CfgS, false>(s, st);
  return al ? launch_al<CfgM, true>(s, st) : launch_al<CfgM, false>(s, st);
}

// ------------------------------------------------------------------ grouped
// BSOI of many independent instances in one persistent launch.  The tiles of
// all instances form one queue: instance by instance, each instance's tiles
// in the (step, row band, column) order of bsoi_persistent_kernel.  A tile
// waits only for tiles of its own instance claimed before it, whose CTAs are
// already running, so progress needs no co-residency; while the last steps of
// one instance finish, idle CTAs claim the next instance's tiles instead of
// idling at a launch boundary.
template <class Cfg, bool ALIGNED>
__global__ void __launch_bounds__(Cfg::THREADS, 1)
    bsoi_grouped_kernel(const __grid_constant__ BsoiGroup g) {
  extern __shared__ __align__(16) double smem_bsoig[];
  __shared__ long long s_tile;
  __shared__ int s_inst, s_ok;
  for (;;) {
    __syncthreads();  // the previous tile's shared memory is no longer read
    if (threadIdx.x == 0) {
      const long long t = atomicAdd(g.next, 1ull);
      int lo = 0, hi = g.count - 1;  // last instance with tile0 <= t
      if (t < g.total) {
        while (lo < hi) {
          const int mid = (lo + hi + 1) / 2;
          if (g.inst[mid].tile0 <= (long long)t) lo = mid;
          else hi = mid - 1;
        }
      }
      s_tile = (long long)t;
      s_inst = lo;
    }
    __syncthreads();
    const long long tile = s_tile;
    if (tile >= g.total) return;
    const BsoiInst& I = g.inst[s_inst];
    const int n2 = 2 * I.n;
    const int RT = (I.N + Cfg::BM - 1) / Cfg::BM, CT = (n2 + Cfg::BN - 1) / Cfg::BN;
    const long long local = tile - I.tile0;
    const int step = (int)(local / ((long long)RT * CT));  // 0 = k = L-2
    const int rem = (int)(local % ((long long)RT * CT));
    const int rb = rem / CT, cb = rem % CT;
    const int k = I.L - 2 - step;
    if (step > 0) {
      if (threadIdx.x == 0) {
        const int* flag = I.done + (long long)(step - 1) * RT + rb;
        long long it = 0;
        int ok = 1;
        while (ld_acq(flag) < CT) {
          if (ld_acq(I.err) != 0 || ++it > g.spin_limit) {
            atomicExch(I.err, 1);
            ok = 0;
            break;
          }
          __nanosleep(64);
        }
        s_ok = ok;
      }
      __syncthreads();
      if (!s_ok) continue;  // this instance failed; its info word reports it
    }
    GemmDims d = {I.N, n2, n2};
    GemmA a;
    a.p0 = I.A + cm(0, (long long)k * I.n, I.ld);
    a.ld0 = I.ld;
    a.p1 = I.carry[(I.L - 2 - k) & 1];
    a.ld1 = I.ldc;
    a.bs0 = a.bs1 = 0;
    a.ksplit = I.n;
    a.rlim0 = (k + 1) * I.n;
    a.roff0 = k * I.n;
    a.rlim1 = INT_MAX;
    a.roff1 = kNoMask;
    GemmB b = {I.G + (long long)k * n2 * n2, n2, 0, kNoMask};
    GemmC c;
    c.p0 = I.carry[(I.L - 1 - k) & 1];
    c.ld0 = I.ldc;
    c.p1 = I.A + cm(0, (long long)(k + 1) * I.n, I.ld);
    c.ld1 = I.ld;
    c.bs0 = c.bs1 = 0;
    c.nsplit = I.n;
    c.alpha = 1.0;
    c.beta0 = c.beta1 = 0.0;
    gemm_tile<Cfg, ALIGNED>(d, a, b, c, rb * Cfg::BM, cb * Cfg::BN, 0, smem_bsoig);
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      asm volatile("red.release.gpu.global.add.s32 [%0], 1;" ::"l"(I.done + (long long)step * RT + rb)
                   : "memory");
    }
  }
}

long long bsoi_group_tiles(int n, int L, bool small) {
  const int BM = small ? CfgS::BM : CfgM::BM, BN = small ? CfgS::BN : CfgM::BN;
  return (long long)(L - 1) * ((n * L + BM - 1) / BM) * ((2 * n + BN - 1) / BN);
}

template <class Cfg, bool AL>
static cudaError_t group_launch(const BsoiGroup& g, cudaStream_t st) {
  static PerDevice once;
  const int pend = once.pending();
  if (pend >= 0) {
    cudaError_t e = cudaFuncSetAttribute(bsoi_grouped_kernel<Cfg, AL>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)Cfg::SMEM);
    if (e != cudaSuccess) return e;
    once.mark(pend);
  }
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, bsoi_grouped_kernel<Cfg, AL>, Cfg::THREADS,
                                                Cfg::SMEM);
  long long grid = (long long)sms * (per > 0 ? per : 1);
  if (g.total < grid) grid = g.total;
  if (grid < 1) return cudaSuccess;
  bsoi_grouped_kernel<Cfg, AL><<<(int)grid, Cfg::THREADS, Cfg::SMEM, st>>>(g);
  return cudaGetLastError();
}

cudaError_t launch_bsoi_grouped(const BsoiGroup& g, bool small, bool aligned, cudaStream_t st) {
  if (small) return aligned ? group_launch<CfgS, true>(g, st) : group_launch<CfgS, false>(g, st);
  return aligned ? group_launch<CfgM, true>(g, st) : group_launch<CfgM, false>(g, st);
}

cudaError_t preload_bsoi(size_t* local) {
  cudaError_t e;
  if ((e = preload_one(bsoi_grouped_kernel<CfgM, true>, local)) != cudaSuccess) return e;
  if ((e = preload_one(bsoi_grouped_kernel<CfgM, false>, local)) != cudaSuccess) return e;
  if ((e = preload_one(bsoi_grouped_kernel<CfgS, true>, local)) != cudaSuccess) return e;
  if ((e = preload_one(bsoi_grouped_kernel<CfgS, false>, local)) != cudaSuccess) return e;
  if ((e = preload_one(bsoi_persistent_kernel<CfgM, true>, local)) != cudaSuccess) return e;
  if ((e = preload_one(bsoi_persistent_kernel<CfgM, false>, local)) != cudaSuccess) return e;
  if ((e = preload_one(bsoi_persistent_kernel<CfgS, true>, local)) != cudaSuccess) return e;
  if ((e = preload_one(bsoi_persistent_kernel<CfgS, false>, local)) != cudaSuccess) return e;
  if ((e = preload_one(bsoi_persistent_kernel<CfgM16, true>, local)) != cudaSuccess) return e;
  if ((e = preload_one(bsoi_persistent_kernel<CfgM16, false>, local)) != cudaSuccess) return e;
  if ((e = preload_one(bsoi_persistent_kernel<CfgS16, true>, local)) != cudaSuccess) return e;
  return preload_one(bsoi_persistent_kernel<CfgS16, false>, local);
}

}  // namespace bsofi
