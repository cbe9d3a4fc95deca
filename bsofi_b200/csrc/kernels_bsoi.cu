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
#include <cuda.h>
#include <atomic>
#include <climits>
#include <mutex>
#include "bsofi_common.cuh"
#include "bsofi_kernels.h"
#include "tcgen05.cuh"

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

// ------------------------------------------------------------------ TMA
// The same persistent BSOI with its tiles' operands loaded by TMA: per
// 32-deep K stage, warp 0's lane 0 issues 16 boxes of 16 rows x 16 k for A
// (from the matrix's block column k, or the carry, per 16 k) and 2 boxes of
// 16 k x BN columns for B = Q_k^T, all with the 128-byte swizzle, into a
// 3-stage ring of full / empty mbarriers; the compute warps read their DMMA
// fragments through the swizzle and never compute copy addresses.  Tiles
// that need a zero-fill mask (the rows of the diagonal block of X(:,k)) take
// the cp.async path on the same shared memory.  The tensor maps cover this
// GPU's memory only; no load uses cluster multicast.
struct BsoiTmaMaps {
  CUtensorMap x;         // the matrix: rows N (inner) x columns N; 16 x 16 boxes
  CUtensorMap carry[2];  // rows N x n; 16 x 16 boxes
  CUtensorMap g;         // G: 2n (k, inner) x 2n (columns) x (L-1); 16 x BN x 1 boxes
};

struct BsoiTmaParams {
  BsoiTmaMaps m;
  BsoiArgs s;
};

struct TmaRing {
  uint64_t full[3];
  uint64_t empty[3];
};

// Abort word of the bounded waits for loads still in flight (never set).
static __device__ int g_tma_no_abort = 0;

constexpr int TMA_STAGES = 3, TMA_A_BYTES = 32768;

// The tile of the TMA kernel: 128 rows x BN columns (BN = 128, or 160 when 2n
// is a multiple of 160 but not of 128, e.g. n = 400), 8 warps of 64 x BN/4.
template <int BN_>
struct TmaTile {
  static constexpr int BM = 128, BN = BN_, BK = 32;
  static constexpr int WTN = BN / CfgM::WARPS_N, NT = WTN / 8;
  // One 16-deep B box (16 k x BN columns) and one stage (A and two B boxes).
  static constexpr int B_BOX_BYTES = 16 * BN * 8;
  static constexpr int STAGE_BYTES = TMA_A_BYTES + 2 * B_BOX_BYTES;
  // The ring, or the cp.async tile of the masked tiles if larger, and 1024
  // bytes to align the swizzled boxes.
  static constexpr size_t SMEM =
      ((size_t)TMA_STAGES * STAGE_BYTES > CfgM::SMEM ? (size_t)TMA_STAGES * STAGE_BYTES
                                                     : CfgM::SMEM) + 1024;
  static_assert(WTN % 8 == 0 && B_BOX_BYTES % 1024 == 0, "TMA tile");
};

// Bounded wait for a ring phase; the (global) error word is read only every
// 256 polls, so a wait whose data is there costs one poll.
BSOFI_DEVINL bool tma_ring_wait(uint64_t* bar, uint32_t parity, const int* err) {
  for (long long i = 0; i < (1ll << 20); i++) {
    if (tc::mbar_try_wait(bar, parity)) return true;
    if ((i & 255) == 255 && *(volatile const int*)err) return false;
  }
  return false;
}

// Byte offset of element (e, r) in a 128-byte-row box with the 128-byte
// swizzle: row r of 128 bytes, its 16-byte chunks permuted by r mod 8.
BSOFI_DEVINL int swz(int r, int e) { return r * 128 + (((e >> 1) ^ (r & 7)) << 4) + (e & 1) * 8; }

// Fragment rows are relabelled so that every 64-bit A fragment read of a
// half-warp meets 16 distinct 8-byte slots of a 128-byte row through the
// swizzle: row g + 8h of a 16-row fragment is tile row frag_row(g, h) (lanes
// 0-15 read rows {2a, 2a+1, 2a+8, 2a+9}).  This permutes output rows only:
// every product and sum is the same, so the results are bitwise those of the
// natural order.  Relabelling B's columns the same way (frag_col) removes
// B's 2-way conflicts too, but measured slower together with the row map
// (BSOI at n = 256, p = 32: 3.350 ms rows only, 3.411 columns only, 3.578
// both, 3.467 neither), so B keeps the natural order.
BSOFI_DEVINL int frag_row(int g, int h) { return (g & 1) + 8 * ((g >> 1) & 1) + 4 * (g >> 2) + 2 * h; }
BSOFI_DEVINL int frag_col(int g) { return g; }

// Stage of K tile kt into ring slot `slot` (lane 0 of warp 0).  below: the
// tile's rows lie under the diagonal block of X(:,k), where X(:,k) is zero;
// a stage that starts before the carry (n not a multiple of 32) then takes
// those 16 k as the carry map's zero fill at column -16.
template <int BN>
BSOFI_DEVINL void tma_issue(const BsoiTmaMaps& M, int k, int n, int src, int m0, int n0, int kt,
                            bool below, char* sa, uint64_t* full) {
  tc::mbar_arrive_expect_tx(full, TmaTile<BN>::STAGE_BYTES);
  char* sb = sa + TMA_A_BYTES;
#pragma unroll
  for (int bk = 0; bk < 2; bk++) {
    const int kk0 = kt * 32 + bk * 16;
#pragma unroll
    for (int bm = 0; bm < 8; bm++) {
      char* dst = sa + (bk * 8 + bm) * 2048;
      if (kk0 < n && !below) tc::tma_load_2d(dst, &M.x, full, m0 + 16 * bm, k * n + kk0);
      else tc::tma_load_2d(dst, &M.carry[src], full, m0 + 16 * bm, kk0 - n);
    }
    tc::tma_load_3d(sb + bk * TmaTile<BN>::B_BOX_BYTES, &M.g, full, kk0, n0, k);
  }
}

// A tile the TMA ring loads: every element its K tiles read is taken as
// stored (tile_clean), or its rows all lie at or below the diagonal block's
// end, where segment 0 (X(:,k)) is zero and read as zero fill, and segment 1
// (the carry) is taken as stored.
template <class T>
BSOFI_DEVINL bool tma_tile_ok(const GemmDims& d, const GemmA& a, const GemmB& b, int m0, int n0,
                              int kt0, int kt1) {
  if (kt1 <= kt0) return false;
  if (tile_clean<T>(d, a, b, m0, n0, kt0, kt1)) return true;
  if (m0 < a.rlim0) return false;
  GemmA z = a;
  z.rlim0 = INT_MAX;
  z.roff0 = kNoMask;
  return tile_clean<T>(d, z, b, m0, n0, kt0, kt1);
}

// One clean tile through the TMA ring; false when a wait gave up (error word
// set).  gstage: stages this CTA has run through the ring (uniform).
template <int BN>
BSOFI_DEVINL bool bsoi_tma_tile(const BsoiTmaMaps& M, const BsoiArgs& s, int k, int src,
                                const GemmC& c, int m0, int n0, int kt0, int kt1, char* tb,
                                TmaRing& ring, unsigned& gstage) {
  using Cfg = CfgM;
  using T = TmaTile<BN>;
  constexpr int NT = T::NT, WTN = T::WTN, STAGE_BYTES = T::STAGE_BYTES;
  const int nkt = kt1 - kt0;
  const bool below = m0 >= (k + 1) * s.n;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = warp % Cfg::WARPS_M, wn = warp / Cfg::WARPS_M;
  const int g = lane >> 2, t = lane & 3;
  bool ok = true;
  int issued = 0, consumed = 0;
  if (warp == 0) {
    for (int i = 0; i < TMA_STAGES && i < nkt && ok; i++) {
      const unsigned gs = gstage + i, slot = gs % TMA_STAGES;
      if (gs >= (unsigned)TMA_STAGES)
        ok = tma_ring_wait(&ring.empty[slot], ((gs / TMA_STAGES) - 1) & 1, s.err);
      if (ok) {
        if (lane == 0)
          tma_issue<BN>(M, k, s.n, src, m0, n0, kt0 + i, below, tb + slot * STAGE_BYTES,
                        &ring.full[slot]);
        issued++;
      } else {
        atomicExch(s.err, 1);
      }
    }
  }
  double acc[Cfg::MT][NT][4];
#pragma unroll
  for (int i = 0; i < Cfg::MT; i++)
#pragma unroll
    for (int j = 0; j < NT; j++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[i][j][q] = 0.0;
  for (int it = 0; it < nkt && ok; it++) {
    const unsigned gs = gstage + it, slot = gs % TMA_STAGES;
    ok = tma_ring_wait(&ring.full[slot], (gs / TMA_STAGES) & 1, s.err);
    if (!ok) {
      atomicExch(s.err, 1);
      break;
    }
    const char* sa = tb + slot * STAGE_BYTES;
    const char* sb = sa + TMA_A_BYTES;
#pragma unroll
    for (int k8 = 0; k8 < 4; k8++) {
      double af[Cfg::MT][4], bf[NT][2];
#pragma unroll
      for (int i = 0; i < Cfg::MT; i++) {
        const int bm = wm * 4 + i;
#pragma unroll
        for (int q = 0; q < 2; q++) {
          const int kk = k8 * 8 + t + 4 * q, bk = kk >> 4, r = kk & 15;
#pragma unroll
          for (int h = 0; h < 2; h++)
            af[i][2 * q + h] = *reinterpret_cast<const double*>(sa + (bk * 8 + bm) * 2048 +
                                                                swz(r, frag_row(g, h)));
        }
      }
#pragma unroll
      for (int j = 0; j < NT; j++) {
        const int jr = wn * WTN + j * 8 + frag_col(g);
#pragma unroll
        for (int q = 0; q < 2; q++) {
          const int kk = k8 * 8 + t + 4 * q;
          bf[j][q] = *reinterpret_cast<const double*>(sb + (kk >> 4) * T::B_BOX_BYTES +
                                                      swz(jr, kk & 15));
        }
      }
#pragma unroll
      for (int i = 0; i < Cfg::MT; i++)
#pragma unroll
        for (int j = 0; j < NT; j++)
          dmma_16x8x8(acc[i][j], af[i][0], af[i][1], af[i][2], af[i][3], bf[j][0], bf[j][1]);
    }
    __syncwarp();
    if (lane == 0) tc::mbar_arrive(&ring.empty[slot]);
    consumed = it + 1;
    if (warp == 0 && it + TMA_STAGES < nkt) {
      // Refill this slot once every warp has consumed it.
      ok = tma_ring_wait(&ring.empty[slot], (gs / TMA_STAGES) & 1, s.err);
      if (ok) {
        if (lane == 0)
          tma_issue<BN>(M, k, s.n, src, m0, n0, kt0 + it + TMA_STAGES, below,
                        tb + slot * STAGE_BYTES, &ring.full[slot]);
        issued++;
      } else {
        atomicExch(s.err, 1);
      }
    }
  }
  if (!ok) {
    // Before the CTA leaves, its loads still in flight land (bounded wait).
    if (warp == 0)
      for (int i = consumed; i < issued; i++) {
        const unsigned gs = gstage + i;
        tma_ring_wait(&ring.full[gs % TMA_STAGES], (gs / TMA_STAGES) & 1, &g_tma_no_abort);
      }
    gstage += nkt;
    return false;
  }
  gstage += nkt;
#pragma unroll
  for (int i = 0; i < Cfg::MT; i++) {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int r = m0 + wm * Cfg::WTM + i * 16 + frag_row(g, h);
#pragma unroll
      for (int j = 0; j < NT; j++) {
#pragma unroll
        for (int q = 0; q < 2; q++) {
          const int col = n0 + wn * WTN + j * 8 + frag_col(2 * t + q);
          const double v = acc[i][j][h * 2 + q];
          if (col < c.nsplit) c.p0[cm(r, col, c.ld0)] = v;
          else c.p1[cm(r, col - c.nsplit, c.ld1)] = v;
        }
      }
    }
  }
  return true;
}

template <int BN>
__global__ void __launch_bounds__(CfgM::THREADS, 1)
    bsoi_tma_kernel(const __grid_constant__ BsoiTmaParams P) {
  using Cfg = CfgM;
  using T = TmaTile<BN>;
  const BsoiArgs& s = P.s;
  extern __shared__ __align__(16) double smem_bsoi[];
  __shared__ int s_tile, s_ok;
  __shared__ TmaRing ring;
  // The 128-byte swizzle wants 1024-byte aligned boxes.
  char* tb = reinterpret_cast<char*>(((uintptr_t)smem_bsoi + 1023) & ~(uintptr_t)1023);
  if (threadIdx.x == 0) {
    for (int i = 0; i < TMA_STAGES; i++) {
      tc::mbar_init(&ring.full[i], 1);
      tc::mbar_init(&ring.empty[i], Cfg::THREADS / 32);
    }
    tc::fence_barrier_init();
    tc::prefetch_tmap(&P.m.x);
    tc::prefetch_tmap(&P.m.carry[0]);
    tc::prefetch_tmap(&P.m.carry[1]);
    tc::prefetch_tmap(&P.m.g);
  }
  unsigned gstage = 0;
  const int n2 = 2 * s.n;
  const int RT = (s.N + T::BM - 1) / T::BM, CT = (n2 + BN - 1) / BN;
  const long long total = (long long)(s.L - 1) * RT * CT;
  for (;;) {
    __syncthreads();  // the previous tile's shared memory is no longer read
    if (threadIdx.x == 0) s_tile = atomicAdd(s.next, 1);
    __syncthreads();
    const long long tile = s_tile;
    if (tile >= total) return;
    const int step = (int)(tile / ((long long)RT * CT));  // 0 = k = L-2
    const int rem = (int)(tile % ((long long)RT * CT));
    const int rb = rem / CT, cb = rem % CT;
    const int k = s.L - 2 - step;
    if (step > 0) {
      if (threadIdx.x == 0) {
        const int* flag = s.done + (long long)(step - 1) * RT + rb;
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
    const int src = (s.L - 2 - k) & 1;
    GemmDims d = {s.N, n2, n2};
    GemmA a;
    a.p0 = s.A + cm(0, (long long)k * s.n, s.ld);
    a.ld0 = s.ld;
    a.p1 = s.carry[src];
    a.ld1 = s.ldc;
    a.bs0 = a.bs1 = 0;
    a.ksplit = s.n;
    a.rlim0 = (k + 1) * s.n;
    a.roff0 = k * s.n;
    a.rlim1 = INT_MAX;
    a.roff1 = kNoMask;
    GemmB b = {s.G + (long long)k * n2 * n2, n2, 0, kNoMask};
    GemmC c = {};
    c.p0 = s.carry[(s.L - 1 - k) & 1];
    c.ld0 = s.ldc;
    c.p1 = s.A + cm(0, (long long)(k + 1) * s.n, s.ld);
    c.ld1 = s.ld;
    c.nsplit = s.n;
    c.alpha = 1.0;
    const int m0 = rb * T::BM, n0 = cb * BN;
    int kt0, kt1;
    tile_k_tiles<T>(d, a, b, m0, n0, kt0, kt1);
    if (tma_tile_ok<T>(d, a, b, m0, n0, kt0, kt1)) {
      const bool ok = bsoi_tma_tile<BN>(P.m, s, k, src, c, m0, n0, kt0, kt1, tb, ring, gstage);
      // Every warp reaches this barrier; a wait that gave up in any warp
      // (error word set) ends the whole CTA.
      if (__syncthreads_or(!ok)) return;
    } else {
      // The cp.async engine in 128-column passes; the last pass's columns
      // end at the tile's (its loads there are zero-filled, its stores
      // skipped).
      GemmDims dc = d;
      dc.N = min(d.N, n0 + BN);
      for (int c0 = 0; c0 < BN; c0 += Cfg::BN) {
        if (c0 > 0) __syncthreads();  // the previous pass's shared memory is read
        gemm_tile<Cfg, true>(dc, a, b, c, m0, n0 + c0, 0, smem_bsoi);
      }
      // The ring's next TMA writes land on bytes these passes wrote.
      tc::fence_proxy_async_smem();
    }
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

// TMA loading of the persistent BSOI's clean tiles (1, the default) or
// cp.async for every tile (0); process-wide.  Measured at n = 256, p = 32:
// BSOI 3.350 against 3.574 ms (30.2 against 28.3 TFLOP/s), bitwise the same.
static std::atomic<int> g_tma{1};
void bsoi_set_tma(int on) { g_tma.store(on ? 1 : 0); }

namespace {

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn tma_encoder() {
  static std::once_flag once;
  static EncodeTiledFn fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// FP64 tensor map of rank 2 or 3 (dims[0] contiguous), 128-byte swizzle.
bool encode_f64(CUtensorMap* m, const double* base, int rank, const cuuint64_t* dims,
                const cuuint64_t* strides_bytes, const cuuint32_t* box) {
  EncodeTiledFn f = tma_encoder();
  if (!f) return false;
  const cuuint32_t es[3] = {1, 1, 1};
  return f(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, rank, const_cast<double*>(base), dims, strides_bytes,
           box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int BN>
cudaError_t launch_tma_bn(const BsoiTmaParams& P, int n, int L, int N, cudaStream_t st) {
  const size_t smem = TmaTile<BN>::SMEM;
  static PerDevice once;
  const int pend = once.pending();
  if (pend >= 0) {
    cudaError_t e = cudaFuncSetAttribute(bsoi_tma_kernel<BN>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    once.mark(pend);
  }
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, bsoi_tma_kernel<BN>, CfgM::THREADS, smem);
  const long long tiles = (long long)(L - 1) * ((N + 127) / 128) * ((2 * n + BN - 1) / BN);
  int grid = sms * (per > 0 ? per : 1);
  if (tiles < grid) grid = (int)tiles;
  bsoi_tma_kernel<BN><<<grid, CfgM::THREADS, smem, st>>>(P);
  return cudaGetLastError();
}

// The TMA launch for a full-range persistent BSOI; false when it does not
// apply (the caller then launches the cp.async kernel): n a multiple of 16
// (the 16-row boxes of A start on block boundaries) and 2n a multiple of 128
// (128 x 128 tiles) or else of 160 (128 x 160 tiles: no ragged column tile
// at n = 400, 2n = 800).
bool launch_tma(const BsoiArgs& s, cudaStream_t st, cudaError_t* err) {
  const int n = s.n, L = s.L, N = s.N;
  if (n % 16 != 0) return false;
  const int bn = (2 * n) % 128 == 0 ? 128 : ((2 * n) % 160 == 0 ? 160 : 0);
  if (bn == 0) return false;
  BsoiTmaParams P;
  P.s = s;
  {
    const cuuint64_t dims[2] = {(cuuint64_t)N, (cuuint64_t)N};
    const cuuint64_t str[1] = {(cuuint64_t)s.ld * sizeof(double)};
    const cuuint32_t box[2] = {16, 16};
    if (!encode_f64(&P.m.x, s.A, 2, dims, str, box)) return false;
  }
  for (int i = 0; i < 2; i++) {
    const cuuint64_t dims[2] = {(cuuint64_t)N, (cuuint64_t)n};
    const cuuint64_t str[1] = {(cuuint64_t)s.ldc * sizeof(double)};
    const cuuint32_t box[2] = {16, 16};
    if (!encode_f64(&P.m.carry[i], s.carry[i], 2, dims, str, box)) return false;
  }
  {
    const cuuint64_t n2 = 2ull * n;
    const cuuint64_t dims[3] = {n2, n2, (cuuint64_t)(L - 1)};
    const cuuint64_t str[2] = {n2 * sizeof(double), n2 * n2 * sizeof(double)};
    const cuuint32_t box[3] = {16, (cuuint32_t)bn, 1};
    if (!encode_f64(&P.m.g, s.G, 3, dims, str, box)) return false;
  }
  *err = bn == 128 ? launch_tma_bn<128>(P, n, L, N, st) : launch_tma_bn<160>(P, n, L, N, st);
  return true;
}

}  // namespace

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
  if (al && g_tma.load() && never == nullptr && s.rb0 == 0 && s.rb1 == s.N) {
    cudaError_t e = cudaSuccess;
    if (launch_tma(s, st, &e)) return e;
  }
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
  if ((e = preload_one(bsoi_tma_kernel<128>, local)) != cudaSuccess) return e;
  if ((e = preload_one(bsoi_tma_kernel<160>, local)) != cudaSuccess) return e;
  if ((e = preload_one(bsoi_persistent_kernel<CfgM16, true>, local)) != cudaSuccess) return e;
  if ((e = preload_one(bsoi_persistent_kernel<CfgM16, false>, local)) != cudaSuccess) return e;
  if ((e = preload_one(bsoi_persistent_kernel<CfgS16, true>, local)) != cudaSuccess) return e;
  return preload_one(bsoi_persistent_kernel<CfgS16, false>, local);
}

}  // namespace bsofi
