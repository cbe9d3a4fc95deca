// FP64 tensor-core tile engine for the BSOF/I contractions (sm_100a).
//
// C = alpha * A * B + beta * C, column-major, strided batch, computed with
// DMMA (mma.sync m16n8k8 f64; tcgen05 has no FP64 kind).  Operands are staged
// in shared memory by cp.async with hardware zero-fill, which also applies the
// structural masks of the block p-cyclic algorithm for free:
//   * A is split along K into two segments with their own base pointers
//     (BSOI reads [X(:,k) | carry] as one operand).  Segment s has a row
//     limit (rows >= rlim are zero) and an upper-triangular mask
//     (element (r,k) is zero when r - roff > k).
//   * B has an upper-triangular mask (element (k,j) is zero when k - koff > j),
//     used for the triangular diagonal blocks of R and R^{-1}, whose strict
//     lower part stores Householder vectors.
//   * C is split along N into two output segments (BSOI writes the carried
//     block column and the finished block column to different buffers), each
//     with its own beta.
// Tiles whose K range is structurally zero are skipped (triangular and
// row-limited operands cost only their nonzero part).
#pragma once
#include "bsofi_common.cuh"

namespace bsofi {

constexpr int kNoMask = 1 << 29;  // roff/koff value that disables a mask

struct GemmA {
  const double* p0;
  const double* p1;
  long long ld0, ld1;
  long long bs0, bs1;  // batch strides (elements)
  int ksplit;          // k < ksplit -> segment 0, else segment 1
  int rlim0, roff0;
  int rlim1, roff1;
};

struct GemmB {
  const double* p;
  long long ld, bs;
  int koff;
};

struct GemmC {
  double* p0;
  double* p1;
  long long ld0, ld1;
  long long bs0, bs1;
  int nsplit;  // j < nsplit -> segment 0, else segment 1 (column j - nsplit)
  double alpha, beta0, beta1;
};

struct GemmDims {
  int M, N, K;
};

// K16: the inner product steps use mma.sync m16n8k16 (16-deep K per
// instruction) instead of m16n8k8.
template <int BM_, int BN_, int WARPS_M_, int WARPS_N_, int STAGES_, int BK_ = 16,
          bool K16_ = false>
struct TileCfg {
  static constexpr int BM = BM_, BN = BN_, BK = BK_;
  static constexpr bool K16 = K16_;
  static_assert(!K16_ || BK_ % 16 == 0, "K16 needs 16-deep stages");
  static constexpr int WARPS_M = WARPS_M_, WARPS_N = WARPS_N_;
  static constexpr int THREADS = 32 * WARPS_M * WARPS_N;
  static constexpr int STAGES = STAGES_;
  static constexpr int WTM = BM / WARPS_M, WTN = BN / WARPS_N;
  static constexpr int MT = WTM / 16, NT = WTN / 8;
  static constexpr int SA = BM + 4;  // k-major A tile row stride (doubles)
  static constexpr int SB = BK + 4;  // n-major B tile row stride (doubles)
  static constexpr int A_STAGE = BK * SA;
  static constexpr int B_STAGE = BN * SB;
  static constexpr size_t SMEM = (size_t)STAGES * (A_STAGE + B_STAGE) * sizeof(double);
  static_assert(WTM % 16 == 0 && WTN % 8 == 0, "warp tile");
  static_assert((BM * BK / 2) % THREADS == 0 && (BN * BK / 2) % THREADS == 0, "loader");
};

using CfgL = TileCfg<128, 128, 2, 4, 3>;  // 256 threads, warp tile 64x32
using CfgM = TileCfg<128, 128, 2, 4, 3, 32>;  // 256 threads, warp tile 64x32, K stage 32
using CfgS = TileCfg<64, 64, 2, 2, 3>;    // 128 threads, warp tile 32x32
// The same tiles with m16n8k16 steps.
using CfgL16 = TileCfg<128, 128, 2, 4, 3, 16, true>;
using CfgM16 = TileCfg<128, 128, 2, 4, 3, 32, true>;
using CfgS16 = TileCfg<64, 64, 2, 2, 3, 16, true>;

BSOFI_DEVINL int clamp02(long long v) { return v < 0 ? 0 : (v > 2 ? 2 : (int)v); }

// Load the A tile (rows m0.., k0..k0+BK) into sA (k-major).  ALIGNED: every
// leading dimension even and every base 16-byte aligned.
template <class Cfg, bool ALIGNED>
BSOFI_DEVINL void load_a_tile(double* sA, const GemmA& a, const double* pa0,
                              const double* pa1, int M, int K, int m0, int k0) {
  if (ALIGNED) {
    constexpr int CH = Cfg::BM * Cfg::BK / 2;
#pragma unroll
    for (int i = 0; i < CH / Cfg::THREADS; i++) {
      int c = threadIdx.x + i * Cfg::THREADS;
      int kk = c / (Cfg::BM / 2);
      int mm = (c % (Cfg::BM / 2)) * 2;
      int k = k0 + kk, r = m0 + mm;
      const double* src;
      long long bound;
      if (k < a.ksplit) {
        bound = min((long long)min(M, a.rlim0), (long long)k + a.roff0 + 1);
        src = pa0 + cm(r, k, a.ld0);
      } else {
        int kl = k - a.ksplit;
        bound = min((long long)min(M, a.rlim1), (long long)kl + a.roff1 + 1);
        src = pa1 + cm(r, kl, a.ld1);
      }
      int nv = (k < K) ? clamp02(bound - r) : 0;
      if (nv == 0) src = pa0;
      cp_async16(sA + kk * Cfg::SA + mm, src, nv * 8);
    }
  } else {
    constexpr int EL = Cfg::BM * Cfg::BK;
#pragma unroll
    for (int i = 0; i < EL / Cfg::THREADS; i++) {
      int e = threadIdx.x + i * Cfg::THREADS;
      int kk = e / Cfg::BM, mm = e % Cfg::BM;
      int k = k0 + kk, r = m0 + mm;
      const double* src;
      bool ok;
      if (k < a.ksplit) {
        ok = r < M && r < a.rlim0 && (long long)r - a.roff0 <= k;
        src = pa0 + cm(r, k, a.ld0);
      } else {
        int kl = k - a.ksplit;
        ok = r < M && r < a.rlim1 && (long long)r - a.roff1 <= kl;
        src = pa1 + cm(r, kl, a.ld1);
      }
      ok = ok && k < K;
      if (!ok) src = pa0;
      cp_async8(sA + kk * Cfg::SA + mm, src, ok ? 8 : 0);
    }
  }
}

template <class Cfg, bool ALIGNED>
BSOFI_DEVINL void load_b_tile(double* sB, const GemmB& b, const double* pb,
                              int N, int K, int k0, int n0) {
  if (ALIGNED) {
    constexpr int CH = Cfg::BN * Cfg::BK / 2;
#pragma unroll
    for (int i = 0; i < CH / Cfg::THREADS; i++) {
      int c = threadIdx.x + i * Cfg::THREADS;
      int jj = c / (Cfg::BK / 2);
      int kk = (c % (Cfg::BK / 2)) * 2;
      int k = k0 + kk, j = n0 + jj;
      long long bound = min((long long)K, (long long)j + b.koff + 1);
      int nv = (j < N) ? clamp02(bound - k) : 0;
      const double* src = nv ? pb + cm(k, j, b.ld) : pb;
      cp_async16(sB + jj * Cfg::SB + kk, src, nv * 8);
    }
  } else {
    constexpr int EL = Cfg::BN * Cfg::BK;
#pragma unroll
    for (int i = 0; i < EL / Cfg::THREADS; i++) {
      int e = threadIdx.x + i * Cfg::THREADS;
      int jj = e / Cfg::BK, kk = e % Cfg::BK;
      int k = k0 + kk, j = n0 + jj;
      bool ok = j < N && k < K && (long long)k - b.koff <= j;
      const double* src = ok ? pb + cm(k, j, b.ld) : pb;
      cp_async8(sB + jj * Cfg::SB + kk, src, ok ? 8 : 0);
    }
  }
}

// K tiles [kt0, kt1) of tile (m0, n0) outside which its K range is
// structurally zero (as gemm_tile computes it).
template <class Cfg>
BSOFI_DEVINL void tile_k_tiles(const GemmDims& d, const GemmA& a, const GemmB& b, int m0, int n0,
                               int& kt0, int& kt1) {
  long long kbeg = 0, kend = d.K;
  if (m0 >= a.rlim0 && a.ksplit < d.K) kbeg = a.ksplit;
  else if (a.ksplit > 0) {
    long long first = (long long)m0 - a.roff0;
    if (first > 0) kbeg = min(first, (long long)a.ksplit);
  }
  {
    long long last = (long long)n0 + Cfg::BN + b.koff;
    if (last < kend) kend = last > 0 ? last : 0;
  }
  kt0 = (int)(kbeg / Cfg::BK);
  kt1 = (int)((kend + Cfg::BK - 1) / Cfg::BK);
}

// True when every element the K tiles [kt0, kt1) of tile (m0, n0) read is
// taken as stored: the tile lies inside M and N, the K tiles inside K, and no
// row limit or triangular mask of A or B reaches into what they load.
template <class Cfg>
BSOFI_DEVINL bool tile_clean(const GemmDims& d, const GemmA& a, const GemmB& b, int m0, int n0,
                             int kt0, int kt1) {
  if (m0 + Cfg::BM > d.M || n0 + Cfg::BN > d.N) return false;
  const long long k_lo = (long long)kt0 * Cfg::BK, k_hi = (long long)kt1 * Cfg::BK;
  if (k_hi > d.K) return false;
  const long long rmax = (long long)m0 + Cfg::BM - 1;
  if (k_lo < a.ksplit) {  // element (r, k) is zero when r >= rlim or r - roff > k
    if (rmax >= a.rlim0) return false;
    if (rmax - a.roff0 > k_lo) return false;
  }
  if (k_hi > a.ksplit) {
    const long long kl = (k_lo > a.ksplit ? k_lo : a.ksplit) - a.ksplit;
    if (rmax >= a.rlim1) return false;
    if (rmax - a.roff1 > kl) return false;
  }
  return k_hi - 1 - b.koff <= n0;  // B element (k, j) is zero when k - koff > j
}

// One CTA computes the BM x BN tile (m0, n0) of batch entry `bz`.
template <class Cfg, bool ALIGNED>
BSOFI_DEVINL void gemm_tile(const GemmDims& d, const GemmA& a, const GemmB& b,
                            const GemmC& c, int m0, int n0, int bz, double* smem) {
  const double* pa0 = a.p0 + (long long)bz * a.bs0;
  const double* pa1 = a.p1 ? a.p1 + (long long)bz * a.bs1 : pa0;
  const double* pb = b.p + (long long)bz * b.bs;

  // Structurally nonzero K range of this tile.
  long long kbeg = 0, kend = d.K;
  if (m0 >= a.rlim0 && a.ksplit < d.K) kbeg = a.ksplit;
  else if (a.ksplit > 0) {
    long long first = (long long)m0 - a.roff0;  // rows >= m0 are zero for k < first
    if (first > 0) kbeg = min(first, (long long)a.ksplit);
  }
  {
    long long last = (long long)n0 + Cfg::BN + b.koff;  // k >= last is zero
    if (last < kend) kend = last > 0 ? last : 0;
  }
  int kt0 = (int)(kbeg / Cfg::BK), kt1 = (int)((kend + Cfg::BK - 1) / Cfg::BK);
  int nkt = kt1 - kt0;

  double* sA = smem;
  double* sB = smem + Cfg::STAGES * Cfg::A_STAGE;

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = warp % Cfg::WARPS_M, wn = warp / Cfg::WARPS_M;
  const int g = lane >> 2, t = lane & 3;

  double acc[Cfg::MT][Cfg::NT][4];
#pragma unroll
  for (int i = 0; i < Cfg::MT; i++)
#pragma unroll
    for (int j = 0; j < Cfg::NT; j++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[i][j][q] = 0.0;

#pragma unroll
  for (int s = 0; s < Cfg::STAGES - 1; s++) {
    if (s < nkt) {
      int k0 = (kt0 + s) * Cfg::BK;
      load_a_tile<Cfg, ALIGNED>(sA + s * Cfg::A_STAGE, a, pa0, pa1, d.M, d.K, m0, k0);
      load_b_tile<Cfg, ALIGNED>(sB + s * Cfg::B_STAGE, b, pb, d.N, d.K, k0, n0);
    }
    cp_async_commit();
  }

  for (int it = 0; it < nkt; it++) {
    cp_async_wait<Cfg::STAGES - 2>();
    __syncthreads();
    const double* tA = sA + (it % Cfg::STAGES) * Cfg::A_STAGE + wm * Cfg::WTM + g;
    const double* tB = sB + (it % Cfg::STAGES) * Cfg::B_STAGE + (wn * Cfg::WTN + g) * Cfg::SB + t;
    if constexpr (Cfg::K16) {
#pragma unroll
      for (int k16 = 0; k16 < Cfg::BK / 16; k16++) {
        // Next stage's loads: after the first 16-deep step's DMMAs when a
        // stage holds two, else first.
        if (k16 == (Cfg::BK >= 32 ? 1 : 0)) {
          const int nx = it + Cfg::STAGES - 1;
          if (nx < nkt) {
            const int s = nx % Cfg::STAGES;
            const int k0 = (kt0 + nx) * Cfg::BK;
            load_b_tile<Cfg, ALIGNED>(sB + s * Cfg::B_STAGE, b, pb, d.N, d.K, k0, n0);
            load_a_tile<Cfg, ALIGNED>(sA + s * Cfg::A_STAGE, a, pa0, pa1, d.M, d.K, m0, k0);
          }
          cp_async_commit();
        }
        double bf[Cfg::NT][4];
#pragma unroll
        for (int j = 0; j < Cfg::NT; j++)
#pragma unroll
          for (int q = 0; q < 4; q++) bf[j][q] = tB[j * 8 * Cfg::SB + k16 * 16 + 4 * q];
#pragma unroll
        for (int i = 0; i < Cfg::MT; i++) {
          double af[8];
#pragma unroll
          for (int q = 0; q < 4; q++) {
            af[2 * q] = tA[(k16 * 16 + t + 4 * q) * Cfg::SA + i * 16];
            af[2 * q + 1] = tA[(k16 * 16 + t + 4 * q) * Cfg::SA + i * 16 + 8];
          }
#pragma unroll
          for (int j = 0; j < Cfg::NT; j++) dmma_16x8x16(acc[i][j], af, bf[j]);
        }
      }
    } else {
#pragma unroll
      for (int k8 = 0; k8 < Cfg::BK / 8; k8++) {
        // With 32-deep stages the next stage's B loads are issued after the
        // first k8 step's DMMAs and its A loads after the second, so the tensor
        // pipe has work queued while the warp computes addresses (measured: -6%
        // on 128x128 K32 tiles; with 16-deep stages issuing them first is
        // faster).
        {
          // One commit group per iteration holding both of the stage's loads:
          // the group is committed after the later of the two.
          constexpr int KA = Cfg::BK >= 32 ? 2 : 0, KB = Cfg::BK >= 32 ? 1 : 0;
          constexpr int KC = KA > KB ? KA : KB;
          int nx = it + Cfg::STAGES - 1;
          if (k8 == KA && nx < nkt) {
            int s = nx % Cfg::STAGES;
            int k0 = (kt0 + nx) * Cfg::BK;
            load_a_tile<Cfg, ALIGNED>(sA + s * Cfg::A_STAGE, a, pa0, pa1, d.M, d.K, m0, k0);
          }
          if (k8 == KB && nx < nkt) {
            int s = nx % Cfg::STAGES;
            int k0 = (kt0 + nx) * Cfg::BK;
            load_b_tile<Cfg, ALIGNED>(sB + s * Cfg::B_STAGE, b, pb, d.N, d.K, k0, n0);
          }
          if (k8 == KC) cp_async_commit();
        }
        double af[Cfg::MT][4], bf[Cfg::NT][2];
#pragma unroll
        for (int i = 0; i < Cfg::MT; i++) {
          af[i][0] = tA[(k8 * 8 + t) * Cfg::SA + i * 16];
          af[i][1] = tA[(k8 * 8 + t) * Cfg::SA + i * 16 + 8];
          af[i][2] = tA[(k8 * 8 + t + 4) * Cfg::SA + i * 16];
          af[i][3] = tA[(k8 * 8 + t + 4) * Cfg::SA + i * 16 + 8];
        }
#pragma unroll
        for (int j = 0; j < Cfg::NT; j++) {
          bf[j][0] = tB[j * 8 * Cfg::SB + k8 * 8];
          bf[j][1] = tB[j * 8 * Cfg::SB + k8 * 8 + 4];
        }
#pragma unroll
        for (int i = 0; i < Cfg::MT; i++)
#pragma unroll
          for (int j = 0; j < Cfg::NT; j++)
            dmma_16x8x8(acc[i][j], af[i][0], af[i][1], af[i][2], af[i][3], bf[j][0], bf[j][1]);
      }
    }
  }
  cp_async_wait<0>();

  // Epilogue.
  double* pc0 = c.p0 + (long long)bz * c.bs0;
  double* pc1 = c.p1 ? c.p1 + (long long)bz * c.bs1 : pc0;
#pragma unroll
  for (int i = 0; i < Cfg::MT; i++) {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      int r = m0 + wm * Cfg::WTM + i * 16 + g + h * 8;
      if (r >= d.M) continue;
#pragma unroll
      for (int j = 0; j < Cfg::NT; j++) {
#pragma unroll
        for (int q = 0; q < 2; q++) {
          int col = n0 + wn * Cfg::WTN + j * 8 + 2 * t + q;
          if (col >= d.N) continue;
          double v = c.alpha * acc[i][j][h * 2 + q];
          double* dst;
          double beta;
          if (col < c.nsplit) {
            dst = pc0 + cm(r, col, c.ld0);
            beta = c.beta0;
          } else {
            dst = pc1 + cm(r, col - c.nsplit, c.ld1);
            beta = c.beta1;
          }
          if (beta != 0.0) v += beta * *dst;
          *dst = v;
        }
      }
    }
  }
}

}  // namespace bsofi
