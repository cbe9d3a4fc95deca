// BSOF as one persistent kernel.
//
// Reference: lapackXbsof, src/bsofi_cpu.c:86-118: for k = 0..L-3, dgeqrf of
// the stacked 2n x n panel [R~_k; B_k] at A_BLK(k,k), dormqr('L','T') of
// A_BLK(k,k+1) and A_BLK(k,L-1); then dgeqrf of the final 2n x 2n block.
//
// Work decomposition.  Every block column is cut into tiles of NB columns
// (the last one may be narrower).  A "leaf" is the Householder QR of one tile
// inside its panel; leaves are numbered s = 0..S-1 in the reference's order
// (panel k, left to right; the final panel has the tiles of block columns L-2
// and L-1).  Leaf s updates a set of target tiles with its block reflector
// (I - V T V^T)^T: the rest of its panel, the next diagonal block column
// (A_BLK(k,k+1)) and the last block column (A_BLK(k,L-1)).
//
// For a physical tile x the leaves that update it form one contiguous range
// [lo(x), hi(x)) of leaf numbers, and hi(x) is the leaf that factors it.  A
// counter cnt[x] holds how many of those updates are done, so leaf s may
// update x once cnt[x] == s - lo(x), and may factor x once cnt[x] == hi - lo.
//
// CTA 0 runs the critical chain: factor leaf s, then immediately apply it to
// the tile of leaf s+1 (target 0).  The other CTAs claim the remaining
// (leaf, target) updates from an ordered task counter.  Every wait depends
// only on tasks earlier in that order and all CTAs are co-resident
// (cooperative launch), so the schedule cannot deadlock; every spin is
// bounded and sets an error word instead of hanging.
#include <atomic>
#include <climits>
#include "bsofi_common.cuh"
#include "bsofi_kernels.h"

namespace bsofi {

constexpr int BT = 256;  // threads per CTA
constexpr int BW = BT / 32;

struct BsofGeom {
  int n, L, NB, nl, S;
  int form_g;  // 1: leaves also update G_k = Q_k^T (identity-initialised by the caller)
};

// Leaf s -> panel k, leaf index l in the panel, tile (m, t), panel column j0.
struct Leaf {
  int k, l, m, t, j0, w;
};

BSOFI_DEVINL Leaf leaf_of(const BsofGeom& g, int s) {
  Leaf f;
  const int reg = (g.L - 2) * g.nl;
  if (s < reg) {
    f.k = s / g.nl;
    f.l = s % g.nl;
    f.m = f.k;
    f.t = f.l;
    f.j0 = f.t * g.NB;
  } else {
    f.k = g.L - 2;
    f.l = s - reg;
    if (f.l < g.nl) {
      f.m = g.L - 2;
      f.t = f.l;
      f.j0 = f.t * g.NB;
    } else {
      f.m = g.L - 1;
      f.t = f.l - g.nl;
      f.j0 = g.n + f.t * g.NB;
    }
  }
  f.w = min(g.NB, g.n - f.t * g.NB);
  return f;
}

BSOFI_DEVINL int tile_id(const BsofGeom& g, int m, int t) { return m * g.nl + t; }

BSOFI_DEVINL void tile_range(const BsofGeom& g, int m, int t, int& lo, int& hi) {
  if (m >= g.L) {  // G_k tile: every leaf of panel k, in order
    const int k = (m - g.L) / 2;
    lo = k * g.nl;
    hi = lo + (k <= g.L - 3 ? g.nl : 2 * g.nl);
    return;
  }
  if (m <= g.L - 2) {
    lo = max(0, (m - 1) * g.nl);
    hi = m * g.nl + t;
  } else {
    lo = 0;
    hi = (g.L - 1) * g.nl + t;
  }
}

// Number of targets of leaf s; target q (0 = tile of leaf s+1).  With
// form_g the 2*nl column tiles of G_k follow the matrix targets; they are
// reported as block columns m = L + 2k + h (h = 0, 1) of a virtual matrix.
BSOFI_DEVINL int ntargets(const BsofGeom& g, const Leaf& f) {
  const int gt = g.form_g ? 2 * g.nl : 0;
  if (f.k <= g.L - 3) return (g.nl - 1 - f.l) + 2 * g.nl + gt;
  return 2 * g.nl - 1 - f.l + gt;
}

BSOFI_DEVINL void target_of(const BsofGeom& g, const Leaf& f, int q, int& m, int& t) {
  const int nmat = (f.k <= g.L - 3) ? (g.nl - 1 - f.l) + 2 * g.nl : 2 * g.nl - 1 - f.l;
  if (q >= nmat) {
    const int u = q - nmat;
    m = g.L + 2 * f.k + u / g.nl;
    t = u % g.nl;
    return;
  }
  if (f.k <= g.L - 3) {
    const int np = g.nl - 1 - f.l;
    if (q < np) {
      m = f.k;
      t = f.l + 1 + q;
    } else if (q < np + g.nl) {
      m = f.k + 1;
      t = q - np;
    } else {
      m = g.L - 1;
      t = q - np - g.nl;
    }
  } else {
    int u = f.l + 1 + q;
    if (u < g.nl) {
      m = g.L - 2;
      t = u;
    } else {
      m = g.L - 1;
      t = u - g.nl;
    }
  }
}

// Worker tasks before leaf s (each leaf contributes ntargets - 1 tasks).
BSOFI_DEVINL long long tasks_before(const BsofGeom& g, int s) {
  const int reg = (g.L - 2) * g.nl;
  const long long nl = g.nl, gt = g.form_g ? 2 * nl : 0;
  const long long per_reg_leaf0 = 3 * nl - 2 + gt;  // tasks of regular leaf l: 3nl - 2 - l + gt
  const long long per_panel = nl * per_reg_leaf0 - nl * (nl - 1) / 2;
  if (s <= reg) {
    long long k = s / g.nl, l = s % g.nl;
    return k * per_panel + l * per_reg_leaf0 - l * (l - 1) / 2;
  }
  long long base = (long long)(g.L - 2) * per_panel;
  long long l = s - reg;  // final leaf l has max(2nl - 2 - l + gt, 0) tasks
  if (gt > 0) return base + l * (2 * nl - 2 + gt) - l * (l - 1) / 2;
  long long full = min(l, 2 * nl - 1);
  return base + full * (2 * nl - 2) - full * (full - 1) / 2;
}

struct BsofState {
  // Block columns 0..L-2 of the matrix at A (leading dimension ld), the last
  // block column at Al (ldl).  The ordinary layout has Al = A + (L-1) n ld;
  // the compact one stores block columns 0..L-2 with ld = 3n (every access
  // of block column m stays in block rows m-1..m+1, so those windows never
  // overlap) and the last block column as its own N x n array.
  double* A;
  long long ld;
  double* Al;
  long long ldl;
  double* G;  // (L-1) x (2n)^2, used when form_g
  double* tau;
  double* T;  // 256 doubles per leaf: (k * maxleaves + l) * 256
  int maxleaves;
  int* cnt;       // per tile
  int* factored;  // per leaf
  int* next_task;
  int* err;       // 0 ok; 1 timeout
  long long spin_limit;
  unsigned long long* timeline;  // 4 stamps per leaf from the panel CTA (diagnostics)
  // This launch factors leaves [s_begin, s_end) and runs their worker tasks;
  // the per-tile and per-leaf counters carry over from an earlier launch of
  // the leaves before s_begin, whose updates are then all done.
  int s_begin, s_end;
};

// Element (row, column col of block column m) of the matrix, and the leading
// dimension there.
BSOFI_DEVINL double* mat_ptr(const BsofGeom& g, const BsofState& st, long long row, int m,
                             int col, long long& ldm) {
  if (m == g.L - 1) {
    ldm = st.ldl;
    return st.Al + cm(row, col, st.ldl);
  }
  ldm = st.ld;
  return st.A + cm(row, (long long)m * g.n + col, st.ld);
}

// Column tile (m, t) of the matrix, or of G_k for m >= L: base pointer at the
// leaf's first row j0 of its panel, and leading dimension.
BSOFI_DEVINL double* tile_ptr(const BsofGeom& g, const BsofState& st, int k, int j0, int m, int t,
                              long long& ldt) {
  if (m >= g.L) {
    const int kk = (m - g.L) / 2, h = (m - g.L) % 2;
    const long long n2 = 2ll * g.n;
    ldt = n2;
    return st.G + (long long)kk * n2 * n2 + cm(j0, (long long)h * g.n + t * g.NB, n2);
  }
  return mat_ptr(g, st, (long long)k * g.n + j0, m, t * g.NB, ldt);
}

BSOFI_DEVINL unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

BSOFI_DEVINL int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

BSOFI_DEVINL void red_release_add(int* p, int v) {
  asm volatile("red.release.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Thread 0 waits until *p >= target (bounded); the result is broadcast.
// Returns false when the wait timed out or another CTA reported an error.
BSOFI_DEVINL bool block_wait_geq(const BsofState& st, const int* p, int target, int* sflag) {
  if (threadIdx.x == 0) {
    int ok = 1;
    long long it = 0;
    while (ld_acquire(p) < target) {
      if (ld_acquire(st.err) != 0) {
        ok = 0;
        break;
      }
      if (++it > st.spin_limit) {
        atomicExch(st.err, 1);
        ok = 0;
        break;
      }
      __nanosleep(64);
    }
    *sflag = ok;
  }
  __syncthreads();
  bool ok = *sflag != 0;
  __syncthreads();
  return ok;
}

// Barrier among the first `count` threads of the CTA (id 1; id 0 is __syncthreads).
BSOFI_DEVINL void named_bar(int count) { asm volatile("bar.sync 1, %0;" ::"r"(count) : "memory"); }
// Barrier id 2: the panel CTA's prefetch warps (concurrent with barrier 1).
BSOFI_DEVINL void named_bar2(int count) { asm volatile("bar.sync 2, %0;" ::"r"(count) : "memory"); }

// Sum NB values per lane over a warp (transpose reduction): lane l ends with
// the warp sum of value (l >> (5 - log2 NB)) & (NB - 1).
template <int NB>
BSOFI_DEVINL double wsum_t(double (&v)[NB], int lane) {
  constexpr int LOG = (NB == 16) ? 4 : 3;
#pragma unroll
  for (int lev = 0; lev < LOG; lev++) {
    const int off = 16 >> lev, half = NB >> (lev + 1);
    const bool up = (lane & off) != 0;
#pragma unroll
    for (int j = 0; j < half; j++) {
      double send = up ? v[j] : v[j + half];
      double keep = up ? v[j + half] : v[j];
      v[j] = keep + __shfl_xor_sync(0xffffffffu, send, off);
    }
  }
  double s = v[0];
#pragma unroll
  for (int off = 16 >> LOG; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  return s;
}

template <int NB>
struct Smem {
  double red[2][BW][NB];
  double coef[2][NB + 4];   // tau*w_c (c < NB), tau, scale, beta
  double prow[2][NB];
  double gsh[2][NB];
  double T[NB][NB + 1];
  double redW[BW][NB][NB + 1];
  double W[NB][NB + 1];
  int flag;
  int task;
  int pflag;  // next-tile prefetch of the panel CTA succeeded
};

// T(0:I, I) = -tau_I T(0:I,0:I) g_I (LAPACK dlarft), run by one warp one
// column behind the factorization; T and g are zero outside their ranges.
template <int NB>
BSOFI_DEVINL void t_column(Smem<NB>& sm, int I, int lane) {
  const int buf = I & 1;
  const double taui = sm.coef[buf][NB];
  if (lane < I) {
    double s0 = 0.0, s1 = 0.0;
#pragma unroll
    for (int b = 0; b < NB; b += 2) {
      s0 = fma(sm.T[lane][b], sm.gsh[buf][b], s0);
      s1 = fma(sm.T[lane][b + 1], sm.gsh[buf][b + 1], s1);
    }
    sm.T[lane][I] = -taui * (s0 + s1);
  }
  if (lane == I) sm.T[I][I] = taui;
  __syncwarp();
}

// Householder QR of one leaf held in registers (thread t owns rows t + BT*i).
// The column loop is a runtime loop over a rotating layout: at step I
// position 0 holds column I, positions 1..NB-1-I the columns not yet
// factored, and positions NB-I..NB-1 the finished reflectors 0..I-1; the
// array rotates left by one position after each step, so every register index
// is a compile-time constant while the loop body exists once (a fully
// unrolled column loop overflows the instruction cache).
//
// One block reduction per column carries, per position, either the dot
// product d_c = sum_{r>I} a_rI a_rc with a pending column (position 0 gives
// ||x||^2) or e_j = sum_{r>I} v_j[r] a_rI with a finished reflector, which
// builds the dlarft factor T(0:I,I) = -tau_I T(0:I,0:I) V^T v_I.
template <int R, int NB, int FW>
BSOFI_DEVINL void factor_leaf(double (&a)[R][NB], Smem<NB>& sm, int m, int w, double* tau_out) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int SH = (NB == 16) ? 1 : 2;
  constexpr int FT = FW * 32;  // threads taking part; thread t owns rows t + FT*i
  auto bar = [&]() {
    if constexpr (FW == BW) __syncthreads();
    else named_bar(FT);
  };
#pragma unroll 1
  for (int I = 0; I < w; I++) {
    const int buf = I & 1;
    const int ndone0 = NB - I;  // first position holding a finished reflector
    if (tid == I) {
#pragma unroll
      for (int p = 0; p < NB; p++) sm.prow[buf][p] = a[0][p];
    }
    double part[NB];
#pragma unroll
    for (int p = 0; p < NB; p++) part[p] = 0.0;
#pragma unroll
    for (int i = 0; i < R; i++) {
      const int r = tid + FT * i;
      const double x = (r > I) ? a[i][0] : 0.0;  // rows >= m hold zeros
#pragma unroll
      for (int p = 0; p < NB; p++) part[p] = fma(x, a[i][p], part[p]);
    }
    {
      double sum = wsum_t<NB>(part, lane);
      if ((lane & ((1 << SH) - 1)) == 0) sm.red[buf][warp][(lane >> SH) & (NB - 1)] = sum;
    }
    bar();
    if (warp == 0) {
      const int slot = lane % NB;
      double tot = 0.0;
#pragma unroll
      for (int k = lane / NB; k < FW; k += 32 / NB) tot += sm.red[buf][k][slot];
#pragma unroll
      for (int off = NB; off < 32; off <<= 1) tot += __shfl_xor_sync(0xffffffffu, tot, off);
      const double xnorm2 = __shfl_sync(0xffffffffu, tot, 0);
      const double alpha = sm.prow[buf][0];
      double beta, taui, scale;
      if (xnorm2 == 0.0) {
        taui = 0.0;
        beta = alpha;
        scale = 1.0;
      } else {
        // beta = -sign(alpha) ||(alpha, x)||, tau = (beta - alpha)/beta = 1 + |alpha|/||.||,
        // scale = 1/(alpha - beta): one reciprocal square root and one division.
        const double s2 = fma(alpha, alpha, xnorm2);
        const double rn = rsqrt(s2);
        beta = -copysign(s2 * rn, alpha);
        taui = fma(fabs(alpha), rn, 1.0);
        scale = 1.0 / (alpha - beta);
      }
      const double val = fma(scale, tot, sm.prow[buf][slot]);
      if (lane < NB) {
        // tau*w_c at pending positions 1..NB-1-I, zero elsewhere, so the row
        // update below needs no predicates.
        sm.coef[buf][slot] = (slot >= 1 && slot < ndone0) ? taui * val : 0.0;
        // g_j = v_j^T v_I for j < I, zero for j >= I.
        // lane slot writes g at index (slot - ndone0) mod NB: indices < I get
        // the reflector dot products, the others zero.
        const int j = (slot + I) & (NB - 1);
        sm.gsh[buf][j] = (slot >= ndone0) ? val : 0.0;
      }
      if (lane == 0) {
        sm.coef[buf][NB] = taui;
        sm.coef[buf][NB + 1] = scale;
        sm.coef[buf][NB + 2] = beta;
        tau_out[I] = taui;
      }
    }
    if (warp == 1 && I > 0) t_column<NB>(sm, I - 1, lane);
    bar();
    const double taui = sm.coef[buf][NB], scale = sm.coef[buf][NB + 1],
                 beta = sm.coef[buf][NB + 2];
    double cf[NB];
#pragma unroll
    for (int p = 1; p < NB; p++) cf[p] = sm.coef[buf][p];
#pragma unroll
    for (int i = 0; i < R; i++) {
      const int r = tid + FT * i;
      const double sv = a[i][0] * scale;
      const double v = (r > I) ? sv : ((r == I) ? 1.0 : 0.0);
      a[i][0] = (r > I) ? sv : ((r == I) ? beta : a[i][0]);
#pragma unroll
      for (int p = 1; p < NB; p++) a[i][p] = fma(-v, cf[p], a[i][p]);
    }
    // Rotate left: the finished column moves to the last position.
#pragma unroll
    for (int i = 0; i < R; i++) {
      const double t0 = a[i][0];
#pragma unroll
      for (int p = 0; p < NB - 1; p++) a[i][p] = a[i][p + 1];
      a[i][NB - 1] = t0;
    }
  }
  bar();
  if (warp == 1) t_column<NB>(sm, w - 1, lane);
  bar();
  // A leaf narrower than NB needs NB - w more rotations to restore column order.
#pragma unroll 1
  for (int k = w; k < NB; k++) {
#pragma unroll
    for (int i = 0; i < R; i++) {
      const double t0 = a[i][0];
#pragma unroll
      for (int p = 0; p < NB - 1; p++) a[i][p] = a[i][p + 1];
      a[i][NB - 1] = t0;
    }
  }
}

// 16-wide block reflector applied with DMMA (mma.sync m16n8k4 f64):
//   W = V^T C (16 x 16, K = rows split over the 8 warps), W <- -T^T W,
//   C <- C + V W (rows split over the warps).
// sV, sC: MP x 20 row-major tiles in shared memory (rows >= m are zero); the
// caller fills sV, this function stages C.  A stride of 20 doubles makes the
// fragment loads of both products bank-conflict free.
constexpr int MS = 20;

// Rows of one staging pass: two thread-owned row slices (R >= 2), i.e. the
// staged tiles never exceed 2 * BT rows whatever the leaf height.
template <int R>
struct Pass {
  static constexpr int SL = R >= 2 ? 2 : 1;      // row slices per pass
  static constexpr int ROWS = SL * BT;           // staged rows per pass
  static constexpr int NP = (R + SL - 1) / SL;   // passes
  // V is staged column-major with this column stride (ROWS + 4: 4 mod 16
  // doubles), so that writes of whole rows by their owning threads and both
  // DMMA fragment patterns read below are free of bank conflicts.
  static constexpr int SV = ROWS + 4;
};

// Fill the staged V rows of pass p.  From registers (the factoring CTA) when
// VREG, else from the stored reflectors in global memory.
template <int R, bool VREG>
BSOFI_DEVINL void stage_v(double* sV, const double (&a)[R][16], const double* P, long long ld,
                          int m, int w, int p) {
  constexpr int SL = Pass<R>::SL;
  const int tid = threadIdx.x;
#pragma unroll
  for (int j = 0; j < SL; j++) {
    const int i = p * SL + j;
    const int lr = tid + BT * j;          // row inside the pass
    const int r = tid + BT * i;           // row of the leaf
#pragma unroll
    for (int c = 0; c < 16; c++) {
      double v = 0.0;
      if (i < R && r < m && c < w) {
        if (r == c) v = 1.0;
        else if (r > c) v = VREG ? a[i < R ? i : 0][c] : __ldcg(P + cm(r, c, ld));
      }
      sV[c * Pass<R>::SV + lr] = v;
    }
  }
}

// Staged C of pass p: row-major with stride MS.  Each warp instruction copies
// an 8-row x 4-column block (lane = 4 * row + column), which reads four 64-byte
// column segments from global memory and writes shared memory without bank
// conflicts.  Staged row lr is row p * ROWS + lr of the tile.  NW warps take
// part; wid is this warp's index among them.
template <int R, int NW = BW>
BSOFI_DEVINL void stage_c(double* sC, const double* C, long long ld, int m, int w, int p,
                          int wid = threadIdx.x >> 5) {
  constexpr int PR = Pass<R>::ROWS, NBK = PR / 8 * 4 / NW;  // blocks per warp
  constexpr int CH = NBK > 32 ? 32 : NBK;                   // loads in flight per chunk
  const int lane = threadIdx.x & 31;
  const int rg = lane >> 2, cg = lane & 3;
#pragma unroll
  for (int q0 = 0; q0 < NBK; q0 += CH) {
    double v[CH];
#pragma unroll
    for (int q = 0; q < CH; q++) {
      const int b = wid + NW * (q0 + q);
      const int lr = (b >> 2) * 8 + rg, cc = (b & 3) * 4 + cg;
      const int r = p * PR + lr;
      v[q] = (r < m && cc < w) ? __ldcg(C + cm(r, cc, ld)) : 0.0;
    }
#pragma unroll
    for (int q = 0; q < CH; q++) {
      const int b = wid + NW * (q0 + q);
      sC[((b >> 2) * 8 + rg) * MS + (b & 3) * 4 + cg] = v[q];
    }
  }
}

// 16-wide block reflector applied with DMMA (mma.sync m16n8k8 f64), in passes
// of at most 2*BT rows staged in shared memory:
//   W = V^T C (16 x 16; K = rows, split over the 8 warps, summed over passes),
//   W <- -T^T W,  C <- C + V W  (second sweep over the passes).
// A stride of MS = 20 doubles makes the fragment loads bank-conflict free.
// wv: width of the leaf (reflector columns), w: width of the target tile.
// VPRE / CPRE: the caller already staged V / C (single pass only).
template <int R, bool VREG, bool VPRE = false, bool CPRE = false>
BSOFI_DEVINL void apply_qt_mma(double* sV, double* sC, const double (&a)[R][16],
                               const double* P, long long ldp, int wv, double* C, long long ld,
                               int m, int w, Smem<16>& sm) {
  static_assert(!VPRE || Pass<R>::NP == 1, "pre-staged V needs a single pass");
  static_assert(!CPRE || Pass<R>::NP == 1, "pre-staged C needs a single pass");
  constexpr int PR = Pass<R>::ROWS, NP = Pass<R>::NP;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  double acc[2][4] = {{0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0}};
#pragma unroll 1
  for (int p = 0; p < NP; p++) {
    if (!VPRE) stage_v<R, VREG>(sV, a, P, ldp, m, wv, p);
    if (!CPRE) stage_c<R>(sC, C, ld, m, w, p);
    __syncthreads();
    constexpr int KW = PR / BW;
    const int r0 = warp * KW;
#pragma unroll 2
    for (int k0 = r0; k0 < r0 + KW; k0 += 8) {
      constexpr int SV = Pass<R>::SV;
      const double a0 = sV[g * SV + k0 + t], a1 = sV[(g + 8) * SV + k0 + t];
      const double a2 = sV[g * SV + k0 + t + 4], a3 = sV[(g + 8) * SV + k0 + t + 4];
      dmma_16x8x8(acc[0], a0, a1, a2, a3, sC[(k0 + t) * MS + g], sC[(k0 + t + 4) * MS + g]);
      dmma_16x8x8(acc[1], a0, a1, a2, a3, sC[(k0 + t) * MS + 8 + g],
                  sC[(k0 + t + 4) * MS + 8 + g]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < 2; j++) {
    sm.redW[warp][g][8 * j + 2 * t] = acc[j][0];
    sm.redW[warp][g][8 * j + 2 * t + 1] = acc[j][1];
    sm.redW[warp][g + 8][8 * j + 2 * t] = acc[j][2];
    sm.redW[warp][g + 8][8 * j + 2 * t + 1] = acc[j][3];
  }
  __syncthreads();
  {
    const int ai = tid & 15, cc = tid >> 4;
    double s2 = 0.0;
#pragma unroll
    for (int k = 0; k < BW; k++) s2 += sm.redW[k][ai][cc];
    sm.W[ai][cc] = s2;
  }
  __syncthreads();
  {  // -(T^T W); T is zero below its diagonal
    const int ai = tid & 15, cc = tid >> 4;
    double s2 = 0.0;
#pragma unroll
    for (int b = 0; b < 16; b++) s2 = fma(sm.T[b][ai], sm.W[b][cc], s2);
    sm.redW[0][ai][cc] = -s2;
  }
  __syncthreads();
#pragma unroll 1
  for (int p = 0; p < NP; p++) {
    if (NP > 1) {  // one pass: sV and sC still hold it
      stage_v<R, VREG>(sV, a, P, ldp, m, wv, p);
      stage_c<R>(sC, C, ld, m, w, p);
      __syncthreads();
    }
    constexpr int RW = PR / BW;
#pragma unroll
    for (int m0 = warp * RW; m0 < (warp + 1) * RW; m0 += 16) {
#pragma unroll
      for (int j = 0; j < 2; j++) {
        double d[4];
        d[0] = sC[(m0 + g) * MS + 8 * j + 2 * t];
        d[1] = sC[(m0 + g) * MS + 8 * j + 2 * t + 1];
        d[2] = sC[(m0 + g + 8) * MS + 8 * j + 2 * t];
        d[3] = sC[(m0 + g + 8) * MS + 8 * j + 2 * t + 1];
        constexpr int SV = Pass<R>::SV;
#pragma unroll
        for (int k8 = 0; k8 < 16; k8 += 8)
          dmma_16x8x8(d, sV[(k8 + t) * SV + m0 + g], sV[(k8 + t) * SV + m0 + g + 8],
                      sV[(k8 + t + 4) * SV + m0 + g], sV[(k8 + t + 4) * SV + m0 + g + 8],
                      sm.redW[0][k8 + t][8 * j + g], sm.redW[0][k8 + t + 4][8 * j + g]);
        const int c0 = 8 * j + 2 * t;
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int lr = m0 + g + 8 * h;            // row inside the pass
          const int i = p * Pass<R>::SL + lr / BT;  // its thread-owned row slice
          const int rr = (lr % BT) + BT * i;        // row of the leaf
          if (i < R && rr < m) {
            if (c0 < w) __stcg(C + cm(rr, c0, ld), d[2 * h]);
            if (c0 + 1 < w) __stcg(C + cm(rr, c0 + 1, ld), d[2 * h + 1]);
          }
        }
      }
    }
    __syncthreads();
  }
}

// 8-wide block reflector with DMMA m8n8k4 (f64), all rows in one pass:
//   W = V^T C (8 x 8; K = the leaf's rows, split over the 8 warps),
//   W <- -T^T W,  C <- C + V W  (rows split over the warps).
// V and C are staged column-major with column stride S8 = R*BT + 4 (4 mod 16
// doubles): the staging writes (one row per thread) and the fragment loads of
// both products are free of bank conflicts.  VREG: V comes from the factoring
// CTA's registers (thread t owns rows t + BT*i), else from the stored leaf.
// wv: width of the leaf, w: width of the target tile.
template <int R>
struct Stage8 {
  static constexpr int S8 = R * BT + 4;
};

template <int R, bool VREG>
BSOFI_DEVINL void apply_qt_mma8(double* sV, double* sC, const double (&a)[R][8],
                                const double* P, long long ldp, int wv, double* C, long long ld,
                                int m, int w, Smem<8>& sm) {
  constexpr int S8 = Stage8<R>::S8, KW = R * BT / BW;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int i = 0; i < R; i++) {
    const int r = tid + BT * i;
#pragma unroll
    for (int c = 0; c < 8; c++) {
      double v = 0.0;
      if (r < m && c < wv) {
        if (r == c) v = 1.0;
        else if (r > c) v = VREG ? a[i][c] : __ldcg(P + cm(r, c, ldp));
      }
      sV[c * S8 + r] = v;
      sC[c * S8 + r] = (r < m && c < w) ? __ldcg(C + cm(r, c, ld)) : 0.0;
    }
  }
  __syncthreads();
  {
    // Four independent accumulators over interleaved 4-deep K steps, so the
    // DMMAs of a warp do not wait on each other's results.
    static_assert(KW % 16 == 0, "8-wide W split");
    double acc[4][2] = {};
    const int k1 = warp * KW;
#pragma unroll
    for (int k0 = k1; k0 < k1 + KW; k0 += 16)
#pragma unroll
      for (int q = 0; q < 4; q++)
        dmma_8x8x4(acc[q], sV[g * S8 + k0 + 4 * q + t], sC[g * S8 + k0 + 4 * q + t]);
    sm.redW[warp][g][2 * t] = (acc[0][0] + acc[1][0]) + (acc[2][0] + acc[3][0]);
    sm.redW[warp][g][2 * t + 1] = (acc[0][1] + acc[1][1]) + (acc[2][1] + acc[3][1]);
  }
  __syncthreads();
  if (tid < 64) {
    const int ai = tid & 7, cc = tid >> 3;
    double s2 = 0.0;
#pragma unroll
    for (int k = 0; k < BW; k++) s2 += sm.redW[k][ai][cc];
    sm.W[ai][cc] = s2;
  }
  __syncthreads();
  if (tid < 64) {  // -(T^T W); T is zero below its diagonal
    const int ai = tid & 7, cc = tid >> 3;
    double s2 = 0.0;
#pragma unroll
    for (int b = 0; b < 8; b++) s2 = fma(sm.T[b][ai], sm.W[b][cc], s2);
    sm.redW[0][ai][cc] = -s2;
  }
  __syncthreads();
#pragma unroll 4
  for (int m0 = warp * KW; m0 < (warp + 1) * KW; m0 += 8) {
    double d[2] = {sC[(2 * t) * S8 + m0 + g], sC[(2 * t + 1) * S8 + m0 + g]};
#pragma unroll
    for (int k0 = 0; k0 < 8; k0 += 4)
      dmma_8x8x4(d, sV[(k0 + t) * S8 + m0 + g], sm.redW[0][k0 + t][g]);
    const int rr = m0 + g;
    if (rr < m) {
      if (2 * t < w) __stcg(C + cm(rr, 2 * t, ld), d[0]);
      if (2 * t + 1 < w) __stcg(C + cm(rr, 2 * t + 1, ld), d[1]);
    }
  }
  __syncthreads();
}

// FW4: 16-wide leaves of at most 2 BT rows are factored by 4 warps while the
// other 4 stage the next leaf's tile (true), or by all 8 warps with the tile
// staged after the factorization (false).
template <int R, int NB, bool FW4 = true>
__global__ void __launch_bounds__(BT, 1) bsof_persistent_kernel(BsofGeom g, BsofState st) {
  __shared__ Smem<NB> sm;
  extern __shared__ __align__(16) double sC[];  // NB x (R*BT) staged tile
  const int tid = threadIdx.x;
  const long long first_task = tasks_before(g, st.s_begin);
  const long long total_tasks = tasks_before(g, st.s_end);

  if (blockIdx.x == 0) {
    // ---------------------------------------------------------- panel chain
    // 16-wide leaves of at most 2*BT rows are factored by 4 warps with 2R rows
    // per thread (the per-column shuffle reduction costs per warp); the other
    // 4 warps meanwhile wait for the next leaf's tile to be ready and stage it
    // in shared memory for the update that follows (PREFETCH).  Taller leaves
    // use all warps for the factorization.
    constexpr int FW = (FW4 && NB == 16 && R <= 2) ? 4 : BW;
    constexpr int FR = R * BW / FW;
    constexpr bool PREFETCH = NB == 16 && FW < BW && Pass<R>::NP == 1;
    const int warp = tid >> 5;
    // own: this CTA applied the last update to the current leaf's tile, so it
    // needs no wait (shared barriers order its own global writes).  A launch
    // that continues at s_begin > 0 starts owning its first tile: the earlier
    // launch, complete before this one starts, applied that tile's last
    // update from its panel CTA, which is never counted.
    bool own = st.s_begin > 0;
    for (int s = st.s_begin; s < st.s_end; s++) {
      const Leaf f = leaf_of(g, s);
      int lo, hi;
      tile_range(g, f.m, f.t, lo, hi);
      if (tid == 0) st.timeline[4 * s + 0] = gtimer();
      if (!own && !block_wait_geq(st, st.cnt + tile_id(g, f.m, f.t), hi - lo, &sm.flag)) return;
      if (tid == 0) st.timeline[4 * s + 1] = gtimer();
      const int mrows = 2 * g.n - f.j0;
      long long ldp;
      double* P = mat_ptr(g, st, (long long)f.k * g.n + f.j0, f.m, f.t * g.NB, ldp);
      // Target 0 of leaf s: the tile of leaf s+1.
      const bool next = ntargets(g, f) > 0;
      int m2 = 0, t2 = 0, lo2 = 0, hi2 = 0;
      if (next) {
        target_of(g, f, 0, m2, t2);
        tile_range(g, m2, t2, lo2, hi2);
      }
      const int x2 = tile_id(g, m2, t2);
      long long ldc = st.ld;
      double* C = next ? tile_ptr(g, st, f.k, f.j0, m2, t2, ldc) : nullptr;
      const int w2 = min(g.NB, g.n - t2 * g.NB);
      for (int e = tid; e < NB * (NB + 1); e += BT) (&sm.T[0][0])[e] = 0.0;
      if (tid < 2 * NB) (&sm.gsh[0][0])[tid] = 0.0;
      if (tid == 0) sm.pflag = 1;
      __syncthreads();
      double a[FR][NB];
      if (tid < FW * 32) {
#pragma unroll
        for (int i = 0; i < FR; i++) {
          const int r = tid + FW * 32 * i;
#pragma unroll
          for (int c = 0; c < NB; c++)
            a[i][c] = (r < mrows && c < f.w) ? __ldcg(P + cm(r, c, ldp)) : 0.0;
        }
        factor_leaf<FR, NB, FW>(a, sm, mrows, f.w, st.tau + (long long)f.k * g.n + f.j0);
#pragma unroll
        for (int i = 0; i < FR; i++) {
          const int r = tid + FW * 32 * i;
          if (r < mrows) {
#pragma unroll
            for (int c = 0; c < NB; c++)
              if (c < f.w) __stcg(P + cm(r, c, ldp), a[i][c]);
          }
          if constexpr (NB == 16 && Pass<R>::NP == 1) {  // reflectors for the next-tile update
            if (r < Pass<R>::ROWS) {
#pragma unroll
              for (int c = 0; c < 16; c++)
                sC[c * Pass<R>::SV + r] = (r >= mrows || c >= f.w) ? 0.0
                                 : (r == c ? 1.0 : (r > c ? a[i][c] : 0.0));
            }
          }
        }
      } else {
        if constexpr (PREFETCH) {
          if (next) {
            // Wait (bounded) until every update of the next tile before leaf
            // s is done, then stage it.
            constexpr int PT = BT - FW * 32;
            if (tid == FW * 32) {
              const int* flag = st.cnt + x2;
              int ok = 1;
              long long it = 0;
              while (ld_acquire(flag) < s - lo2) {
                if (ld_acquire(st.err) != 0 || ++it > st.spin_limit) {
                  atomicExch(st.err, 1);
                  ok = 0;
                  break;
                }
                __nanosleep(64);
              }
              sm.pflag = ok;
            }
            named_bar2(PT);
            if (sm.pflag)
              stage_c<R, BW - FW>(sC + Pass<R>::ROWS * MS, C, ldc, mrows, w2, 0, warp - FW);
          }
        }
      }
      __syncthreads();
      if (!sm.pflag) return;
      double* Tout = st.T + ((long long)f.k * st.maxleaves + f.l) * 256;
      for (int e = tid; e < 256; e += BT) {
        const int rr = e % 16, cc = e / 16;
        Tout[e] = (rr < NB && cc < NB && rr < f.w && cc < f.w) ? sm.T[rr][cc] : 0.0;
      }
      __syncthreads();
      // Apply leaf s to the tile of leaf s+1.  That is the tile's last update
      // and only this CTA reads the tile next, so it is not published; the
      // leaf itself (reflectors and T) is published after the update, with one
      // fence for both.
      if (next) {
        if (!PREFETCH && !block_wait_geq(st, st.cnt + x2, s - lo2, &sm.flag)) return;
        if (tid == 0) st.timeline[4 * s + 3] = gtimer();
        if constexpr (NB == 16) {
          // V is staged from the factor's registers when one pass covers the
          // leaf, else re-read from L2 (just written by this CTA).
          double none[R][16];
          apply_qt_mma<R, false, Pass<R>::NP == 1, PREFETCH>(
              sC, sC + Pass<R>::ROWS * MS, none, P, ldp, f.w, C, ldc, mrows, w2, sm);
        } else {
          apply_qt_mma8<R, true>(sC, sC + 8 * Stage8<R>::S8, a, P, ldp, f.w, C, ldc, mrows, w2,
                                 sm);
        }
      }
      if (tid == 0) {
        __threadfence();
        red_release_add(st.factored + s, 1);
        st.timeline[4 * s + 2] = gtimer();
      }
      own = next;
    }
    return;
  }

  // ------------------------------------------------------------ workers
  for (;;) {
    if (tid == 0) sm.task = first_task + atomicAdd(st.next_task, 1);
    __syncthreads();
    const long long task = sm.task;
    __syncthreads();
    if (task >= total_tasks) return;
    // Leaf of this task: largest s with tasks_before(s) <= task.
    int lo_s = 0, hi_s = g.S - 1;
    while (lo_s < hi_s) {
      const int mid = (lo_s + hi_s + 1) / 2;
      if (tasks_before(g, mid) <= task) lo_s = mid;
      else hi_s = mid - 1;
    }
    const int s = lo_s;
    const int q = 1 + (int)(task - tasks_before(g, s));
    const Leaf f = leaf_of(g, s);
    int m2, t2;
    target_of(g, f, q, m2, t2);
    int lo2, hi2;
    tile_range(g, m2, t2, lo2, hi2);
    const int x2 = tile_id(g, m2, t2);
    if (!block_wait_geq(st, st.factored + s, 1, &sm.flag)) return;
    const int mrows = 2 * g.n - f.j0;
    const double* T = st.T + ((long long)f.k * st.maxleaves + f.l) * 256;
    for (int e = tid; e < NB * NB; e += BT) sm.T[e % NB][e / NB] = __ldcg(T + (e % NB) + 16 * (e / NB));
    long long ldp, ldc;
    const double* P = mat_ptr(g, st, (long long)f.k * g.n + f.j0, f.m, f.t * g.NB, ldp);
    double* C = tile_ptr(g, st, f.k, f.j0, m2, t2, ldc);
    const int w2 = min(g.NB, g.n - t2 * g.NB);
    if constexpr (NB == 16) {
      if (!block_wait_geq(st, st.cnt + x2, s - lo2, &sm.flag)) return;
      double none[R][16];
      apply_qt_mma<R, false>(sC, sC + Pass<R>::ROWS * MS, none, P, ldp, f.w, C, ldc, mrows, w2,
                             sm);
    } else {
      if (!block_wait_geq(st, st.cnt + x2, s - lo2, &sm.flag)) return;
      double none[R][8];
      apply_qt_mma8<R, false>(sC, sC + 8 * Stage8<R>::S8, none, P, ldp, f.w, C, ldc, mrows, w2,
                              sm);
    }
    if (tid == 0) {
      __threadfence();
      red_release_add(st.cnt + x2, 1);
    }
  }
}

// ------------------------------------------------------------------ launcher
// 16-wide leaves (DMMA block-reflector update, one 512-row staging pass) up
// to 2n = 512 rows; taller panels use 8-wide leaves (up to 2n = 1536 rows,
// six rows per thread), whose CUDA-core update streams rows from registers.
// (16-wide leaves with two staging passes measured slower at n = 400.)
int bsof_leaf_width(int n) { return n <= 256 ? 16 : 8; }

int bsof_tiles(int n) { return (n + bsof_leaf_width(n) - 1) / bsof_leaf_width(n); }

template <int R, int NB>
static size_t dyn_smem() {
  return NB == 16 ? sizeof(double) * 2 * (size_t)Pass<R>::ROWS * MS
                  : sizeof(double) * 2 * 8 * (size_t)Stage8<R>::S8;
}

template <int R, int NB, bool FW4 = true>
static cudaError_t launch_R(const BsofGeom& g, const BsofState& st, int grid, cudaStream_t s) {
  void* args[] = {(void*)&g, (void*)&st};
  return cudaLaunchCooperativeKernel((const void*)bsof_persistent_kernel<R, NB, FW4>, dim3(grid),
                                     dim3(BT), args, dyn_smem<R, NB>(), s);
}

template <int R, int NB, bool FW4 = true>
static int max_grid() {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaFuncSetAttribute(bsof_persistent_kernel<R, NB, FW4>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn_smem<R, NB>());
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, bsof_persistent_kernel<R, NB, FW4>, BT,
                                                dyn_smem<R, NB>());
  return sms * (per > 0 ? per : 1);
}

// Factor warps of 16-wide leaves: 4 with the next tile staged meanwhile (the
// default), or 8; process-wide.
static std::atomic<int> g_factor8{0};
void bsof_set_factor_warps(int w) { g_factor8.store(w == 8 ? 1 : 0); }

cudaError_t launch_bsof_persistent(double* A, long long ld, int n, int L, double* tau, double* T,
                                   double* G, int maxleaves, int* cnt, int* factored,
                                   int* next_task, int* err, unsigned long long* timeline,
                                   int workers, cudaStream_t st, int s_begin, int s_end,
                                   double* Al, long long ldl) {
  BsofGeom g;
  g.form_g = G != nullptr;
  g.n = n;
  g.L = L;
  g.NB = bsof_leaf_width(n);
  g.nl = bsof_tiles(n);
  g.S = (L - 2) * g.nl + 2 * g.nl;
  BsofState s;
  s.A = A;
  s.ld = ld;
  s.Al = Al ? Al : A + cm(0, (long long)(L - 1) * n, ld);
  s.ldl = Al ? ldl : ld;
  s.G = G;
  s.tau = tau;
  s.T = T;
  s.maxleaves = maxleaves;
  s.cnt = cnt;
  s.factored = factored;
  s.next_task = next_task;
  s.err = err;
  s.timeline = timeline;
  s.spin_limit = 1ll << 22;  // polls of ~0.5 us each: a few seconds at most
  s.s_begin = s_begin > 0 ? s_begin : 0;
  s.s_end = (s_end < 0 || s_end > g.S) ? g.S : s_end;
  if (s.s_begin >= s.s_end) return cudaSuccess;
  const int R = (2 * n + BT - 1) / BT;
  int grid = 1 + workers;
  if (g.NB == 16) {
    switch (R) {
      case 1:
        if (g_factor8.load()) {
          grid = min(grid, max_grid<1, 16, false>());
          return launch_R<1, 16, false>(g, s, grid, st);
        }
        grid = min(grid, max_grid<1, 16>());
        return launch_R<1, 16>(g, s, grid, st);
      case 2:
        if (g_factor8.load()) {
          grid = min(grid, max_grid<2, 16, false>());
          return launch_R<2, 16, false>(g, s, grid, st);
        }
        grid = min(grid, max_grid<2, 16>());
        return launch_R<2, 16>(g, s, grid, st);
      default: return cudaErrorInvalidValue;
    }
  }
  switch (R) {
    case 3: grid = min(grid, max_grid<3, 8>()); return launch_R<3, 8>(g, s, grid, st);
    case 4: grid = min(grid, max_grid<4, 8>()); return launch_R<4, 8>(g, s, grid, st);
    case 5: grid = min(grid, max_grid<5, 8>()); return launch_R<5, 8>(g, s, grid, st);
    case 6: grid = min(grid, max_grid<6, 8>()); return launch_R<6, 8>(g, s, grid, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t preload_bsof(size_t* local) {
  cudaError_t e;
  if ((e = preload_one(bsof_persistent_kernel<1, 16>, local)) != cudaSuccess) return e;
  if ((e = preload_one(bsof_persistent_kernel<2, 16>, local)) != cudaSuccess) return e;
  if ((e = preload_one(bsof_persistent_kernel<1, 16, false>, local)) != cudaSuccess) return e;
  if ((e = preload_one(bsof_persistent_kernel<2, 16, false>, local)) != cudaSuccess) return e;
  if ((e = preload_one(bsof_persistent_kernel<3, 8>, local)) != cudaSuccess) return e;
  if ((e = preload_one(bsof_persistent_kernel<4, 8>, local)) != cudaSuccess) return e;
  if ((e = preload_one(bsof_persistent_kernel<5, 8>, local)) != cudaSuccess) return e;
  return preload_one(bsof_persistent_kernel<6, 8>, local);
}

}  // namespace bsofi
