// Device pipeline of BSOF/I: the order of kernels for BSOF, BSTRI and BSOI.
//
// Reference algorithm: src/bsofi_cpu.c:86-248 (lapackXbsof, lapackXbstri,
// lapackXbsoi_ormqr).  All data stays in HBM; nothing runs on the host.
//
// Workspace (one allocation, regions 256-byte aligned):
//   info   int                      first exactly-zero diagonal of R (1-based)
//   T      (L-1) x leaves x 16x16   compact-WY factors of every panel leaf
//   G      (L-1) x (2n x 2n)        explicit Q_k^T of every panel
//   W      (L-2) x (n x n)          BSTRI row multipliers  W_i = -R_ii^{-1} R_{i,i+1}
//   Y      (L-1) x (n x n)          BSTRI scratch  R_{i,L-1} R_{L-1,L-1}^{-1}
//   carry  2 x (ldd x n)            BSOI ping-pong block column
#include <climits>
#include <atomic>
#include <map>
#include <mutex>
#include <utility>
#include <vector>
#include "bsofi_device.h"
#include "bsofi_kernels.h"

using namespace bsofi;

namespace {

thread_local long long g_launches = 0;

// Optional CUDA-event timing of every BSOI step GEMM launch (the dominant
// kernel), recorded on the launching stream.
struct GemmTimer {
  bool on = false;
  std::vector<cudaEvent_t> ev;  // pairs (start, stop)
  size_t used = 0;
  cudaError_t mark(cudaStream_t st) {
    if (used == ev.size()) {
      cudaEvent_t e;
      cudaError_t r = cudaEventCreate(&e);
      if (r != cudaSuccess) return r;
      ev.push_back(e);
    }
    return cudaEventRecord(ev[used++], st);
  }
};
thread_local GemmTimer g_timer;

// Launch plan of one problem size: how BSOI runs (0 / 5: one persistent
// launch of 128x128 / 64x64 tiles; 1: one GEMM launch per step with the tile
// shape chosen by tile count; 2, 3, 4: per step with 64x64, 128x128 K32,
// 128x128 K16 tiles), the BSTRI
// row recurrence (launch_gemm's cfg per step, or 4: one persistent launch),
// the number of BSOF worker CTAs of a single inversion, and the BSTRI row
// group (0: one recurrence step per block row; 2..8: that many block rows per
// step of the blocked recurrence, one persistent launch when bstri_cfg is 4,
// else one launch per group).  Tuned plans
// (bsofi_autotune) live in a process-wide table; other sizes use the default
// below.
struct Plan {
  int bsoi, bstri_cfg, workers, bstri_group;
};
constexpr int kMaxBstriGroup = 8;
std::mutex g_plan_mu;
std::map<std::pair<int, int>, Plan> g_plans;

Plan default_plan(int n, int L) {
  // From autotuned sizes (n, p): 128 x 128 tiles pay off when 2n is a
  // multiple of 128 and a step fills the GPU (256, 32: persistent); otherwise
  // 64 x 64 tiles waste less of the 2n columns: one persistent launch for
  // mid-size N (100/64, 196/40, 324/40), per-step launches for N of 20k and
  // more (400/64, 576/80) and for small N (64/16, 144/20).  The persistent
  // recurrence helped at 64/16 and 400/64 and tied elsewhere.  The blocked
  // BSTRI recurrence, persistent with 4 rows per step, gained 2-7% for N
  // between 2048 and 20000 (256/32, 196/40, 100/64, 324/40); at 64/16 one
  // launch per group of 2 rows was best; at 400/64 no group size beat the
  // persistent one-row recurrence.
  // When 2n is a multiple of 160 (and n of 16), the persistent launch runs
  // 128 x 160 tiles loaded by TMA; its BSOI against the 64 x 64 plans: 50.5
  // against 56.0 ms at 400/64, 53.7 against 57.5 ms at 560/40 (per step),
  // 4.63 against 5.43 ms at 240/40 (persistent).
  const int N = n * L;
  const int tiles = ((N + 127) / 128) * ((2 * n + 127) / 128);
  const int tiles160 = ((N + 127) / 128) * ((2 * n) / 160);
  int bsoi;
  if ((2 * n) % 128 == 0 && tiles >= 148) bsoi = 0;
  else if ((2 * n) % 160 == 0 && n % 16 == 0 && tiles160 >= 148) bsoi = 0;
  else if (N >= 20000) bsoi = 2;
  else if (N >= 4000) bsoi = 5;
  else bsoi = 1;
  int rec, group;
  if (N <= 2048) {
    rec = 2;
    group = 2;
  } else if (N < 20000) {
    rec = 4;
    group = 4;
  } else {
    rec = N < 40000 ? 4 : 2;
    group = 0;
  }
  return Plan{bsoi, rec, 32, group};
}

// Plans of this thread's launches without persistent GEMM kernels (set by
// pipelined batches): a persistent launch keeps every SM until it ends, so
// another instance's cooperative BSOF launch could not start meanwhile.
thread_local bool g_nonpersistent = false;

Plan plan_for(int n, int L) {
  Plan p;
  {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    auto it = g_plans.find({n, L});
    p = it == g_plans.end() ? default_plan(n, L) : it->second;
  }
  if (g_nonpersistent) {
    if (p.bsoi == 0) p.bsoi = 3;  // per-step 128 x 128 (K stage 32)
    if (p.bsoi == 5) p.bsoi = 2;  // per-step 64 x 64
    if (p.bstri_cfg == 4) p.bstri_cfg = 0;  // per-step (or per-group) launches
  }
  return p;
}

// Diagnostics override of the BSOF worker count (0 = the plan's).
thread_local int g_workers_override = 0;
// Diagnostics: persistent BSOI launches of this thread wait on a word that
// nothing writes (the spare int after the BSOI tile counter), so their
// bounded waits give up.
thread_local bool g_wait_test = false;

// Worker CTAs of one BSOF launch: the caller's count, else the override, else
// the plan's.
int bsof_workers(int n, int L, int requested) {
  if (requested > 0) return requested;
  if (g_workers_override > 0) return g_workers_override;
  return plan_for(n, L).workers;
}

struct Layout {
  size_t info, sync, bsync, rsync, tl, T, G, W, Y, C0, C1, total;
  int nbw, maxleaves, tiles, leaves, sync_ints, bsync_ints, rsync_ints;
};

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

Layout layout(int n, int L, int ldd) {
  Layout l;
  l.nbw = leaf_width(n);
  l.tiles = bsof_tiles(n);
  l.leaves = (L - 2) * l.tiles + 2 * l.tiles;
  l.maxleaves = max((2 * n + l.nbw - 1) / l.nbw, 2 * l.tiles);
  l.sync_ints = (L + 2 * (L - 1)) * l.tiles + l.leaves + 2;
  size_t off = 0;
  l.info = off;  // BSTRI info, BSOF / BSOI / BSTRI wait error words
  off += 256;
  l.sync = off;  // tile counters, leaf flags, task counter, spare
  off += align256(sizeof(int) * (size_t)l.sync_ints);
  l.bsync_ints = (L - 1) * bsoi_row_bands(n * L) + 2;
  l.bsync = off;  // BSOI: finished tiles per (step, row band), tile counter
  off += align256(sizeof(int) * (size_t)l.bsync_ints);
  l.rsync_ints = (L > 2 ? (L - 2) * bstri_recurrence_ctmax(n, L) : 0) + 2;
  l.rsync = off;  // BSTRI recurrence: finished row tiles per (step, column tile), tile counter
  off += align256(sizeof(int) * (size_t)l.rsync_ints);
  l.tl = off;    // BSOF timeline: 4 globaltimer stamps per leaf
  off += align256(sizeof(unsigned long long) * 4 * (size_t)l.leaves);
  l.T = off;
  off += align256(sizeof(double) * (size_t)(L - 1) * l.maxleaves * 256);
  l.G = off;
  off += align256(sizeof(double) * (size_t)(L - 1) * 4 * n * n);
  l.W = off;
  off += align256(sizeof(double) * (size_t)(L > 2 ? L - 2 : 1) * n * n);
  l.Y = off;
  off += align256(sizeof(double) * (size_t)(L - 1) * n * n);
  l.C0 = off;
  off += align256(sizeof(double) * (size_t)ldd * n);
  l.C1 = off;
  off += align256(sizeof(double) * (size_t)ldd * n);
  l.total = off;
  return l;
}

template <class T>
T* at(void* ws, size_t off) {
  return reinterpret_cast<T*>(reinterpret_cast<char*>(ws) + off);
}

// CK: a kernel launch (counted); CKM: a memset/copy (not a kernel).
#define CK(x)                              \
  do {                                     \
    cudaError_t _e = (x);                  \
    if (_e != cudaSuccess) return (int)_e; \
    g_launches++;                          \
  } while (0)
#define CKM(x)                             \
  do {                                     \
    cudaError_t _e = (x);                  \
    if (_e != cudaSuccess) return (int)_e; \
  } while (0)

// Compact-WY factor of one panel leaf from its stored reflectors and tau
// (LAPACK dlarft, forward/columnwise): T(0:i,i) = -tau_i T(0:i,0:i) V^T v_i.
// grid (leaves, panels); rebuilt in BSOI so that the split entry points work
// from the caller's (A, tau) alone.
__global__ void __launch_bounds__(256) build_leaf_t_kernel(const double* __restrict__ A,
                                                           long long ld, int n, int L,
                                                           const double* __restrict__ tau,
                                                           double* __restrict__ Tbase,
                                                           int maxleaves, int nbw) {
  __shared__ double sV[64][17];
  __shared__ double sG[16][17];
  __shared__ double sT[16][17];
  const int l = blockIdx.x, k = blockIdx.y, tid = threadIdx.x;
  const int ncp = (k < L - 2) ? n : 2 * n;
  const int j0 = l * nbw;
  double* Tout = Tbase + ((size_t)k * maxleaves + l) * 256;
  if (j0 >= ncp) return;
  const int nc = min(nbw, ncp - j0), m = 2 * n - j0;
  const double* V = A + cm((long long)k * n + j0, (long long)k * n + j0, ld);
  const double* tl = tau + (size_t)k * n + j0;
  const int ga = tid % 16, gb = tid / 16;
  double acc = 0.0;
  for (int r0 = 0; r0 < m; r0 += 64) {
    __syncthreads();
    for (int e = tid; e < 64 * 16; e += 256) {
      int rr = e % 64, aa = e / 64, r = r0 + rr;
      double v = 0.0;
      if (r < m && aa < nc) v = (r == aa) ? 1.0 : (r > aa ? V[cm(r, aa, ld)] : 0.0);
      sV[rr][aa] = v;
    }
    __syncthreads();
#pragma unroll 8
    for (int rr = 0; rr < 64; rr++) acc = fma(sV[rr][ga], sV[rr][gb], acc);
  }
  sG[ga][gb] = acc;
  sT[ga][gb] = 0.0;
  __syncthreads();
  if (tid < 32) {
    for (int i = 0; i < nc; i++) {
      double ti = tl[i];
      double s = 0.0;
      if (tid < i)
        for (int b = tid; b < i; b++) s = fma(sT[tid][b], sG[b][i], s);
      __syncwarp();
      if (tid < i) sT[tid][i] = -ti * s;
      if (tid == i) sT[i][i] = ti;
      __syncwarp();
    }
  }
  __syncthreads();
  Tout[tid] = sT[tid % 16][tid / 16];
}

// BSOF.  form_q: the persistent kernel also forms G_k = Q_k^T for BSOI.
// workers: worker CTAs for 16-wide leaves (four times as many for 8-wide).
// Al, ldl (optional): the last block column in its own array (the compact
// layout of the storage-sharded inversion); the workspace regions used here
// lie before the carries, so their offsets do not depend on ldd.
int run_bsof(int n, int L, double* dA, int ldd, double* dtau, void* ws, cudaStream_t st,
             bool form_q, int base_workers, double* Al = nullptr, long long ldl = 0) {
  Layout ly = layout(n, L, ldd);
  double* Tb = at<double>(ws, ly.T);
  double* G = at<double>(ws, ly.G);
  int* sync = at<int>(ws, ly.sync);
  const int ntiles = (L + 2 * (L - 1)) * ly.tiles;
  CKM(cudaMemsetAsync(sync, 0, sizeof(int) * ly.sync_ints, st));
  CKM(cudaMemsetAsync(at<int>(ws, ly.info) + 1, 0, sizeof(int), st));
  if (form_q) CK(launch_set_identity(G, 2 * n, 2 * n, 4ll * n * n, L - 1, st));
  // 16-wide leaves apply with DMMA and need few workers; 8-wide leaves
  // (n > 256) have three times the tasks per leaf and use every SM.
  int workers = bsof_leaf_width(n) == 16 ? base_workers : 4 * base_workers;
  if (form_q) workers *= 2;
  CK(launch_bsof_persistent(dA, ldd, n, L, dtau, Tb, form_q ? G : nullptr, ly.maxleaves, sync,
                            sync + ntiles, sync + ntiles + ly.leaves, at<int>(ws, ly.info) + 1,
                            at<unsigned long long>(ws, ly.tl), workers, st, 0, -1, Al, ldl));
  return 0;
}

// Blocked BSTRI row recurrence.  The block rows i = L-3 .. 0 are taken in
// groups of grp from the bottom; group g holds rows t..b (b = L-3-g grp).
// Inside a group, X_{r,c} = W_r W_{r+1} ... W_b X_{b+1,c} for every column c
// beyond b, so with the stacked products P_r = W_r P_{r+1} (P_b = W_b) one
// GEMM of (b-t+1) n rows computes the whole group from row b+1:
//   X_{t:b, b+1:L} = [P_t; ...; P_b] X_{b+1, b+1:L}  (+ Zc on block column L-1),
// where Zc_r = Z_r + W_r Zc_{r+1} (Zc_b = Z_b) carries the Z terms.  The
// columns inside the group, X_{r, r+1:b} = W_r X_{r+1, r+1:b}, and P and Zc
// need only the group's own W_i, Z_i and X_ii, so every group forms them at
// once, in grp - 1 batched rounds, before the ceil((L-2)/grp) group steps run
// in order.  Same per-block products as the one-row recurrence, grouped
// differently; the serial chain is grp times shorter and every step grp times
// taller.  P (grp n x n per group, leading dimension grp n; a short top group
// uses the bottom rows of its block) lives in the BSOI carry buffers, which
// are idle until BSOI.
struct RowGroups {
  int n, L, grp, ngr, mlast, b0;
  long long nn, pld, pbs;
  RowGroups(int n_, int L_, int grp_) : n(n_), L(L_), grp(grp_) {
    b0 = L - 3;
    ngr = (L - 2 + grp - 1) / grp;
    mlast = (L - 2) - (ngr - 1) * grp;
    nn = (long long)n * n;
    pld = (long long)grp * n;
    pbs = pld * n;
  }
  int b(int g) const { return b0 - g * grp; }
  int m(int g) const { return b(g) + 1 < grp ? b(g) + 1 : grp; }
  int t(int g) const { return b(g) - m(g) + 1; }
};

GemmA plain_a(const double* p, long long ld, long long bs) {
  GemmA a = {};
  a.p0 = p;
  a.ld0 = ld;
  a.bs0 = bs;
  a.ld1 = 2;
  a.rlim0 = INT_MAX;
  a.roff0 = kNoMask;
  a.rlim1 = INT_MAX;
  a.roff1 = kNoMask;
  return a;
}

// P_b = W_b at the bottom of the blocks of groups [g0, g1).
int groups_seed(const RowGroups& G, const double* W, double* P, int g0, int g1, cudaStream_t st) {
  for (int g = g0; g < g1; g++)
    CKM(cudaMemcpy2DAsync(P + g * G.pbs + (long long)(G.grp - 1) * G.n, sizeof(double) * G.pld,
                          W + (long long)G.b(g) * G.nn, sizeof(double) * G.n,
                          sizeof(double) * G.n, G.n, cudaMemcpyDeviceToDevice, st));
  return 0;
}

enum { kRoundP = 1, kRoundIntra = 2, kRoundZc = 4 };

// The in-group rounds of groups [g0, g1): round q forms, for row r = b_g - q
// of every group that has it, P_r (kRoundP), X_{r, r+1:r+q} (kRoundIntra) and
// Zc_r in place in block column L-1 (kRoundZc), batched over the groups.
int groups_rounds(const RowGroups& G, double* dA, int ldd, const double* W, double* P, int g0,
                  int g1, int what, cudaStream_t st) {
  const int n = G.n, grp = G.grp, L = G.L;
  const long long rstep = -(long long)grp * n;             // row offset from one group to the next
  const long long dstep = rstep + rstep * (long long)ldd;  // the same along the diagonal
  for (int q = 1; q < grp; q++) {
    // Only the top group (ngr - 1) can be short.
    const int batch = (g1 - g0) - ((g1 == G.ngr && G.mlast <= q) ? 1 : 0);
    if (batch <= 0) break;
    const int r = G.b(g0) - q;  // in group g0
    GemmDims d1 = {n, n, n};
    GemmA a = plain_a(W + (long long)r * G.nn, n, -(long long)grp * G.nn);
    a.ksplit = n;
    if (what & kRoundP) {  // P_r = W_r P_{r+1}
      GemmB b = {P + g0 * G.pbs + (long long)(grp - q) * n, G.pld, G.pbs, kNoMask};
      GemmC c = {};
      c.p0 = P + g0 * G.pbs + (long long)(grp - 1 - q) * n;
      c.ld0 = G.pld;
      c.bs0 = G.pbs;
      c.ld1 = 1;
      c.nsplit = n;
      c.alpha = 1.0;
      CK(launch_gemm(d1, a, b, c, batch, 2, st));
    }
    if (what & kRoundIntra) {  // X_{r, r+1:r+q} = W_r X_{r+1, r+1:r+q}; X_{r+1,r+1} is upper triangular
      GemmDims dq = {n, q * n, n};
      GemmB b = {dA + cm((long long)(r + 1) * n, (long long)(r + 1) * n, ldd), ldd, dstep, 0};
      GemmC c = {};
      c.p0 = dA + cm((long long)r * n, (long long)(r + 1) * n, ldd);
      c.ld0 = ldd;
      c.bs0 = dstep;
      c.ld1 = 1;
      c.nsplit = q * n;
      c.alpha = 1.0;
      CK(launch_gemm(dq, a, b, c, batch, 2, st));
    }
    if (what & kRoundZc) {  // Zc_r = Z_r + W_r Zc_{r+1}, in place in block column L-1
      GemmB b = {dA + cm((long long)(r + 1) * n, (long long)(L - 1) * n, ldd), ldd, rstep, kNoMask};
      GemmC c = {};
      c.p0 = dA + cm((long long)r * n, (long long)(L - 1) * n, ldd);
      c.ld0 = ldd;
      c.bs0 = rstep;
      c.ld1 = 1;
      c.nsplit = n;
      c.alpha = 1.0;
      c.beta0 = 1.0;
      CK(launch_gemm(d1, a, b, c, batch, 2, st));
    }
  }
  return 0;
}

// Group steps g0 .. g1-1 in order, one launch each, over block columns
// [max(b+1, cfrom), cto); cto = L includes block column L-1 with its Zc.
int groups_steps(const RowGroups& G, double* dA, int ldd, const double* P, int g0, int g1,
                 int cfrom, int cto, int cfg, cudaStream_t st) {
  const int n = G.n, L = G.L;
  for (int g = g0; g < g1; g++) {
    const int b = G.b(g), m = G.m(g), t = G.t(g);
    const int cs = b + 1 > cfrom ? b + 1 : cfrom;
    if (cto <= cs) continue;
    const int ncol = (cto - cs) * n;
    GemmDims d = {m * n, ncol, n};
    GemmA a = plain_a(P + g * G.pbs + (long long)(G.grp - m) * n, G.pld, 0);
    a.ksplit = n;
    GemmB bb = {dA + cm((long long)(b + 1) * n, (long long)cs * n, ldd), ldd, 0,
                cs == b + 1 ? 0 : kNoMask};
    GemmC c = {};
    c.p0 = dA + cm((long long)t * n, (long long)cs * n, ldd);
    c.ld0 = ldd;
    c.alpha = 1.0;
    c.beta0 = 0.0;
    if (cto == L) {
      c.p1 = dA + cm((long long)t * n, (long long)(L - 1) * n, ldd);
      c.ld1 = ldd;
      c.nsplit = ncol - n;
      c.beta1 = 1.0;
    } else {
      c.ld1 = 1;
      c.nsplit = ncol;
    }
    CK(launch_gemm(d, a, bb, c, 1, cfg, st));
  }
  return 0;
}

int bstri_blocked(int n, int L, double* dA, int ldd, const double* W, double* P, int grp,
                  bool persistent, int* rsync, int rsync_ints, int* err, cudaStream_t st) {
  const RowGroups G(n, L, grp);
  if (int e = groups_seed(G, W, P, 0, G.ngr, st)) return e;
  if (int e = groups_rounds(G, dA, ldd, W, P, 0, G.ngr, kRoundP | kRoundIntra | kRoundZc, st))
    return e;
  if (persistent) {
    // All group steps in one launch, column tiles pipelined across the steps.
    CKM(cudaMemsetAsync(rsync, 0, sizeof(int) * rsync_ints, st));
    CK(launch_bstri_recurrence_blocked(dA, ldd, P, G.pld, G.pbs, grp, n, L, rsync,
                                       rsync + rsync_ints - 2, err, st));
    return 0;
  }
  return groups_steps(G, dA, ldd, P, 0, G.ngr, 0, L, 0, st);
}

// X_ii = R_ii^{-1} for the diagonal blocks [i0, i1) (tmp: the recursive
// inversion's scratch, n^2/4 doubles per block).
int diag_inverse(int n, double* dA, int ldd, int* info, double* tmp, int i0, int i1,
                 cudaStream_t st) {
  if (i1 <= i0) return 0;
  const long long diag = (long long)n * (ldd + 1);
  CK(launch_trtri_blocks(dA + i0 * diag, ldd, n, diag, i1 - i0, info, tmp, st, i0));
  return 0;
}

// W_i = -X_ii R_{i,i+1} for i in [i0, i1).
int w_products(int n, double* dA, int ldd, double* W, int i0, int i1, cudaStream_t st) {
  if (i1 <= i0) return 0;
  const long long nn = (long long)n * n, diag = (long long)n * (ldd + 1);
  GemmDims d = {n, n, n};
  GemmA a = plain_a(dA + i0 * diag, ldd, diag);
  a.ksplit = n;
  a.roff0 = 0;
  GemmB b = {dA + i0 * diag + cm(0, n, ldd), ldd, diag, kNoMask};
  GemmC c = {};
  c.p0 = W + i0 * nn;
  c.ld0 = n;
  c.bs0 = nn;
  c.ld1 = 1;
  c.nsplit = n;
  c.alpha = -1.0;
  CK(launch_gemm(d, a, b, c, i1 - i0, 0, st));
  return 0;
}

// Y_i = R_{i,L-1} X_{L-1,L-1} and Z_i = -X_ii Y_i -> A(i, L-1), i = 0..L-2.
// The last block column is at Al (leading dimension ldl): A's block column
// L-1, or its own array in the compact layout.
int yz_products(int n, int L, double* dA, int ldd, double* Al, long long ldl, double* Y,
                cudaStream_t st) {
  const long long nn = (long long)n * n, diag = (long long)n * (ldd + 1);
  GemmDims d = {n, n, n};
  {
    GemmA a = plain_a(Al, ldl, n);
    a.ksplit = n;
    GemmB b = {Al + cm((long long)(L - 1) * n, 0, ldl), ldl, 0, 0};
    GemmC c = {};
    c.p0 = Y;
    c.ld0 = n;
    c.bs0 = nn;
    c.ld1 = 1;
    c.nsplit = n;
    c.alpha = 1.0;
    CK(launch_gemm(d, a, b, c, L - 1, 0, st));
  }
  {
    GemmA a = plain_a(dA, ldd, diag);
    a.ksplit = n;
    a.roff0 = 0;
    GemmB b = {Y, n, nn, kNoMask};
    GemmC c = {};
    c.p0 = Al;
    c.ld0 = ldl;
    c.bs0 = n;
    c.ld1 = 1;
    c.nsplit = n;
    c.alpha = -1.0;
    CK(launch_gemm(d, a, b, c, L - 1, 0, st));
  }
  return 0;
}

int run_bstri(int n, int L, double* dA, int ldd, void* ws, cudaStream_t st) {
  Layout ly = layout(n, L, ldd);
  int* info = at<int>(ws, ly.info);
  double* W = at<double>(ws, ly.W);
  double* Y = at<double>(ws, ly.Y);
  const long long nn = (long long)n * n;
  CKM(cudaMemsetAsync(info, 0x7f, sizeof(int), st));
  // X_ii = R_ii^{-1} for every diagonal block (Y, not yet used, is the
  // scratch of the recursive inversion).
  if (int e = diag_inverse(n, dA, ldd, info, Y, 0, L, st)) return e;
  double* last = dA + cm(0, (long long)(L - 1) * n, ldd);
  if (int e = yz_products(n, L, dA, ldd, last, ldd, Y, st)) return e;
  if (int e = w_products(n, dA, ldd, W, 0, L - 2, st)) return e;
  // Row recurrence: X_{i, i+1:L} = W_i X_{i+1, i+1:L} (+ Z_i on the last block).
  const Plan plan = plan_for(n, L);
  const int rec = plan.bstri_cfg;
  CKM(cudaMemsetAsync(info + 3, 0, sizeof(int), st));
  // At most L-2 rows per group: the stacked P then takes at most (2L-5) n^2
  // doubles, inside the two carry buffers (2 ldd n >= 2 L n^2).
  const int grp = plan.bstri_group < L - 2 ? plan.bstri_group : L - 2;
  if (grp >= 2)
    return bstri_blocked(n, L, dA, ldd, W, at<double>(ws, ly.C0), grp, rec == 4,
                         at<int>(ws, ly.rsync), ly.rsync_ints, info + 3, st);
  if (rec == 4) {
    // One persistent launch, column tiles pipelined across the steps.
    if (L >= 3) {
      int* rs = at<int>(ws, ly.rsync);
      CKM(cudaMemsetAsync(rs, 0, sizeof(int) * ly.rsync_ints, st));
      CK(launch_bstri_recurrence(dA, ldd, W, n, L, rs, rs + ly.rsync_ints - 2, info + 3, st));
    }
    return 0;
  }
  for (int i = L - 3; i >= 0; i--) {
    const int ncol = (L - 1 - i) * n;
    GemmDims dr = {n, ncol, n};
    GemmA a = plain_a(W + (size_t)i * nn, n, 0);
    a.ksplit = n;
    GemmB b = {dA + cm((long long)(i + 1) * n, (long long)(i + 1) * n, ldd), ldd, 0, 0};
    GemmC c = {};
    c.p0 = dA + cm((long long)i * n, (long long)(i + 1) * n, ldd);
    c.ld0 = ldd;
    c.p1 = dA + cm((long long)i * n, (long long)(L - 1) * n, ldd);
    c.ld1 = ldd;
    c.nsplit = ncol - n;
    c.alpha = 1.0;
    c.beta0 = 0.0;
    c.beta1 = 1.0;
    CK(launch_gemm(dr, a, b, c, 1, rec, st));
  }
  return 0;
}

// BSOF + BSTRI with BSTRI's leading rows overlapped with the end of the
// factorization.  Block row i of R (R_ii, R_{i,i+1}, R_{i,L-1}) is final once
// panel i is factored, and the leading block of X = R^{-1} above row h, the
// columns left of h, depends only on R's rows above h.  So the factorization
// runs as two launches split at panel h; after the first, a low-priority side
// stream inverts the diagonal blocks above h, forms their W_i, the row-group
// products P and in-group columns of the groups above h, and those groups'
// steps over the columns left of h, on the SMs the factorization leaves idle,
// while the second launch (on a high-priority side stream, so its
// cooperative CTAs are placed first) factors the remaining panels.  The two
// touch disjoint data: the second launch reads and writes rows from h n down.
// Once both are done the rest of BSTRI runs: the remaining diagonal blocks,
// Y and Z, the other groups' rounds, every group's Zc, and one persistent
// launch of all group steps over the columns from h on.  Every product is the
// one the unsplit path computes, so the results are the same.  Used for
// 16-wide leaves (n <= 256: the factorization occupies under half the SMs)
// with the persistent blocked recurrence; h is the top row of the fourth of
// the row groups nearest the bottom (at least two groups).
struct SideStreams {
  cudaStream_t hi = nullptr, lo = nullptr;
  cudaEvent_t e1 = nullptr, e2 = nullptr, e3 = nullptr;
};
thread_local std::map<int, SideStreams> g_side;
std::atomic<int> g_overlap_enabled{1};

// This thread's side streams on the current device, created on first use
// (never while `st` is being captured into a graph: then nullptr and the
// unsplit path runs).
SideStreams* side_streams(cudaStream_t st) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  auto it = g_side.find(dev);
  if (it != g_side.end()) return &it->second;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
    cudaGetLastError();
    return nullptr;
  }
  SideStreams x;
  int least = 0, greatest = 0;
  bool ok = cudaDeviceGetStreamPriorityRange(&least, &greatest) == cudaSuccess &&
            cudaStreamCreateWithPriority(&x.hi, cudaStreamNonBlocking, greatest) == cudaSuccess &&
            cudaStreamCreateWithPriority(&x.lo, cudaStreamNonBlocking, least) == cudaSuccess &&
            cudaEventCreateWithFlags(&x.e1, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&x.e2, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&x.e3, cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    if (x.hi) cudaStreamDestroy(x.hi);
    if (x.lo) cudaStreamDestroy(x.lo);
    if (x.e1) cudaEventDestroy(x.e1);
    if (x.e2) cudaEventDestroy(x.e2);
    cudaGetLastError();
    return nullptr;
  }
  return &(g_side[dev] = x);
}

// Row groups and split row h of the overlapped path, or false when it does
// not apply to (n, L).
bool overlap_split(int n, int L, int* grp_out, int* tailg_out, int* h_out) {
  if (!g_overlap_enabled.load() || bsof_leaf_width(n) != 16 || L < 4) return false;
  const Plan plan = plan_for(n, L);
  const int grp = plan.bstri_group < L - 2 ? plan.bstri_group : L - 2;
  if (plan.bstri_cfg != 4 || grp < 2) return false;
  const int ngr = (L - 2 + grp - 1) / grp;
  const int tailg = (ngr + 3) / 4 > 2 ? (ngr + 3) / 4 : 2;
  if (ngr <= tailg) return false;
  *grp_out = grp;
  *tailg_out = tailg;
  *h_out = L - 2 - tailg * grp;
  return true;
}

int run_bsoftri_overlap(int n, int L, double* dA, int ldd, double* dtau, void* ws, cudaStream_t st,
                        bool form_q, int base_workers, int grp, int tailg, int h,
                        SideStreams* ss) {
  Layout ly = layout(n, L, ldd);
  const RowGroups G(n, L, grp);
  int* info = at<int>(ws, ly.info);
  double* W = at<double>(ws, ly.W);
  double* Y = at<double>(ws, ly.Y);
  double* P = at<double>(ws, ly.C0);
  double* Tb = at<double>(ws, ly.T);
  double* Gq = at<double>(ws, ly.G);
  int* sync = at<int>(ws, ly.sync);
  const int ntiles = (L + 2 * (L - 1)) * ly.tiles;
  int* next_task = sync + ntiles + ly.leaves;
  // Counters and info words before either side stream starts.
  CKM(cudaMemsetAsync(sync, 0, sizeof(int) * ly.sync_ints, st));
  CKM(cudaMemsetAsync(info + 1, 0, sizeof(int), st));
  CKM(cudaMemsetAsync(info, 0x7f, sizeof(int), st));
  CKM(cudaMemsetAsync(info + 3, 0, sizeof(int), st));
  if (form_q) CK(launch_set_identity(Gq, 2 * n, 2 * n, 4ll * n * n, L - 1, st));
  int workers = base_workers;
  if (form_q) workers *= 2;
  const int sh = h * ly.tiles;  // first leaf of panel h
  CK(launch_bsof_persistent(dA, ldd, n, L, dtau, Tb, form_q ? Gq : nullptr, ly.maxleaves, sync,
                            sync + ntiles, next_task, info + 1, at<unsigned long long>(ws, ly.tl),
                            workers, st, 0, sh));
  CKM(cudaEventRecord(ss->e1, st));
  // From here on both side streams are always joined back into st, so that
  // nothing of this call is still queued on them when it returns, error or not.
  int err = 0;
  // Panels h .. L-2.
  err = (int)cudaStreamWaitEvent(ss->hi, ss->e1, 0);
  if (!err) err = (int)cudaMemsetAsync(next_task, 0, sizeof(int), ss->hi);
  if (!err) {
    err = (int)launch_bsof_persistent(dA, ldd, n, L, dtau, Tb, form_q ? Gq : nullptr, ly.maxleaves,
                                      sync, sync + ntiles, next_task, info + 1,
                                      at<unsigned long long>(ws, ly.tl), workers, ss->hi, sh, -1);
    if (!err) g_launches++;
  }
  // BSTRI of the rows above h (W_{h-1} uses R_{h-1,h}, final after panel h-1).
  if (!err) err = (int)cudaStreamWaitEvent(ss->lo, ss->e1, 0);
  if (!err) err = diag_inverse(n, dA, ldd, info, Y, 0, h, ss->lo);
  if (!err) err = w_products(n, dA, ldd, W, 0, h, ss->lo);
  if (!err) err = groups_seed(G, W, P, tailg, G.ngr, ss->lo);
  if (!err) err = groups_rounds(G, dA, ldd, W, P, tailg, G.ngr, kRoundP | kRoundIntra, ss->lo);
  if (!err) err = groups_steps(G, dA, ldd, P, tailg + 1, G.ngr, 0, h, 3, ss->lo);
  // Join (the events are recorded even after an error).
  const int j1 = (int)cudaEventRecord(ss->e3, ss->hi);
  const int j2 = (int)cudaEventRecord(ss->e2, ss->lo);
  const int j3 = j1 ? j1 : (int)cudaStreamWaitEvent(st, ss->e3, 0);
  const int j4 = j2 ? j2 : (int)cudaStreamWaitEvent(st, ss->e2, 0);
  if (err) return err;
  if (j3) return j3;
  if (j4) return j4;
  // The rest of BSTRI.
  if (int e = diag_inverse(n, dA, ldd, info, Y, h, L, st)) return e;
  double* last = dA + cm(0, (long long)(L - 1) * n, ldd);
  if (int e = yz_products(n, L, dA, ldd, last, ldd, Y, st)) return e;
  if (int e = w_products(n, dA, ldd, W, h, L - 2, st)) return e;
  if (int e = groups_seed(G, W, P, 0, tailg, st)) return e;
  if (int e = groups_rounds(G, dA, ldd, W, P, 0, tailg, kRoundP | kRoundIntra, st)) return e;
  if (int e = groups_rounds(G, dA, ldd, W, P, 0, G.ngr, kRoundZc, st)) return e;
  int* rs = at<int>(ws, ly.rsync);
  CKM(cudaMemsetAsync(rs, 0, sizeof(int) * ly.rsync_ints, st));
  CK(launch_bstri_recurrence_blocked(dA, ldd, P, G.pld, G.pbs, grp, n, L, rs,
                                     rs + ly.rsync_ints - 2, info + 3, st, h));
  return 0;
}

// BSOF + BSTRI of one inversion: overlapped where it applies, else in order.
int run_bsoftri(int n, int L, double* dA, int ldd, double* dtau, void* ws, cudaStream_t st,
                bool form_q, int base_workers, bool allow_overlap) {
  int grp = 0, tailg = 0, h = 0;
  if (allow_overlap && overlap_split(n, L, &grp, &tailg, &h)) {
    SideStreams* ss = side_streams(st);
    if (ss)
      return run_bsoftri_overlap(n, L, dA, ldd, dtau, ws, st, form_q, base_workers, grp, tailg,
                                 h, ss);
  }
  int e = run_bsof(n, L, dA, ldd, dtau, ws, st, form_q, base_workers);
  if (e) return e;
  return run_bstri(n, L, dA, ldd, ws, st);
}

// G_k = Q_k^T of every panel from the stored reflectors and tau: compact-WY
// factors first, then the block reflectors applied to identity matrices.
int bsoi_form_q(int n, int L, double* dA, int ldd, const double* dtau, void* ws, cudaStream_t st) {
  Layout ly = layout(n, L, ldd);
  double* Tb = at<double>(ws, ly.T);
  double* G = at<double>(ws, ly.G);
  const int n2 = 2 * n;
  const long long g2 = (long long)n2 * n2;
  build_leaf_t_kernel<<<dim3(ly.maxleaves, L - 1), 256, 0, st>>>(dA, ldd, n, L, dtau, Tb,
                                                                  ly.maxleaves, ly.nbw);
  CK(cudaGetLastError());
  CK(launch_set_identity(G, n2, n2, g2, L - 1, st));
  for (int l = 0, j0 = 0; j0 < n2; l++, j0 += ly.nbw) {
    // Regular panels k = 0..L-3 have n reflectors, the last one 2n.
    for (int part = 0; part < 2; part++) {
      const int k0 = (part == 0) ? 0 : L - 2;
      const int batch = (part == 0) ? L - 2 : 1;
      const int ncp = (part == 0) ? n : n2;
      if (batch <= 0 || j0 >= ncp) continue;
      WyArgs a = {};
      a.V = dA + cm((long long)k0 * n + j0, (long long)k0 * n + j0, ldd);
      a.ldv = ldd;
      a.vbs = (long long)n * (ldd + 1);
      a.T = Tb + ((size_t)k0 * ly.maxleaves + l) * 256;
      a.tbs = (long long)ly.maxleaves * 256;
      a.m = n2 - j0;
      a.nb = min(ly.nbw, ncp - j0);
      a.trans = 1;
      a.seg[0] = {G + (size_t)k0 * g2 + j0, n2, g2, n2};
      CK(launch_wy_apply(a, batch, st));
    }
  }
  return 0;
}

// Carry for the first BSOI step: X(:, L-1) with the triangular diagonal
// block; also clears the BSOI error word.
int bsoi_carry(int n, int L, double* dA, int ldd, void* ws, cudaStream_t st) {
  Layout ly = layout(n, L, ldd);
  const int N = n * L;
  CK(launch_copy_masked(at<double>(ws, ly.C0), ldd, dA + cm(0, (long long)(L - 1) * n, ldd), ldd,
                        N, n, (L - 1) * n, st));
  CKM(cudaMemsetAsync(at<int>(ws, ly.info) + 2, 0, sizeof(int), st));
  return 0;
}

// BSOI step k as one GEMM launch: [X(:,k) | carry] Q_k^T -> [carry' | X(:,k+1)]
// (cfg: launch_gemm's tile shape, 0 = by tile count).
int bsoi_step(int n, int L, int k, double* dA, int ldd, void* ws, cudaStream_t st, int cfg = 0) {
  Layout ly = layout(n, L, ldd);
  double* G = at<double>(ws, ly.G);
  double* C[2] = {at<double>(ws, ly.C0), at<double>(ws, ly.C1)};
  const int N = n * L, n2 = 2 * n;
  const long long g2 = (long long)n2 * n2;
  const int rd = (L - 2 - k) & 1;
  GemmDims d = {N, n2, n2};
  GemmA a = {};
  a.p0 = dA + cm(0, (long long)k * n, ldd);
  a.ld0 = ldd;
  a.p1 = C[rd];
  a.ld1 = ldd;
  a.ksplit = n;
  a.rlim0 = (k + 1) * n;
  a.roff0 = k * n;
  a.rlim1 = INT_MAX;
  a.roff1 = kNoMask;
  GemmB b = {G + (size_t)k * g2, n2, 0, kNoMask};
  GemmC c = {};
  c.p0 = C[rd ^ 1];
  c.ld0 = ldd;
  c.p1 = dA + cm(0, (long long)(k + 1) * n, ldd);
  c.ld1 = ldd;
  c.nsplit = n;
  c.alpha = 1.0;
  if (g_timer.on) CKM(g_timer.mark(st));
  CK(launch_gemm(d, a, b, c, 1, cfg, st));
  if (g_timer.on) CKM(g_timer.mark(st));
  return 0;
}

// X(:, 0) from the last carry; the info word absorbs the wait error words.
int bsoi_finish(int n, int L, double* dA, int ldd, void* ws, cudaStream_t st) {
  Layout ly = layout(n, L, ldd);
  double* C[2] = {at<double>(ws, ly.C0), at<double>(ws, ly.C1)};
  const int cur = (L - 1) & 1;  // carry buffer written by step 0
  CK(launch_copy_masked(dA, ldd, C[cur], ldd, n * L, n, kNoMask, st, at<int>(ws, ly.info)));
  return 0;
}

// BSOI of the rows [row0, row1) only (every column): the share of one GPU
// when an inversion's BSOI is split by rows.  Q formation is repeated in
// full; the carry seed, the persistent launch and the final copy cover only
// those rows.  Each computed tile is the one the full launch of the same tile
// shape computes.  row0 a multiple of 128, row1 too unless it is N.
int run_bsoi_rows(int n, int L, double* dA, int ldd, const double* dtau, void* ws, cudaStream_t st,
                  int row0, int row1) {
  Layout ly = layout(n, L, ldd);
  const int N = n * L;
  if (row0 < 0 || row1 > N || row0 >= row1 || row0 % 128 != 0 || (row1 % 128 != 0 && row1 != N))
    return (int)cudaErrorInvalidValue;
  double* G = at<double>(ws, ly.G);
  double* C[2] = {at<double>(ws, ly.C0), at<double>(ws, ly.C1)};
  if (int e = bsoi_form_q(n, L, dA, ldd, dtau, ws, st)) return e;
  const int rows = row1 - row0;
  CK(launch_copy_masked(C[0] + row0, ldd, dA + cm(row0, (long long)(L - 1) * n, ldd), ldd, rows, n,
                        (L - 1) * n - row0, st));
  CKM(cudaMemsetAsync(at<int>(ws, ly.info) + 2, 0, sizeof(int), st));
  // Persistent with the plan's tile shape when it has one, else 64 x 64.
  const Plan plan = plan_for(n, L);
  int* bs = at<int>(ws, ly.bsync);
  CKM(cudaMemsetAsync(bs, 0, sizeof(int) * ly.bsync_ints, st));
  CK(launch_bsoi_persistent(dA, ldd, C[0], C[1], ldd, G, n, L, bs, bs + ly.bsync_ints - 2,
                            at<int>(ws, ly.info) + 2, plan.bsoi != 0, st, row0, row1));
  const int cur = (L - 1) & 1;  // carry buffer written by step 0
  CK(launch_copy_masked(dA + row0, ldd, C[cur] + row0, ldd, rows, n, kNoMask, st,
                        at<int>(ws, ly.info)));
  return 0;
}

// BSOI with every step's product on the int8 tensor cores (Ozaki scheme with
// S slices; kernels_ozaki.cu): the same steps, operands and output segments
// as bsoi_step, the zero structure applied while the operand is sliced.
// oz: the product's scratch (ozaki_scratch_bytes(N, 2n, 2n, S)), reused by
// every step (the steps run in order on `st`).
int run_bsoi_mixed(int n, int L, double* dA, int ldd, void* ws, void* oz, int S, cudaStream_t st) {
  Layout ly = layout(n, L, ldd);
  double* G = at<double>(ws, ly.G);
  double* C[2] = {at<double>(ws, ly.C0), at<double>(ws, ly.C1)};
  const int N = n * L, n2 = 2 * n;
  const long long g2 = (long long)n2 * n2;
  int e = bsoi_carry(n, L, dA, ldd, ws, st);
  if (e) return e;
  for (int k = L - 2; k >= 0; k--) {
    const int rd = (L - 2 - k) & 1;
    OzProduct p = {};
    p.a0 = dA + cm(0, (long long)k * n, ldd);
    p.lda0 = ldd;
    p.a1 = C[rd];
    p.lda1 = ldd;
    p.ksplit = n;
    p.rlim0 = (k + 1) * n;
    p.roff0 = k * n;
    p.M = N;
    p.K = n2;
    p.b = G + (size_t)k * g2;
    p.ldb = n2;
    p.N = n2;
    p.c0 = C[rd ^ 1];
    p.ldc0 = ldd;
    p.c1 = dA + cm(0, (long long)(k + 1) * n, ldd);
    p.ldc1 = ldd;
    p.nsplit = n;
    p.S = S;
    p.scratch = oz;
    p.err = at<int>(ws, ly.info) + 2;
    if (g_timer.on) CKM(g_timer.mark(st));
    CKM(launch_ozaki_product(p, st));
    g_launches += 3;  // the row maxima, the split and the product
    if (g_timer.on) CKM(g_timer.mark(st));
  }
  return bsoi_finish(n, L, dA, ldd, ws, st);
}

int run_bsoi(int n, int L, double* dA, int ldd, const double* dtau, void* ws, cudaStream_t st,
             bool q_ready) {
  Layout ly = layout(n, L, ldd);
  double* G = at<double>(ws, ly.G);
  double* C[2] = {at<double>(ws, ly.C0), at<double>(ws, ly.C1)};
  // G_k = Q_k^T unless the factorization already formed it.
  if (!q_ready) {
    int e = bsoi_form_q(n, L, dA, ldd, dtau, ws, st);
    if (e) return e;
  }
  int e = bsoi_carry(n, L, dA, ldd, ws, st);
  if (e) return e;
  const Plan plan = plan_for(n, L);
  if (plan.bsoi == 0 || plan.bsoi == 5) {
    // One persistent launch over all steps (rows flow from step to step).
    int* bs = at<int>(ws, ly.bsync);
    CKM(cudaMemsetAsync(bs, 0, sizeof(int) * ly.bsync_ints, st));
    if (g_timer.on) CKM(g_timer.mark(st));
    CK(launch_bsoi_persistent(dA, ldd, C[0], C[1], ldd, G, n, L, bs, bs + ly.bsync_ints - 2,
                              at<int>(ws, ly.info) + 2, plan.bsoi == 5, st, 0, -1,
                              g_wait_test ? bs + ly.bsync_ints - 1 : nullptr));
    if (g_timer.on) CKM(g_timer.mark(st));
  } else {
    // One launch per step (small problems: more, smaller tiles per step).
    static const int cfg_of[5] = {0, 0, 2, 3, 1};
    const int cfg = cfg_of[plan.bsoi >= 1 && plan.bsoi <= 4 ? plan.bsoi : 1];
    for (int k = L - 2; k >= 0; k--)
      if ((e = bsoi_step(n, L, k, dA, ldd, ws, st, cfg)) != 0) return e;
  }
  return bsoi_finish(n, L, dA, ldd, ws, st);
}

// ------------------------------------------------------ storage-sharded
// One inversion over several GPUs with no GPU holding M or M^{-1} whole.
// The factorization's state is O(L n^2): R has three nonzero blocks per block
// row (diagonal, superdiagonal, last column) and the reflectors fill the
// panels, so every rank factors the whole matrix in a compact layout:
//   band  block columns 0..L-2 with leading dimension 3n: BSOF and BSTRI's
//         diagonal and row-multiplier products touch only block rows m-1..m+1
//         of block column m, and with ld = 3n those windows of consecutive
//         columns never overlap (column j's window starts 3n elements after
//         column j-1's, and n further at a block boundary);
//   last  the last block column, N x n (R_{i,L-1} and then Z_i for every i);
//   tau   N doubles;
// plus the workspace regions of the fused pipeline (G_k = Q_k^T, W_i, Y_i,
// the BSOI carries).  BSTRI's block columns are then independent given W_i
// and Z_i (X_{i,c} = W_i X_{i+1,c} (+ Z_i for c = L-1)), and BSOI's rows are
// independent (X(rows, k:k+1) Q_k^T), so a rank computes the block columns it
// owns, the ranks exchange them for row bands, and each finishes its rows.
struct ShardLayout {
  size_t ws, band, last, tau, total;
  size_t band_doubles;
};

ShardLayout shard_layout(int n, int L) {
  const size_t N = (size_t)n * L;
  ShardLayout s;
  s.ws = 0;
  // Carries for a row band of up to N rows with an even leading dimension.
  size_t off = layout(n, L, (int)N + 1).total;
  s.band_doubles = 3 * (size_t)n * (size_t)(L - 1) * n + N;
  s.band = off;
  off += align256(sizeof(double) * s.band_doubles);
  s.last = off;
  off += align256(sizeof(double) * N * n);
  s.tau = off;
  off += align256(sizeof(double) * N);
  s.total = off;
  return s;
}

// Compact input, BSOF with every Q_k^T formed, the diagonal inverses
// X_ii = R_ii^{-1}, Z_i (into last) and W_i: everything BSTRI's column
// recurrence and BSOI read.
int shard_factor(int n, int L, const double* dD, const double* dS, const double* dExpK,
                 const double* dh, double lambda, void* state, cudaStream_t st) {
  const ShardLayout sl = shard_layout(n, L);
  const int N = n * L;
  Layout ly = layout(n, L, N + 1);
  double* band = at<double>(state, sl.band);
  double* last = at<double>(state, sl.last);
  double* tau = at<double>(state, sl.tau);
  int* info = at<int>(state, ly.info);
  double* W = at<double>(state, ly.W);
  double* Y = at<double>(state, ly.Y);
  const int ldb = 3 * n;
  if (int e = bsofi_dev_assemble_compact(n, L, dD, dS, dExpK, dh, lambda, band, sl.band_doubles,
                                         last, st))
    return e;
  g_launches++;
  if (int e = run_bsof(n, L, band, ldb, tau, state, st, true, bsof_workers(n, L, 0), last, N))
    return e;
  CKM(cudaMemsetAsync(info, 0x7f, sizeof(int), st));
  CKM(cudaMemsetAsync(info + 3, 0, sizeof(int), st));
  if (int e = diag_inverse(n, band, ldb, info, Y, 0, L - 1, st)) return e;
  CK(launch_trtri_blocks(last + cm((long long)(L - 1) * n, 0, N), N, n, 0, 1, info, Y, st,
                         L - 1));
  if (int e = yz_products(n, L, band, ldb, last, N, Y, st)) return e;
  return w_products(n, band, ldb, W, 0, L - 2, st);
}

// Block columns [c0, c1) of X = R^{-1}, rows 0..c1 n - 1 (X is block upper
// triangular), into X (leading dimension ldx >= c1 n), from the state of
// shard_factor: the diagonal blocks and Z_i copied in, then for
// i = min(c1-2, L-3) .. 0 one GEMM X_{i, c} = W_i X_{i+1, c} (+ Z_i for
// c = L-1) over the owned columns c > i.
int shard_bstri_columns(int n, int L, int c0, int c1, double* X, long long ldx, void* state,
                        cudaStream_t st) {
  const ShardLayout sl = shard_layout(n, L);
  const int N = n * L;
  Layout ly = layout(n, L, N + 1);
  const double* band = at<double>(state, sl.band);
  const double* last = at<double>(state, sl.last);
  const double* W = at<double>(state, ly.W);
  const long long nn = (long long)n * n, ldb = 3ll * n;
  const bool has_last = c1 == L;
  CKM(cudaMemset2DAsync(X, sizeof(double) * ldx, 0, sizeof(double) * (size_t)c1 * n,
                        (size_t)(c1 - c0) * n, st));
  for (int c = c0; c < c1 && c < L - 1; c++)
    CK(launch_copy_masked(X + cm((long long)c * n, (long long)(c - c0) * n, ldx), ldx,
                          band + cm((long long)c * n, (long long)c * n, ldb), ldb, n, n, 0, st));
  if (has_last)
    CK(launch_copy_masked(X + cm(0, (long long)(L - 1 - c0) * n, ldx), ldx, last, N, N, n,
                          (L - 1) * n, st));
  for (int i = min(c1 - 2, L - 3); i >= 0; i--) {
    const int cs = max(i + 1, c0);
    if (cs >= c1) continue;
    const int ncol = (c1 - cs) * n;
    GemmDims d = {n, ncol, n};
    GemmA a = plain_a(W + (size_t)i * nn, n, 0);
    a.ksplit = n;
    GemmB b = {X + cm((long long)(i + 1) * n, (long long)(cs - c0) * n, ldx), ldx, 0, kNoMask};
    GemmC c = {};
    c.p0 = X + cm((long long)i * n, (long long)(cs - c0) * n, ldx);
    c.ld0 = ldx;
    c.alpha = 1.0;
    c.beta0 = 0.0;
    if (has_last) {
      c.p1 = X + cm((long long)i * n, (long long)(L - 1 - c0) * n, ldx);
      c.ld1 = ldx;
      c.nsplit = ncol - n;
      c.beta1 = 1.0;
    } else {
      c.p1 = c.p0;
      c.ld1 = ldx;
      c.nsplit = ncol;
    }
    CK(launch_gemm(d, a, b, c, 1, 0, st));
  }
  return 0;
}

// Rows [r0, r1) of M^{-1} from the same rows of X in every column, in place
// in B (leading dimension ldb >= r1 - r0): BSOI's persistent launch over
// that row range, with B and the carries addressed by global row (shifted
// base pointers; every access stays inside [r0, r1)).
int shard_bsoi_rows(int n, int L, int r0, int r1, double* B, long long ldb, void* state,
                    cudaStream_t st) {
  const int N = n * L;
  Layout ly = layout(n, L, N + 1);
  const int rows = r1 - r0;
  const long long ldc = (rows + 1) & ~1;
  double* Bs = B - r0;
  double* C[2] = {at<double>(state, ly.C0) - r0, at<double>(state, ly.C1) - r0};
  const double* G = at<double>(state, ly.G);
  int* info = at<int>(state, ly.info);
  CK(launch_copy_masked(C[0] + r0, ldc, Bs + cm(r0, (long long)(L - 1) * n, ldb), ldb, rows, n,
                        (L - 1) * n - r0, st));
  CKM(cudaMemsetAsync(info + 2, 0, sizeof(int), st));
  const Plan plan = plan_for(n, L);
  int* bs = at<int>(state, ly.bsync);
  CKM(cudaMemsetAsync(bs, 0, sizeof(int) * ly.bsync_ints, st));
  CK(launch_bsoi_persistent(Bs, ldb, C[0], C[1], ldc, G, n, L, bs, bs + ly.bsync_ints - 2,
                            info + 2, plan.bsoi != 0, st, r0, r1));
  const int cur = (L - 1) & 1;  // carry buffer written by step 0
  CK(launch_copy_masked(B, ldb, C[cur] + r0, ldc, rows, n, kNoMask, st, info));
  return 0;
}

}  // namespace

extern "C" {

size_t bsofi_dev_ws_bytes(int n, int L, int ldd) { return layout(n, L, ldd).total; }

size_t bsofi_dev_ws_bytes_mixed(int n, int L, int ldd, int slices) {
  return layout(n, L, ldd).total + ozaki_scratch_bytes(n * L, 2 * n, 2 * n, slices);
}

int bsofi_dev_invert_mixed(int n, int L, double* dA, int ldd, double* dtau, void* dws,
                           void* stream, int workers, int slices) {
  g_launches = 0;
  if (slices < kOzakiMinSlices || slices > kOzakiMaxSlices || 2 * n > kOzakiMaxK)
    return (int)cudaErrorInvalidValue;
  int e = run_bsoftri(n, L, dA, ldd, dtau, dws, (cudaStream_t)stream, true,
                      bsof_workers(n, L, workers), workers == 0);
  if (e) return e;
  void* oz = at<char>(dws, layout(n, L, ldd).total);
  return run_bsoi_mixed(n, L, dA, ldd, dws, oz, slices, (cudaStream_t)stream);
}

int bsofi_dev_invert_gated(int n, int L, double* dA, int ldd, double* dtau, void* dws,
                           void* stream, int workers, int slices, void* wait_ev, void* done_ev) {
  g_launches = 0;
  const cudaStream_t st = (cudaStream_t)stream;
  if (slices != 0 &&
      (slices < kOzakiMinSlices || slices > kOzakiMaxSlices || 2 * n > kOzakiMaxK))
    return (int)cudaErrorInvalidValue;
  if (wait_ev) CKM(cudaStreamWaitEvent(st, (cudaEvent_t)wait_ev, 0));
  int e = run_bsof(n, L, dA, ldd, dtau, dws, st, true, bsof_workers(n, L, workers));
  if (e) return e;
  if (done_ev) CKM(cudaEventRecord((cudaEvent_t)done_ev, st));
  if ((e = run_bstri(n, L, dA, ldd, dws, st)) != 0) return e;
  if (slices != 0)
    return run_bsoi_mixed(n, L, dA, ldd, dws, at<char>(dws, layout(n, L, ldd).total), slices, st);
  return run_bsoi(n, L, dA, ldd, dtau, dws, st, true);
}

int bsofi_dev_invert_two_streams(int n, int L, double* dA, int ldd, double* dtau, void* dws,
                                 void* chain_stream, void* gemm_stream, void* handoff,
                                 int workers, int slices) {
  g_launches = 0;
  const cudaStream_t hs = (cudaStream_t)chain_stream, gs = (cudaStream_t)gemm_stream;
  if (slices != 0 &&
      (slices < kOzakiMinSlices || slices > kOzakiMaxSlices || 2 * n > kOzakiMaxK))
    return (int)cudaErrorInvalidValue;
  int e = run_bsof(n, L, dA, ldd, dtau, dws, hs, true, bsof_workers(n, L, workers));
  if (e) return e;
  CKM(cudaEventRecord((cudaEvent_t)handoff, hs));
  CKM(cudaStreamWaitEvent(gs, (cudaEvent_t)handoff, 0));
  if ((e = run_bstri(n, L, dA, ldd, dws, gs)) != 0) return e;
  if (slices != 0)
    return run_bsoi_mixed(n, L, dA, ldd, dws, at<char>(dws, layout(n, L, ldd).total), slices, gs);
  return run_bsoi(n, L, dA, ldd, dtau, dws, gs, true);
}

void bsofi_dev_set_nonpersistent(int on) { g_nonpersistent = on != 0; }

void bsofi_dev_set_gemm_k16(int on) { gemm_set_k16(on); }

void bsofi_dev_set_bsoi_tma(int on) { bsoi_set_tma(on); }

int bsofi_dev_bsoftri_q_ex(int n, int L, double* dA, int ldd, double* dtau, void* dws,
                           void* stream, int workers) {
  g_launches = 0;
  return run_bsoftri(n, L, dA, ldd, dtau, dws, (cudaStream_t)stream, true,
                     bsof_workers(n, L, workers), false);
}

int bsofi_dev_bsoi_group_prepare(int n, int L, double* dA, int ldd, void* dws, void* stream) {
  const Layout ly = layout(n, L, ldd);
  int e = bsoi_carry(n, L, dA, ldd, dws, (cudaStream_t)stream);
  if (e) return e;
  CKM(cudaMemsetAsync(at<int>(dws, ly.bsync), 0, sizeof(int) * ly.bsync_ints,
                      (cudaStream_t)stream));
  return 0;
}

int bsofi_dev_bsoi_group_finish(int n, int L, double* dA, int ldd, void* dws, void* stream) {
  return bsoi_finish(n, L, dA, ldd, dws, (cudaStream_t)stream);
}

// Tile counters of the grouped launches: at most two tile shapes, each in
// chunks of kBsoiGroupMax instances.
static int group_launches_max(int count) { return 2 * ((count + kBsoiGroupMax - 1) / kBsoiGroupMax); }

size_t bsofi_dev_bsoi_group_bytes(int count) {
  return align256(sizeof(unsigned long long) * (size_t)group_launches_max(count));
}

int bsofi_dev_bsoi_group_run(int count, const int* n, const int* L, double* const* dA,
                             const int* ldd, void* const* dws, void* gws, void* stream_small,
                             void* stream_large) {
  // Instances with 2n a multiple of 128 run on 128 x 128 tiles, the others on
  // 64 x 64 tiles (the persistent single-instance plans choose the same way);
  // each tile shape on its own stream, kBsoiGroupMax instances per launch, the
  // descriptors in the launch's parameters (so the launches need no host
  // staging and can be captured into a graph).
  static thread_local BsoiGroup grp[2];
  g_launches = 0;
  unsigned long long* counters = static_cast<unsigned long long*>(gws);
  cudaStream_t sts[2] = {(cudaStream_t)stream_small, (cudaStream_t)stream_large};
  int used = 0;
  for (int g = 0; g < 2; g++) {
    BsoiGroup& G = grp[g];
    G.count = 0;
    G.total = 0;
    bool al = true;
    for (int i = 0; i <= count; i++) {
      if (i == count || G.count == kBsoiGroupMax) {
        if (G.count > 0) {  // launch the chunk gathered so far
          if (used >= group_launches_max(count)) return (int)cudaErrorInvalidValue;
          G.next = counters + used++;
          G.spin_limit = 1ll << 22;
          CKM(cudaMemsetAsync(G.next, 0, sizeof(unsigned long long), sts[g]));
          CK(launch_bsoi_grouped(G, g == 0, al, sts[g]));
        }
        G.count = 0;
        G.total = 0;
        al = true;
        if (i == count) break;
      }
      if (((2 * n[i]) % 128 == 0 ? 1 : 0) != g) continue;
      const Layout ly = layout(n[i], L[i], ldd[i]);
      BsoiInst& I = G.inst[G.count++];
      I.A = dA[i];
      I.ld = ldd[i];
      I.carry[0] = at<double>(dws[i], ly.C0);
      I.carry[1] = at<double>(dws[i], ly.C1);
      I.ldc = ldd[i];
      I.G = at<double>(dws[i], ly.G);
      I.n = n[i];
      I.L = L[i];
      I.N = n[i] * L[i];
      I.done = at<int>(dws[i], ly.bsync);
      I.err = at<int>(dws[i], ly.info) + 2;
      I.tile0 = G.total;
      G.total += bsoi_group_tiles(n[i], L[i], g == 0);
      al = al && ((uintptr_t)I.A % 16 == 0) && ((uintptr_t)I.carry[0] % 16 == 0) &&
           ((uintptr_t)I.carry[1] % 16 == 0) && ((uintptr_t)I.G % 16 == 0) && I.ld % 2 == 0 &&
           I.n % 2 == 0;
    }
  }
  return 0;
}

size_t bsofi_dev_ozaki_scratch_bytes(int M, int N, int K, int slices) {
  return ozaki_scratch_bytes(M, N, K, slices);
}

int bsofi_dev_selftest_ozaki(int M, int N, int K, const double* dA, int lda, const double* dB,
                             int ldb, double* dC, int ldc, int slices, void* scratch, int* derr,
                             void* stream) {
  OzProduct p = {};
  p.a0 = dA;
  p.lda0 = lda;
  p.a1 = dA;
  p.lda1 = lda;
  p.ksplit = K;
  p.rlim0 = INT_MAX;
  p.roff0 = kNoMask;
  p.M = M;
  p.K = K;
  p.b = dB;
  p.ldb = ldb;
  p.N = N;
  p.c0 = dC;
  p.ldc0 = ldc;
  p.c1 = dC;
  p.ldc1 = ldc;
  p.nsplit = N;
  p.S = slices;
  p.scratch = scratch;
  p.err = derr;
  g_launches = 3;
  return (int)launch_ozaki_product(p, (cudaStream_t)stream);
}

int bsofi_dev_prepare(void) { return (int)gemm_init_attributes(); }

int bsofi_dev_preload(void) {
  size_t local = 0;
  cudaError_t e;
  if ((e = gemm_init_attributes()) != cudaSuccess) return (int)e;
  if ((e = preload_bsof(&local)) != cudaSuccess) return (int)e;
  if ((e = preload_bsoi(&local)) != cudaSuccess) return (int)e;
  if ((e = preload_bstri(&local)) != cudaSuccess) return (int)e;
  if ((e = preload_gemm(&local)) != cudaSuccess) return (int)e;
  if ((e = preload_panel(&local)) != cudaSuccess) return (int)e;
  if ((e = preload_tri(&local)) != cudaSuccess) return (int)e;
  if ((e = preload_ozaki(&local)) != cudaSuccess) return (int)e;
  if ((e = preload_one(build_leaf_t_kernel, &local)) != cudaSuccess) return (int)e;
  // The context's local-memory reservation grows at the launch of a kernel
  // that needs more than it holds; growing it here keeps later launches from
  // allocating.
  size_t stack = 0;
  if ((e = cudaDeviceGetLimit(&stack, cudaLimitStackSize)) != cudaSuccess) return (int)e;
  if (local > stack && (e = cudaDeviceSetLimit(cudaLimitStackSize, local)) != cudaSuccess)
    return (int)e;
  return 0;
}

int bsofi_dev_zero_structural(int n, int L, double* dA, int ldd, void* stream) {
  g_launches = 0;
  CK(launch_zero_structural(dA, ldd, n, L, (cudaStream_t)stream));
  return 0;
}

int bsofi_dev_bsof(int n, int L, double* dA, int ldd, double* dtau, void* dws, void* stream) {
  g_launches = 0;
  return run_bsof(n, L, dA, ldd, dtau, dws, (cudaStream_t)stream, false, bsof_workers(n, L, 0));
}

int bsofi_dev_bstri(int n, int L, double* dA, int ldd, void* dws, void* stream) {
  g_launches = 0;
  return run_bstri(n, L, dA, ldd, dws, (cudaStream_t)stream);
}

int bsofi_dev_bsoftri(int n, int L, double* dA, int ldd, double* dtau, void* dws,
                      void* stream) {
  g_launches = 0;
  int e = run_bsof(n, L, dA, ldd, dtau, dws, (cudaStream_t)stream, false, bsof_workers(n, L, 0));
  if (e) return e;
  return run_bstri(n, L, dA, ldd, dws, (cudaStream_t)stream);
}

int bsofi_dev_bsoi(int n, int L, double* dA, int ldd, const double* dtau, void* dws,
                   void* stream) {
  g_launches = 0;
  return run_bsoi(n, L, dA, ldd, dtau, dws, (cudaStream_t)stream, false);
}

int bsofi_dev_bsoftri_q(int n, int L, double* dA, int ldd, double* dtau, void* dws,
                        void* stream) {
  g_launches = 0;
  return run_bsoftri(n, L, dA, ldd, dtau, dws, (cudaStream_t)stream, true, bsof_workers(n, L, 0),
                     true);
}

int bsofi_dev_bsoi_rows(int n, int L, double* dA, int ldd, const double* dtau, void* dws,
                        void* stream, int row0, int row1) {
  g_launches = 0;
  return run_bsoi_rows(n, L, dA, ldd, dtau, dws, (cudaStream_t)stream, row0, row1);
}

int bsofi_dev_bsoi_ex(int n, int L, double* dA, int ldd, const double* dtau, void* dws,
                      void* stream, int q_ready) {
  g_launches = 0;
  return run_bsoi(n, L, dA, ldd, dtau, dws, (cudaStream_t)stream, q_ready != 0);
}

size_t bsofi_dev_state_ref_doubles(int n, int L) {
  return 2ull * n * n * L + (size_t)n * L;
}

int bsofi_dev_state_ref(int n, int L, const double* dA, int ldd, const double* dtau, double* ref,
                        int mode, int* dflag, void* stream) {
  CK(launch_state_ref(dA, ldd, n, L, dtau, ref, mode, dflag, (cudaStream_t)stream));
  return 0;
}

int bsofi_dev_bsoi_form_q(int n, int L, double* dA, int ldd, const double* dtau, void* dws,
                          void* stream) {
  return bsoi_form_q(n, L, dA, ldd, dtau, dws, (cudaStream_t)stream);
}

int bsofi_dev_bsoi_carry(int n, int L, double* dA, int ldd, void* dws, void* stream) {
  return bsoi_carry(n, L, dA, ldd, dws, (cudaStream_t)stream);
}

int bsofi_dev_bsoi_step(int n, int L, int k, double* dA, int ldd, void* dws, void* stream) {
  return bsoi_step(n, L, k, dA, ldd, dws, (cudaStream_t)stream);
}

int bsofi_dev_bsoi_finish(int n, int L, double* dA, int ldd, void* dws, void* stream) {
  return bsoi_finish(n, L, dA, ldd, dws, (cudaStream_t)stream);
}

size_t bsofi_dev_shard_state_bytes(int n, int L) { return shard_layout(n, L).total; }

int bsofi_dev_shard_factor(int n, int L, const double* dD, const double* dS,
                           const double* dExpK, const double* dh, double lambda, void* dstate,
                           void* stream) {
  g_launches = 0;
  return shard_factor(n, L, dD, dS, dExpK, dh, lambda, dstate, (cudaStream_t)stream);
}

int bsofi_dev_shard_bstri_columns(int n, int L, int c0, int c1, double* dX, long long ldx,
                                  void* dstate, void* stream) {
  g_launches = 0;
  return shard_bstri_columns(n, L, c0, c1, dX, ldx, dstate, (cudaStream_t)stream);
}

int bsofi_dev_shard_bsoi_rows(int n, int L, int r0, int r1, double* dB, long long ldb,
                              void* dstate, void* stream) {
  g_launches = 0;
  return shard_bsoi_rows(n, L, r0, r1, dB, ldb, dstate, (cudaStream_t)stream);
}

int bsofi_dev_shard_logdet(int n, int L, const void* dstate, double* dout, void* stream) {
  const ShardLayout sl = shard_layout(n, L);
  void* s = const_cast<void*>(dstate);
  // After shard_factor the diagonal blocks hold R_ii^{-1}.
  return bsofi_dev_logdet_compact(n, L, at<double>(s, sl.band), at<double>(s, sl.last),
                                  at<double>(s, sl.tau), 1, dout, stream);
}

const double* bsofi_dev_shard_tau(const void* dstate, int n, int L) {
  return at<double>(const_cast<void*>(dstate), shard_layout(n, L).tau);
}

int bsofi_dev_invert(int n, int L, double* dA, int ldd, double* dtau, void* dws, void* stream) {
  return bsofi_dev_invert_ex(n, L, dA, ldd, dtau, dws, stream, 0);
}

int bsofi_dev_invert_ex(int n, int L, double* dA, int ldd, double* dtau, void* dws, void* stream,
                        int workers) {
  g_launches = 0;
  // The overlapped BSTRI uses this thread's side streams: only for a single
  // inversion (workers == 0), not for the pooled ones of batches and servers.
  int e = run_bsoftri(n, L, dA, ldd, dtau, dws, (cudaStream_t)stream, true,
                      bsof_workers(n, L, workers), workers == 0);
  if (!e) e = run_bsoi(n, L, dA, ldd, dtau, dws, (cudaStream_t)stream, true);
  return e;
}

int* bsofi_dev_info_ptr(void* dws) { return at<int>(dws, 0); }

int bsofi_dev_bsof_timeline(int n, int L, int ldd, void* dws, unsigned long long** ptr) {
  Layout ly = layout(n, L, ldd);
  *ptr = at<unsigned long long>(dws, ly.tl);
  return ly.leaves;
}

void bsofi_dev_set_bsof_workers(int w) { g_workers_override = w > 0 ? w : 0; }

void bsofi_dev_set_bsof_factor_warps(int w) { bsof_set_factor_warps(w); }

void bsofi_dev_set_wait_test(int on) { g_wait_test = on != 0; }

void bsofi_dev_set_bstri_overlap(int on) { g_overlap_enabled.store(on ? 1 : 0); }

int bsofi_dev_plan_get(int n, int L, int* plan) {
  std::lock_guard<std::mutex> lk(g_plan_mu);
  auto it = g_plans.find({n, L});
  const Plan p = it == g_plans.end() ? default_plan(n, L) : it->second;
  plan[0] = p.bsoi;
  plan[1] = p.bstri_cfg;
  plan[2] = p.workers;
  plan[3] = p.bstri_group;
  return it == g_plans.end() ? 0 : 1;
}

int bsofi_dev_plan_set(int n, int L, const int* plan) {
  if (n < 1 || L < 2 || plan[0] < 0 || plan[0] > 5 || plan[1] < 0 || plan[1] > 4 ||
      plan[2] < 1 || plan[2] > 1024 || plan[3] < 0 || plan[3] == 1 || plan[3] > kMaxBstriGroup)
    return -1;
  std::lock_guard<std::mutex> lk(g_plan_mu);
  g_plans[{n, L}] = Plan{plan[0], plan[1], plan[2], plan[3]};
  return 0;
}

void bsofi_dev_plan_clear(void) {
  std::lock_guard<std::mutex> lk(g_plan_mu);
  g_plans.clear();
}

void bsofi_dev_plan_clear_one(int n, int L) {
  std::lock_guard<std::mutex> lk(g_plan_mu);
  g_plans.erase({n, L});
}

int bsofi_dev_selftest_gemm(int M, int N, int K, double alpha, const double* dA, int lda,
                            int upper_a, const double* dB, int ldb, int upper_b, double beta,
                            double* dC, int ldc, int tile, void* stream) {
  GemmDims d = {M, N, K};
  GemmA a = {};
  a.p0 = dA;
  a.ld0 = lda;
  a.ld1 = 2;
  a.ksplit = K;
  a.rlim0 = INT_MAX;
  a.roff0 = upper_a ? 0 : kNoMask;
  a.rlim1 = INT_MAX;
  a.roff1 = kNoMask;
  GemmB b = {dB, ldb, 0, upper_b ? 0 : kNoMask};
  GemmC c = {};
  c.p0 = dC;
  c.ld0 = ldc;
  c.ld1 = 1;
  c.nsplit = N;
  c.alpha = alpha;
  c.beta0 = beta;
  g_launches = 0;
  CK(launch_gemm(d, a, b, c, 1, tile, (cudaStream_t)stream));
  return 0;
}

long long bsofi_dev_launch_count(void) { return g_launches; }

void bsofi_dev_add_launches(long long c) { g_launches += c; }

void bsofi_dev_timing(int on) {
  g_timer.on = on != 0;
  g_timer.used = 0;
}

int bsofi_dev_timing_read(double* ms, long long* launches) {
  double tot = 0.0;
  for (size_t i = 0; i + 1 < g_timer.used; i += 2) {
    float t = 0.f;
    cudaError_t e = cudaEventSynchronize(g_timer.ev[i + 1]);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, g_timer.ev[i], g_timer.ev[i + 1]);
    if (e != cudaSuccess) return (int)e;
    tot += t;
  }
  *ms = tot;
  *launches = (long long)(g_timer.used / 2);
  g_timer.used = 0;
  return 0;
}

}  // extern "C"
