// Internal C++ interface between the device pipeline and the kernel files.
#pragma once
#include <cuda_runtime.h>
#include "gemm.cuh"

namespace bsofi {

// Kernel attributes (cudaFuncSetAttribute) apply to the current device only:
// set-up that is done once is done once per device.  Devices beyond the table
// redo it every time (harmless: the call is idempotent).
constexpr int kMaxDevices = 64;
struct PerDevice {
  bool done[kMaxDevices] = {};
  // Device index whose set-up is still to do, or -1 if it is done.
  int pending() const {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (dev < 0 || dev >= kMaxDevices) return dev;
    return done[dev] ? -1 : dev;
  }
  void mark(int dev) {
    if (dev >= 0 && dev < kMaxDevices) done[dev] = true;
  }
};

struct WySeg {
  double* p;
  long long ld, bs;
  int ncols;
};

struct WyArgs {
  const double* V;  // leaf top-left (unit lower trapezoidal reflectors)
  long long ldv, vbs;
  const double* T;  // 16 x 16 compact-WY factor (ld 16)
  long long tbs;
  int m, nb, trans;
  WySeg seg[3];
};

int leaf_width(int n);
cudaError_t launch_wy_apply(const WyArgs& a, int batch, cudaStream_t st);

// Persistent BSOF (kernels_bsof.cu).  cnt: (L + 2(L-1))*tiles ints,
// factored: leaves ints, next_task and err: one int each, all zeroed before
// the launch.  G (optional): (L-1) x (2n)^2 identity matrices that become
// Q_k^T.  [s_begin, s_end): the leaves this launch factors (-1: to the end);
// a later launch continues with the counters the earlier one left, after
// next_task is zeroed again.  Al, ldl (optional): the last block column in
// its own array (rows 0..N-1), with block columns 0..L-2 at A; without them
// it is A's block column L-1.
int bsof_leaf_width(int n);
void bsof_set_factor_warps(int w);
// TMA loading of the persistent BSOI's clean 128 x 128 tiles; process-wide.
void bsoi_set_tma(int on);
int bsof_tiles(int n);
cudaError_t launch_bsof_persistent(double* A, long long ld, int n, int L, double* tau, double* T,
                                   double* G, int maxleaves, int* cnt, int* factored,
                                   int* next_task, int* err, unsigned long long* timeline,
                                   int workers, cudaStream_t st, int s_begin = 0,
                                   int s_end = -1, double* Al = nullptr, long long ldl = 0);

// Persistent BSTRI row recurrence (kernels_bstri.cu): done is (L-2) x
// bstri_recurrence_ctmax(n, L) ints and next one int, zeroed before.
int bstri_recurrence_ctmax(int n, int L);
cudaError_t launch_bstri_recurrence(double* A, long long ld, const double* W, int n, int L,
                                    int* done, int* next, int* err, cudaStream_t st);
// The blocked form: grp rows per step, step g's left operand the stacked
// products at P + g pstep (leading dimension pld), 128x128 tiles; block
// columns left of hfloor are not computed (already final).
cudaError_t launch_bstri_recurrence_blocked(double* A, long long ld, const double* P,
                                            long long pld, long long pstep, int grp, int n, int L,
                                            int* done, int* next, int* err, cudaStream_t st,
                                            int hfloor = 0);

// Persistent BSOI (kernels_bsoi.cu): all p-1 steps in one launch.
// done: (L-1) * bsoi_row_bands(N) ints and next: one int, zeroed before;
// small: 64 x 64 tiles instead of 128 x 128.  never (diagnostics): a zeroed
// word that nothing writes; when given, every step wait polls it under a short
// limit, so the waits give up and report through err.
int bsoi_row_bands(int N);
// [row0, row1): the rows computed (row1 = -1: to N); row0 a multiple of the
// tile height (128, or 64 when small), row1 too unless it is N.
cudaError_t launch_bsoi_persistent(double* A, long long ld, double* carry0, double* carry1,
                                   long long ldc, const double* G, int n, int L, int* done,
                                   int* next, int* err, bool small, cudaStream_t st,
                                   int row0 = 0, int row1 = -1, const int* never = nullptr);

// BSOI of many instances in one persistent launch (kernels_bsoi.cu).  Each
// instance: its matrix, carries, G_k, sizes, its done counters ((L-1) *
// bsoi_row_bands(N) ints, zeroed) and BSOI error word, and the global index
// of its first tile (prefix sums of bsoi_group_tiles, instance order).
struct BsoiInst {
  double* A;
  long long ld;
  double* carry[2];
  long long ldc;
  const double* G;
  int n, L, N;
  int* done;
  int* err;
  long long tile0;
};
// Passed by value as the kernel's (__grid_constant__) parameter: up to
// kBsoiGroupMax instances per launch (kernel parameters may take 32,764 bytes).
constexpr int kBsoiGroupMax = 256;
struct BsoiGroup {
  BsoiInst inst[kBsoiGroupMax];
  int count;
  long long total;           // tiles of all instances
  unsigned long long* next;  // tile counter, zeroed
  long long spin_limit;
};
static_assert(sizeof(BsoiGroup) <= 32764, "kernel parameter limit");
long long bsoi_group_tiles(int n, int L, bool small);
cudaError_t launch_bsoi_grouped(const BsoiGroup& g, bool small, bool aligned, cudaStream_t st);

// In-place inversion of the upper triangles of nblk n x n blocks (block b at
// A + b * bstride); tmp: device scratch of nblk * n * n / 4 doubles.  A zero
// diagonal is reported as the global index of diagonal block boff + b.
cudaError_t launch_trtri_blocks(double* A, long long ld, int n, long long bstride,
                                int nblk, int* info, double* tmp, cudaStream_t st, int boff = 0);

// cfg: 0 = choose by tile count, 1 = 128x128 (K stage 16), 2 = 64x64, 3 = 128x128 (K stage 32).
// Tile engine steps of every later launch: m16n8k8 (0, the default) or
// m16n8k16 (1); process-wide.
void gemm_set_k16(int on);
bool gemm_k16();
cudaError_t launch_gemm(const GemmDims& d, const GemmA& a, const GemmB& b,
                        const GemmC& c, int batch, int cfg, cudaStream_t st);
cudaError_t gemm_init_attributes();

cudaError_t launch_set_identity(double* G, long long ld, int m, long long bs, int batch,
                                cudaStream_t st);
// Info word value when a bounded wait inside a persistent kernel gave up:
// BSOFI_INFO_CUDA - cudaErrorLaunchTimeout.
constexpr int kInfoWaitFailed = -1000 - (int)cudaErrorLaunchTimeout;
// dst(r,c) = src(r,c), or 0 where r - roff > c (roff = kNoMask copies all).
// fold (optional): info words {info, BSOF error, BSOI error, BSTRI error};
// info becomes kInfoWaitFailed when any error word is set.
cudaError_t launch_copy_masked(double* dst, long long ldd, const double* src, long long lds,
                               int rows, int cols, int roff, cudaStream_t st,
                               int* fold = nullptr);
// Pack (mode 0) or compare (mode 1, *mismatch set on a difference) the
// reflector rows of every block column and tau; ref holds 2 n^2 L + n L doubles.
cudaError_t launch_state_ref(const double* A, long long ld, int n, int L, const double* tau,
                             double* ref, int mode, int* mismatch, cudaStream_t st);
// Zero the n x n blocks of A that BSOF reads as structural zeros:
// superdiagonal blocks (k,k+1) and last-column blocks (k,L-1), 1 <= k <= L-2.
cudaError_t launch_zero_structural(double* A, long long ld, int n, int L, cudaStream_t st);

// Loading every kernel onto the current device ahead of use.  Under lazy
// module loading (the CUDA 12 default) a kernel's code is loaded, and device
// memory taken for it, at its first launch; cudaFuncGetAttributes loads it
// now.  *local is raised to the kernel's per-thread local memory.
template <class F>
cudaError_t preload_one(F* f, size_t* local) {
  cudaFuncAttributes at;
  cudaError_t e = cudaFuncGetAttributes(&at, (const void*)f);
  if (e == cudaSuccess && at.localSizeBytes > *local) *local = at.localSizeBytes;
  return e;
}
// FP64 product C = A B on the int8 tensor cores by the Ozaki splitting
// scheme with S slices (kernels_ozaki.cu).  A (M x K) has two K segments as
// GemmA (k < ksplit: a0 with the row limit rlim0 and the mask r - roff0 > k;
// else a1), B is K x N column-major, C goes to two column segments as GemmC
// (j < nsplit: c0, else c1).  C must not overlap A or B.  scratch: 256-byte
// aligned, ozaki_scratch_bytes(M, N, K, S).  err: set to 1 when a bounded
// wait inside the kernel gives up.
constexpr int kOzakiMinSlices = 3, kOzakiMaxSlices = 8, kOzakiMaxK = 1536;
struct OzProduct {
  const double* a0;
  const double* a1;
  long long lda0, lda1;
  int ksplit, rlim0, roff0;
  int M, K;
  const double* b;
  long long ldb;
  int N;
  double* c0;
  double* c1;
  long long ldc0, ldc1;
  int nsplit;
  int S;
  void* scratch;
  int* err;
};
size_t ozaki_scratch_bytes(int M, int N, int K, int S);
cudaError_t launch_ozaki_product(const OzProduct& p, cudaStream_t st);

// One per kernel file: every kernel (each template instance) it launches.
cudaError_t preload_bsof(size_t* local);
cudaError_t preload_bsoi(size_t* local);
cudaError_t preload_bstri(size_t* local);
cudaError_t preload_gemm(size_t* local);
cudaError_t preload_panel(size_t* local);
cudaError_t preload_tri(size_t* local);
cudaError_t preload_ozaki(size_t* local);

}  // namespace bsofi
