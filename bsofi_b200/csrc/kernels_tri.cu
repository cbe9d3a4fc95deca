// BSTRI building blocks: batched inversion of the upper-triangular diagonal
// blocks of R, and small utility kernels.
//
// Reference: lapackXbstri, src/bsofi_cpu.c:146-177 (dtrtri of the 3n corner
// and of each n x n diagonal block).  The diagonal blocks are independent of
// the block recurrence, so all of them are inverted together, in place in the
// upper triangle; the strict lower part, which holds Householder vectors, is
// never touched (as with LAPACK dtrtri).
#include <climits>
#include <vector>
#include "bsofi_common.cuh"
#include "bsofi_kernels.h"

namespace bsofi {

// Recursive inversion of the upper-triangular diagonal blocks, in place:
//   inv([U11 U12; 0 U22]) = [X11, -X11 U12 X22; 0, X22],  X = inv(U),
// split at a multiple of 32 near the middle down to leaves of at most 32
// columns.  Every leaf of every block is independent (one warp each, the
// column loop of LAPACK dtrti2 in shared memory); then, bottom-up, each split
// is two GEMMs batched over the blocks on the FP64 DMMA tile engine (the
// triangular factors are masked operands): T = U12 X22, X12 = -X11 T.
constexpr int TLEAF = 32;

// One warp inverts one leaf (rows/columns [32 l, 32 l + w) of block b).  An
// exactly zero diagonal entry leaves the leaf as it is and records the
// smallest 1-based global index ((boff + block) * n + i + 1) in *info; the block's
// inverse is then not formed.
__global__ void __launch_bounds__(128) trtri_leaves_kernel(double* A, long long ld, int n,
                                                           long long bstride, int nblk, int* info,
                                                           int boff) {
  __shared__ double sU[4][TLEAF][TLEAF + 1];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nleaf = (n + TLEAF - 1) / TLEAF;
  const long long gw = (long long)blockIdx.x * 4 + warp;
  if (gw >= (long long)nblk * nleaf) return;  // whole warps only: no block barrier below
  const int b = (int)(gw / nleaf), o = (int)(gw % nleaf) * TLEAF;
  const int w = min(TLEAF, n - o);
  double* U = A + (long long)b * bstride + cm(o, o, ld);
  double(*X)[TLEAF + 1] = sU[warp];
  for (int c = 0; c < TLEAF; c++)
    X[lane][c] = (lane <= c && c < w) ? U[cm(lane, c, ld)] : 0.0;
  __syncwarp();
  const unsigned zero = __ballot_sync(0xffffffffu, lane < w && X[lane][lane] == 0.0);
  if (zero != 0u) {
    if (lane == __ffs(zero) - 1) atomicMin(info, (boff + b) * n + o + lane + 1);
    return;
  }
  // dtrti2 ('U'): X(j,j) = 1/U(j,j), X(0:j,j) = -X(j,j) X(0:j,0:j) U(0:j,j).
  for (int j = 0; j < w; j++) {
    const double xjj = 1.0 / X[j][j];
    double s = 0.0;
    if (lane < j)
      for (int k = lane; k < j; k++) s = fma(X[lane][k], X[k][j], s);
    __syncwarp();
    if (lane < j) X[lane][j] = -xjj * s;
    if (lane == j) X[j][j] = xjj;
    __syncwarp();
  }
  for (int c = 0; c < w; c++)
    if (lane <= c) U[cm(lane, c, ld)] = X[lane][c];
}

namespace {
struct TriNode {
  int off, size, h;
};

// Splits of an n-column triangle in post order (children before parents).
void tri_nodes(int off, int size, std::vector<TriNode>& out) {
  if (size <= TLEAF) return;
  const int h = TLEAF * ((size + 2 * TLEAF - 1) / (2 * TLEAF));
  tri_nodes(off, h, out);
  tri_nodes(off + h, size - h, out);
  out.push_back({off, size, h});
}
}  // namespace

cudaError_t launch_trtri_blocks(double* A, long long ld, int n, long long bstride, int nblk,
                                int* info, double* tmp, cudaStream_t st, int boff) {
  if (nblk <= 0 || n <= 0) return cudaSuccess;
  const long long leaves = (long long)nblk * ((n + TLEAF - 1) / TLEAF);
  trtri_leaves_kernel<<<(int)((leaves + 3) / 4), 128, 0, st>>>(A, ld, n, bstride, nblk, info, boff);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  std::vector<TriNode> nodes;
  tri_nodes(0, n, nodes);
  for (const TriNode& q : nodes) {
    const int h = q.h, r = q.size - q.h;
    double* U12 = A + cm(q.off, q.off + h, ld);
    const double* X11 = A + cm(q.off, q.off, ld);
    const double* X22 = A + cm(q.off + h, q.off + h, ld);
    // T = U12 X22 (X22 upper triangular), T is h x r with leading dimension h.
    {
      GemmDims d = {h, r, r};
      GemmA a = {};
      a.p0 = U12;
      a.ld0 = ld;
      a.bs0 = bstride;
      a.ld1 = 2;
      a.ksplit = r;
      a.rlim0 = INT_MAX;
      a.roff0 = kNoMask;
      a.rlim1 = INT_MAX;
      a.roff1 = kNoMask;
      GemmB b = {X22, ld, bstride, 0};
      GemmC c = {};
      c.p0 = tmp;
      c.ld0 = h;
      c.bs0 = (long long)h * r;
      c.ld1 = 1;
      c.nsplit = r;
      c.alpha = 1.0;
      if ((e = launch_gemm(d, a, b, c, nblk, 0, st)) != cudaSuccess) return e;
    }
    // X12 = -X11 T (X11 upper triangular), written over U12.
    {
      GemmDims d = {h, r, h};
      GemmA a = {};
      a.p0 = X11;
      a.ld0 = ld;
      a.bs0 = bstride;
      a.ld1 = 2;
      a.ksplit = h;
      a.rlim0 = INT_MAX;
      a.roff0 = 0;
      a.rlim1 = INT_MAX;
      a.roff1 = kNoMask;
      GemmB b = {tmp, h, (long long)h * r, kNoMask};
      GemmC c = {};
      c.p0 = U12;
      c.ld0 = ld;
      c.bs0 = bstride;
      c.ld1 = 1;
      c.nsplit = r;
      c.alpha = -1.0;
      if ((e = launch_gemm(d, a, b, c, nblk, 0, st)) != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

// ------------------------------------------------------------------ utilities
// The part of the BSOF/I state that Q formation reads: rows [k n, (k+2) n)
// of block column k (the reflectors under each panel's diagonal, with the
// diagonal block), packed block after block with a 2n x n stride, then tau.
// mode 0 packs it into ref; mode 1 compares it with ref and sets *mismatch on
// any difference (bitwise: NaN never matches).
__global__ void state_ref_kernel(const double* A, long long ld, int n, int L, const double* tau,
                                 double* ref, int mode, int* mismatch) {
  const int k = blockIdx.y;
  const long long N = (long long)n * L;
  if (k < L) {
    const long long r0 = (long long)k * n;
    const int rows = (int)min(2ll * n, N - r0);
    const long long cnt = (long long)rows * n;
    const double* src = A + r0 + r0 * ld;
    double* dst = ref + (long long)k * 2 * n * n;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < cnt;
         e += (long long)gridDim.x * blockDim.x) {
      const double v = src[(e % rows) + (e / rows) * ld];
      if (mode == 0) dst[e] = v;
      else if (!(v == dst[e])) *mismatch = 1;
    }
  } else {
    double* dt = ref + 2ll * n * n * L;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < N;
         e += (long long)gridDim.x * blockDim.x) {
      const double v = tau[e];
      if (mode == 0) dt[e] = v;
      else if (!(v == dt[e])) *mismatch = 1;
    }
  }
}

cudaError_t launch_state_ref(const double* A, long long ld, int n, int L, const double* tau,
                             double* ref, int mode, int* mismatch, cudaStream_t st) {
  const long long per = 2ll * n * n;
  const int gx = (int)min((per + 255) / 256, 256ll);
  state_ref_kernel<<<dim3(gx, L + 1), 256, 0, st>>>(A, ld, n, L, tau, ref, mode, mismatch);
  return cudaGetLastError();
}


__global__ void set_identity_kernel(double* G, long long ld, int m, long long bs) {
  double* g = G + (long long)blockIdx.y * bs;
  long long total = (long long)m * m;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int r = (int)(e % m), c = (int)(e / m);
    g[cm(r, c, ld)] = (r == c) ? 1.0 : 0.0;
  }
}

cudaError_t launch_set_identity(double* G, long long ld, int m, long long bs, int batch,
                                cudaStream_t st) {
  if (batch <= 0 || m <= 0) return cudaSuccess;
  long long total = (long long)m * m;
  int gx = (int)min((total + 255) / 256, (long long)1024);
  set_identity_kernel<<<dim3(gx, batch), 256, 0, st>>>(G, ld, m, bs);
  return cudaGetLastError();
}

__global__ void copy_masked_kernel(double* dst, long long ldd, const double* src, long long lds,
                                   int rows, int cols, int roff, int* fold) {
  // fold (optional): the workspace info words {BSTRI info, BSOF error, BSOI
  // error, BSTRI error}; a bounded wait that gave up turns the info word into
  // an error.
  if (fold != nullptr && blockIdx.x == 0 && threadIdx.x == 0 && (fold[1] | fold[2] | fold[3]) != 0)
    fold[0] = kInfoWaitFailed;
  long long total = (long long)rows * cols;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int r = (int)(e % rows), c = (int)(e / rows);
    double v = ((long long)r - roff > c) ? 0.0 : src[cm(r, c, lds)];
    dst[cm(r, c, ldd)] = v;
  }
}

cudaError_t launch_copy_masked(double* dst, long long ldd, const double* src, long long lds,
                               int rows, int cols, int roff, cudaStream_t st, int* fold) {
  long long total = (long long)rows * cols;
  if (total <= 0) return cudaSuccess;
  int gx = (int)min((total + 255) / 256, (long long)4096);
  copy_masked_kernel<<<gx, 256, 0, st>>>(dst, ldd, src, lds, rows, cols, roff, fold);
  return cudaGetLastError();
}

__global__ void zero_structural_kernel(double* A, long long ld, int n, int L) {
  // blockIdx.y < L-1: superdiagonal block (k, k+1); else last-column block (k, L-1).
  int b = blockIdx.y, bi, bj;
  if (b < L - 1) {
    bi = b;
    bj = b + 1;
  } else {
    bi = b - (L - 1) + 1;
    bj = L - 1;
  }
  long long total = (long long)n * n;
  double* blk = A + cm((long long)bi * n, (long long)bj * n, ld);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x)
    blk[cm(e % n, e / n, ld)] = 0.0;
}

cudaError_t launch_zero_structural(double* A, long long ld, int n, int L, cudaStream_t st) {
  int nb = (L - 1) + (L >= 3 ? L - 2 : 0);
  if (nb <= 0) return cudaSuccess;
  long long total = (long long)n * n;
  int gx = (int)min((total + 255) / 256, (long long)64);
  zero_structural_kernel<<<dim3(gx, nb), 256, 0, st>>>(A, ld, n, L);
  return cudaGetLastError();
}

cudaError_t preload_tri(size_t* local) {
  cudaError_t e;
  if ((e = preload_one(trtri_leaves_kernel, local)) != cudaSuccess) return e;
  if ((e = preload_one(state_ref_kernel, local)) != cudaSuccess) return e;
  if ((e = preload_one(set_identity_kernel, local)) != cudaSuccess) return e;
  if ((e = preload_one(copy_masked_kernel, local)) != cudaSuccess) return e;
  return preload_one(zero_structural_kernel, local);
}

}  // namespace bsofi
