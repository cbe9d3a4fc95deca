// DQMC producer and consumer steps around the inversion, on the device.
//
// Producer: a DQMC code builds M from p small blocks (B_k = expm(dtau t K)
// diag(exp(lambda h_k)), n x n each), not from a dense N x N matrix.  The
// reference takes the dense matrix on the host (src/bsofi_callback.c:130-144,
// filled by examples/ftest_hybrid/ftest_hybrid.f90:12-52), so a caller pays an
// N^2 copy for 2 p n^2 numbers of content.  These kernels write the p-cyclic
// blocks straight into the device matrix from packed blocks (or from expm(K)
// and the fields), together with the zero blocks the factorization reads.
//
// Consumer: the Metropolis ratio needs sign(det M) and log|det M| between the
// factorization and the inverse (ftest_hybrid.f90:141-145 reads tau and
// diag(A) after hybridXbsoftriH).  With M = Q R, Q a product of N Householder
// reflectors H_j = I - tau_j v_j v_j^T (det H_j = -1 when tau_j != 0, +1 when
// tau_j = 0) and R triangular:
//   sign(det M) = (-1)^{#(tau_j != 0)} prod sign(R_jj),  log|det M| = sum log|R_jj|.
// After BSTRI the diagonal holds 1/R_jj (same sign, log negated).
#include <climits>

#include <cuda_runtime.h>

#include "bsofi_common.cuh"
#include "bsofi_kernels.h"

#define BSOFI_API extern "C" __attribute__((visibility("default")))
#define BSOFI_INFO_CUDA (-1000)

namespace bsofi {
namespace {

struct AssembleArgs {
  int n, L;
  long long ldd;
  double* A;
  double* Al;         // the last block column (rows 0..N-1), leading dimension ldl
  long long ldl;
  const double* D;    // L packed diagonal blocks, or nullptr = identity
  const double* S;    // L packed coupling blocks (packed mode)
  const double* E;    // expm(dtau t K), n x n (Hubbard mode)
  const double* h;    // L x n fields, h[k*n + j] (Hubbard mode)
  double lambda;
  int hubbard;
};

// blockIdx.y < L: diagonal block y; otherwise coupling block k = y - L, placed
// at (k+1, k) for k < L-1 and at (0, L-1) for k = L-1.  Column-major element
// order, so reads of the packed block and writes into A are both coalesced.
__global__ void assemble_kernel(AssembleArgs s) {
  const int y = blockIdx.y, n = s.n;
  const long long nn = (long long)n * n;
  const bool diag = y < s.L;
  const int k = diag ? y : y - s.L;
  const int bi = diag ? k : (k + 1) % s.L, bj = k;
  const bool last = bj == s.L - 1;
  double* blk = last ? s.Al + cm((long long)bi * n, 0, s.ldl)
                     : s.A + cm((long long)bi * n, (long long)bj * n, s.ldd);
  const long long ld = last ? s.ldl : s.ldd;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nn;
       e += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(e % n), c = (int)(e / n);
    double v;
    if (diag) {
      v = s.D ? s.D[(long long)k * nn + e] : (r == c ? 1.0 : 0.0);
    } else if (s.hubbard) {
      // B_{k+1} = E diag(exp(lambda h_k)); -B below the diagonal, +B_p in the corner.
      const double b = s.E[e] * exp(s.lambda * s.h[(long long)k * n + c]);
      v = (k == s.L - 1) ? b : -b;
    } else {
      v = s.S[(long long)k * nn + e];
    }
    blk[cm(r, c, ld)] = v;
  }
}

// Into the ordinary layout (s.Al unset): the structural zero blocks the
// factorization reads, then the p-cyclic blocks.  Into the compact one
// (s.Al set; the caller zeroed both arrays): the p-cyclic blocks only.
cudaError_t launch_assemble(AssembleArgs s, cudaStream_t st) {
  if (s.Al == nullptr) {
    cudaError_t e = launch_zero_structural(s.A, s.ldd, s.n, s.L, st);
    if (e != cudaSuccess) return e;
    s.Al = s.A + cm(0, (long long)(s.L - 1) * s.n, s.ldd);
    s.ldl = s.ldd;
  }
  const long long nn = (long long)s.n * s.n;
  const int gx = (int)((nn + 255) / 256 < 64 ? (nn + 255) / 256 : 64);
  assemble_kernel<<<dim3(gx, 2 * s.L), 256, 0, st>>>(s);
  return cudaGetLastError();
}

// One CTA: sum of log|d_j|, count of d_j < 0, of d_j == 0 (or not finite) and
// of tau_j != 0 over the N diagonal entries.
// Diagonal entries j < jsplit at A (leading dimension ldd), the rest at Al
// (ldl), whose column 0 is column jsplit of the matrix (jsplit = N: all in A).
__global__ void __launch_bounds__(1024) logdet_kernel(const double* A, long long ldd, int N,
                                                      const double* tau, int inverted,
                                                      double* out, const double* Al = nullptr,
                                                      long long ldl = 0, int jsplit = INT_MAX) {
  __shared__ double s_log[32];
  __shared__ int s_cnt[32][3];
  double lsum = 0.0;
  int neg = 0, bad = 0, refl = 0;
  for (int j = threadIdx.x; j < N; j += blockDim.x) {
    const double d = j < jsplit ? A[(long long)j * ldd + j] : Al[cm(j, j - jsplit, ldl)];
    const double ad = fabs(d);
    if (d < 0.0) neg++;
    if (!(ad > 0.0) || isinf(ad)) bad++;
    else lsum += log(ad);
    if (tau[j] != 0.0) refl++;
  }
  lsum = warp_sum(lsum);
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    neg += __shfl_xor_sync(0xffffffffu, neg, off);
    bad += __shfl_xor_sync(0xffffffffu, bad, off);
    refl += __shfl_xor_sync(0xffffffffu, refl, off);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    s_log[warp] = lsum;
    s_cnt[warp][0] = neg;
    s_cnt[warp][1] = bad;
    s_cnt[warp][2] = refl;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    int cn = 0, cb = 0, cr = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      t += s_log[w];
      cn += s_cnt[w][0];
      cb += s_cnt[w][1];
      cr += s_cnt[w][2];
    }
    if (cb > 0) {
      out[0] = 0.0;  // singular R (or an overflowed diagonal): no finite log-determinant
      out[1] = -INFINITY;
    } else {
      out[0] = ((cn + cr) & 1) ? -1.0 : 1.0;
      out[1] = inverted ? -t : t;
    }
  }
}

}  // namespace
}  // namespace bsofi

using namespace bsofi;

static int api_err(cudaError_t e) { return e == cudaSuccess ? 0 : BSOFI_INFO_CUDA - (int)e; }

BSOFI_API int bsofi_device_assemble(int n, int L, const double* dD, const double* dS, double* dA,
                                    int ldda, void* stream) {
  if (n < 1 || L < 2 || ldda < n * L || dS == nullptr || dA == nullptr) return -1;
  AssembleArgs s = {};
  s.n = n;
  s.L = L;
  s.ldd = ldda;
  s.A = dA;
  s.D = dD;
  s.S = dS;
  return api_err(launch_assemble(s, (cudaStream_t)stream));
}

BSOFI_API int bsofi_device_hubbard_assemble(int n, int L, const double* dExpK, const double* dh,
                                            double lambda, double* dA, int ldda, void* stream) {
  if (n < 1 || L < 2 || ldda < n * L || dExpK == nullptr || dh == nullptr || dA == nullptr)
    return -1;
  AssembleArgs s = {};
  s.n = n;
  s.L = L;
  s.ldd = ldda;
  s.A = dA;
  s.E = dExpK;
  s.h = dh;
  s.lambda = lambda;
  s.hubbard = 1;
  return api_err(launch_assemble(s, (cudaStream_t)stream));
}

BSOFI_API int bsofi_device_logdet(int n, int L, const double* dA, int ldda, const double* dtau,
                                  int inverted, double* dout, void* stream) {
  if (n < 1 || L < 2 || ldda < n * L || dA == nullptr || dtau == nullptr || dout == nullptr)
    return -1;
  logdet_kernel<<<1, 1024, 0, (cudaStream_t)stream>>>(dA, ldda, n * L, dtau, inverted ? 1 : 0,
                                                      dout);
  return api_err(cudaGetLastError());
}

// Compact storage of the storage-sharded inversion: block columns 0..L-2 at
// band (leading dimension 3n, band_doubles in all), the last block column at
// last (N x n, leading dimension N).  Both arrays are zeroed, then the
// p-cyclic blocks written: packed (dS, and dD or identity diagonal blocks) or
// Hubbard (dExpK set: dh and lambda as for bsofi_device_hubbard_assemble).
extern "C" int bsofi_dev_assemble_compact(int n, int L, const double* dD, const double* dS,
                                          const double* dExpK, const double* dh, double lambda,
                                          double* band, size_t band_doubles, double* last,
                                          void* stream) {
  const cudaStream_t st = (cudaStream_t)stream;
  const long long N = (long long)n * L;
  cudaError_t e = cudaMemsetAsync(band, 0, sizeof(double) * band_doubles, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(last, 0, sizeof(double) * (size_t)N * n, st);
  if (e != cudaSuccess) return (int)e;
  AssembleArgs s = {};
  s.n = n;
  s.L = L;
  s.ldd = 3ll * n;
  s.A = band;
  s.Al = last;
  s.ldl = N;
  s.D = dD;
  s.S = dS;
  s.E = dExpK;
  s.h = dh;
  s.lambda = lambda;
  s.hubbard = dExpK != nullptr;
  return (int)launch_assemble(s, st);
}

// Sign and log|det M| from the compact state (as bsofi_device_logdet).
extern "C" int bsofi_dev_logdet_compact(int n, int L, const double* band, const double* last,
                                        const double* tau, int inverted, double* out,
                                        void* stream) {
  const int N = n * L;
  logdet_kernel<<<1, 1024, 0, (cudaStream_t)stream>>>(band, 3ll * n, N, tau, inverted ? 1 : 0,
                                                      out, last, N, (L - 1) * n);
  return (int)cudaGetLastError();
}
