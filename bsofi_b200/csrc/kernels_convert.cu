// FP32 <-> FP64 conversion of the parts of a block p-cyclic matrix that the
// single-precision API moves (libbsofi_b200_fp32.so).
//
// The single-precision build of the reference (scalar_t = float,
// config.h:132-136) keeps every entry point and storage contract of the
// double one.  Here the caller's float arrays are widened on the device into
// the FP64 working matrix, the FP64 pipeline runs, and the results are
// rounded back to float.  Regions (column block k = column / n, N = n L):
//   0 full      rows [0, N) of every column;
//   1 state     rows [0, min((k+2) n, N)): the block upper triangle plus the
//               reflector rows of each block column (the BSOF/BSTRI state);
//   2 p-cyclic  rows [k n, (k+2) n) for k < L-1, and rows [0, n) and
//               [(L-1) n, N) of the last block column (the 2L input blocks).
// One CTA per column; consecutive threads take consecutive rows, so both the
// float and the double side are read and written coalesced.  The caller
// counts these launches (they do not touch the pipeline's launch counter).
#include <cuda_runtime.h>

#include "bsofi_device.h"

namespace {

struct Range {
  int lo0, hi0, lo1, hi1;
};

__device__ __forceinline__ Range column_rows(int j, int n, int L, int region) {
  const int N = n * L, k = j / n;
  Range r = {0, 0, 0, 0};
  if (region == 0) {
    r.hi0 = N;
  } else if (region == 1) {
    r.hi0 = (k + 2) * n < N ? (k + 2) * n : N;
  } else if (k < L - 1) {
    r.lo0 = k * n;
    r.hi0 = (k + 2) * n;
  } else {
    r.hi0 = n;
    r.lo1 = (L - 1) * n;
    r.hi1 = N;
  }
  return r;
}

__global__ void widen_kernel(const float* __restrict__ f, long long ldf, double* __restrict__ d,
                             long long ldd, int n, int L, int region) {
  const int j = blockIdx.x;
  const Range r = column_rows(j, n, L, region);
  const float* fc = f + (long long)j * ldf;
  double* dc = d + (long long)j * ldd;
  for (int i = r.lo0 + threadIdx.x; i < r.hi0; i += blockDim.x) dc[i] = (double)fc[i];
  for (int i = r.lo1 + threadIdx.x; i < r.hi1; i += blockDim.x) dc[i] = (double)fc[i];
}

__global__ void narrow_kernel(const double* __restrict__ d, long long ldd, float* __restrict__ f,
                              long long ldf, int n, int L, int region) {
  const int j = blockIdx.x;
  const Range r = column_rows(j, n, L, region);
  const double* dc = d + (long long)j * ldd;
  float* fc = f + (long long)j * ldf;
  for (int i = r.lo0 + threadIdx.x; i < r.hi0; i += blockDim.x) fc[i] = (float)dc[i];
  for (int i = r.lo1 + threadIdx.x; i < r.hi1; i += blockDim.x) fc[i] = (float)dc[i];
}

__global__ void widen_vec_kernel(const float* __restrict__ f, double* __restrict__ d, int len) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < len) d[i] = (double)f[i];
}

__global__ void narrow_vec_kernel(const double* __restrict__ d, float* __restrict__ f, int len) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < len) f[i] = (float)d[i];
}

}  // namespace

extern "C" int bsofi_dev_convert(int n, int L, float* f, int ldf, double* d, int ldd, int region,
                                 int to_float, void* stream) {
  const int N = n * L;
  if (n < 1 || L < 2 || ldf < N || ldd < N || region < 0 || region > 2 || !f || !d)
    return (int)cudaErrorInvalidValue;
  cudaStream_t st = (cudaStream_t)stream;
  if (to_float)
    narrow_kernel<<<N, 256, 0, st>>>(d, ldd, f, ldf, n, L, region);
  else
    widen_kernel<<<N, 256, 0, st>>>(f, ldf, d, ldd, n, L, region);
  return (int)cudaGetLastError();
}

extern "C" int bsofi_dev_convert_vec(float* f, double* d, int len, int to_float, void* stream) {
  if (len <= 0) return 0;
  if (!f || !d) return (int)cudaErrorInvalidValue;
  cudaStream_t st = (cudaStream_t)stream;
  const int grid = (len + 255) / 256;
  if (to_float)
    narrow_vec_kernel<<<grid, 256, 0, st>>>(d, f, len);
  else
    widen_vec_kernel<<<grid, 256, 0, st>>>(f, d, len);
  return (int)cudaGetLastError();
}
