// Allocation-free variant of the device-resident inversion.
//
// Some callers cannot allocate device memory when they invert: a DQMC code
// whose memory pool has already reserved nearly all of HBM (a fresh
// cudaMalloc fails), or a caller that must not let cudaMalloc/cudaFree
// synchronize the device in the middle of a Monte Carlo sweep while other
// streams are busy.  bsofi_device_invert_noalloc serves them: it runs the same
// BSOF + BSTRI + BSOI kernels as bsofi_device_invert, but its workspace is the
// file-scope array below instead of a caller buffer, and it calls no
// cudaMalloc, cudaFree or allocating library routine.
//
// The array is BSOFI_NOALLOC_SCRATCH_BYTES (32 MiB).  The driver reserves it
// when it loads this file's module on a device, which under lazy module
// loading (the CUDA 12 default) is the first time the module is used there;
// kernel code and local memory are likewise taken at first use.
// bsofi_noalloc_prepare does all of that up front, so that a caller can run it
// before its own pool takes the rest of HBM.  After that the device holds the
// array until the process exits.  All calls share it and it keeps the previous
// call's contents: the pipeline writes every scratch region before reading it
// (the BSTRI info word is reset at the start of each call), so nothing needs
// clearing between calls, but calls that overlap on the GPU (different streams
// or threads on the same device) race on it.
#include <cuda_runtime.h>

#include "bsofi_device.h"

#define BSOFI_NOALLOC_SCRATCH_BYTES (32ull << 20)
#define BSOFI_INFO_CUDA (-1000)
#define BSOFI_NOALLOC_TOO_LARGE (-2000)

static __device__ __align__(256) unsigned char g_noalloc_scratch[BSOFI_NOALLOC_SCRATCH_BYTES];

namespace {

// Device address of the scratch array on the current device.  In host code
// the array's name is only a host-side stand-in; the address is looked up on
// every call (cheap once the module is loaded), so a context that was reset
// and reloaded the module at another address is never handed a stale one.
cudaError_t scratch_address(void** out) {
  *out = nullptr;
  return cudaGetSymbolAddress(out, g_noalloc_scratch);
}

}  // namespace

extern "C" __attribute__((visibility("default"))) unsigned long long
bsofi_noalloc_scratch_bytes(void) {
  return BSOFI_NOALLOC_SCRATCH_BYTES;
}

extern "C" __attribute__((visibility("default"))) int bsofi_noalloc_prepare(void) {
  void* ws = nullptr;
  cudaError_t e = scratch_address(&ws);
  if (e != cudaSuccess) return BSOFI_INFO_CUDA - (int)e;
  const int r = bsofi_dev_preload();
  return r ? BSOFI_INFO_CUDA - r : 0;
}

extern "C" __attribute__((visibility("default"))) int bsofi_device_invert_noalloc(
    int n, int L, double* dA, int ldda, double* dtau, int* dinfo, void* stream) {
  if (n < 1 || n > 768 || L < 2 || ldda < n * L || dA == nullptr || dtau == nullptr) return -1;
  if (bsofi_dev_ws_bytes(n, L, ldda) > BSOFI_NOALLOC_SCRATCH_BYTES) return BSOFI_NOALLOC_TOO_LARGE;
  void* ws = nullptr;
  cudaError_t e = scratch_address(&ws);
  if (e != cudaSuccess) return BSOFI_INFO_CUDA - (int)e;
  int r = bsofi_dev_prepare();
  if (r == 0) r = bsofi_dev_bsoftri(n, L, dA, ldda, dtau, ws, stream);
  if (r == 0) {
    long long c = bsofi_dev_launch_count();
    r = bsofi_dev_bsoi(n, L, dA, ldda, dtau, ws, stream);
    bsofi_dev_add_launches(c);
  }
  if (r) return BSOFI_INFO_CUDA - r;
  // The info word after BSOI also carries the BSOF/BSOI wait errors.
  if (dinfo != nullptr)
    r = (int)cudaMemcpyAsync(dinfo, bsofi_dev_info_ptr(ws), sizeof(int), cudaMemcpyDeviceToDevice,
                             (cudaStream_t)stream);
  if (r) return BSOFI_INFO_CUDA - r;
  if (dinfo != nullptr) return 0;
  // No device word to receive it: wait for the stream and return the info
  // word itself (0, i > 0 for an exactly zero R(i,i), or the wait-failure code).
  int info = 0;
  r = (int)cudaMemcpyAsync(&info, bsofi_dev_info_ptr(ws), sizeof(int), cudaMemcpyDeviceToHost,
                           (cudaStream_t)stream);
  if (r == 0) r = (int)cudaStreamSynchronize((cudaStream_t)stream);
  if (r) return BSOFI_INFO_CUDA - r;
  return info >= 0x7f7f7f7f ? 0 : info;
}
