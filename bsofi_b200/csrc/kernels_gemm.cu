// Launch wrappers for the FP64 DMMA tile engine (gemm.cuh).
#include <atomic>

#include "bsofi_kernels.h"

namespace bsofi {

// Tile engine steps: m16n8k8 (0, the default) or m16n8k16 (1); process-wide.
static std::atomic<int> g_k16{0};
void gemm_set_k16(int on) { g_k16.store(on ? 1 : 0); }
bool gemm_k16() { return g_k16.load() != 0; }

template <class Cfg, bool ALIGNED>
__global__ void __launch_bounds__(Cfg::THREADS) gemm_kernel(GemmDims d, GemmA a, GemmB b,
                                                            GemmC c) {
  extern __shared__ __align__(16) double smem_gemm[];
  gemm_tile<Cfg, ALIGNED>(d, a, b, c, blockIdx.x * Cfg::BM, blockIdx.y * Cfg::BN, blockIdx.z,
                          smem_gemm);
}

template <class Cfg, bool AL>
static cudaError_t set_attr() {
  return cudaFuncSetAttribute(gemm_kernel<Cfg, AL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)Cfg::SMEM);
}

cudaError_t gemm_init_attributes() {
  static PerDevice once;
  const int dev = once.pending();
  if (dev < 0) return cudaSuccess;
  cudaError_t e;
  if ((e = set_attr<CfgL, true>()) != cudaSuccess) return e;
  if ((e = set_attr<CfgL, false>()) != cudaSuccess) return e;
  if ((e = set_attr<CfgM, true>()) != cudaSuccess) return e;
  if ((e = set_attr<CfgM, false>()) != cudaSuccess) return e;
  if ((e = set_attr<CfgS, true>()) != cudaSuccess) return e;
  if ((e = set_attr<CfgS, false>()) != cudaSuccess) return e;
  if ((e = set_attr<CfgL16, true>()) != cudaSuccess) return e;
  if ((e = set_attr<CfgL16, false>()) != cudaSuccess) return e;
  if ((e = set_attr<CfgM16, true>()) != cudaSuccess) return e;
  if ((e = set_attr<CfgM16, false>()) != cudaSuccess) return e;
  if ((e = set_attr<CfgS16, true>()) != cudaSuccess) return e;
  if ((e = set_attr<CfgS16, false>()) != cudaSuccess) return e;
  once.mark(dev);
  return cudaSuccess;
}

static bool al16(const void* p) { return ((uintptr_t)p & 15) == 0; }

template <class Cfg>
static cudaError_t run(const GemmDims& d, const GemmA& a, const GemmB& b, const GemmC& c,
                       int batch, cudaStream_t st) {
  dim3 grid((d.M + Cfg::BM - 1) / Cfg::BM, (d.N + Cfg::BN - 1) / Cfg::BN, batch);
  bool aligned = al16(a.p0) && (a.p1 == nullptr || al16(a.p1)) && al16(b.p) &&
                 (a.ld0 % 2 == 0) && (a.ld1 % 2 == 0) && (b.ld % 2 == 0) &&
                 (a.bs0 % 2 == 0) && (a.bs1 % 2 == 0) && (b.bs % 2 == 0) &&
                 (a.ksplit % 2 == 0);
  if (aligned)
    gemm_kernel<Cfg, true><<<grid, Cfg::THREADS, Cfg::SMEM, st>>>(d, a, b, c);
  else
    gemm_kernel<Cfg, false><<<grid, Cfg::THREADS, Cfg::SMEM, st>>>(d, a, b, c);
  return cudaGetLastError();
}

cudaError_t launch_gemm(const GemmDims& d, const GemmA& a, const GemmB& b, const GemmC& c,
                        int batch, int cfg, cudaStream_t st) {
  if (d.M <= 0 || d.N <= 0 || batch <= 0) return cudaSuccess;
  cudaError_t e = gemm_init_attributes();
  if (e != cudaSuccess) return e;
  if (cfg == 0) {
    long long tilesL = (long long)((d.M + 127) / 128) * ((d.N + 127) / 128) * batch;
    cfg = (tilesL >= 148) ? 3 : 2;
  }
  if (gemm_k16()) {
    if (cfg == 1) return run<CfgL16>(d, a, b, c, batch, st);
    if (cfg == 3) return run<CfgM16>(d, a, b, c, batch, st);
    return run<CfgS16>(d, a, b, c, batch, st);
  }
  if (cfg == 1) return run<CfgL>(d, a, b, c, batch, st);
  if (cfg == 3) return run<CfgM>(d, a, b, c, batch, st);
  return run<CfgS>(d, a, b, c, batch, st);
}

cudaError_t preload_gemm(size_t* local) {
  cudaError_t e;
  if ((e = preload_one(gemm_kernel<CfgL, true>, local)) != cudaSuccess) return e;
  if ((e = preload_one(gemm_kernel<CfgL, false>, local)) != cudaSuccess) return e;
  if ((e = preload_one(gemm_kernel<CfgM, true>, local)) != cudaSuccess) return e;
  if ((e = preload_one(gemm_kernel<CfgM, false>, local)) != cudaSuccess) return e;
  if ((e = preload_one(gemm_kernel<CfgS, true>, local)) != cudaSuccess) return e;
  if ((e = preload_one(gemm_kernel<CfgS, false>, local)) != cudaSuccess) return e;
  if ((e = preload_one(gemm_kernel<CfgL16, true>, local)) != cudaSuccess) return e;
  if ((e = preload_one(gemm_kernel<CfgL16, false>, local)) != cudaSuccess) return e;
  if ((e = preload_one(gemm_kernel<CfgM16, true>, local)) != cudaSuccess) return e;
  if ((e = preload_one(gemm_kernel<CfgM16, false>, local)) != cudaSuccess) return e;
  if ((e = preload_one(gemm_kernel<CfgS16, true>, local)) != cudaSuccess) return e;
  return preload_one(gemm_kernel<CfgS16, false>, local);
}

}  // namespace bsofi
