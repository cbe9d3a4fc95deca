// Autotuner of the per-size launch plan (no reference counterpart).
//
// Which BSOI form is fastest (one persistent launch, or one GEMM launch per
// step with a given tile shape), which tile shape suits the BSTRI
// row-recurrence GEMMs and how many worker CTAs the BSOF kernel wants depend
// on (n, L): the persistent BSOI kernel wins once a step fills the GPU with
// 128 x 128 tiles, per-step launches of smaller tiles win below that, and the
// crossover is not sharp.  bsofi_autotune times the candidates on the device
// for one (n, L), one knob at a time (coordinate descent from the default
// plan), on a synthetic p-cyclic matrix of that size, and stores the fastest
// plan in the process-wide table every later inversion of that size uses.
#include <cuda_runtime.h>

#include <cmath>

#include "bsofi_device.h"

#define BSOFI_API extern "C" __attribute__((visibility("default")))
#define BSOFI_INFO_CUDA (-1000)

extern "C" int bsofi_device_assemble(int n, int L, const double* dD, const double* dS,
                                     double* dA, int ldda, void* stream);

namespace {

// Coupling blocks with entries uniform in (-1, 1) / sqrt(n) from a hash of
// the index: a nonsingular p-cyclic matrix with an identity diagonal.
__global__ void synthetic_blocks_kernel(double* S, long long count, double scale) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x) {
    unsigned long long z = (unsigned long long)i * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const double u = (double)(z >> 11) * (1.0 / 9007199254740992.0);  // [0, 1)
    S[i] = (2.0 * u - 1.0) * scale;
  }
}

struct Buffers {
  double *A = nullptr, *tau = nullptr, *S = nullptr;
  void* ws = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  ~Buffers() {
    if (A) cudaFree(A);
    if (tau) cudaFree(tau);
    if (S) cudaFree(S);
    if (ws) cudaFree(ws);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  }
};

// The fastest of `reps` inversions after one warm-up.
cudaError_t time_plan(int n, int L, int ldd, Buffers& b, cudaStream_t st, const int* plan,
                      int reps, float* best) {
  if (bsofi_dev_plan_set(n, L, plan) != 0) return cudaErrorInvalidValue;
  *best = 1e30f;
  for (int r = 0; r <= reps; r++) {
    int e = bsofi_device_assemble(n, L, nullptr, b.S, b.A, ldd, st);
    if (e) return cudaErrorLaunchFailure;
    cudaError_t c = cudaEventRecord(b.e0, st);
    if (c != cudaSuccess) return c;
    e = bsofi_dev_invert(n, L, b.A, ldd, b.tau, b.ws, st);
    if (e) return (cudaError_t)e;
    if ((c = cudaEventRecord(b.e1, st)) != cudaSuccess) return c;
    if ((c = cudaEventSynchronize(b.e1)) != cudaSuccess) return c;
    float ms = 0.f;
    if ((c = cudaEventElapsedTime(&ms, b.e0, b.e1)) != cudaSuccess) return c;
    if (r > 0 && ms < *best) *best = ms;
  }
  return cudaSuccess;
}

}  // namespace

BSOFI_API int bsofi_autotune(int n, int L, int reps, void* stream, int* plan_out) {
  if (n < 1 || n > 768 || L < 2) return -1;
  if (reps < 1) reps = 3;
  int e = bsofi_dev_prepare();
  if (e) return BSOFI_INFO_CUDA - e;
  cudaStream_t st = (cudaStream_t)stream;
  const int N = n * L, ldd = (N + 31) / 32 * 32;
  Buffers b;
  cudaError_t c;
  const long long nsb = (long long)L * n * n;
  if ((c = cudaMalloc((void**)&b.A, sizeof(double) * (size_t)ldd * N)) != cudaSuccess ||
      (c = cudaMalloc((void**)&b.tau, sizeof(double) * (size_t)N)) != cudaSuccess ||
      (c = cudaMalloc((void**)&b.S, sizeof(double) * (size_t)nsb)) != cudaSuccess ||
      (c = cudaMalloc(&b.ws, bsofi_dev_ws_bytes(n, L, ldd))) != cudaSuccess ||
      (c = cudaMemsetAsync(b.ws, 0, 256, st)) != cudaSuccess ||
      (c = cudaEventCreate(&b.e0)) != cudaSuccess || (c = cudaEventCreate(&b.e1)) != cudaSuccess)
    return BSOFI_INFO_CUDA - (int)c;
  synthetic_blocks_kernel<<<1024, 256, 0, st>>>(b.S, nsb, 1.0 / std::sqrt((double)n));
  if ((c = cudaGetLastError()) != cudaSuccess) return BSOFI_INFO_CUDA - (int)c;

  int plan[4];
  bsofi_dev_plan_clear_one(n, L);
  bsofi_dev_plan_get(n, L, plan);
  float best;
  if ((c = time_plan(n, L, ldd, b, st, plan, reps, &best)) != cudaSuccess) goto fail;
  {
    // Knob 0: BSOI form; knob 3: BSTRI row group; knob 1: BSTRI one-row
    // recurrence tiles (only used with row group 0); knob 2: BSOF workers.
    static const int cand0[] = {0, 5, 1, 2, 3, 4};
    static const int cand1[] = {2, 4, 0, 3, 1};
    static const int cand2[] = {32, 48, 16, 64};
    static const int cand3[] = {0, 4, 2, 6};
    const int* cands[4] = {cand0, cand1, cand2, cand3};
    const int ncand[4] = {6, 5, 4, 4};
    static const int order[4] = {0, 3, 1, 2};
    for (int o = 0; o < 4; o++) {
      const int knob = order[o];
      if (knob == 1 && plan[3] >= 2) continue;
      for (int i = 0; i < ncand[knob]; i++) {
        if (cands[knob][i] == plan[knob]) continue;
        int trial[4] = {plan[0], plan[1], plan[2], plan[3]};
        trial[knob] = cands[knob][i];
        float t;
        if ((c = time_plan(n, L, ldd, b, st, trial, reps, &t)) != cudaSuccess) goto fail;
        if (t < best * 0.99f) {  // keep the incumbent unless clearly faster
          best = t;
          plan[knob] = trial[knob];
        }
      }
    }
  }
  bsofi_dev_plan_set(n, L, plan);
  if (plan_out)
    for (int i = 0; i < 4; i++) plan_out[i] = plan[i];
  return 0;
fail:
  bsofi_dev_plan_clear_one(n, L);
  cudaGetLastError();
  return BSOFI_INFO_CUDA - (int)c;
}

BSOFI_API int bsofi_plan_get(int n, int L, int* plan) { return bsofi_dev_plan_get(n, L, plan); }

BSOFI_API int bsofi_plan_set(int n, int L, const int* plan) {
  return bsofi_dev_plan_set(n, L, plan);
}

BSOFI_API void bsofi_plan_clear(void) { bsofi_dev_plan_clear(); }
