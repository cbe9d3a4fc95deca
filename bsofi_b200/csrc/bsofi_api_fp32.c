/*
 * bsofi_api_fp32.c -- host C layer of libbsofi_b200_fp32.so: the
 * reference's single-precision build (scalar_t = float, config.h:132-136)
 * over the FP64 device pipeline.
 *
 * Reference interface: src/bsofi_callback.c:24-218 (handle API, Fortran
 * twins, timers), include/bsofi_cpu.h:24-72, include/bsofi_hybrid.h:110-130,
 * include/bsofi_gpu.h:34-62, with float arrays.  Every call moves the same
 * regions as the double library, in float, between the caller's arrays and
 * a float device matrix, and widens / rounds them on the GPU around the
 * FP64 pipeline:
 *   XbsoftriH  H2D the 2L p-cyclic blocks, D2H the state (block upper
 *              triangle plus reflector rows) and tau;
 *   XbsoiH     H2D the state and tau, D2H the dense M^{-1}.
 */
#include <limits.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>
#include <cuda_runtime_api.h>

#include "../../include/bsofi_b200_fp32.h"
#include "bsofi_device.h"

#define HANDLE_MAGIC 0x34465342u /* "BSF4" */
#define HANDLE_VERSION 1u
#define CTX_MAGIC 0x34544342u

enum { REGION_FULL = 0, REGION_STATE = 1, REGION_PCYCLIC = 2 };
enum { PH_BSOF = 0, PH_BSTRI = 1, PH_BSOFTRI = 2, PH_BSOI = 3 };

typedef struct f32_ctx {
  uint32_t magic;
  int device;
  int n, L, ldd;
  cudaStream_t stream;
  double *dA, *dtau; /* FP64 working matrix and tau */
  float *fA, *ftau;  /* float copies the host transfers use (pitch ldd) */
  void *dws;
} f32_ctx;

typedef struct f32_handle {
  uint32_t magic;
  uint32_t version;
  uint64_t ctx;
  int32_t n, L, lda;
  int32_t reserved[3];
} f32_handle;

typedef char f32_handle_fits_in_40_bytes[(sizeof(f32_handle) <= 40) ? 1 : -1];

static __thread long long t_launches = 0;

static int cuda_info(cudaError_t e) { return BSOFI_INFO_CUDA - (int)e; }
static int round_up(int v, int m) { return (v + m - 1) / m * m; }

/* Device workspace length in floats for the -2 queries. */
static int device_floats(int n, int L) {
  const int N = n * L, ldd = round_up(N, 32);
  const size_t bytes = (size_t)ldd * N * (sizeof(double) + sizeof(float)) +
                       (size_t)N * (sizeof(double) + sizeof(float)) + bsofi_dev_ws_bytes(n, L, ldd);
  const size_t fl = bytes / sizeof(float);
  return fl > (size_t)INT_MAX ? INT_MAX : (int)fl;
}

static void ctx_free_buffers(f32_ctx *c) {
  if (c->dA) cudaFree(c->dA);
  if (c->dtau) cudaFree(c->dtau);
  if (c->fA) cudaFree(c->fA);
  if (c->ftau) cudaFree(c->ftau);
  if (c->dws) cudaFree(c->dws);
  c->dA = c->dtau = NULL;
  c->fA = c->ftau = NULL;
  c->dws = NULL;
  c->n = c->L = c->ldd = 0;
}

static cudaError_t ctx_fit(f32_ctx *c, int n, int L) {
  cudaError_t e;
  const int N = n * L;
  int ldd;
  if (c->dA && c->n == n && c->L == L) return cudaSuccess;
  ctx_free_buffers(c);
  ldd = round_up(N, 32);
  if ((e = cudaMalloc((void **)&c->dA, sizeof(double) * (size_t)ldd * N)) != cudaSuccess) goto fail;
  if ((e = cudaMalloc((void **)&c->fA, sizeof(float) * (size_t)ldd * N)) != cudaSuccess) goto fail;
  if ((e = cudaMalloc((void **)&c->dtau, sizeof(double) * (size_t)N)) != cudaSuccess) goto fail;
  if ((e = cudaMalloc((void **)&c->ftau, sizeof(float) * (size_t)N)) != cudaSuccess) goto fail;
  if ((e = cudaMalloc(&c->dws, bsofi_dev_ws_bytes(n, L, ldd))) != cudaSuccess) goto fail;
  if ((e = cudaMemset(c->dws, 0, 256)) != cudaSuccess) goto fail;
  c->n = n;
  c->L = L;
  c->ldd = ldd;
  return cudaSuccess;
fail:
  ctx_free_buffers(c);
  cudaGetLastError();
  return e;
}

static f32_ctx *ctx_create(int n, int L, cudaError_t *err) {
  cudaError_t e;
  f32_ctx *c = (f32_ctx *)calloc(1, sizeof(f32_ctx));
  if (!c) {
    *err = cudaErrorMemoryAllocation;
    return NULL;
  }
  c->magic = CTX_MAGIC;
  if ((e = cudaGetDevice(&c->device)) != cudaSuccess ||
      (e = (cudaError_t)bsofi_dev_prepare()) != cudaSuccess ||
      (e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) {
    free(c);
    *err = e;
    return NULL;
  }
  if ((e = ctx_fit(c, n, L)) != cudaSuccess) {
    cudaStreamDestroy(c->stream);
    free(c);
    *err = e;
    return NULL;
  }
  *err = cudaSuccess;
  return c;
}

static void ctx_destroy(f32_ctx *c) {
  if (!c) return;
  if (c->stream) cudaStreamSynchronize(c->stream);
  ctx_free_buffers(c);
  if (c->stream) cudaStreamDestroy(c->stream);
  c->magic = 0;
  free(c);
}

static f32_ctx *handle_ctx(const int *h) {
  f32_handle hd;
  f32_ctx *c;
  if (!h) return NULL;
  memcpy(&hd, h, sizeof(hd));
  if (hd.magic != HANDLE_MAGIC || hd.version != HANDLE_VERSION) return NULL;
  c = (f32_ctx *)(uintptr_t)hd.ctx;
  if (!c || c->magic != CTX_MAGIC) return NULL;
  return c;
}

/* ------------------------------------------------------------- transfers */
/* One region between the caller's host float array (pitch lda) and the
 * context's float device matrix (pitch ldd), block column by block column. */
static cudaError_t copy_region(f32_ctx *c, float *A, int lda, int region, int to_host) {
  const int n = c->n, L = c->L, N = n * L;
  const size_t es = sizeof(float), sh = es * (size_t)lda, sd = es * (size_t)c->ldd;
  const enum cudaMemcpyKind kind = to_host ? cudaMemcpyDeviceToHost : cudaMemcpyHostToDevice;
  cudaError_t e = cudaSuccess;
  int k;
#define SPAN(r0, r1, k0)                                                                      \
  do {                                                                                        \
    float *h_ = A + (size_t)(k0) * n * lda + (r0);                                            \
    float *d_ = c->fA + (size_t)(k0) * n * c->ldd + (r0);                                     \
    e = to_host ? cudaMemcpy2DAsync(h_, sh, d_, sd, es * ((r1) - (r0)), n, kind, c->stream)   \
                : cudaMemcpy2DAsync(d_, sd, h_, sh, es * ((r1) - (r0)), n, kind, c->stream);  \
  } while (0)
  if (region == REGION_FULL) {
    return to_host ? cudaMemcpy2DAsync(A, sh, c->fA, sd, es * N, N, kind, c->stream)
                   : cudaMemcpy2DAsync(c->fA, sd, A, sh, es * N, N, kind, c->stream);
  }
  for (k = 0; k < L && e == cudaSuccess; k++) {
    if (region == REGION_STATE) {
      SPAN(0, (k + 2) * n < N ? (k + 2) * n : N, k);
    } else if (k < L - 1) {
      SPAN(k * n, (k + 2) * n, k);
    } else {
      SPAN(0, n, k);
      if (e == cudaSuccess) SPAN((L - 1) * n, N, k);
    }
  }
#undef SPAN
  return e;
}

static cudaError_t convert(f32_ctx *c, float *f, int ldf, int region, int to_float) {
  cudaError_t e =
      (cudaError_t)bsofi_dev_convert(c->n, c->L, f, ldf, c->dA, c->ldd, region, to_float, c->stream);
  if (e == cudaSuccess) t_launches++;
  return e;
}

static cudaError_t convert_tau(f32_ctx *c, int to_float) {
  cudaError_t e = (cudaError_t)bsofi_dev_convert_vec(c->ftau, c->dtau, c->n * c->L, to_float,
                                                    c->stream);
  if (e == cudaSuccess) t_launches++;
  return e;
}

/* Reads the BSTRI info word and the wait-error words after synchronising. */
static int read_info(f32_ctx *c) {
  int v[4] = {0, 0, 0, 0};
  cudaError_t e = cudaMemcpyAsync(v, bsofi_dev_info_ptr(c->dws), sizeof(v),
                                  cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_info(e);
  if (v[1] != 0 || v[2] != 0 || v[3] != 0) return cuda_info(cudaErrorLaunchTimeout);
  return v[0] >= 0x7f7f7f7f ? 0 : v[0];
}

/* One phase on the FP64 working matrix, which holds its input. */
static cudaError_t run_phase(f32_ctx *c, int phase) {
  const int n = c->n, L = c->L;
  int r;
  if (phase == PH_BSOF)
    r = bsofi_dev_bsof(n, L, c->dA, c->ldd, c->dtau, c->dws, c->stream);
  else if (phase == PH_BSTRI)
    r = bsofi_dev_bstri(n, L, c->dA, c->ldd, c->dws, c->stream);
  else if (phase == PH_BSOFTRI)
    r = bsofi_dev_bsoftri(n, L, c->dA, c->ldd, c->dtau, c->dws, c->stream);
  else
    r = bsofi_dev_bsoi(n, L, c->dA, c->ldd, c->dtau, c->dws, c->stream);
  t_launches += bsofi_dev_launch_count();
  return (cudaError_t)r;
}

/* Load the phase's input into the FP64 working matrix from the float
 * device matrix f (pitch ldf; the context's own after a host upload). */
static cudaError_t load_input(f32_ctx *c, float *f, int ldf, int phase) {
  cudaError_t e;
  if (phase == PH_BSOF || phase == PH_BSOFTRI) {
    /* Zero first: with L = 2 the corner block (0, L-1) is also the
     * superdiagonal block the zeroing clears. */
    e = (cudaError_t)bsofi_dev_zero_structural(c->n, c->L, c->dA, c->ldd, c->stream);
    t_launches += bsofi_dev_launch_count();
    if (e != cudaSuccess) return e;
    return convert(c, f, ldf, REGION_PCYCLIC, 0);
  }
  if ((e = convert(c, f, ldf, REGION_STATE, 0)) != cudaSuccess) return e;
  return phase == PH_BSOI ? convert_tau(c, 0) : cudaSuccess;
}

/* A phase on a host float array: returns info. */
static int drive_host(f32_ctx *c, int n, int L, float *A, int lda, float *tau, int phase) {
  const int N = n * L;
  const int in_region = (phase == PH_BSOF || phase == PH_BSOFTRI) ? REGION_PCYCLIC : REGION_STATE;
  const int out_region = phase == PH_BSOI ? REGION_FULL : REGION_STATE;
  cudaError_t e;
  int info;
  t_launches = 0;
  if ((e = ctx_fit(c, n, L)) != cudaSuccess) return cuda_info(e);
  if ((e = copy_region(c, A, lda, in_region, 0)) != cudaSuccess) return cuda_info(e);
  if (phase == PH_BSOI &&
      (e = cudaMemcpyAsync(c->ftau, tau, sizeof(float) * N, cudaMemcpyHostToDevice, c->stream)) !=
          cudaSuccess)
    return cuda_info(e);
  if ((e = load_input(c, c->fA, c->ldd, phase)) != cudaSuccess) return cuda_info(e);
  if ((e = run_phase(c, phase)) != cudaSuccess) return cuda_info(e);
  if ((e = convert(c, c->fA, c->ldd, out_region, 1)) != cudaSuccess) return cuda_info(e);
  if ((e = copy_region(c, A, lda, out_region, 1)) != cudaSuccess) return cuda_info(e);
  if (phase == PH_BSOF || phase == PH_BSOFTRI) {
    if ((e = convert_tau(c, 1)) != cudaSuccess) return cuda_info(e);
    e = cudaMemcpyAsync(tau, c->ftau, sizeof(float) * N, cudaMemcpyDeviceToHost, c->stream);
    if (e != cudaSuccess) return cuda_info(e);
  }
  info = read_info(c);
  /* A phase that only factors or only applies Q reports its own errors, not
   * BSTRI's info word. */
  if (phase == PH_BSOF || phase == PH_BSOI) return info < 0 ? info : 0;
  return info;
}

/* ---------------------------------------------------------------- checks */
static int check_args(int n, int L, const float *A, int lda, const float *tau, const float *work,
                      int lwork, int first_arg) {
  if (n < 1 || n > BSOFI_MAX_BLOCK) return -(first_arg);
  if (L < 2 || (long long)n * L > 1000000) return -(first_arg + 1);
  if (!A) return -(first_arg + 2);
  if (lda < n * L) return -(first_arg + 3);
  if (!tau) return -(first_arg + 4);
  if ((lwork == -1 || lwork == -2) && !work) return -(first_arg + 5);
  if (lwork < 1 && lwork != -1 && lwork != -2) return -(first_arg + 6);
  return 0;
}

/* ================================================================ handle API */
int hybridxinith_(int *handle, int *n, int *L, int *lda) {
  f32_handle hd;
  f32_ctx *c;
  cudaError_t e;
  if (!handle || !n || !L || !lda) return -1;
  if (*n < 1 || *n > BSOFI_MAX_BLOCK || *L < 2 || *lda < (*n) * (*L)) return -1;
  c = ctx_create(*n, *L, &e);
  if (!c) return -1;
  memset(&hd, 0, sizeof(hd));
  hd.magic = HANDLE_MAGIC;
  hd.version = HANDLE_VERSION;
  hd.ctx = (uint64_t)(uintptr_t)c;
  hd.n = *n;
  hd.L = *L;
  hd.lda = *lda;
  memcpy(handle, &hd, sizeof(hd));
  return 0;
}

int hybridxbsofilworkh_(int *handle, int *n, int *L, int *lda) {
  (void)handle;
  (void)n;
  (void)L;
  (void)lda;
  return 1;
}

static int handle_phase(int *handle, int *n, int *L, float *A, int *lda, float *tau, float *work,
                        int *lwork, int *info, int phase) {
  f32_ctx *c = handle_ctx(handle);
  int r;
  if (!info) return -9;
  if (!n || !L || !lda || !lwork) return *info = !n ? -2 : !L ? -3 : !lda ? -5 : -8;
  if (!c) return *info = -1;
  r = check_args(*n, *L, A, *lda, tau, work, *lwork, 2);
  if (r) return *info = r;
  if (*lwork == -1 || *lwork == -2) {
    work[0] = *lwork == -1 ? 1.0f : (float)device_floats(*n, *L);
    return *info = 0;
  }
  return *info = drive_host(c, *n, *L, A, *lda, tau, phase);
}

int hybridxbsoftrih_(int *handle, int *n, int *L, float *A, int *lda, float *tau, float *work,
                     int *lwork, int *info) {
  return handle_phase(handle, n, L, A, lda, tau, work, lwork, info, PH_BSOFTRI);
}

int hybridxbsoih_(int *handle, int *n, int *L, float *A, int *lda, float *tau, float *work,
                  int *lwork, int *info) {
  return handle_phase(handle, n, L, A, lda, tau, work, lwork, info, PH_BSOI);
}

int hybridxfinalizeh_(int *handle) {
  f32_ctx *c = handle_ctx(handle);
  if (c) ctx_destroy(c);
  if (handle) memset(handle, 0, sizeof(f32_handle));
  return 0;
}

void fgetwalltime_(double tv[2]) {
  struct timeval t;
  gettimeofday(&t, NULL);
  tv[0] = (double)t.tv_sec;
  tv[1] = (double)t.tv_usec;
}

double felapsed_(double t1[2], double t0[2]) {
  return (t1[0] - t0[0]) + (t1[1] - t0[1]) / 1000000.0;
}

/* ================================================================ C names */
static __thread f32_ctx *t_ctx = NULL;

static f32_ctx *thread_ctx(int n, int L, int *info) {
  cudaError_t e;
  if (t_ctx) {
    int dev = -1;
    if (cudaGetDevice(&dev) == cudaSuccess && dev == t_ctx->device) return t_ctx;
    ctx_destroy(t_ctx);
    t_ctx = NULL;
  }
  t_ctx = ctx_create(n, L, &e);
  if (!t_ctx) *info = cuda_info(e);
  return t_ctx;
}

int lapackXbsofiLWork(int n, int L, int lda) {
  (void)n;
  (void)L;
  (void)lda;
  return 1;
}

int hybridXbsofiLWork(int n, int L, int lda, int lworkHostDevice) {
  (void)lda;
  return lworkHostDevice == -2 ? device_floats(n, L) : 1;
}

static int c_phase(int n, int L, float *A, int lda, float *tau, float *work, int lwork, int *info,
                   int phase) {
  int r, tmp = 0;
  f32_ctx *c;
  if (!info) info = &tmp;
  r = check_args(n, L, A, lda, phase == PH_BSTRI ? A : tau, work, lwork, 1);
  if (r) return *info = r;
  if (lwork == -1 || lwork == -2) {
    work[0] = lwork == -1 ? 1.0f : (float)device_floats(n, L);
    return *info = 0;
  }
  c = thread_ctx(n, L, info);
  if (!c) return *info;
  return *info = drive_host(c, n, L, A, lda, tau, phase);
}

int lapackXbsof(int n, int L, float A[], int lda, float tau[], float work[], int lwork,
                int *info) {
  return c_phase(n, L, A, lda, tau, work, lwork, info, PH_BSOF);
}

int lapackXbstri(int n, int L, float A[], int lda, int *info) {
  float w = 0.0f;
  return c_phase(n, L, A, lda, NULL, &w, 1, info, PH_BSTRI);
}

int lapackXbsoi_ormqr(int n, int L, float A[], int lda, float tau[], float work[], int lwork,
                      int *info) {
  return c_phase(n, L, A, lda, tau, work, lwork, info, PH_BSOI);
}

int lapackXbsoi_orgqr(int n, int L, float A[], int lda, float tau[], float work[], int lwork,
                      int *info) {
  return c_phase(n, L, A, lda, tau, work, lwork, info, PH_BSOI);
}

int lapackxbsofilwork_(int *n, int *L, int *lda) { return lapackXbsofiLWork(*n, *L, *lda); }
int lapackxbsof_(int *n, int *L, float A[], int *lda, float tau[], float work[], int *lwork,
                 int *info) {
  return lapackXbsof(*n, *L, A, *lda, tau, work, *lwork, info);
}
int lapackxbstri_(int *n, int *L, float A[], int *lda, int *info) {
  return lapackXbstri(*n, *L, A, *lda, info);
}
int lapackxbsoi_ormqr_(int *n, int *L, float A[], int *lda, float tau[], float work[], int *lwork,
                       int *info) {
  return lapackXbsoi_ormqr(*n, *L, A, *lda, tau, work, *lwork, info);
}
int lapackxbsoi_orgqr_(int *n, int *L, float A[], int *lda, float tau[], float work[], int *lwork,
                       int *info) {
  return lapackXbsoi_orgqr(*n, *L, A, *lda, tau, work, *lwork, info);
}

int hybridXbsoftri(int handle, int n, int L, float A[], int lda, float tau[], float work[],
                   int lwork, float dwork[], int ldwork, int *info) {
  (void)handle;
  (void)dwork;
  (void)ldwork;
  return c_phase(n, L, A, lda, tau, work, lwork, info, PH_BSOFTRI);
}

int hybridXbsoi(int handle, int n, int L, float A[], int lda, float tau[], float work[],
                int lwork, float dwork[], int ldwork, int *info) {
  (void)handle;
  (void)dwork;
  (void)ldwork;
  return c_phase(n, L, A, lda, tau, work, lwork, info, PH_BSOI);
}

/* Fortran twins of the hybridX names (the reference's cb_hybridXbsofiLWork,
 * cb_hybridXbsoftri, cb_hybridXbsoi, src/bsofi_callback.c:62-87): every
 * argument by pointer; the cuBLAS handle is not passed. */
int hybridxbsofilwork_(int *n, int *L, int *lda, int *lworkHostDevice) {
  if (!n || !L || !lda || !lworkHostDevice) return 1;
  return hybridXbsofiLWork(*n, *L, *lda, *lworkHostDevice);
}
int hybridxbsoftri_(int *n, int *L, float A[], int *lda, float tau[], float work[], int *lwork,
                    float dwork[], int *ldwork, int *info) {
  if (!info) return -10;
  if (!n || !L || !lda || !lwork || !ldwork) {
    *info = !n ? -1 : !L ? -2 : !lda ? -4 : !lwork ? -7 : -9;
    return *info;
  }
  return hybridXbsoftri(0, *n, *L, A, *lda, tau, work, *lwork, dwork, *ldwork, info);
}
int hybridxbsoi_(int *n, int *L, float A[], int *lda, float tau[], float work[], int *lwork,
                 float dwork[], int *ldwork, int *info) {
  if (!info) return -10;
  if (!n || !L || !lda || !lwork || !ldwork) {
    *info = !n ? -1 : !L ? -2 : !lda ? -4 : !lwork ? -7 : -9;
    return *info;
  }
  return hybridXbsoi(0, *n, *L, A, *lda, tau, work, *lwork, dwork, *ldwork, info);
}

/* ------------------------------------------------------ device-pointer API */
/* A phase on the caller's float device matrix dA (pitch ldda), in place;
 * tau is host memory as in the reference. */
static int gpu_phase(int n, int L, float *dA, int ldda, float *tau, int *info, int phase) {
  int tmp = 0, N = n * L, r;
  f32_ctx *c;
  cudaError_t e;
  if (!info) info = &tmp;
  if (n < 1 || n > BSOFI_MAX_BLOCK) return *info = -1;
  if (L < 2) return *info = -2;
  if (!dA) return *info = -3;
  if (ldda < N) return *info = -4;
  if (phase != PH_BSTRI && !tau) return *info = -5;
  c = thread_ctx(n, L, info);
  if (!c) return *info;
  t_launches = 0;
  if ((e = ctx_fit(c, n, L)) != cudaSuccess) return *info = cuda_info(e);
  if (phase == PH_BSOI &&
      (e = cudaMemcpyAsync(c->ftau, tau, sizeof(float) * N, cudaMemcpyHostToDevice, c->stream)) !=
          cudaSuccess)
    return *info = cuda_info(e);
  if ((e = load_input(c, dA, ldda, phase)) != cudaSuccess) return *info = cuda_info(e);
  if ((e = run_phase(c, phase)) != cudaSuccess) return *info = cuda_info(e);
  if ((e = convert(c, dA, ldda, phase == PH_BSOI ? REGION_FULL : REGION_STATE, 1)) != cudaSuccess)
    return *info = cuda_info(e);
  if (phase == PH_BSOF) {
    if ((e = convert_tau(c, 1)) != cudaSuccess) return *info = cuda_info(e);
    e = cudaMemcpyAsync(tau, c->ftau, sizeof(float) * N, cudaMemcpyDeviceToHost, c->stream);
    if (e != cudaSuccess) return *info = cuda_info(e);
  }
  r = read_info(c);
  if (phase != PH_BSTRI && r > 0) r = 0;
  return *info = r;
}

int gpuXbsof(int n, int L, float dA[], int ldda, float tau[], float work[], int lwork, float *dT,
             int *info) {
  (void)dT;
  if (lwork == -1 || lwork == -2) {
    if (!work) return info ? (*info = -6) : -6;
    work[0] = lwork == -1 ? 1.0f : (float)device_floats(n, L);
    return info ? (*info = 0) : 0;
  }
  return gpu_phase(n, L, dA, ldda, tau, info, PH_BSOF);
}

int gpuXbstri_rseq(int n, int L, float dA[], int ldda, float dwork[], int ldwork, int *info) {
  (void)dwork;
  (void)ldwork;
  return gpu_phase(n, L, dA, ldda, NULL, info, PH_BSTRI);
}

int gpuXbstri_rbatched(int n, int L, float dA[], int ldda, float dwork[], int ldwork, int *info) {
  return gpuXbstri_rseq(n, L, dA, ldda, dwork, ldwork, info);
}

int gpuXbsoi_ormqr(int n, int L, float dA[], int ldda, float tau[], float work[], int lwork,
                   float *dT, float dwork[], int ldwork, int *info) {
  (void)dT;
  (void)dwork;
  (void)ldwork;
  if (lwork == -1 || lwork == -2) {
    if (!work) return info ? (*info = -6) : -6;
    work[0] = lwork == -1 ? 1.0f : (float)device_floats(n, L);
    return info ? (*info = 0) : 0;
  }
  return gpu_phase(n, L, dA, ldda, tau, info, PH_BSOI);
}

int gpuXbsoi_orgqr(int n, int L, float dA[], int ldda, float tau[], float work[], int lwork,
                   float *dT, float dwork[], int ldwork, int *info) {
  return gpuXbsoi_ormqr(n, L, dA, ldda, tau, work, lwork, dT, dwork, ldwork, info);
}

int gpuXbsoi_batched(int n, int L, float dA[], int ldda, float tau[], float work[], int lwork,
                     float *dT, float dwork[], int ldwork, int *info) {
  return gpuXbsoi_ormqr(n, L, dA, ldda, tau, work, lwork, dT, dwork, ldwork, info);
}

long long bsofi_fp32_last_launches(void) { return t_launches; }
