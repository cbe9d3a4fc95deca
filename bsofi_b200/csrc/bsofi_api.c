/*
 * bsofi_api.c -- host C layer of libbsofi_b200.so: the reference's handle
 * API, C names and Fortran bindings over the device pipeline.
 *
 * Reference interface: src/bsofi_callback.c:1-220 (handle API and timers),
 * include/bsofi_cpu.h, include/bsofi_hybrid.h, include/bsofi_gpu.h.
 * Unlike the reference there is no host/device switch (KAPPA split) and no
 * LAPACK fallback: every call runs the sm_100a kernels.  Host <-> device
 * traffic per call is what the storage contract needs:
 *   XbsoftriH  H2D the 2L p-cyclic blocks, D2H the block upper triangle plus
 *              the reflector blocks, D2H tau;
 *   XbsoiH     H2D that same region and tau, D2H the dense M^{-1}.
 */
#include <pthread.h>
#include <stdint.h>
#include <limits.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>
#include <unistd.h>
#include <cuda_runtime_api.h>

#include "../../include/bsofi_b200.h"
#include "bsofi_device.h"

#define HANDLE_MAGIC 0x49465342u /* "BSFI" */
#define HANDLE_VERSION 1u
#define CTX_MAGIC 0x58544342u

/* ------------------------------------------------------------------------
 * Host staging.  Pageable caller arrays are copied through two pinned
 * buffers (double buffering against the DMA engine), packed and unpacked
 * column by column by a small pool of host threads so that host memory
 * bandwidth, not one core, bounds the transfer.  Page-locked caller arrays
 * (cudaMallocHost, cudaHostRegister) are copied by the DMA engine directly.
 * ---------------------------------------------------------------------- */
#define STAGE_BYTES ((size_t)64 << 20)
#define MAX_COPY_THREADS 16
#define PAR_MIN_BYTES ((size_t)1 << 20)

typedef struct copy_pool {
  int nthreads;
  pthread_t th[MAX_COPY_THREADS];
  pthread_mutex_t mu;
  pthread_cond_t cv_work, cv_done;
  unsigned long generation;
  int remaining, stop;
  char *dst;
  const char *src;
  size_t dpitch, spitch, width, height;
} copy_pool;

typedef struct {
  copy_pool *p;
  int index;
} copy_arg;

static void copy_rows(char *dst, size_t dpitch, const char *src, size_t spitch, size_t width,
                      size_t h0, size_t h1) {
  size_t i;
  for (i = h0; i < h1; i++) memcpy(dst + i * dpitch, src + i * spitch, width);
}

static void *copy_worker(void *arg) {
  copy_arg *a = (copy_arg *)arg;
  copy_pool *p = a->p;
  unsigned long seen = 0;
  for (;;) {
    size_t h0, h1;
    pthread_mutex_lock(&p->mu);
    while (p->generation == seen && !p->stop) pthread_cond_wait(&p->cv_work, &p->mu);
    if (p->stop) {
      pthread_mutex_unlock(&p->mu);
      break;
    }
    seen = p->generation;
    h0 = p->height * (size_t)a->index / (size_t)(p->nthreads + 1);
    h1 = p->height * (size_t)(a->index + 1) / (size_t)(p->nthreads + 1);
    pthread_mutex_unlock(&p->mu);
    copy_rows(p->dst, p->dpitch, p->src, p->spitch, p->width, h0, h1);
    pthread_mutex_lock(&p->mu);
    if (--p->remaining == 0) pthread_cond_signal(&p->cv_done);
    pthread_mutex_unlock(&p->mu);
  }
  free(a);
  return NULL;
}

static copy_pool *copy_pool_create(void) {
  copy_pool *p = (copy_pool *)calloc(1, sizeof(copy_pool));
  long nproc = sysconf(_SC_NPROCESSORS_ONLN);
  int i, want;
  if (!p) return NULL;
  want = (int)(nproc > 1 ? nproc - 1 : 0);
  if (want > MAX_COPY_THREADS - 1) want = MAX_COPY_THREADS - 1;
  pthread_mutex_init(&p->mu, NULL);
  pthread_cond_init(&p->cv_work, NULL);
  pthread_cond_init(&p->cv_done, NULL);
  for (i = 0; i < want; i++) {
    copy_arg *a = (copy_arg *)malloc(sizeof(copy_arg));
    if (!a) break;
    a->p = p;
    a->index = i;
    if (pthread_create(&p->th[i], NULL, copy_worker, a) != 0) {
      free(a);
      break;
    }
    p->nthreads++;
  }
  return p;
}

static void copy_pool_destroy(copy_pool *p) {
  int i;
  if (!p) return;
  pthread_mutex_lock(&p->mu);
  p->stop = 1;
  pthread_cond_broadcast(&p->cv_work);
  pthread_mutex_unlock(&p->mu);
  for (i = 0; i < p->nthreads; i++) pthread_join(p->th[i], NULL);
  pthread_mutex_destroy(&p->mu);
  pthread_cond_destroy(&p->cv_work);
  pthread_cond_destroy(&p->cv_done);
  free(p);
}

/* height rows of `width` bytes, split over the pool and the calling thread. */
static void par_copy2d(copy_pool *p, char *dst, size_t dpitch, const char *src, size_t spitch,
                       size_t width, size_t height) {
  size_t h0;
  if (!p || p->nthreads == 0 || width * height < PAR_MIN_BYTES) {
    copy_rows(dst, dpitch, src, spitch, width, 0, height);
    return;
  }
  pthread_mutex_lock(&p->mu);
  p->dst = dst;
  p->src = src;
  p->dpitch = dpitch;
  p->spitch = spitch;
  p->width = width;
  p->height = height;
  p->remaining = p->nthreads;
  p->generation++;
  pthread_cond_broadcast(&p->cv_work);
  pthread_mutex_unlock(&p->mu);
  h0 = height * (size_t)p->nthreads / (size_t)(p->nthreads + 1);
  copy_rows(dst, dpitch, src, spitch, width, h0, height);
  pthread_mutex_lock(&p->mu);
  while (p->remaining > 0) pthread_cond_wait(&p->cv_done, &p->mu);
  pthread_mutex_unlock(&p->mu);
}

typedef struct bsofi_ctx {
  uint32_t magic;
  int device;
  int n, L, ldd;
  cudaStream_t stream;
  double *dA;
  double *dtau;
  void *dws;
  size_t ws_bytes;
  char *stage[2];       /* pinned host staging buffers */
  cudaEvent_t stage_ev[2];
  int stage_next;
  copy_pool *pool;
  /* Pipelined BSOI on page-locked caller arrays: copy-in and copy-out
   * streams and per-column-block events (created on first use). */
  cudaStream_t s_in, s_out;
  cudaEvent_t *ev;      /* 2 * nev: [0, nev) uploaded, [nev, 2 nev) finished */
  cudaEvent_t ev_refl, ev_start;
  int nev;
  /* G_k = Q_k^T formed by the last hybridxbsoftrih_ stay in the workspace;
   * dref holds the reflector rows and tau they were formed from, so that
   * hybridxbsoih_ skips Q formation when it gets the same state back. */
  double *dref;
  int *dflag, *hflag;
  int g_valid;
} bsofi_ctx;

/* Layout of the caller's integer handler(10) (40 bytes). */
typedef struct bsofi_handle {
  uint32_t magic;
  uint32_t version;
  uint64_t ctx;
  int32_t n, L, lda;
  int32_t reserved[3];
} bsofi_handle;

typedef char handle_fits_in_40_bytes[(sizeof(bsofi_handle) <= 40) ? 1 : -1];

static int cuda_info(cudaError_t e) { return BSOFI_INFO_CUDA - (int)e; }

static int round_up(int v, int m) { return (v + m - 1) / m * m; }

/* Device workspace of the lwork = -2 query in doubles: the N x N matrix (leading
 * dimension rounded up to 32), tau and the pipeline workspace.  As a double it
 * is exact at every supported size (2.1e9 doubles at n = 576, L = 80 is past
 * INT_MAX, so the int-returning query saturates). */
static double device_lwork(int n, int L) {
  int ldd = round_up(n * L, 32), N = n * L;
  return (double)((size_t)ldd * N + N + bsofi_dev_ws_bytes(n, L, ldd) / sizeof(double));
}

static void ctx_free_buffers(bsofi_ctx *c) {
  if (c->dA) cudaFree(c->dA);
  if (c->dtau) cudaFree(c->dtau);
  if (c->dws) cudaFree(c->dws);
  if (c->dref) cudaFree(c->dref);
  c->dA = NULL;
  c->dtau = NULL;
  c->dws = NULL;
  c->dref = NULL;
  c->g_valid = 0;
  c->n = c->L = c->ldd = 0;
}

/* Make the context's buffers fit (n, L).  Returns cudaError_t. */
static cudaError_t ctx_fit(bsofi_ctx *c, int n, int L) {
  cudaError_t e;
  int N = n * L, ldd;
  if (c->dA && c->n == n && c->L == L) return cudaSuccess;
  ctx_free_buffers(c);
  ldd = round_up(N, 32);
  if ((e = cudaMalloc((void **)&c->dA, sizeof(double) * (size_t)ldd * N)) != cudaSuccess) goto fail;
  if ((e = cudaMalloc((void **)&c->dtau, sizeof(double) * (size_t)N)) != cudaSuccess) goto fail;
  c->ws_bytes = bsofi_dev_ws_bytes(n, L, ldd);
  if ((e = cudaMalloc(&c->dws, c->ws_bytes)) != cudaSuccess) goto fail;
  /* info words (BSTRI info, BSOF and BSOI error words) start cleared */
  if ((e = cudaMemset(c->dws, 0, 256)) != cudaSuccess) goto fail;
  if ((e = cudaMalloc((void **)&c->dref, sizeof(double) * bsofi_dev_state_ref_doubles(n, L))) !=
      cudaSuccess)
    goto fail;
  if (!c->dflag && (e = cudaMalloc((void **)&c->dflag, sizeof(int))) != cudaSuccess) goto fail;
  if (!c->hflag && (e = cudaMallocHost((void **)&c->hflag, sizeof(int))) != cudaSuccess) goto fail;
  c->n = n;
  c->L = L;
  c->ldd = ldd;
  return cudaSuccess;
fail:
  ctx_free_buffers(c);
  cudaGetLastError();
  return e;
}

static bsofi_ctx *ctx_create(int n, int L, cudaError_t *err) {
  cudaError_t e;
  bsofi_ctx *c = (bsofi_ctx *)calloc(1, sizeof(bsofi_ctx));
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
  {
    int b;
    for (b = 0; b < 2; b++) {
      if ((e = cudaMallocHost((void **)&c->stage[b], STAGE_BYTES)) != cudaSuccess ||
          (e = cudaEventCreateWithFlags(&c->stage_ev[b], cudaEventDisableTiming)) != cudaSuccess) {
        c->stage[b] = NULL;
        cudaGetLastError();
        break;
      }
    }
    c->pool = copy_pool_create();
  }
  *err = cudaSuccess;
  return c;
}

static void ctx_destroy(bsofi_ctx *c) {
  int b;
  if (!c) return;
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (b = 0; b < 2; b++) {
    if (c->stage[b]) cudaFreeHost(c->stage[b]);
    if (c->stage_ev[b]) cudaEventDestroy(c->stage_ev[b]);
  }
  copy_pool_destroy(c->pool);
  ctx_free_buffers(c);
  if (c->s_in) {
    cudaStreamSynchronize(c->s_in);
    cudaStreamDestroy(c->s_in);
  }
  if (c->s_out) {
    cudaStreamSynchronize(c->s_out);
    cudaStreamDestroy(c->s_out);
  }
  for (b = 0; b < 2 * c->nev; b++) cudaEventDestroy(c->ev[b]);
  free(c->ev);
  if (c->ev_refl) cudaEventDestroy(c->ev_refl);
  if (c->ev_start) cudaEventDestroy(c->ev_start);
  if (c->dflag) cudaFree(c->dflag);
  if (c->hflag) cudaFreeHost(c->hflag);
  if (c->stream) cudaStreamDestroy(c->stream);
  c->magic = 0;
  free(c);
}

static bsofi_ctx *handle_ctx(const int *h) {
  bsofi_handle hd;
  bsofi_ctx *c;
  if (!h) return NULL;
  memcpy(&hd, h, sizeof(hd));
  if (hd.magic != HANDLE_MAGIC || hd.version != HANDLE_VERSION) return NULL;
  c = (bsofi_ctx *)(uintptr_t)hd.ctx;
  if (!c || c->magic != CTX_MAGIC) return NULL;
  return c;
}

/* ---------------------------------------------------------------- copies */
/* Host (pitch lda) -> device (pitch ldd): `rows` doubles of `cols` columns,
 * through the pinned staging buffers. */
/* True when the host range [p, p + bytes) is page-locked (cudaMallocHost or
 * cudaHostRegister): the DMA engine then reads or writes it directly. */
static int host_pinned(const void *p, size_t bytes) {
  struct cudaPointerAttributes a;
  const char *q = (const char *)p;
  if (bytes == 0) return 0;
  if (cudaPointerGetAttributes(&a, q) != cudaSuccess || a.type != cudaMemoryTypeHost) {
    cudaGetLastError();
    return 0;
  }
  if (cudaPointerGetAttributes(&a, q + bytes - 1) != cudaSuccess || a.type != cudaMemoryTypeHost) {
    cudaGetLastError();
    return 0;
  }
  return 1;
}

/* Span of a column-major host block (rows x cols, pitch lda doubles). */
static size_t host_span(int lda, int rows, int cols) {
  return cols > 0 ? ((size_t)(cols - 1) * lda + rows) * sizeof(double) : 0;
}

static cudaError_t h2d_cols(bsofi_ctx *c, double *dst, int ldd, const double *src, int lda,
                            int rows, int cols) {
  const size_t es = sizeof(double), w = (size_t)rows * es;
  int c0, cpc;
  cudaError_t e;
  if (cols <= 0 || rows <= 0) return cudaSuccess;
  if (!c->stage[1] || host_pinned(src, host_span(lda, rows, cols)))
    return cudaMemcpy2DAsync(dst, es * ldd, src, es * lda, w, cols, cudaMemcpyHostToDevice,
                             c->stream);
  cpc = (int)(STAGE_BYTES / w);
  if (cpc < 1) cpc = 1;
  for (c0 = 0; c0 < cols; c0 += cpc) {
    const int nc = cols - c0 < cpc ? cols - c0 : cpc, b = c->stage_next;
    c->stage_next ^= 1;
    if ((e = cudaEventSynchronize(c->stage_ev[b])) != cudaSuccess) return e;
    par_copy2d(c->pool, c->stage[b], w, (const char *)(src + (size_t)c0 * lda), es * lda, w, nc);
    e = cudaMemcpy2DAsync(dst + (size_t)c0 * ldd, es * ldd, c->stage[b], w, w, nc,
                          cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaEventRecord(c->stage_ev[b], c->stream);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

/* Device (pitch ldd) -> host (pitch lda), pipelined: the DMA of chunk i+1
 * runs while the host threads unpack chunk i.  Returns when all of it is on
 * the host. */
static cudaError_t d2h_cols(bsofi_ctx *c, double *dst, int lda, const double *src, int ldd,
                            int rows, int cols) {
  const size_t es = sizeof(double), w = (size_t)rows * es;
  int i, nchunks, cpc, prev_c0 = 0, prev_nc = 0, prev_b = 0;
  cudaError_t e;
  if (cols <= 0 || rows <= 0) return cudaSuccess;
  if (!c->stage[1] || host_pinned(dst, host_span(lda, rows, cols))) {
    e = cudaMemcpy2DAsync(dst, es * lda, src, es * ldd, w, cols, cudaMemcpyDeviceToHost,
                          c->stream);
    return e == cudaSuccess ? cudaStreamSynchronize(c->stream) : e;
  }
  cpc = (int)(STAGE_BYTES / w);
  if (cpc < 1) cpc = 1;
  nchunks = (cols + cpc - 1) / cpc;
  /* Iteration i issues the DMA of chunk i (if any) and unpacks chunk i-1. */
  for (i = 0; i <= nchunks; i++) {
    if (i < nchunks) {
      const int c0 = i * cpc, nc = cols - c0 < cpc ? cols - c0 : cpc, b = c->stage_next;
      c->stage_next ^= 1;
      if ((e = cudaEventSynchronize(c->stage_ev[b])) != cudaSuccess) return e;
      e = cudaMemcpy2DAsync(c->stage[b], w, src + (size_t)c0 * ldd, es * ldd, w, nc,
                            cudaMemcpyDeviceToHost, c->stream);
      if (e == cudaSuccess) e = cudaEventRecord(c->stage_ev[b], c->stream);
      if (e != cudaSuccess) return e;
      if (i > 0) {
        if ((e = cudaEventSynchronize(c->stage_ev[prev_b])) != cudaSuccess) return e;
        par_copy2d(c->pool, (char *)(dst + (size_t)prev_c0 * lda), es * lda, c->stage[prev_b], w,
                   w, prev_nc);
      }
      prev_c0 = c0;
      prev_nc = nc;
      prev_b = b;
    } else {
      if ((e = cudaEventSynchronize(c->stage_ev[prev_b])) != cudaSuccess) return e;
      par_copy2d(c->pool, (char *)(dst + (size_t)prev_c0 * lda), es * lda, c->stage[prev_b], w, w,
                 prev_nc);
    }
  }
  return cudaSuccess;
}

/* H2D of the p-cyclic blocks of the host matrix (every other block zero). */
static cudaError_t upload_pcyclic(bsofi_ctx *c, const double *A, int lda) {
  int n = c->n, L = c->L, k;
  size_t es = sizeof(double);
  cudaError_t e = (cudaError_t)bsofi_dev_zero_structural(n, L, c->dA, c->ldd, c->stream);
  if (e != cudaSuccess) return e;
  (void)es;
  for (k = 0; k < L - 1; k++) { /* diagonal + sub-diagonal block of column block k */
    size_t off_h = (size_t)k * n * lda + (size_t)k * n;
    size_t off_d = (size_t)k * n * c->ldd + (size_t)k * n;
    if ((e = h2d_cols(c, c->dA + off_d, c->ldd, A + off_h, lda, 2 * n, n)) != cudaSuccess)
      return e;
  }
  /* last column block: corner (0, L-1) and diagonal (L-1, L-1) */
  {
    size_t col_h = (size_t)(L - 1) * n * lda, col_d = (size_t)(L - 1) * n * c->ldd;
    if ((e = h2d_cols(c, c->dA + col_d, c->ldd, A + col_h, lda, n, n)) != cudaSuccess) return e;
    e = h2d_cols(c, c->dA + col_d + (size_t)(L - 1) * n, c->ldd, A + col_h + (size_t)(L - 1) * n,
                 lda, n, n);
  }
  return e;
}

/* The BSOFTRI state: rows 0 .. min(N, (k+2)n) of every column block k. */
static cudaError_t copy_state(bsofi_ctx *c, double *A, int lda, int to_host) {
  int n = c->n, L = c->L, N = n * L, k;
  size_t es = sizeof(double);
  cudaError_t e = cudaSuccess;
  if (host_pinned(A, host_span(lda, N, N))) {
    /* Page-locked caller array: direct DMA of every block column, one wait. */
    for (k = 0; k < L && e == cudaSuccess; k++) {
      int rows = (k + 2) * n < N ? (k + 2) * n : N;
      double *h = A + (size_t)k * n * lda;
      double *d = c->dA + (size_t)k * n * c->ldd;
      if (to_host)
        e = cudaMemcpy2DAsync(h, es * lda, d, es * c->ldd, es * rows, n, cudaMemcpyDeviceToHost,
                              c->stream);
      else
        e = cudaMemcpy2DAsync(d, es * c->ldd, h, es * lda, es * rows, n, cudaMemcpyHostToDevice,
                              c->stream);
    }
    if (e == cudaSuccess && to_host) e = cudaStreamSynchronize(c->stream);
    return e;
  }
  for (k = 0; k < L; k++) {
    int rows = (k + 2) * n < N ? (k + 2) * n : N;
    double *h = A + (size_t)k * n * lda;
    double *d = c->dA + (size_t)k * n * c->ldd;
    if (to_host)
      e = d2h_cols(c, h, lda, d, c->ldd, rows, n);
    else
      e = h2d_cols(c, d, c->ldd, h, lda, rows, n);
    if (e != cudaSuccess) return e;
  }
  return e;
}

/* ---------------------------------------------------------------- checks */
static int check_args(const int *h_ok, int n, int L, const double *A, int lda,
                      const double *tau, const double *work, int lwork, int first_arg) {
  /* first_arg: position of n in the argument list (2 with a handle). */
  if (h_ok && !*h_ok) return -1;
  if (n < 1 || n > BSOFI_MAX_BLOCK) return -(first_arg);
  if (L < 2 || (long long)n * L > 1000000) return -(first_arg + 1);
  if (!A) return -(first_arg + 2);
  if (lda < n * L) return -(first_arg + 3);
  if (!tau) return -(first_arg + 4);
  if ((lwork == -1 || lwork == -2) && !work) return -(first_arg + 5);
  if (lwork < 1 && lwork != -1 && lwork != -2) return -(first_arg + 6);
  return 0;
}

/* Reads the BSTRI info word and the BSOF and BSOI error words (a bounded
 * wait inside a persistent kernel that gave up) after synchronising the
 * stream. */
static int read_info(bsofi_ctx *c, int *info) {
  int v[4] = {0, 0, 0, 0};
  cudaError_t e = cudaMemcpyAsync(v, bsofi_dev_info_ptr(c->dws), sizeof(v),
                                  cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    *info = cuda_info(e);
    return *info;
  }
  if (v[1] != 0 || v[2] != 0 || v[3] != 0) {
    *info = cuda_info(cudaErrorLaunchTimeout);
    return *info;
  }
  *info = v[0] >= 0x7f7f7f7f ? 0 : v[0];
  return *info;
}

/* ------------------------------------------------------- phase drivers */
/* BSOF (+ BSTRI when do_tri) on host A; returns info. */
static int drive_bsoftri(bsofi_ctx *c, int n, int L, double *A, int lda, double *tau,
                         int do_bsof, int do_tri) {
  cudaError_t e;
  int info = 0, N = n * L;
  if ((e = ctx_fit(c, n, L)) != cudaSuccess) return cuda_info(e);
  if (do_bsof) {
    if ((e = upload_pcyclic(c, A, lda)) != cudaSuccess) return cuda_info(e);
  } else {
    if ((e = copy_state(c, A, lda, 0)) != cudaSuccess) return cuda_info(e);
  }
  c->g_valid = 0;
  if (do_bsof && do_tri) {
    /* The workers also form every G_k (off the critical chain) for the BSOI
     * call that usually follows; dref records what they were formed from. */
    e = (cudaError_t)bsofi_dev_bsoftri_q(n, L, c->dA, c->ldd, c->dtau, c->dws, c->stream);
    if (e == cudaSuccess)
      e = (cudaError_t)bsofi_dev_state_ref(n, L, c->dA, c->ldd, c->dtau, c->dref, 0, c->dflag,
                                           c->stream);
    if (e == cudaSuccess) c->g_valid = 1;
  } else if (do_bsof)
    e = (cudaError_t)bsofi_dev_bsof(n, L, c->dA, c->ldd, c->dtau, c->dws, c->stream);
  else
    e = (cudaError_t)bsofi_dev_bstri(n, L, c->dA, c->ldd, c->dws, c->stream);
  if (e != cudaSuccess) return cuda_info(e);
  if ((e = copy_state(c, A, lda, 1)) != cudaSuccess) return cuda_info(e);
  if (do_bsof) {
    e = cudaMemcpyAsync(tau, c->dtau, sizeof(double) * N, cudaMemcpyDeviceToHost, c->stream);
    if (e != cudaSuccess) return cuda_info(e);
  }
  if (do_tri) return read_info(c, &info);
  if (do_bsof) {
    read_info(c, &info);
    return info < 0 ? info : 0;
  }
  e = cudaStreamSynchronize(c->stream);
  return e == cudaSuccess ? 0 : cuda_info(e);
}

/* After the reflector rows and tau of a state are on the device (ordered
 * before `st`): 1 if they are the ones the workspace's G_k were formed from. */
static int state_matches(bsofi_ctx *c, int n, int L, cudaStream_t st) {
  if (!c->g_valid) return 0;
  if (cudaMemsetAsync(c->dflag, 0, sizeof(int), st) != cudaSuccess) return 0;
  if (bsofi_dev_state_ref(n, L, c->dA, c->ldd, c->dtau, c->dref, 1, c->dflag, st) != 0) return 0;
  if (cudaMemcpyAsync(c->hflag, c->dflag, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return 0;
  if (cudaStreamSynchronize(st) != cudaSuccess) return 0;
  return *c->hflag == 0;
}

/* Streams and L events of each kind for the pipelined BSOI. */
static cudaError_t pipe_fit(bsofi_ctx *c, int L) {
  cudaError_t e = cudaSuccess;
  int i;
  if (!c->s_in && (e = cudaStreamCreateWithFlags(&c->s_in, cudaStreamNonBlocking)) != cudaSuccess)
    return e;
  if (!c->s_out && (e = cudaStreamCreateWithFlags(&c->s_out, cudaStreamNonBlocking)) != cudaSuccess)
    return e;
  if (!c->ev_refl && (e = cudaEventCreateWithFlags(&c->ev_refl, cudaEventDisableTiming)) != cudaSuccess)
    return e;
  if (!c->ev_start && (e = cudaEventCreateWithFlags(&c->ev_start, cudaEventDisableTiming)) != cudaSuccess)
    return e;
  if (c->nev >= L) return cudaSuccess;
  for (i = 0; i < 2 * c->nev; i++) cudaEventDestroy(c->ev[i]);
  free(c->ev);
  c->nev = 0;
  c->ev = (cudaEvent_t *)calloc(2 * (size_t)L, sizeof(cudaEvent_t));
  if (!c->ev) return cudaErrorMemoryAllocation;
  for (i = 0; i < 2 * L; i++) {
    if ((e = cudaEventCreateWithFlags(&c->ev[i], cudaEventDisableTiming)) != cudaSuccess) {
      while (--i >= 0) cudaEventDestroy(c->ev[i]);
      free(c->ev);
      c->ev = NULL;
      return e;
    }
  }
  c->nev = L;
  return cudaSuccess;
}

/* BSOI on a page-locked caller array, as a three-stream pipeline:
 *   copy-in:  tau and the reflector rows of every block column (what Q
 *             formation reads), then the rest of block columns L-1, ..., 0;
 *   compute:  Q formation, then step k as soon as block column k is on the
 *             device (one GEMM launch per step);
 *   copy-out: block column k+1 as soon as step k has finished it.
 * The upload of later block columns and the download of finished ones run
 * under the GEMM steps. */
static cudaError_t bsoi_pipelined(bsofi_ctx *c, int n, int L, double *A, int lda,
                                  const double *tau) {
  const size_t es = sizeof(double), sh = es * (size_t)lda, sd = es * (size_t)c->ldd;
  const int N = n * L;
  cudaError_t e;
  int k, r;
  if ((e = pipe_fit(c, L)) != cudaSuccess) return e;
  cudaEvent_t *up = c->ev, *done = c->ev + c->nev;
  /* Copies start after whatever the context's stream still has queued. */
  if ((e = cudaEventRecord(c->ev_start, c->stream)) != cudaSuccess) return e;
  if ((e = cudaStreamWaitEvent(c->s_in, c->ev_start, 0)) != cudaSuccess) goto drain;
  if ((e = cudaStreamWaitEvent(c->s_out, c->ev_start, 0)) != cudaSuccess) goto drain;
  e = cudaMemcpyAsync(c->dtau, tau, es * N, cudaMemcpyHostToDevice, c->s_in);
  for (k = 0; k < L && e == cudaSuccess; k++) {
    const int r0 = k * n, r1 = (k + 2) * n < N ? (k + 2) * n : N;
    e = cudaMemcpy2DAsync(c->dA + (size_t)k * n * c->ldd + r0, sd, A + (size_t)k * n * lda + r0,
                          sh, es * (r1 - r0), n, cudaMemcpyHostToDevice, c->s_in);
  }
  if (e == cudaSuccess) e = cudaEventRecord(c->ev_refl, c->s_in);
  for (k = L - 1; k >= 0 && e == cudaSuccess; k--) {
    if (k > 0)
      e = cudaMemcpy2DAsync(c->dA + (size_t)k * n * c->ldd, sd, A + (size_t)k * n * lda, sh,
                            es * (size_t)k * n, n, cudaMemcpyHostToDevice, c->s_in);
    if (e == cudaSuccess) e = cudaEventRecord(up[k], c->s_in);
  }
  if (e != cudaSuccess) goto drain;
  /* compute */
  if ((e = cudaStreamWaitEvent(c->stream, c->ev_refl, 0)) != cudaSuccess) goto drain;
  if (!state_matches(c, n, L, c->stream)) {
    if ((r = bsofi_dev_bsoi_form_q(n, L, c->dA, c->ldd, c->dtau, c->dws, c->stream)) != 0) {
      e = (cudaError_t)r;
      goto drain;
    }
    /* The workspace's G_k now belong to this state. */
    if ((r = bsofi_dev_state_ref(n, L, c->dA, c->ldd, c->dtau, c->dref, 0, c->dflag,
                                 c->stream)) != 0) {
      e = (cudaError_t)r;
      goto drain;
    }
    c->g_valid = 1;
  }
  if ((e = cudaStreamWaitEvent(c->stream, up[L - 1], 0)) != cudaSuccess) goto drain;
  if ((r = bsofi_dev_bsoi_carry(n, L, c->dA, c->ldd, c->dws, c->stream)) != 0) {
    e = (cudaError_t)r;
    goto drain;
  }
  for (k = L - 2; k >= 0; k--) {
    if ((e = cudaStreamWaitEvent(c->stream, up[k], 0)) != cudaSuccess) goto drain;
    if ((r = bsofi_dev_bsoi_step(n, L, k, c->dA, c->ldd, c->dws, c->stream)) != 0) {
      e = (cudaError_t)r;
      goto drain;
    }
    if ((e = cudaEventRecord(done[k + 1], c->stream)) != cudaSuccess) goto drain;
  }
  if ((r = bsofi_dev_bsoi_finish(n, L, c->dA, c->ldd, c->dws, c->stream)) != 0) {
    e = (cudaError_t)r;
    goto drain;
  }
  if ((e = cudaEventRecord(done[0], c->stream)) != cudaSuccess) goto drain;
  /* copy-out, right to left as the block columns finish */
  for (k = L - 1; k >= 0 && e == cudaSuccess; k--) {
    e = cudaStreamWaitEvent(c->s_out, done[k], 0);
    if (e == cudaSuccess)
      e = cudaMemcpy2DAsync(A + (size_t)k * n * lda, sh, c->dA + (size_t)k * n * c->ldd, sd,
                            es * N, n, cudaMemcpyDeviceToHost, c->s_out);
  }
drain: {
  /* Nothing may still touch the caller's arrays when this returns. */
  cudaError_t e1 = cudaStreamSynchronize(c->s_in);
  cudaError_t e2 = cudaStreamSynchronize(c->s_out);
  cudaError_t e3 = cudaStreamSynchronize(c->stream);
  if (e == cudaSuccess) e = e1 != cudaSuccess ? e1 : (e2 != cudaSuccess ? e2 : e3);
}
  return e;
}

static int drive_bsoi(bsofi_ctx *c, int n, int L, double *A, int lda, const double *tau) {
  cudaError_t e;
  int N = n * L;
  if ((e = ctx_fit(c, n, L)) != cudaSuccess) return cuda_info(e);
  if (L >= 2 && host_pinned(A, host_span(lda, N, N))) {
    int info = 0;
    if ((e = bsoi_pipelined(c, n, L, A, lda, tau)) != cudaSuccess) return cuda_info(e);
    return read_info(c, &info) < 0 ? info : 0;
  }
  if ((e = copy_state(c, A, lda, 0)) != cudaSuccess) return cuda_info(e);
  e = cudaMemcpyAsync(c->dtau, tau, sizeof(double) * N, cudaMemcpyHostToDevice, c->stream);
  if (e != cudaSuccess) return cuda_info(e);
  {
    const int q_ready = state_matches(c, n, L, c->stream);
    if (!q_ready) c->g_valid = 0;
    e = (cudaError_t)bsofi_dev_bsoi_ex(n, L, c->dA, c->ldd, c->dtau, c->dws, c->stream, q_ready);
  }
  if (e != cudaSuccess) return cuda_info(e);
  e = d2h_cols(c, A, lda, c->dA, c->ldd, N, N);
  if (e != cudaSuccess) return cuda_info(e);
  {
    int info = 0;
    return read_info(c, &info) < 0 ? info : 0;
  }
}

/* ================================================================ handle API */
int hybridxinith_(int *handle, int *n, int *L, int *lda) {
  bsofi_handle hd;
  bsofi_ctx *c;
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

int hybridxbsoftrih_(int *handle, int *n, int *L, double *A, int *lda, double *tau,
                     double *work, int *lwork, int *info) {
  bsofi_ctx *c = handle_ctx(handle);
  int ok = c != NULL, r;
  if (!info) return -9;
  if (!n || !L || !lda || !lwork) {
    *info = !n ? -2 : !L ? -3 : !lda ? -5 : -8;
    return *info;
  }
  r = check_args(&ok, *n, *L, A, *lda, tau, work, *lwork, 2);
  if (r) return *info = r;
  if (*lwork == -1) {
    work[0] = 1.0;
    return *info = 0;
  }
  if (*lwork == -2) {
    work[0] = device_lwork(*n, *L);
    return *info = 0;
  }
  return *info = drive_bsoftri(c, *n, *L, A, *lda, tau, 1, 1);
}

int hybridxbsoih_(int *handle, int *n, int *L, double *A, int *lda, double *tau, double *work,
                  int *lwork, int *info) {
  bsofi_ctx *c = handle_ctx(handle);
  int ok = c != NULL, r;
  if (!info) return -9;
  if (!n || !L || !lda || !lwork) {
    *info = !n ? -2 : !L ? -3 : !lda ? -5 : -8;
    return *info;
  }
  r = check_args(&ok, *n, *L, A, *lda, tau, work, *lwork, 2);
  if (r) return *info = r;
  if (*lwork == -1) {
    work[0] = 1.0;
    return *info = 0;
  }
  if (*lwork == -2) {
    work[0] = device_lwork(*n, *L);
    return *info = 0;
  }
  return *info = drive_bsoi(c, *n, *L, A, *lda, tau);
}

int hybridxfinalizeh_(int *handle) {
  bsofi_ctx *c = handle_ctx(handle);
  if (c) ctx_destroy(c);
  if (handle) memset(handle, 0, sizeof(bsofi_handle));
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
static __thread bsofi_ctx *t_ctx = NULL;

static bsofi_ctx *thread_ctx(int n, int L, int *info) {
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
  if (lworkHostDevice == -2) {
    const double w = device_lwork(n, L);
    return w > (double)INT_MAX ? INT_MAX : (int)w;
  }
  return 1;
}

static int c_phase(int n, int L, double *A, int lda, double *tau, double *work, int lwork,
                   int *info, int phase) {
  int r, tmp = 0;
  bsofi_ctx *c;
  if (!info) info = &tmp;
  r = check_args(NULL, n, L, A, lda, phase == 1 ? A : tau, work, lwork, 1);
  if (r) return *info = r;
  if (lwork == -1 || lwork == -2) {
    work[0] = lwork == -1 ? 1.0 : device_lwork(n, L);
    return *info = 0;
  }
  c = thread_ctx(n, L, info);
  if (!c) return *info;
  if (phase == 0) return *info = drive_bsoftri(c, n, L, A, lda, tau, 1, 0);
  if (phase == 1) return *info = drive_bsoftri(c, n, L, A, lda, tau, 0, 1);
  if (phase == 2) return *info = drive_bsoftri(c, n, L, A, lda, tau, 1, 1);
  return *info = drive_bsoi(c, n, L, A, lda, tau);
}

int lapackXbsof(int n, int L, double A[], int lda, double tau[], double work[], int lwork,
                int *info) {
  return c_phase(n, L, A, lda, tau, work, lwork, info, 0);
}

int lapackXbstri(int n, int L, double A[], int lda, int *info) {
  double w = 0.0;
  return c_phase(n, L, A, lda, NULL, &w, 1, info, 1);
}

int lapackXbsoi_ormqr(int n, int L, double A[], int lda, double tau[], double work[], int lwork,
                      int *info) {
  return c_phase(n, L, A, lda, tau, work, lwork, info, 3);
}

int lapackXbsoi_orgqr(int n, int L, double A[], int lda, double tau[], double work[], int lwork,
                      int *info) {
  return c_phase(n, L, A, lda, tau, work, lwork, info, 3);
}

int lapackxbsofilwork_(int *n, int *L, int *lda) { return lapackXbsofiLWork(*n, *L, *lda); }
int lapackxbsof_(int *n, int *L, double A[], int *lda, double tau[], double work[], int *lwork,
                 int *info) {
  return lapackXbsof(*n, *L, A, *lda, tau, work, *lwork, info);
}
int lapackxbstri_(int *n, int *L, double A[], int *lda, int *info) {
  return lapackXbstri(*n, *L, A, *lda, info);
}
int lapackxbsoi_ormqr_(int *n, int *L, double A[], int *lda, double tau[], double work[],
                       int *lwork, int *info) {
  return lapackXbsoi_ormqr(*n, *L, A, *lda, tau, work, *lwork, info);
}
int lapackxbsoi_orgqr_(int *n, int *L, double A[], int *lda, double tau[], double work[],
                       int *lwork, int *info) {
  return lapackXbsoi_orgqr(*n, *L, A, *lda, tau, work, *lwork, info);
}

int hybridXbsoftri(int handle, int n, int L, double A[], int lda, double tau[], double work[],
                   int lwork, double dwork[], int ldwork, int *info) {
  (void)handle;
  (void)dwork;
  (void)ldwork;
  return c_phase(n, L, A, lda, tau, work, lwork, info, 2);
}

int hybridXbsoi(int handle, int n, int L, double A[], int lda, double tau[], double work[],
                int lwork, double dwork[], int ldwork, int *info) {
  (void)handle;
  (void)dwork;
  (void)ldwork;
  return c_phase(n, L, A, lda, tau, work, lwork, info, 3);
}

/* Fortran twins of the hybridX names (the reference's cb_hybridXbsofiLWork,
 * cb_hybridXbsoftri, cb_hybridXbsoi, src/bsofi_callback.c:62-87): every
 * argument by pointer; the cuBLAS handle is not passed. */
int hybridxbsofilwork_(int *n, int *L, int *lda, int *lworkHostDevice) {
  if (!n || !L || !lda || !lworkHostDevice) return 1;
  return hybridXbsofiLWork(*n, *L, *lda, *lworkHostDevice);
}
int hybridxbsoftri_(int *n, int *L, double A[], int *lda, double tau[], double work[], int *lwork,
                    double dwork[], int *ldwork, int *info) {
  if (!info) return -10;
  if (!n || !L || !lda || !lwork || !ldwork) {
    *info = !n ? -1 : !L ? -2 : !lda ? -4 : !lwork ? -7 : -9;
    return *info;
  }
  return hybridXbsoftri(0, *n, *L, A, *lda, tau, work, *lwork, dwork, *ldwork, info);
}
int hybridxbsoi_(int *n, int *L, double A[], int *lda, double tau[], double work[], int *lwork,
                 double dwork[], int *ldwork, int *info) {
  if (!info) return -10;
  if (!n || !L || !lda || !lwork || !ldwork) {
    *info = !n ? -1 : !L ? -2 : !lda ? -4 : !lwork ? -7 : -9;
    return *info;
  }
  return hybridXbsoi(0, *n, *L, A, *lda, tau, work, *lwork, dwork, *ldwork, info);
}

/* ------------------------------------------------------ device-pointer API */
static int gpu_phase(int n, int L, double *dA, int ldda, double *tau, int *info, int phase) {
  int tmp = 0, N = n * L;
  bsofi_ctx *c;
  cudaError_t e;
  if (!info) info = &tmp;
  if (n < 1 || n > BSOFI_MAX_BLOCK) return *info = -1;
  if (L < 2) return *info = -2;
  if (!dA) return *info = -3;
  if (ldda < N) return *info = -4;
  if (phase != 1 && !tau) return *info = -5;
  c = thread_ctx(n, L, info);
  if (!c) return *info;
  if ((e = ctx_fit(c, n, L)) != cudaSuccess) return *info = cuda_info(e);
  if (phase == 0) {
    e = (cudaError_t)bsofi_dev_bsof(n, L, dA, ldda, c->dtau, c->dws, c->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(tau, c->dtau, sizeof(double) * N, cudaMemcpyDeviceToHost, c->stream);
  } else if (phase == 1) {
    e = (cudaError_t)bsofi_dev_bstri(n, L, dA, ldda, c->dws, c->stream);
    if (e == cudaSuccess) return read_info(c, info);
  } else {
    e = cudaMemcpyAsync(c->dtau, tau, sizeof(double) * N, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
      e = (cudaError_t)bsofi_dev_bsoi(n, L, dA, ldda, c->dtau, c->dws, c->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  return *info = (e == cudaSuccess ? 0 : cuda_info(e));
}

int gpuXbsof(int n, int L, double dA[], int ldda, double tau[], double work[], int lwork,
             double *dT, int *info) {
  (void)dT;
  if (lwork == -1 || lwork == -2) {
    if (!work) return info ? (*info = -6) : -6;
    work[0] = lwork == -1 ? 1.0 : (double)bsofi_dev_ws_bytes(n, L, ldda) / sizeof(double);
    return info ? (*info = 0) : 0;
  }
  return gpu_phase(n, L, dA, ldda, tau, info, 0);
}

int gpuXbstri_rseq(int n, int L, double dA[], int ldda, double dwork[], int ldwork, int *info) {
  (void)dwork;
  (void)ldwork;
  return gpu_phase(n, L, dA, ldda, NULL, info, 1);
}

int gpuXbstri_rbatched(int n, int L, double dA[], int ldda, double dwork[], int ldwork,
                       int *info) {
  return gpuXbstri_rseq(n, L, dA, ldda, dwork, ldwork, info);
}

int gpuXbsoi_ormqr(int n, int L, double dA[], int ldda, double tau[], double work[], int lwork,
                   double *dT, double dwork[], int ldwork, int *info) {
  (void)dT;
  (void)dwork;
  (void)ldwork;
  if (lwork == -1 || lwork == -2) {
    if (!work) return info ? (*info = -6) : -6;
    work[0] = lwork == -1 ? 1.0 : (double)bsofi_dev_ws_bytes(n, L, ldda) / sizeof(double);
    return info ? (*info = 0) : 0;
  }
  return gpu_phase(n, L, dA, ldda, tau, info, 2);
}

int gpuXbsoi_orgqr(int n, int L, double dA[], int ldda, double tau[], double work[], int lwork,
                   double *dT, double dwork[], int ldwork, int *info) {
  return gpuXbsoi_ormqr(n, L, dA, ldda, tau, work, lwork, dT, dwork, ldwork, info);
}

int gpuXbsoi_batched(int n, int L, double dA[], int ldda, double tau[], double work[],
                     int lwork, double *dT, double dwork[], int ldwork, int *info) {
  return gpuXbsoi_ormqr(n, L, dA, ldda, tau, work, lwork, dT, dwork, ldwork, info);
}

/* ------------------------------------------------------ async device API */
unsigned long long bsofi_device_workspace_bytes(int n, int L, int ldda) {
  return (unsigned long long)bsofi_dev_ws_bytes(n, L, ldda);
}

/* Sizes and pointers every device entry point requires. */
static int device_args_ok(int n, int L, const double *dA, int ldda, const double *dtau,
                          const void *dwork) {
  return n >= 1 && n <= BSOFI_MAX_BLOCK && L >= 2 && ldda >= n * L && dA && dtau && dwork;
}

int bsofi_device_bsoftri(int n, int L, double *dA, int ldda, double *dtau, void *dwork,
                         void *stream) {
  int e;
  if (!device_args_ok(n, L, dA, ldda, dtau, dwork)) return -1;
  e = bsofi_dev_prepare();
  if (e) return cuda_info((cudaError_t)e);
  e = bsofi_dev_bsoftri(n, L, dA, ldda, dtau, dwork, stream);
  return e ? cuda_info((cudaError_t)e) : 0;
}

int bsofi_device_bsoi(int n, int L, double *dA, int ldda, const double *dtau, void *dwork,
                      void *stream) {
  int e;
  if (!device_args_ok(n, L, dA, ldda, dtau, dwork)) return -1;
  e = bsofi_dev_prepare();
  if (e) return cuda_info((cudaError_t)e);
  e = bsofi_dev_bsoi(n, L, dA, ldda, dtau, dwork, stream);
  return e ? cuda_info((cudaError_t)e) : 0;
}

int bsofi_device_bsoi_rows(int n, int L, double *dA, int ldda, const double *dtau, void *dwork,
                           int row0, int row1, void *stream) {
  int e, N = n * L;
  if (!device_args_ok(n, L, dA, ldda, dtau, dwork)) return -1;
  if (row0 < 0 || row1 > N || row0 >= row1 || row0 % 128 != 0 || (row1 % 128 != 0 && row1 != N))
    return -1;
  e = bsofi_dev_prepare();
  if (!e) e = bsofi_dev_bsoi_rows(n, L, dA, ldda, dtau, dwork, stream, row0, row1);
  return e ? cuda_info((cudaError_t)e) : 0;
}

/* ---------------------------------------------- storage-sharded inversion */

unsigned long long bsofi_shard_state_bytes(int n, int L) {
  if (n < 1 || n > BSOFI_MAX_BLOCK || L < 2) return 0;
  return (unsigned long long)bsofi_dev_shard_state_bytes(n, L);
}

static int shard_run(int e) { return e ? cuda_info((cudaError_t)e) : 0; }

int bsofi_shard_factor(int n, int L, const double *dD, const double *dS, void *dstate,
                       void *stream) {
  int e;
  if (n < 1 || n > BSOFI_MAX_BLOCK || L < 2 || dS == NULL || dstate == NULL) return -1;
  e = bsofi_dev_prepare();
  if (!e) e = bsofi_dev_shard_factor(n, L, dD, dS, NULL, NULL, 0.0, dstate, stream);
  return shard_run(e);
}

int bsofi_shard_hubbard_factor(int n, int L, const double *dExpK, const double *dh,
                               double lambda, void *dstate, void *stream) {
  int e;
  if (n < 1 || n > BSOFI_MAX_BLOCK || L < 2 || dExpK == NULL || dh == NULL || dstate == NULL)
    return -1;
  e = bsofi_dev_prepare();
  if (!e) e = bsofi_dev_shard_factor(n, L, NULL, NULL, dExpK, dh, lambda, dstate, stream);
  return shard_run(e);
}

int bsofi_shard_bstri_columns(int n, int L, int c0, int c1, double *dX, long long ldx,
                              void *dstate, void *stream) {
  int e;
  if (n < 1 || n > BSOFI_MAX_BLOCK || L < 2 || c0 < 0 || c1 > L || c0 >= c1 || dX == NULL ||
      dstate == NULL || ldx < (long long)c1 * n)
    return -1;
  e = bsofi_dev_prepare();
  if (!e) e = bsofi_dev_shard_bstri_columns(n, L, c0, c1, dX, ldx, dstate, stream);
  return shard_run(e);
}

int bsofi_shard_bsoi_rows(int n, int L, int row0, int row1, double *dB, long long ldb,
                          void *dstate, void *stream) {
  int e, N = n * L;
  if (n < 1 || n > BSOFI_MAX_BLOCK || L < 2 || dB == NULL || dstate == NULL) return -1;
  if (row0 < 0 || row1 > N || row0 >= row1 || row0 % 128 != 0 || (row1 % 128 != 0 && row1 != N) ||
      ldb < row1 - row0)
    return -1;
  e = bsofi_dev_prepare();
  if (!e) e = bsofi_dev_shard_bsoi_rows(n, L, row0, row1, dB, ldb, dstate, stream);
  return shard_run(e);
}

int bsofi_shard_logdet(int n, int L, const void *dstate, double *dout, void *stream) {
  if (n < 1 || n > BSOFI_MAX_BLOCK || L < 2 || dstate == NULL || dout == NULL) return -1;
  return shard_run(bsofi_dev_shard_logdet(n, L, dstate, dout, stream));
}

int *bsofi_shard_info(void *dstate) { return dstate ? bsofi_dev_info_ptr(dstate) : NULL; }

const double *bsofi_shard_tau(const void *dstate, int n, int L) {
  if (dstate == NULL || n < 1 || n > BSOFI_MAX_BLOCK || L < 2) return NULL;
  return bsofi_dev_shard_tau(dstate, n, L);
}

int bsofi_device_invert(int n, int L, double *dA, int ldda, double *dtau, void *dwork,
                        void *stream) {
  int e;
  if (!device_args_ok(n, L, dA, ldda, dtau, dwork)) return -1;
  e = bsofi_dev_prepare();
  if (!e) e = bsofi_dev_invert(n, L, dA, ldda, dtau, dwork, stream);
  return e ? cuda_info((cudaError_t)e) : 0;
}

static int mixed_slices(int slices) { return slices == 0 ? BSOFI_MIXED_SLICES : slices; }

unsigned long long bsofi_device_workspace_bytes_mixed(int n, int L, int ldda, int slices) {
  slices = mixed_slices(slices);
  if (n < 1 || n > BSOFI_MAX_BLOCK || L < 2 || ldda < n * L || slices < 3 || slices > 8) return 0;
  return (unsigned long long)bsofi_dev_ws_bytes_mixed(n, L, ldda, slices);
}

int bsofi_device_invert_mixed(int n, int L, double *dA, int ldda, double *dtau, void *dwork,
                              int slices, void *stream) {
  int e;
  slices = mixed_slices(slices);
  if (!device_args_ok(n, L, dA, ldda, dtau, dwork) || slices < 3 || slices > 8) return -1;
  e = bsofi_dev_prepare();
  if (!e) e = bsofi_dev_invert_mixed(n, L, dA, ldda, dtau, dwork, stream, 0, slices);
  return e ? cuda_info((cudaError_t)e) : 0;
}

unsigned long long bsofi_selftest_ozaki_scratch_bytes(int M, int N, int K, int slices) {
  return (unsigned long long)bsofi_dev_ozaki_scratch_bytes(M, N, K, mixed_slices(slices));
}

int bsofi_selftest_ozaki(int M, int N, int K, const double *dA, int lda, const double *dB, int ldb,
                         double *dC, int ldc, int slices, void *dscratch, int *derr,
                         void *stream) {
  int e;
  slices = mixed_slices(slices);
  if (M < 1 || N < 1 || K < 1 || K > 1536 || lda < M || ldb < K || ldc < M || !dA || !dB ||
      !dC || !dscratch || !derr || slices < 3 || slices > 8)
    return -1;
  e = bsofi_dev_selftest_ozaki(M, N, K, dA, lda, dB, ldb, dC, ldc, slices, dscratch, derr,
                               stream);
  return e ? cuda_info((cudaError_t)e) : 0;
}

int *bsofi_device_info(void *dwork) { return bsofi_dev_info_ptr(dwork); }

long long bsofi_device_last_launches(void) { return bsofi_dev_launch_count(); }

int bsofi_selftest_gemm(int M, int N, int K, double alpha, const double *dA, int lda,
                        int upper_a, const double *dB, int ldb, int upper_b, double beta,
                        double *dC, int ldc, int tile, void *stream) {
  int e = bsofi_dev_prepare();
  if (!e)
    e = bsofi_dev_selftest_gemm(M, N, K, alpha, dA, lda, upper_a, dB, ldb, upper_b, beta, dC,
                                ldc, tile, stream);
  return e ? cuda_info((cudaError_t)e) : 0;
}

void bsofi_device_timing(int on) { bsofi_dev_timing(on); }

int bsofi_device_timing_read(double *ms, long long *launches) {
  int e = bsofi_dev_timing_read(ms, launches);
  return e ? cuda_info((cudaError_t)e) : 0;
}

int bsofi_device_bsof_timeline(int n, int L, int ldda, void *dwork, unsigned long long *host,
                               int max_leaves) {
  unsigned long long *d = NULL;
  int leaves = bsofi_dev_bsof_timeline(n, L, ldda, dwork, &d);
  int cnt = leaves < max_leaves ? leaves : max_leaves;
  cudaError_t e = cudaMemcpy(host, d, sizeof(unsigned long long) * 4 * (size_t)cnt,
                             cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? cnt : cuda_info(e);
}

void bsofi_device_set_bsof_workers(int workers) { bsofi_dev_set_bsof_workers(workers); }

void bsofi_device_set_bstri_overlap(int on) { bsofi_dev_set_bstri_overlap(on); }

void bsofi_device_set_bsof_factor_warps(int warps) { bsofi_dev_set_bsof_factor_warps(warps); }

void bsofi_device_set_gemm_k16(int on) { bsofi_dev_set_gemm_k16(on); }

void bsofi_device_set_bsoi_tma(int on) { bsofi_dev_set_bsoi_tma(on); }

void bsofi_device_set_wait_test(int on) { bsofi_dev_set_wait_test(on); }
