/*
 * server.c -- continuous-batching inversion server.
 *
 * DQMC production runs and parameter sweeps produce a stream of inversion
 * requests of different sizes (n = lattice sites, L = time slices).  The
 * reference has no serving layer: each call is synchronous
 * (src/bsofi_callback.c:130-157).  This server keeps every request's matrix
 * and result resident in HBM (the caller owns them), runs up to `slots`
 * requests at once (one stream each, so their kernels overlap on the
 * device), and admits queued requests as slots and workspace memory free up:
 *   * workspace comes from one device pool allocated at creation, handed out
 *     first-fit; a request is admitted only when its workspace fits
 *     (admission by memory footprint);
 *   * admission is FIFO, but a request that does not fit may be passed by
 *     smaller ones behind it at most BYPASS_LIMIT times, after which nothing
 *     is admitted until it fits (no starvation);
 *   * a request whose workspace exceeds the whole pool fails at submission.
 * Two kinds of request:
 *   * caller-owned (bsofi_server_submit): the caller's matrix is inverted in
 *     place; the pool holds only the workspace;
 *   * server-owned (bsofi_server_submit_blocks): the request is given by its
 *     packed p-cyclic blocks; at admission the pool supplies the matrix, tau
 *     and the workspace together (admission by the full memory footprint, up
 *     to 17 GB for n = 576, L = 80), the matrix is assembled in the pool and
 *     inverted there; the workspace returns to the pool when the inversion
 *     ends, the matrix and tau stay resident until bsofi_server_release.
 * Precision 0 runs the FP64 pipeline, 1 the mixed one (BSOI on the int8
 * tensor cores, bsofi_device_invert_mixed).
 * Progress is driven by bsofi_server_poll (no background thread): it retires
 * finished requests (event query, no device synchronisation) and admits new
 * ones.  One server is used by one host thread at a time.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <cuda_runtime_api.h>

#include "../../include/bsofi_b200.h"
#include "bsofi_device.h"

#define MAX_SLOTS 64
#define BYPASS_LIMIT 16

typedef struct {
  long long id;
  int n, L, ldda, precision;
  double *dA, *dtau;  /* caller-owned request: the caller's buffers */
  const double *dD, *dS; /* server-owned request: packed blocks (until admission) */
  int owned;
  size_t ws;  /* workspace bytes */
  size_t mat; /* server-owned: matrix + tau bytes, 0 otherwise */
} request;

typedef struct {
  int busy;
  long long id;
  size_t off, len;         /* workspace in the pool */
  size_t moff, mlen;       /* server-owned matrix + tau in the pool (mlen 0: none) */
  int ldda, n, L;
  cudaStream_t stream;
  cudaStream_t hi;       /* highest priority: the request's factorization chain */
  cudaEvent_t handoff;   /* chain done on hi -> BSTRI and BSOI on stream */
  cudaEvent_t done;
  int *hinfo; /* pinned: BSTRI info word, BSOF / BSOI / BSTRI wait error words */
} slot;

/* A finished server-owned request whose matrix and tau are still resident. */
typedef struct {
  long long id;
  size_t moff, mlen;
  int ldda, N;
} resident;

typedef struct {
  size_t off, len;
} span;

struct bsofi_server {
  int device, nslots;
  slot s[MAX_SLOTS];
  char *pool;
  size_t pool_bytes;
  span *free_list;
  int nfree, cap_free;
  request *queue;
  int qhead, qlen, qcap;
  int bypassed;
  long long next_id;
  resident *res;
  int nres, cap_res;
};

typedef struct bsofi_server bsofi_server;

static size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

/* ------------------------------------------------------------ pool */
static int pool_alloc(bsofi_server *sv, size_t len, size_t *off) {
  int i;
  for (i = 0; i < sv->nfree; i++) {
    if (sv->free_list[i].len >= len) {
      *off = sv->free_list[i].off;
      sv->free_list[i].off += len;
      sv->free_list[i].len -= len;
      if (sv->free_list[i].len == 0) {
        memmove(&sv->free_list[i], &sv->free_list[i + 1], sizeof(span) * (sv->nfree - i - 1));
        sv->nfree--;
      }
      return 1;
    }
  }
  return 0;
}

static int pool_free(bsofi_server *sv, size_t off, size_t len) {
  int i = 0, j;
  while (i < sv->nfree && sv->free_list[i].off < off) i++;
  if (sv->nfree == sv->cap_free) {
    span *nl = (span *)realloc(sv->free_list, sizeof(span) * 2 * sv->cap_free);
    if (!nl) return 0;
    sv->free_list = nl;
    sv->cap_free *= 2;
  }
  memmove(&sv->free_list[i + 1], &sv->free_list[i], sizeof(span) * (sv->nfree - i));
  sv->free_list[i].off = off;
  sv->free_list[i].len = len;
  sv->nfree++;
  /* merge with neighbours */
  for (j = (i > 0 ? i - 1 : 0); j + 1 < sv->nfree && j <= i;) {
    if (sv->free_list[j].off + sv->free_list[j].len == sv->free_list[j + 1].off) {
      sv->free_list[j].len += sv->free_list[j + 1].len;
      memmove(&sv->free_list[j + 1], &sv->free_list[j + 2], sizeof(span) * (sv->nfree - j - 2));
      sv->nfree--;
    } else {
      j++;
    }
  }
  return 1;
}

/* ------------------------------------------------------------ queue */
static int queue_push(bsofi_server *sv, const request *r) {
  if (sv->qlen == sv->qcap) {
    int ncap = sv->qcap ? 2 * sv->qcap : 64, i;
    request *nq = (request *)malloc(sizeof(request) * ncap);
    if (!nq) return 0;
    for (i = 0; i < sv->qlen; i++) nq[i] = sv->queue[(sv->qhead + i) % sv->qcap];
    free(sv->queue);
    sv->queue = nq;
    sv->qcap = ncap;
    sv->qhead = 0;
  }
  sv->queue[(sv->qhead + sv->qlen) % sv->qcap] = *r;
  sv->qlen++;
  return 1;
}

static void queue_remove(bsofi_server *sv, int pos) {
  int i;
  for (i = pos; i > 0; i--)
    sv->queue[(sv->qhead + i) % sv->qcap] = sv->queue[(sv->qhead + i - 1) % sv->qcap];
  sv->qhead = (sv->qhead + 1) % sv->qcap;
  sv->qlen--;
}

/* ------------------------------------------------------------ API */
bsofi_server *bsofi_server_create(int slots, unsigned long long pool_bytes) {
  bsofi_server *sv;
  int i, least = 0, greatest = 0;
  if (slots < 1 || slots > MAX_SLOTS || pool_bytes < 4096) return NULL;
  if (bsofi_dev_prepare() != 0) return NULL;
  sv = (bsofi_server *)calloc(1, sizeof(bsofi_server));
  if (!sv) return NULL;
  if (cudaGetDevice(&sv->device) != cudaSuccess) goto fail;
  sv->nslots = slots;
  sv->pool_bytes = (size_t)pool_bytes & ~(size_t)255;
  if (cudaMalloc((void **)&sv->pool, sv->pool_bytes) != cudaSuccess) goto fail;
  sv->cap_free = 64;
  sv->free_list = (span *)malloc(sizeof(span) * sv->cap_free);
  if (!sv->free_list) goto fail;
  sv->free_list[0].off = 0;
  sv->free_list[0].len = sv->pool_bytes;
  sv->nfree = 1;
  if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess) goto fail;
  for (i = 0; i < slots; i++) {
    if (cudaStreamCreateWithFlags(&sv->s[i].stream, cudaStreamNonBlocking) != cudaSuccess) goto fail;
    if (cudaStreamCreateWithPriority(&sv->s[i].hi, cudaStreamNonBlocking, greatest) != cudaSuccess)
      goto fail;
    if (cudaEventCreateWithFlags(&sv->s[i].handoff, cudaEventDisableTiming) != cudaSuccess)
      goto fail;
    if (cudaEventCreateWithFlags(&sv->s[i].done, cudaEventDisableTiming) != cudaSuccess) goto fail;
    if (cudaMallocHost((void **)&sv->s[i].hinfo, 4 * sizeof(int)) != cudaSuccess) goto fail;
  }
  return sv;
fail:
  bsofi_server_destroy(sv);
  return NULL;
}

void bsofi_server_destroy(bsofi_server *sv) {
  int i;
  if (!sv) return;
  for (i = 0; i < MAX_SLOTS; i++) {
    if (sv->s[i].stream) {
      cudaStreamSynchronize(sv->s[i].stream);
      cudaStreamDestroy(sv->s[i].stream);
    }
    if (sv->s[i].hi) {
      cudaStreamSynchronize(sv->s[i].hi);
      cudaStreamDestroy(sv->s[i].hi);
    }
    if (sv->s[i].handoff) cudaEventDestroy(sv->s[i].handoff);
    if (sv->s[i].done) cudaEventDestroy(sv->s[i].done);
    if (sv->s[i].hinfo) cudaFreeHost(sv->s[i].hinfo);
  }
  if (sv->pool) cudaFree(sv->pool);
  free(sv->free_list);
  free(sv->queue);
  free(sv->res);
  free(sv);
}

static size_t ws_bytes(int n, int L, int ldda, int precision) {
  return align256(precision == 1 ? bsofi_dev_ws_bytes_mixed(n, L, ldda, BSOFI_MIXED_SLICES)
                                 : bsofi_dev_ws_bytes(n, L, ldda));
}

static int owned_ldda(int n, int L) { return (n * L + 31) / 32 * 32; }

static size_t mat_bytes(int n, int L) {
  const int N = n * L;
  return align256(sizeof(double) * (size_t)owned_ldda(n, L) * N) + align256(sizeof(double) * N);
}

unsigned long long bsofi_server_request_bytes(int n, int L, int ldda) {
  return ws_bytes(n, L, ldda, 0);
}

unsigned long long bsofi_server_footprint_bytes(int n, int L, int precision) {
  if (n < 1 || n > BSOFI_MAX_BLOCK || L < 2 || (precision != 0 && precision != 1)) return 0;
  return ws_bytes(n, L, owned_ldda(n, L), precision) + mat_bytes(n, L);
}

long long bsofi_server_submit(bsofi_server *sv, int n, int L, double *dA, int ldda,
                              double *dtau, int precision) {
  request r;
  if (!sv) return -1;
  if (n < 1 || n > BSOFI_MAX_BLOCK || L < 2 || ldda < n * L || !dA || !dtau) return -2;
  if (precision != 0 && precision != 1) return -3;
  memset(&r, 0, sizeof(r));
  r.ws = ws_bytes(n, L, ldda, precision);
  if (r.ws > sv->pool_bytes) return -4; /* can never be admitted */
  r.id = sv->next_id++;
  r.n = n;
  r.L = L;
  r.ldda = ldda;
  r.precision = precision;
  r.dA = dA;
  r.dtau = dtau;
  if (!queue_push(sv, &r)) return -5;
  return r.id;
}

long long bsofi_server_submit_blocks(bsofi_server *sv, int n, int L, const double *dD,
                                     const double *dS, int precision) {
  request r;
  if (!sv) return -1;
  if (n < 1 || n > BSOFI_MAX_BLOCK || L < 2 || !dS) return -2;
  if (precision != 0 && precision != 1) return -3;
  memset(&r, 0, sizeof(r));
  r.ldda = owned_ldda(n, L);
  r.ws = ws_bytes(n, L, r.ldda, precision);
  r.mat = mat_bytes(n, L);
  if (r.ws + r.mat > sv->pool_bytes) return -4;
  r.id = sv->next_id++;
  r.n = n;
  r.L = L;
  r.precision = precision;
  r.dD = dD;
  r.dS = dS;
  r.owned = 1;
  if (!queue_push(sv, &r)) return -5;
  return r.id;
}

static int find_resident(bsofi_server *sv, long long id) {
  int i;
  for (i = 0; i < sv->nres; i++)
    if (sv->res[i].id == id) return i;
  return -1;
}

int bsofi_server_result(bsofi_server *sv, long long id, double **dA, int *ldda, double **dtau) {
  int i;
  if (!sv || !dA || !ldda || !dtau) return -1;
  i = find_resident(sv, id);
  if (i < 0) return -1;
  *dA = (double *)(sv->pool + sv->res[i].moff);
  *ldda = sv->res[i].ldda;
  *dtau = (double *)(sv->pool + sv->res[i].moff +
                     align256(sizeof(double) * (size_t)sv->res[i].ldda * sv->res[i].N));
  return 0;
}

int bsofi_server_release(bsofi_server *sv, long long id) {
  int i;
  if (!sv) return -1;
  i = find_resident(sv, id);
  if (i < 0) return -1;
  if (!pool_free(sv, sv->res[i].moff, sv->res[i].mlen)) return -1;
  sv->res[i] = sv->res[sv->nres - 1];
  sv->nres--;
  return 0;
}

/* A request runs pipelined like a batch instance (bsofi_device_set_batch_
 * pipelined): the assembly and the factorization chain on the slot's
 * highest-priority stream, then BSTRI and BSOI as per-step launches on its
 * ordinary stream, so the other slots' chains are never held back by a
 * persistent GEMM kernel; otherwise the whole pipeline on the ordinary one. */
static int launch(bsofi_server *sv, slot *sl, const request *r) {
  const int pipelined = bsofi_batch_pipelined_now();
  int e = 0, workers = bsofi_batch_workers_for(r->n);
  void *ws = sv->pool + sl->off;
  double *dA = r->dA, *dtau = r->dtau;
  cudaStream_t first = pipelined ? sl->hi : sl->stream;
  if (r->owned) {
    dA = (double *)(sv->pool + sl->moff);
    dtau = (double *)(sv->pool + sl->moff +
                      align256(sizeof(double) * (size_t)r->ldda * r->n * r->L));
    e = bsofi_device_assemble(r->n, r->L, r->dD, r->dS, dA, r->ldda, first);
    if (e) return e <= BSOFI_INFO_CUDA ? BSOFI_INFO_CUDA - e : (int)cudaErrorInvalidValue;
  }
  if (pipelined) {
    bsofi_dev_set_nonpersistent(1);
    e = bsofi_dev_invert_two_streams(r->n, r->L, dA, r->ldda, dtau, ws, sl->hi, sl->stream,
                                     sl->handoff, workers,
                                     r->precision == 1 ? BSOFI_MIXED_SLICES : 0);
    bsofi_dev_set_nonpersistent(0);
  } else if (r->precision == 1)
    e = bsofi_dev_invert_mixed(r->n, r->L, dA, r->ldda, dtau, ws, sl->stream, workers,
                               BSOFI_MIXED_SLICES);
  else
    e = bsofi_dev_invert_ex(r->n, r->L, dA, r->ldda, dtau, ws, sl->stream, workers);
  if (!e)
    e = (int)cudaMemcpyAsync(sl->hinfo, bsofi_dev_info_ptr(ws), 4 * sizeof(int),
                             cudaMemcpyDeviceToHost, sl->stream);
  if (!e) e = (int)cudaEventRecord(sl->done, sl->stream);
  return e;
}

/* Admit queued requests into free slots while their workspace fits. */
static int admit(bsofi_server *sv, long long *done_ids, int *done_status, int max, int *ndone) {
  int pos = 0, i;
  while (pos < sv->qlen) {
    slot *sl = NULL;
    request *r = &sv->queue[(sv->qhead + pos) % sv->qcap];
    size_t off;
    for (i = 0; i < sv->nslots; i++)
      if (!sv->s[i].busy) {
        sl = &sv->s[i];
        break;
      }
    if (!sl) break;
    {
      /* The whole footprint or nothing: workspace, then the owned matrix. */
      size_t moff = 0;
      int fits = pool_alloc(sv, r->ws, &off);
      if (fits && r->mat > 0 && !pool_alloc(sv, r->mat, &moff)) {
        pool_free(sv, off, r->ws);
        fits = 0;
      }
      if (!fits) {
        if (pos == 0 && sv->bypassed >= BYPASS_LIMIT) break; /* hold for the head */
        pos++;
        continue;
      }
      sl->moff = moff;
      sl->mlen = r->mat;
    }
    if (pos > 0) sv->bypassed++;
    else sv->bypassed = 0;
    sl->busy = 1;
    sl->id = r->id;
    sl->off = off;
    sl->len = r->ws;
    sl->ldda = r->ldda;
    sl->n = r->n;
    sl->L = r->L;
    {
      const int e = launch(sv, sl, r);
      if (e != 0) { /* a launch error retires the request at once */
        sl->busy = 0;
        pool_free(sv, off, r->ws);
        if (sl->mlen) pool_free(sv, sl->moff, sl->mlen);
        sl->mlen = 0;
        if (*ndone < max) {
          done_ids[*ndone] = r->id;
          done_status[*ndone] = BSOFI_INFO_CUDA - e;
          (*ndone)++;
        }
      }
    }
    queue_remove(sv, pos);
  }
  return 0;
}

int bsofi_server_poll(bsofi_server *sv, long long *done_ids, int *done_status, int max) {
  int i, ndone = 0;
  if (!sv || max < 0) return -1;
  for (i = 0; i < sv->nslots && ndone < max; i++) {
    slot *sl = &sv->s[i];
    cudaError_t q;
    if (!sl->busy) continue;
    q = cudaEventQuery(sl->done);
    if (q == cudaErrorNotReady) continue;
    done_ids[ndone] = sl->id;
    if (q != cudaSuccess) done_status[ndone] = BSOFI_INFO_CUDA - (int)q;
    else if (sl->hinfo[1] != 0 || sl->hinfo[2] != 0 || sl->hinfo[3] != 0)
      done_status[ndone] = BSOFI_INFO_CUDA - (int)cudaErrorLaunchTimeout;
    else done_status[ndone] = sl->hinfo[0] >= 0x7f7f7f7f ? 0 : sl->hinfo[0];
    ndone++;
    sl->busy = 0;
    pool_free(sv, sl->off, sl->len);
    if (sl->mlen) {
      /* The owned matrix and tau stay resident until bsofi_server_release. */
      if (sv->nres == sv->cap_res) {
        const int ncap = sv->cap_res ? 2 * sv->cap_res : 64;
        resident *nr = (resident *)realloc(sv->res, sizeof(resident) * ncap);
        if (!nr) { /* no host memory to track it: give the memory back */
          pool_free(sv, sl->moff, sl->mlen);
          done_status[ndone - 1] = BSOFI_INFO_CUDA - (int)cudaErrorMemoryAllocation;
          sl->mlen = 0;
          continue;
        }
        sv->res = nr;
        sv->cap_res = ncap;
      }
      sv->res[sv->nres].id = sl->id;
      sv->res[sv->nres].moff = sl->moff;
      sv->res[sv->nres].mlen = sl->mlen;
      sv->res[sv->nres].ldda = sl->ldda;
      sv->res[sv->nres].N = sl->n * sl->L;
      sv->nres++;
      sl->mlen = 0;
    }
  }
  admit(sv, done_ids, done_status, max, &ndone);
  return ndone;
}

int bsofi_server_pending(bsofi_server *sv) {
  int i, busy = 0;
  if (!sv) return -1;
  for (i = 0; i < sv->nslots; i++) busy += sv->s[i].busy;
  return busy + sv->qlen;
}
