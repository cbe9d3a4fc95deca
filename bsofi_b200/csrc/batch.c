/*
 * batch.c -- batched inversion of independent block p-cyclic matrices.
 *
 * DQMC runs many Monte Carlo walkers, each with its own Green's-function
 * matrix M (n, L differ between walkers only through the lattice and the
 * number of time slices).  The reference inverts them one call at a time
 * (src/bsofi_callback.c:130-157).  Here a batch is one call: instances are
 * ordered by their flop count (largest first) and dealt over a pool of
 * streams owned by the calling thread; each instance runs the fused device
 * pipeline with a small BSOF worker pool, so the latency-bound panel chains
 * of several instances overlap each other and the GEMM phases of the rest.
 * The caller's stream waits for the whole batch (event fork/join), so the
 * call is asynchronous like the single-instance device API.
 */
#include <stdint.h>
#include <stdlib.h>
#include <cuda_runtime_api.h>

#include "../../include/bsofi_b200.h"
#include "bsofi_device.h"

#define MAX_STREAMS 32

/* Ring of events bounding the factorization chains in flight. */
#define MAX_GATE 32

typedef struct {
  int ready, count, device, gates, hi_count;
  cudaStream_t s[MAX_STREAMS];
  cudaStream_t hi[MAX_STREAMS];  /* highest priority: factorization chains */
  cudaEvent_t ev[MAX_STREAMS + 1];
  cudaEvent_t gate[MAX_GATE];
} stream_pool;

static __thread stream_pool t_pool;

static size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

static cudaError_t pool_get(int want, stream_pool **out) {
  stream_pool *p = &t_pool;
  int dev = -1, i;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (p->ready && p->device != dev) {
    for (i = 0; i < p->count; i++) cudaStreamDestroy(p->s[i]);
    for (i = 0; i <= p->count; i++) cudaEventDestroy(p->ev[i]);
    for (i = 0; i < p->gates; i++) cudaEventDestroy(p->gate[i]);
    for (i = 0; i < p->hi_count; i++) cudaStreamDestroy(p->hi[i]);
    p->ready = 0;
    p->count = 0;
    p->gates = 0;
    p->hi_count = 0;
  }
  if (!p->ready) {
    if ((e = cudaEventCreateWithFlags(&p->ev[0], cudaEventDisableTiming)) != cudaSuccess) return e;
    p->ready = 1;
    p->device = dev;
  }
  while (p->count < want && p->count < MAX_STREAMS) {
    if ((e = cudaStreamCreateWithFlags(&p->s[p->count], cudaStreamNonBlocking)) != cudaSuccess)
      return e;
    if ((e = cudaEventCreateWithFlags(&p->ev[p->count + 1], cudaEventDisableTiming)) != cudaSuccess)
      return e;
    p->count++;
  }
  while (p->gates < MAX_GATE) {
    if ((e = cudaEventCreateWithFlags(&p->gate[p->gates], cudaEventDisableTiming)) != cudaSuccess)
      return e;
    p->gates++;
  }
  if (p->hi_count < p->count) {
    int least = 0, greatest = 0;
    if ((e = cudaDeviceGetStreamPriorityRange(&least, &greatest)) != cudaSuccess) return e;
    while (p->hi_count < p->count) {
      if ((e = cudaStreamCreateWithPriority(&p->hi[p->hi_count], cudaStreamNonBlocking,
                                            greatest)) != cudaSuccess)
        return e;
      p->hi_count++;
    }
  }
  *out = p;
  return cudaSuccess;
}

static double cost(int n, int L) { return 7.0 * (double)n * (double)n * (double)n * L * L; }

/* Workspace of one instance at `precision` (0 FP64, 1 mixed). */
static size_t inst_ws(int n, int L, int ldda, int precision) {
  return precision == 1 ? bsofi_dev_ws_bytes_mixed(n, L, ldda, BSOFI_MIXED_SLICES)
                        : bsofi_dev_ws_bytes(n, L, ldda);
}

/* Process-wide switches, set and read from any thread. */
static void flag_set(int *f, int v) { __atomic_store_n(f, v, __ATOMIC_RELAXED); }
static int flag_get(int *f) { return __atomic_load_n(f, __ATOMIC_RELAXED); }

/* FP64 batches run each instance's BSOI as its own launch (0, the default:
 * it overlaps the other instances' latency-bound factorization chains) or all
 * BSOI as one grouped persistent launch per tile shape after every
 * factorization (1: no wave tails between instances, but no overlap with the
 * chains; measured slower on a 256-instance batch of mixed sizes, 227.8
 * against 248.5 inversions/s). */
static int g_grouped = 0;
void bsofi_device_set_batch_grouped(int on) { flag_set(&g_grouped, on ? 1 : 0); }

/* At most this many instances' factorization chains run at once in
 * one-stream-per-instance batches (0, the default: as many as there are
 * streams).  Every bound measured slower (the batch is held by the chains'
 * latency, not by the SMs their launches occupy); kept for diagnostics. */
static int g_chains = 0;
void bsofi_device_set_batch_chains(int k) {
  flag_set(&g_chains, k < 0 ? 0 : (k > MAX_GATE ? MAX_GATE : k));
}

/* Pipelined batches (1, the default): each instance's factorization chain
 * runs on a highest-priority stream, chains of the instances dealt to one
 * slot back to back, and hands over by an event to the slot's ordinary
 * stream for BSTRI and BSOI, launched without persistent kernels (per-step
 * GEMMs, whose CTAs retire tile by tile, so that the next chains' cooperative
 * launches find SMs).  Measured on the 256-instance batch of mixed sizes:
 * 265.4 against 249.5 inversions/s (16 streams); 16 instances of one size
 * unchanged.  0: each instance's whole pipeline on one stream. */
static int g_pipelined = 1;
void bsofi_device_set_batch_pipelined(int on) { flag_set(&g_pipelined, on ? 1 : 0); }

/* BSOF worker CTAs per instance of a batch (0: by block size).  Measured on
 * pipelined batches: 16 x (n = 256, p = 32) ran 134 inversions/s with 6
 * workers and 142 with 12; the 256 instances of mixed sizes (n = 64..256)
 * ran 268.5/s with 6 for all, 253/s with 12 for all, 251/s with 3.  So the
 * largest 16-wide instances take 12, smaller ones 6, 8-wide ones 24. */
static int g_batch_workers = 0;
void bsofi_device_set_batch_workers(int w) { flag_set(&g_batch_workers, w < 0 ? 0 : w); }
static int batch_workers(int n) {
  const int w = flag_get(&g_batch_workers);
  if (w > 0) return w;
  return n > 256 ? 24 : (n >= 224 ? 12 : 6);
}

/* The same settings for the server's requests (server.c). */
int bsofi_batch_pipelined_now(void) { return flag_get(&g_pipelined); }
int bsofi_batch_workers_for(int n) { return batch_workers(n); }

unsigned long long bsofi_batch_workspace_bytes_ex(int count, const int *n, const int *L,
                                                  const int *ldda, int precision) {
  unsigned long long tot = 0;
  int i;
  if (precision != 0 && precision != 1) return 0;
  for (i = 0; i < count; i++) tot += align256(inst_ws(n[i], L[i], ldda[i], precision));
  if (precision == 0) tot += align256(bsofi_dev_bsoi_group_bytes(count));
  return tot;
}

unsigned long long bsofi_batch_workspace_bytes(int count, const int *n, const int *L,
                                               const int *ldda) {
  return bsofi_batch_workspace_bytes_ex(count, n, L, ldda, 0);
}

typedef struct {
  double c;
  int i;
} order_t;

static int by_cost_desc(const void *a, const void *b) {
  double x = ((const order_t *)a)->c, y = ((const order_t *)b)->c;
  return x < y ? 1 : (x > y ? -1 : 0);
}

/* Join the `used` pool streams into streams a and b (a == b allowed). */
static cudaError_t join2(stream_pool *p, int used, cudaStream_t a, cudaStream_t b) {
  cudaError_t e;
  int i;
  for (i = 0; i < used; i++) {
    if ((e = cudaEventRecord(p->ev[i + 1], p->s[i])) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(a, p->ev[i + 1], 0)) != cudaSuccess) return e;
    if (b != a && (e = cudaStreamWaitEvent(b, p->ev[i + 1], 0)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

/* FP64 batch with a grouped BSOI: BSOF + BSTRI (forming every Q_k^T) and the
 * first BSOI carry per instance over the pool streams; all streams joined;
 * the grouped BSOI launches on pool streams 0 and 1; forked again for each
 * instance's last BSOI copy.  Returns 0 or a cudaError_t value. */
static int grouped_fp64(stream_pool *p, int used, int count, const int *n, const int *L,
                        double *const *dA, const int *ldda, double *const *dtau, void *dwork,
                        const order_t *ord, const size_t *off, long long *launches) {
  void **ws = (void **)malloc(sizeof(void *) * count);
  cudaStream_t a = p->s[0], b = p->s[used > 1 ? 1 : 0];
  size_t end = 0;
  cudaError_t e;
  int i, r = 0;
  if (!ws) return (int)cudaErrorMemoryAllocation;
  for (i = 0; i < count; i++) {
    ws[i] = (char *)dwork + off[i];
    end = off[i] + align256(inst_ws(n[i], L[i], ldda[i], 0)) > end
              ? off[i] + align256(inst_ws(n[i], L[i], ldda[i], 0))
              : end;
  }
  for (i = 0; i < count && !r; i++) {
    const int k = ord[i].i;
    const int workers = batch_workers(n[k]);
    r = bsofi_dev_bsoftri_q_ex(n[k], L[k], dA[k], ldda[k], dtau[k], ws[k], p->s[i % used],
                               workers);
    *launches += bsofi_dev_launch_count();
    if (!r) r = bsofi_dev_bsoi_group_prepare(n[k], L[k], dA[k], ldda[k], ws[k], p->s[i % used]);
    *launches += 1;
  }
  if (!r && (e = join2(p, used, a, b)) != cudaSuccess) r = (int)e;
  if (!r) {
    r = bsofi_dev_bsoi_group_run(count, n, L, dA, ldda, ws, (char *)dwork + end, a, b);
    *launches += bsofi_dev_launch_count();
  }
  /* fork: every stream waits for both grouped launches */
  if (!r && (e = cudaEventRecord(p->ev[1], a)) != cudaSuccess) r = (int)e;
  if (!r && b != a && (e = cudaEventRecord(p->ev[2], b)) != cudaSuccess) r = (int)e;
  for (i = 0; i < used && !r; i++) {
    if ((e = cudaStreamWaitEvent(p->s[i], p->ev[1], 0)) != cudaSuccess) r = (int)e;
    else if (b != a && (e = cudaStreamWaitEvent(p->s[i], p->ev[2], 0)) != cudaSuccess) r = (int)e;
  }
  for (i = 0; i < count && !r; i++) {
    r = bsofi_dev_bsoi_group_finish(n[i], L[i], dA[i], ldda[i], ws[i], p->s[i % used]);
    *launches += 1;
  }
  free(ws);
  return r;
}

int bsofi_device_invert_batched(int count, const int *n, const int *L, double *const *dA,
                                const int *ldda, double *const *dtau, void *dwork, int streams,
                                void *stream) {
  return bsofi_device_invert_batched_ex(count, n, L, dA, ldda, dtau, dwork, streams, 0, stream);
}

int bsofi_device_invert_batched_ex(int count, const int *n, const int *L, double *const *dA,
                                   const int *ldda, double *const *dtau, void *dwork, int streams,
                                   int precision, void *stream) {
  stream_pool *p;
  order_t *ord;
  size_t *off;
  cudaError_t e;
  int i, used, r = 0, grouped, pipelined, chains;
  long long launches = 0;
  if (count < 0 || (count > 0 && (!n || !L || !dA || !ldda || !dtau || !dwork))) return -1;
  if (precision != 0 && precision != 1) return -1;
  for (i = 0; i < count; i++)
    if (n[i] < 1 || n[i] > BSOFI_MAX_BLOCK || L[i] < 2 || ldda[i] < n[i] * L[i] || !dA[i] ||
        !dtau[i])
      return -1;
  if (count == 0) return 0;
  grouped = flag_get(&g_grouped);
  pipelined = flag_get(&g_pipelined);
  chains = flag_get(&g_chains);
  if ((e = (cudaError_t)bsofi_dev_prepare()) != cudaSuccess) return BSOFI_INFO_CUDA - (int)e;
  if (streams < 1) streams = 8;
  if (streams > MAX_STREAMS) streams = MAX_STREAMS;
  if ((e = pool_get(streams, &p)) != cudaSuccess) return BSOFI_INFO_CUDA - (int)e;
  used = streams < count ? streams : count;
  ord = (order_t *)malloc(sizeof(order_t) * count);
  off = (size_t *)malloc(sizeof(size_t) * count);
  if (!ord || !off) {
    free(ord);
    free(off);
    return BSOFI_INFO_CUDA - (int)cudaErrorMemoryAllocation;
  }
  {
    size_t o = 0;
    for (i = 0; i < count; i++) {
      ord[i].c = cost(n[i], L[i]);
      ord[i].i = i;
      off[i] = o;
      o += align256(inst_ws(n[i], L[i], ldda[i], precision));
    }
  }
  qsort(ord, count, sizeof(order_t), by_cost_desc);
  if ((e = cudaEventRecord(p->ev[0], (cudaStream_t)stream)) != cudaSuccess) goto fail;
  for (i = 0; i < used; i++)
    if ((e = cudaStreamWaitEvent(p->s[i], p->ev[0], 0)) != cudaSuccess) goto fail;
  if (precision == 0 && grouped) {
    r = grouped_fp64(p, used, count, n, L, dA, ldda, dtau, dwork, ord, off, &launches);
    if (r) {
      e = (cudaError_t)r;
      goto fail;
    }
  }
  if (pipelined && !(precision == 0 && grouped)) {
    for (i = 0; i < used; i++)
      if ((e = cudaStreamWaitEvent(p->hi[i], p->ev[0], 0)) != cudaSuccess) goto fail;
    bsofi_dev_set_nonpersistent(1);
    for (i = 0; i < count && !r; i++) {
      const int k = ord[i].i, slot = i % used;
      const int workers = batch_workers(n[k]);
      r = bsofi_dev_invert_two_streams(n[k], L[k], dA[k], ldda[k], dtau[k],
                                       (char *)dwork + off[k], p->hi[slot], p->s[slot],
                                       p->gate[slot], workers,
                                       precision == 1 ? BSOFI_MIXED_SLICES : 0);
      launches += bsofi_dev_launch_count();
    }
    bsofi_dev_set_nonpersistent(0);
    if (r) {
      e = (cudaError_t)r;
      goto fail;
    }
  }
  for (i = 0; i < count && !(precision == 0 && grouped) && !pipelined; i++) {
    const int k = ord[i].i;
    /* Few BSOF workers per instance: the batch supplies the parallelism. */
    const int workers = batch_workers(n[k]);
    /* Gate: instance i waits for the chain of instance i - K (ring slot
     * i % K, recorded by that instance after its BSOF) and records the slot
     * after its own; the host issues them in that order. */
    const int K = (chains > 0 && chains < used) ? chains : 0;
    if (K > 0)
      r = bsofi_dev_invert_gated(n[k], L[k], dA[k], ldda[k], dtau[k], (char *)dwork + off[k],
                                 p->s[i % used], workers, precision == 1 ? BSOFI_MIXED_SLICES : 0,
                                 i >= K ? (void *)p->gate[i % K] : NULL, (void *)p->gate[i % K]);
    else if (precision == 1)
      r = bsofi_dev_invert_mixed(n[k], L[k], dA[k], ldda[k], dtau[k], (char *)dwork + off[k],
                                 p->s[i % used], workers, BSOFI_MIXED_SLICES);
    else
      r = bsofi_dev_invert_ex(n[k], L[k], dA[k], ldda[k], dtau[k], (char *)dwork + off[k],
                              p->s[i % used], workers);
    if (r) {
      e = (cudaError_t)r;
      goto fail;
    }
    launches += bsofi_dev_launch_count();
  }
  for (i = 0; i < used; i++) {
    if ((e = cudaEventRecord(p->ev[i + 1], p->s[i])) != cudaSuccess) goto fail;
    if ((e = cudaStreamWaitEvent((cudaStream_t)stream, p->ev[i + 1], 0)) != cudaSuccess) goto fail;
    /* The chain streams too (their last work is already ordered before the
     * ordinary streams' by the hand-over events; joining them as well keeps
     * a stream capture of the batch complete). */
    if (pipelined && !(precision == 0 && grouped)) {
      if ((e = cudaEventRecord(p->gate[i], p->hi[i])) != cudaSuccess) goto fail;
      if ((e = cudaStreamWaitEvent((cudaStream_t)stream, p->gate[i], 0)) != cudaSuccess)
        goto fail;
    }
  }
  free(ord);
  free(off);
  bsofi_dev_add_launches(launches - bsofi_dev_launch_count());
  return 0;
fail:
  free(ord);
  free(off);
  return BSOFI_INFO_CUDA - (int)e;
}

/* ------------------------------------------------------------ graph */
struct bsofi_batch_graph {
  cudaGraph_t graph;
  cudaGraphExec_t exec;
};

bsofi_batch_graph *bsofi_batch_graph_create(int count, const int *n, const int *L,
                                            double *const *dA, const int *ldda,
                                            double *const *dtau, void *dwork, int streams) {
  bsofi_batch_graph *g;
  cudaStream_t cs = NULL;
  cudaError_t e;
  int r;
  if (count < 1) return NULL;
  /* Kernel attributes and the stream pool are set up outside the capture. */
  if (bsofi_dev_prepare() != 0) return NULL;
  {
    stream_pool *p;
    int want = streams < 1 ? 8 : (streams > MAX_STREAMS ? MAX_STREAMS : streams);
    if (pool_get(want, &p) != cudaSuccess) return NULL;
  }
  g = (bsofi_batch_graph *)calloc(1, sizeof(bsofi_batch_graph));
  if (!g) return NULL;
  if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) goto fail;
  if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed) != cudaSuccess) goto fail;
  r = bsofi_device_invert_batched(count, n, L, dA, ldda, dtau, dwork, streams, cs);
  e = cudaStreamEndCapture(cs, &g->graph);
  if (r != 0 || e != cudaSuccess) goto fail;
  if (cudaGraphInstantiate(&g->exec, g->graph, 0) != cudaSuccess) goto fail;
  cudaStreamDestroy(cs);
  return g;
fail:
  if (cs) {
    enum cudaStreamCaptureStatus st;
    if (cudaStreamIsCapturing(cs, &st) == cudaSuccess && st != cudaStreamCaptureStatusNone) {
      cudaGraph_t junk = NULL;
      cudaStreamEndCapture(cs, &junk);
      if (junk) cudaGraphDestroy(junk);
    }
    cudaStreamDestroy(cs);
  }
  cudaGetLastError();
  bsofi_batch_graph_destroy(g);
  return NULL;
}

int bsofi_batch_graph_launch(bsofi_batch_graph *g, void *stream) {
  cudaError_t e;
  if (!g || !g->exec || !stream) return -1;
  e = cudaGraphLaunch(g->exec, (cudaStream_t)stream);
  return e == cudaSuccess ? 0 : BSOFI_INFO_CUDA - (int)e;
}

void bsofi_batch_graph_destroy(bsofi_batch_graph *g) {
  if (!g) return;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  free(g);
}
