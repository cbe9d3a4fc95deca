/*
 * bsofi_b200.h -- C ABI of the B200-native BSOF/I library (libbsofi_b200.so).
 *
 * BSOF/I: structured orthogonal factorization and explicit inversion of an
 * N x N block p-cyclic matrix (N = n*L): identity-like diagonal blocks A_k,
 * sub-diagonal blocks at (k+1, k) and a corner block at (0, L-1).  All
 * arithmetic is FP64 on the GPU; there is no CPU fallback.
 *
 * The entry points keep the reference's names, argument lists and meaning
 * (scalar_t = double, Fortran symbols lowercase with a trailing underscore,
 * every Fortran argument by pointer).  Each declaration cites the reference
 * interface it replaces.
 *
 * Storage contract (reference src/bsofi_cpu.c:58-85):
 *   A      column-major, leading dimension lda >= n*L, overwritten in place.
 *          Only the p-cyclic blocks (diagonal, sub-diagonal, corner) of the
 *          input are read; every other block is taken as zero (the
 *          reference reads them and assumes they are zero).
 *   after XbsoftriH: the Householder vectors of panel k are stored below the
 *          diagonal of A(kn:(k+2)n, kn:(k+1)n) (unit entry implicit), tau(kn+i)
 *          their scalars (the last panel has 2n of them), and the block upper
 *          triangle of A holds R^{-1}.
 *   after XbsoiH: A holds M^{-1} (dense).
 *
 * Errors: info = 0 success; info = -i the i-th argument is illegal (LAPACK
 * convention; i counts the handle as argument 1 in the handle API);
 * info = i > 0 after BSTRI: R(i,i) is exactly zero (1-based global index,
 * the inverse was not formed); info <= BSOFI_INFO_CUDA: a CUDA runtime error
 * (BSOFI_INFO_CUDA - cudaError_t).  No entry point exits the process.
 *
 * Threading: every handle owns its own stream and device buffers, so calls
 * on different handles may run from different threads.  The C names without
 * a handle (lapackX*, hybridX*, gpuX*) share one context per thread.
 */
#ifndef BSOFI_B200_H
#define BSOFI_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define BSOFI_INFO_CUDA (-1000)
#define BSOFI_MAX_BLOCK 768 /* largest supported block size n */

/* ------------------------------------------------------------------------
 * Fortran handle API (primary drop-in).  `handle` is the caller's
 * integer handler(10) array (40 bytes); it stores a context pointer.
 * ---------------------------------------------------------------------- */

/* Replaces cb_hybridXinitH, src/bsofi_callback.c:101-128 (bsofi.h:282).
 * Allocates the device context for (n, L, lda).  Returns 0, or -1 on an
 * illegal argument or a device failure (as the reference). */
int hybridxinith_(int *handle, int *n, int *L, int *lda);

/* Replaces cb_hybridXbsofiLWorkH, src/bsofi_callback.c:170-180
 * (bsofi.h:290).  Returns the host workspace length in doubles for `work`
 * of XbsoftriH / XbsoiH.  The GPU path keeps its workspace on the device,
 * so this is 1. */
int hybridxbsofilworkh_(int *handle, int *n, int *L, int *lda);

/* Replaces cb_hybridXbsoftriH, src/bsofi_callback.c:130-144 (bsofi.h:283).
 * BSOF + BSTRI.  lwork = -1: work[0] <- host workspace length;
 * lwork = -2: work[0] <- device workspace length (doubles).  Returns *info. */
int hybridxbsoftrih_(int *handle, int *n, int *L, double *A, int *lda, double *tau,
                     double *work, int *lwork, int *info);

/* Replaces cb_hybridXbsoiH, src/bsofi_callback.c:146-157 (bsofi.h:286).
 * BSOI: A (reflectors + R^{-1}, tau) <- M^{-1}.  Returns *info. */
int hybridxbsoih_(int *handle, int *n, int *L, double *A, int *lda, double *tau,
                  double *work, int *lwork, int *info);

/* Replaces cb_hybridXfinalizeH, src/bsofi_callback.c:159-168 (bsofi.h:289).
 * Frees the context and clears the handle.  Returns 0. */
int hybridxfinalizeh_(int *handle);

/* Replace the timer callbacks fgetwalltime/felapsed,
 * src/bsofi_callback.c:189-218. */
void fgetwalltime_(double tv[2]);
double felapsed_(double t1[2], double t0[2]);

/* ------------------------------------------------------------------------
 * C names of the reference (thin wrappers over the same device pipeline).
 * ---------------------------------------------------------------------- */

/* Replaces lapackXbsofiLWork, src/bsofi_cpu.c:31-42 (include/bsofi_cpu.h:24). */
int lapackXbsofiLWork(int n, int L, int lda);
/* Replaces lapackXbsof, src/bsofi_cpu.c:86-118 (include/bsofi_cpu.h:26). */
int lapackXbsof(int n, int L, double A[], int lda, double tau[], double work[], int lwork,
                int *info);
/* Replaces lapackXbstri, src/bsofi_cpu.c:146-177 (include/bsofi_cpu.h:38). */
int lapackXbstri(int n, int L, double A[], int lda, int *info);
/* Replace lapackXbsoi_ormqr / lapackXbsoi_orgqr, src/bsofi_cpu.c:211-248 and
 * 283-333 (include/bsofi_cpu.h:30-36).  Both compute M^{-1} = R^{-1} Q^T. */
int lapackXbsoi_ormqr(int n, int L, double A[], int lda, double tau[], double work[],
                      int lwork, int *info);
int lapackXbsoi_orgqr(int n, int L, double A[], int lda, double tau[], double work[],
                      int lwork, int *info);

/* Fortran twins, include/bsofi_cpu.h:48-72 (src/bsofi_callback.c:24-56). */
int lapackxbsofilwork_(int *n, int *L, int *lda);
int lapackxbsof_(int *n, int *L, double A[], int *lda, double tau[], double work[],
                 int *lwork, int *info);
int lapackxbstri_(int *n, int *L, double A[], int *lda, int *info);
int lapackxbsoi_ormqr_(int *n, int *L, double A[], int *lda, double tau[], double work[],
                       int *lwork, int *info);
int lapackxbsoi_orgqr_(int *n, int *L, double A[], int *lda, double tau[], double work[],
                       int *lwork, int *info);

/* Replaces hybridXbsofiLWork, src/bsofi_hybrid_adaptive.c:43-57
 * (include/bsofi_hybrid.h:110).  lworkHostDevice = -1: host length,
 * -2: device length (doubles). */
int hybridXbsofiLWork(int n, int L, int lda, int lworkHostDevice);
/* Replace hybridXbsoftri / hybridXbsoi, src/bsofi_hybrid_adaptive.c:108-213,
 * 255-403 (include/bsofi_hybrid.h:120-130).  `handle` is the reference's
 * cublasHandle_t slot (an int when cuBLAS is absent) and is ignored; dwork
 * and ldwork are accepted for ABI compatibility and not used. */
int hybridXbsoftri(int handle, int n, int L, double A[], int lda, double tau[], double work[],
                   int lwork, double dwork[], int ldwork, int *info);
int hybridXbsoi(int handle, int n, int L, double A[], int lda, double tau[], double work[],
                int lwork, double dwork[], int ldwork, int *info);
/* Fortran twins of the three names above: cb_hybridXbsofiLWork,
 * cb_hybridXbsoftri, cb_hybridXbsoi, src/bsofi_callback.c:62-87
 * (include/bsofi_hybrid.h:57-69).  Every argument by pointer, no cuBLAS
 * handle; a NULL argument gives info = -(its position). */
int hybridxbsofilwork_(int *n, int *L, int *lda, int *lworkHostDevice);
int hybridxbsoftri_(int *n, int *L, double A[], int *lda, double tau[], double work[], int *lwork,
                    double dwork[], int *ldwork, int *info);
int hybridxbsoi_(int *n, int *L, double A[], int *lda, double tau[], double work[], int *lwork,
                 double dwork[], int *ldwork, int *info);

/* Device-pointer API, include/bsofi_gpu.h:34-62 (src/bsofi_gpu.c:74-414).
 * dA is device memory (ldda >= n*L), tau is HOST memory as in the reference
 * (MAGMA returns tau on the host).  dT / dwork are accepted and not used.
 * Synchronous. */
int gpuXbsof(int n, int L, double dA[], int ldda, double tau[], double work[], int lwork,
             double *dT, int *info);
int gpuXbstri_rseq(int n, int L, double dA[], int ldda, double dwork[], int ldwork, int *info);
int gpuXbstri_rbatched(int n, int L, double dA[], int ldda, double dwork[], int ldwork,
                       int *info);
int gpuXbsoi_ormqr(int n, int L, double dA[], int ldda, double tau[], double work[], int lwork,
                   double *dT, double dwork[], int ldwork, int *info);
int gpuXbsoi_orgqr(int n, int L, double dA[], int ldda, double tau[], double work[], int lwork,
                   double *dT, double dwork[], int ldwork, int *info);
int gpuXbsoi_batched(int n, int L, double dA[], int ldda, double tau[], double work[],
                     int lwork, double *dT, double dwork[], int ldwork, int *info);

/* ------------------------------------------------------------------------
 * Asynchronous device-resident API.  No reference counterpart: the
 * reference's GPU routines are synchronous and keep tau on the host.  Used
 * by callers that hold M in HBM (batched walkers, the benchmark).
 * ---------------------------------------------------------------------- */

/* Device workspace bytes for (n, L, ldda). */
unsigned long long bsofi_device_workspace_bytes(int n, int L, int ldda);

/* BSOF + BSTRI + BSOI on device memory, enqueued on `stream`
 * (cudaStream_t, 0 = legacy default stream); dtau is device memory (N
 * doubles), dwork device memory of bsofi_device_workspace_bytes.  dA must
 * hold the p-cyclic input (no other block is read).  Returns 0, -1 for an
 * illegal argument (n outside 1..BSOFI_MAX_BLOCK, L < 2, ldda < n*L, a NULL
 * pointer) or BSOFI_INFO_CUDA - cudaError_t; the BSTRI info word is at
 * bsofi_device_info(dwork) (device int, values >= 0x7f7f7f7f mean 0; after
 * bsofi_device_invert or bsofi_device_bsoi it is BSOFI_INFO_CUDA -
 * cudaErrorLaunchTimeout if a bounded wait inside a persistent kernel gave
 * up; words 1, 2 and 3 are the BSOF, BSOI and BSTRI wait error flags). */
int bsofi_device_invert(int n, int L, double *dA, int ldda, double *dtau, void *dwork,
                        void *stream);
int bsofi_device_bsoftri(int n, int L, double *dA, int ldda, double *dtau, void *dwork,
                         void *stream);
int bsofi_device_bsoi(int n, int L, double *dA, int ldda, const double *dtau, void *dwork,
                      void *stream);

/* BSOI of the rows [row0, row1) of M^{-1} only, every column (no reference
 * counterpart; one inversion over several GPUs: the factorization on every
 * GPU, BSOI by rows, since rows of X are independent in X(:,k:k+1) Q_k^T,
 * src/bsofi_cpu.c:211-248).  dA holds the BSOF +
 * BSTRI state as for bsofi_device_bsoi; rows outside the range are left as
 * they were.  row0 must be a multiple of 128 and row1 too unless it is n*L.
 * Returns 0, -1 for an illegal argument or range, or BSOFI_INFO_CUDA -
 * cudaError_t.  bsofi_b200/shard.py runs it on every rank of a
 * torch.distributed group and all-gathers the rows. */
int bsofi_device_bsoi_rows(int n, int L, double *dA, int ldda, const double *dtau, void *dwork,
                           int row0, int row1, void *stream);
int *bsofi_device_info(void *dwork);

/* Storage-sharded inversion: one inversion over several GPUs with no GPU
 * holding M or M^{-1} whole, for N beyond one GPU's memory (no reference
 * counterpart; the reference inverts on one device, src/bsofi_callback.c:
 * 130-157).  The split follows the algorithm's structure:
 *   - BSOF's state is small: R has three nonzero blocks per block row and the
 *     reflectors fill the 2n x n panels (src/bsofi_cpu.c:86-118), so every
 *     rank factors the whole matrix in a compact layout (3 L n^2 + N n
 *     doubles instead of N^2) and holds the same state;
 *   - BSTRI's block columns are independent once the diagonal inverses
 *     X_ii = R_ii^{-1}, the row multipliers W_i = -X_ii R_{i,i+1} and
 *     Z_i = -X_ii R_{i,L-1} X_{L-1,L-1} are known (the row recurrence of
 *     src/bsofi_cpu.c:146-177 read by columns: X_{i,c} = W_i X_{i+1,c}, plus
 *     Z_i in the last column), so each rank computes the block columns it owns;
 *   - BSOI's rows are independent (X(:,k:k+1) Q_k^T, src/bsofi_cpu.c:211-248),
 *     so after the ranks exchange their columns for row bands each finishes
 *     its rows of M^{-1}.
 * Per rank: bsofi_shard_state_bytes(n, L) of device state, the owned block
 * columns (c1 n x (c1 - c0) n doubles) and the row band ((r1 - r0) x N).
 *
 * bsofi_shard_factor: the state from the packed p-cyclic blocks (dD, dS as
 * bsofi_device_assemble takes them); bsofi_shard_hubbard_factor from expm(K)
 * and the fields (as bsofi_device_hubbard_assemble).
 * bsofi_shard_bstri_columns: block columns [c0, c1) of X = R^{-1}, rows
 * 0 .. c1 n - 1 (the rest of those columns is zero), into dX (column-major,
 * leading dimension ldx >= c1 n).
 * bsofi_shard_bsoi_rows: dB holds rows [row0, row1) of X in all N columns
 * (column-major, leading dimension ldb >= row1 - row0) and is overwritten
 * with the same rows of M^{-1}; row0 a multiple of 128, row1 too unless it
 * is N.  Calls on one state run in order (they share its workspace).
 * bsofi_shard_logdet: sign and log|det M| as bsofi_device_logdet, from the
 * state.  bsofi_shard_info: the state's info word (as bsofi_device_info);
 * bsofi_shard_tau: the N reflector scalars inside the state.
 * All enqueue on `stream` and return 0, -1 for an illegal argument, or
 * BSOFI_INFO_CUDA - cudaError_t.  bsofi_b200/shard.py drives them over a
 * torch.distributed group (all-to-all of columns into row bands). */
unsigned long long bsofi_shard_state_bytes(int n, int L);
int bsofi_shard_factor(int n, int L, const double *dD, const double *dS, void *dstate,
                       void *stream);
int bsofi_shard_hubbard_factor(int n, int L, const double *dExpK, const double *dh,
                               double lambda, void *dstate, void *stream);
int bsofi_shard_bstri_columns(int n, int L, int c0, int c1, double *dX, long long ldx,
                              void *dstate, void *stream);
int bsofi_shard_bsoi_rows(int n, int L, int row0, int row1, double *dB, long long ldb,
                          void *dstate, void *stream);
int bsofi_shard_logdet(int n, int L, const void *dstate, double *dout, void *stream);
int *bsofi_shard_info(void *dstate);
const double *bsofi_shard_tau(const void *dstate, int n, int L);

/* Mixed-precision inversion (no reference counterpart; the reference's
 * BSOI products are FP64 LAPACK/MAGMA calls, src/bsofi_cpu.c:234-245 and
 * src/bsofi_gpu.c:397-411).  The factorization (BSOF), the triangular
 * inverse (BSTRI), tau, the reflectors and the diagonal TRTRI stay FP64; the
 * p-1 BSOI products X(:,k:k+1) Q_k^T run on the int8 tensor cores by the
 * Ozaki splitting scheme: each row of X and each column of Q_k^T is scaled by
 * a power of two and cut into `slices` signed 7-bit integers, the slice
 * products are summed exactly in int32 in tensor memory, and the result is
 * formed in FP64 (slices = 0 means BSOFI_MIXED_SLICES = 8; valid 3..8).  With 8
 * slices ||M X - I||_F / ||X||_F stays at the FP64 path's level (about 1e-14 on
 * the Hubbard matrices); with 7 about 1e-12.  The result is deterministic.
 * dwork holds bsofi_device_workspace_bytes_mixed bytes (the FP64 workspace
 * plus the slices of one N x 2n operand; returns 0 for illegal arguments).
 * Returns as bsofi_device_invert; the info word is at bsofi_device_info(dwork). */
#define BSOFI_MIXED_SLICES 8
unsigned long long bsofi_device_workspace_bytes_mixed(int n, int L, int ldda, int slices);
int bsofi_device_invert_mixed(int n, int L, double *dA, int ldda, double *dtau, void *dwork,
                              int slices, void *stream);
/* Kernels launched by the last bsofi_device_* call on this thread. */
long long bsofi_device_last_launches(void);

/* DQMC producer and consumer on the device (no reference counterpart: the
 * reference takes the dense N x N matrix on the host and leaves the
 * determinant to the caller, examples/ftest_hybrid/ftest_hybrid.f90:12-52
 * and :141-145).
 *
 * bsofi_device_assemble writes the p-cyclic input into dA from packed blocks:
 * dD holds the L diagonal blocks (n x n column-major, block k at dD + k n^2;
 * NULL = identity blocks), dS the L coupling blocks, dS[k] placed at block
 * (k+1, k) for k < L-1 and dS[L-1] at block (0, L-1).  It also zeroes the
 * blocks the factorization reads as zeros; no other block is written (none
 * other is read by bsofi_device_*).
 *
 * bsofi_device_hubbard_assemble builds the DQMC matrix itself: identity
 * diagonal, -B_k at block (k, k-1) (k = 1..L-1) and +B_L at block (0, L-1),
 * with B_k = dExpK diag(exp(lambda h_k)); dExpK is expm(dtau t K) (n x n,
 * times exp(dtau mu) if mu != 0), dh the L x n fields (h_k = dh + (k-1) n).
 *
 * bsofi_device_logdet writes dout[0] = sign(det M) (+1, -1, or 0 when a
 * diagonal entry of R is zero or not finite) and dout[1] = log|det M| from
 * the factorization state: diag(dA) holds R_jj after bsofi_device_bsoftri's
 * BSOF phase only (inverted = 0) or 1/R_jj after BSTRI (inverted = 1, the
 * state bsofi_device_bsoftri and hybridxbsoftrih_ leave), and
 * sign(det M) = (-1)^{#(tau_j != 0)} prod sign(R_jj).  (The reference example
 * flips the sign for tau_j == 0 instead; the two agree when N is even.)
 * All three enqueue on `stream` and return 0, -1 for an illegal argument or
 * BSOFI_INFO_CUDA - cudaError_t. */
int bsofi_device_assemble(int n, int L, const double *dD, const double *dS, double *dA, int ldda,
                          void *stream);
int bsofi_device_hubbard_assemble(int n, int L, const double *dExpK, const double *dh,
                                  double lambda, double *dA, int ldda, void *stream);
int bsofi_device_logdet(int n, int L, const double *dA, int ldda, const double *dtau,
                        int inverted, double *dout, void *stream);

/* Batched inversion of `count` independent matrices (no reference
 * counterpart: the reference inverts one walker per call).  Instance i has
 * block size n[i], L[i] blocks, device matrix dA[i] (ldda[i]) and device tau
 * dtau[i]; dwork is one device workspace of bsofi_batch_workspace_bytes
 * bytes.  Instances run largest first over `streams` internal streams
 * (0 = 8, at most 32) owned by the calling thread; `stream` waits for the
 * whole batch.  Returns 0, -1 for an illegal argument, or
 * BSOFI_INFO_CUDA - cudaError_t. */
unsigned long long bsofi_batch_workspace_bytes(int count, const int *n, const int *L,
                                               const int *ldda);
int bsofi_device_invert_batched(int count, const int *n, const int *L, double *const *dA,
                                const int *ldda, double *const *dtau, void *dwork, int streams,
                                void *stream);
/* How FP64 batches run BSOI (no reference counterpart; process-wide).
 * on = 0, the default: each instance's BSOI is its own persistent launch on
 * the instance's stream, overlapping the other instances' factorizations.
 * on = 1: BSOF + BSTRI of every instance over the stream pool first, then BSOI
 * of all instances as one persistent launch per tile shape over one queue of
 * every instance's tiles (at most 256 instances per launch), then each
 * instance's last BSOI copy: no wave tails between instances, but the
 * latency-bound factorizations no longer overlap the GEMM work (measured
 * slower on a 256-instance batch of mixed sizes). */
void bsofi_device_set_batch_grouped(int on);
/* At most k instances' factorization chains (BSOF) of a batch in flight at
 * once (0, the default: no bound beyond the stream count; at most 32), for
 * batches with bsofi_device_set_batch_pipelined(0); process-wide, no
 * reference counterpart.  Results are unchanged.  (Measured: every bound
 * slowed the batch; the chains' latency, not their SMs, limits it.) */
void bsofi_device_set_batch_chains(int k);
/* Pipelined batches and server requests (on = 1, the default; process-wide,
 * no reference counterpart): each instance's factorization chain runs on a
 * highest-priority stream of the pool, the chains dealt to one stream back
 * to back, and hands over by an event to an ordinary stream for BSTRI and
 * BSOI, which then run as per-step launches instead of persistent kernels (a
 * persistent kernel holds every SM until it ends, so the next chains could
 * not start).  on = 0: each instance's whole pipeline on one stream.  The two
 * agree to the launch plans' rounding (tau bitwise). */
void bsofi_device_set_batch_pipelined(int on);
/* BSOF worker CTAs per batch instance (diagnostics; 0, the default: 6 for
 * n < 224, 12 for 224 <= n <= 256, 24 above); process-wide. */
void bsofi_device_set_batch_workers(int workers);
/* The same batch at a chosen precision: 0 FP64 (as above), 1 mixed (every
 * instance as bsofi_device_invert_mixed with BSOFI_MIXED_SLICES slices).  The
 * workspace query returns 0 for an unknown precision. */
unsigned long long bsofi_batch_workspace_bytes_ex(int count, const int *n, const int *L,
                                                  const int *ldda, int precision);
int bsofi_device_invert_batched_ex(int count, const int *n, const int *L, double *const *dA,
                                   const int *ldda, double *const *dtau, void *dwork, int streams,
                                   int precision, void *stream);

/* The same batch captured once into a CUDA graph and replayed (no reference
 * counterpart).  A Monte Carlo sweep re-inverts the same walkers' buffers
 * every step; a graph replays the ~40 launches per walker with one call.
 * bsofi_batch_graph_create captures the batch (arguments as for
 * bsofi_device_invert_batched; the buffers are bound into the graph) and
 * returns NULL on failure; bsofi_batch_graph_launch enqueues one replay on
 * `stream` (not the legacy default stream) and returns 0 or
 * BSOFI_INFO_CUDA - cudaError_t; the caller refills dA between replays. */
typedef struct bsofi_batch_graph bsofi_batch_graph;
bsofi_batch_graph *bsofi_batch_graph_create(int count, const int *n, const int *L,
                                            double *const *dA, const int *ldda,
                                            double *const *dtau, void *dwork, int streams);
int bsofi_batch_graph_launch(bsofi_batch_graph *graph, void *stream);
void bsofi_batch_graph_destroy(bsofi_batch_graph *graph);

/* Launch plans and the autotuner (no reference counterpart).  A plan is
 * four ints: [0] BSOI form (0 / 5 one persistent launch over all steps with
 * 128x128 / 64x64 tiles; 1 one
 * GEMM launch per step, tile shape by tile count; 2 / 3 / 4 per step with
 * 64x64 / 128x128 with 32-deep K stages / 128x128 with 16-deep K stages),
 * [1] the BSTRI row recurrence (one GEMM launch per step with tiles 0 by
 * tile count, 1 128x128 K16, 2 64x64, 3 128x128 K32; or 4: one persistent
 * launch of 64x64 tiles pipelined across the steps), [2] BSOF worker CTAs of
 * a single inversion, [3] the BSTRI row group: 0 one recurrence step per
 * block row, g in 2..8 the blocked recurrence with g block rows per step
 * (products of g consecutive W_i formed for all groups at once, then one
 * GEMM of g n rows per group: all groups in one persistent launch of 128x128
 * tiles when [1] is 4, else one launch per group).
 * Every inversion of block size n with L blocks uses the tuned plan of (n, L)
 * if there is one, else a default fitted to the sizes tuned on a B200
 * (bsofi_plan_get shows it).  bsofi_autotune times the candidates one knob at a time on a
 * synthetic matrix of that size (reps timed runs each, fastest kept; it
 * allocates its own buffers) on `stream`, stores the winner and copies it to
 * plan_out (may be NULL); it returns 0, -1 for an illegal size or
 * BSOFI_INFO_CUDA - cudaError_t.  While it runs, other inversions of the same
 * size see its trial plans.  bsofi_plan_get fills plan and returns 1 for a
 * tuned plan, 0 for the default; bsofi_plan_set stores a plan (e.g. one saved
 * from an earlier run) and returns -1 if it is invalid; bsofi_plan_clear
 * forgets every tuned plan. */
int bsofi_autotune(int n, int L, int reps, void *stream, int *plan_out);
int bsofi_plan_get(int n, int L, int *plan);
int bsofi_plan_set(int n, int L, const int *plan);
void bsofi_plan_clear(void);

/* Continuous-batching inversion server (no reference counterpart: the
 * reference's calls are synchronous, one matrix at a time).  Requests invert
 * caller-owned device-resident matrices; up to `slots` run at once, each on
 * its own stream, with workspace taken first-fit from a device pool of
 * `pool_bytes` allocated at creation (admission by memory footprint, FIFO
 * with bounded bypass so large requests are not starved).  Progress is made
 * in bsofi_server_poll, which retires finished requests (writing up to `max`
 * ids and statuses: 0, info > 0 for an exactly singular R, or
 * BSOFI_INFO_CUDA - cudaError_t) and admits queued ones; it never blocks.
 * submit returns the request id (>= 0) or -1 bad server, -2 illegal size,
 * -3 unsupported precision (0 = FP64, 1 = mixed as bsofi_device_invert_mixed
 * with BSOFI_MIXED_SLICES slices), -4 workspace larger than the pool, -5 out
 * of host memory.  One host thread per server. */
typedef struct bsofi_server bsofi_server;
bsofi_server *bsofi_server_create(int slots, unsigned long long pool_bytes);
unsigned long long bsofi_server_request_bytes(int n, int L, int ldda);
long long bsofi_server_submit(bsofi_server *server, int n, int L, double *dA, int ldda,
                              double *dtau, int precision);
/* Server-owned requests.  The request is given by its packed p-cyclic blocks
 * in device memory (dD: L diagonal blocks or NULL for identity blocks, dS: L
 * coupling blocks, as bsofi_device_assemble takes them; both must stay valid
 * until the request completes).  At admission the pool supplies the matrix
 * (leading dimension n*L rounded up to 32), tau and the workspace together,
 * bsofi_server_footprint_bytes(n, L, precision) bytes in all: admission is by
 * the request's full memory footprint.  After the request completes, the
 * workspace returns to the pool and bsofi_server_result gives the device
 * addresses of M^{-1} and tau (0, or -1 for an unknown or released id);
 * they stay resident, and count against the pool, until
 * bsofi_server_release (0 or -1).  submit_blocks returns the id or the
 * submit error codes above (-4: the footprint exceeds the pool). */
unsigned long long bsofi_server_footprint_bytes(int n, int L, int precision);
long long bsofi_server_submit_blocks(bsofi_server *server, int n, int L, const double *dD,
                                     const double *dS, int precision);
int bsofi_server_result(bsofi_server *server, long long id, double **dA, int *ldda,
                        double **dtau);
int bsofi_server_release(bsofi_server *server, long long id);
int bsofi_server_poll(bsofi_server *server, long long *done_ids, int *done_status, int max);
int bsofi_server_pending(bsofi_server *server);
void bsofi_server_destroy(bsofi_server *server);

/* Allocation-free inversion.  No counterpart in the reference.  For callers
 * that cannot allocate device memory at inversion time: a code whose memory
 * pool already holds nearly all of HBM (cudaMalloc would fail), or one that
 * cannot let cudaMalloc/cudaFree synchronize the device mid-sweep.  Same
 * kernels and result as bsofi_device_invert, but the workspace is a static
 * device array of bsofi_noalloc_scratch_bytes() (32 MiB) instead of a caller
 * buffer, and the call makes no cudaMalloc, cudaFree or other allocating call.
 *
 * bsofi_noalloc_prepare: call it once per device, with that device current,
 * before the caller's pool reserves HBM and before any stream capture.  Under
 * lazy module loading (the CUDA 12 default) the driver reserves the static
 * array, loads kernel code and grows the local-memory reservation the first
 * time each is used; prepare does all of it now (it looks up the array's
 * device address and loads every kernel of the pipeline).  Without it the
 * first inversion on a device does that work and can fail for lack of memory
 * (BSOFI_INFO_CUDA - cudaErrorMemoryAllocation).  From then on the device holds
 * the array until the process exits.  Returns 0 or BSOFI_INFO_CUDA -
 * cudaError_t.
 *
 * Size limit: the workspace grows with n, L and ldda; problems with
 * bsofi_device_workspace_bytes(n, L, ldda) > bsofi_noalloc_scratch_bytes()
 * are rejected with BSOFI_NOALLOC_TOO_LARGE before any device work.  With
 * ldda = n*L that allows L up to 120 at n = 64, 50 at n = 100, 31 at n = 128,
 * 14 at n = 196 and 8 at n = 256; compare the two functions for other sizes.
 *
 * All calls share the array and it keeps the last call's contents (the
 * pipeline writes every region before reading it): calls that overlap on the
 * GPU (other streams or threads on the same device) race.  dinfo (device int)
 * receives the info word as bsofi_device_info describes it (values >=
 * 0x7f7f7f7f mean 0), enqueued on `stream`, and the call returns without
 * waiting.  With dinfo = NULL the call waits for `stream` and returns the info
 * word itself: 0, i > 0 for an exactly zero R(i,i), or BSOFI_INFO_CUDA -
 * cudaErrorLaunchTimeout when a bounded wait inside a kernel gave up.
 * Returns 0 (or that info word), -1 for an illegal argument,
 * BSOFI_NOALLOC_TOO_LARGE, or BSOFI_INFO_CUDA - cudaError_t. */
#define BSOFI_NOALLOC_TOO_LARGE (-2000)
unsigned long long bsofi_noalloc_scratch_bytes(void);
int bsofi_noalloc_prepare(void);
int bsofi_device_invert_noalloc(int n, int L, double *dA, int ldda, double *dtau, int *dinfo,
                                void *stream);

/* Diagnostics (no reference counterpart): when on, every BSOI step GEMM
 * launch (the dominant kernel) made by this thread is bracketed by CUDA
 * events on its stream; bsofi_device_timing_read waits for them and returns
 * the summed kernel time in ms and the number of timed launches, then clears
 * the record. */
void bsofi_device_timing(int on);
int bsofi_device_timing_read(double *ms, long long *launches);

/* Diagnostics (no reference counterpart): the BSOF timeline of the last
 * factorization that used `dwork` -- four globaltimer stamps (ns) per leaf
 * from the CTA that runs the critical chain: loop start, tile ready, leaf
 * published, next-tile update start.  Copies up to max_leaves leaves to host
 * and returns the number copied.  set_bsof_workers sets the number of worker
 * CTAs of the persistent BSOF kernel (default 32) for this process. */
int bsofi_device_bsof_timeline(int n, int L, int ldda, void *dwork, unsigned long long *host,
                               int max_leaves);
void bsofi_device_set_bsof_workers(int workers);
/* Single inversions with n <= 256 whose plan runs the persistent blocked BSTRI
 * recurrence split the factorization at a panel and overlap BSTRI's leading
 * rows with the rest of it on two side streams of the calling thread (created
 * on first use, never during a graph capture of the caller's stream; the
 * results are the same as without the split).  on = 0 turns this off for the
 * process, 1 (the default) on. */
void bsofi_device_set_bstri_overlap(int on);
/* Diagnostics (no reference counterpart): warps that factor a 16-wide leaf of
 * the BSOF chain (n <= 256): 4 (the default; the CTA's other 4 warps stage the
 * next leaf's tile meanwhile) or 8 (the tile is staged after the
 * factorization).  Results are the same either way to rounding.  Process-wide. */
void bsofi_device_set_bsof_factor_warps(int warps);
/* FP64 tile engine instruction shape (diagnostics, no reference
 * counterpart; process-wide): mma.sync m16n8k8 steps (0, the default) or
 * m16n8k16 (1: half the instructions, each 16 deep in K), for every GEMM
 * launch and persistent BSOI launch that follows. */
void bsofi_device_set_gemm_k16(int on);
/* Operand loading of the persistent 128-row BSOI kernel (no reference
 * counterpart; process-wide): on = 1, the default, loads by TMA every tile
 * that needs no zero-fill mask, and every tile under the diagonal block of
 * X(:,k), whose zeros come from the tensor map's fill (2-D and 3-D tensor
 * maps of the matrix, the carries and Q_k^T, 16 x 16 and 16 x BN boxes with
 * the 128-byte swizzle, a 3-stage ring of mbarriers filled by one thread),
 * the rest by cp.async; on = 0 loads every tile by cp.async in 128 x 128
 * tiles.  Same products in the same order: the same results bit for bit.
 * Applies to full-range launches with even leading dimensions, n a multiple
 * of 16 and 2n a multiple of 128 (128 x 128 tiles) or of 160 (128 x 160
 * tiles, which need TMA: with on = 0 such sizes run 128 x 128 tiles). */
void bsofi_device_set_bsoi_tma(int on);
/* Diagnostics (no reference counterpart): with on = 1, the persistent BSOI
 * launches made by this thread wait, in every step after the first, on a
 * zeroed workspace word that nothing writes, under a short poll limit (about
 * a millisecond).  The waits give up, the kernel returns, and the inversion's
 * info word reads BSOFI_INFO_CUDA - cudaErrorLaunchTimeout, exactly as when a
 * real wait runs out; the device and the workspace stay usable.  Lets a test
 * check that path without any fault.  on = 0 (the default) turns it off. */
void bsofi_device_set_wait_test(int on);

/* Diagnostic entry point (no reference counterpart): one call of the FP64
 * DMMA tile engine, C = alpha*A*B + beta*C on device memory (column-major),
 * with the optional upper-triangular masks the pipeline uses (upper_a: A(i,k)
 * = 0 for i > k; upper_b: B(k,j) = 0 for k > j).  tile: 0 auto, 1 128x128,
 * 2 64x64.  Enqueued on `stream`; returns 0 or BSOFI_INFO_CUDA - error. */
int bsofi_selftest_gemm(int M, int N, int K, double alpha, const double *dA, int lda,
                        int upper_a, const double *dB, int ldb, int upper_b, double beta,
                        double *dC, int ldc, int tile, void *stream);

/* Diagnostic entry point (no reference counterpart): one product C = A B
 * (column-major, M x K times K x N, K <= 1536) on the int8 tensor cores by the
 * Ozaki scheme with `slices` slices (0 = 8), as the mixed-precision BSOI
 * computes each step.  dscratch: device memory of
 * bsofi_selftest_ozaki_scratch_bytes (256-byte aligned); derr: a device int
 * set to 1 if a bounded wait inside the kernel gave up.  Enqueued on
 * `stream`; returns 0, -1 for an illegal argument or BSOFI_INFO_CUDA - error. */
unsigned long long bsofi_selftest_ozaki_scratch_bytes(int M, int N, int K, int slices);
int bsofi_selftest_ozaki(int M, int N, int K, const double *dA, int lda, const double *dB, int ldb,
                         double *dC, int ldc, int slices, void *dscratch, int *derr, void *stream);

#ifdef __cplusplus
}
#endif
#endif
