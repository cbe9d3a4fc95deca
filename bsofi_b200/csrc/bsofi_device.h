/*
 * bsofi_device.h -- device-side BSOF/I pipeline, plain C interface.
 *
 * Used by the host C layer (bsofi_api.c).  Every function enqueues work on
 * `stream` (a cudaStream_t passed as void*) and returns a cudaError_t value
 * (0 = success) without synchronising.  Matrices are column-major FP64 in
 * device memory with leading dimension ldd >= n*L.
 */
#ifndef BSOFI_DEVICE_H
#define BSOFI_DEVICE_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Bytes of device workspace the pipeline needs for (n, L, ldd). */
size_t bsofi_dev_ws_bytes(int n, int L, int ldd);

/* One-time per-process set-up (kernel attributes).  Call before capturing
 * the pipeline into a CUDA graph. */
int bsofi_dev_prepare(void);
/* bsofi_dev_prepare plus loading every kernel of the pipeline onto the
 * current device now (under lazy module loading each kernel is otherwise
 * loaded, and device memory taken, at its first launch) and reserving the
 * largest per-thread local memory any of them needs. */
int bsofi_dev_preload(void);

/* Zero the blocks of A that the factorization reads as structural zeros
 * (superdiagonal blocks and the last block column except its first and last
 * blocks).  Used after copying only the p-cyclic blocks to the device. */
int bsofi_dev_zero_structural(int n, int L, double *dA, int ldd, void *stream);

/* BSOF + BSTRI: A <- reflectors + R^{-1}, tau <- reflector scalars.
 * Resets the workspace info word first; read it with bsofi_dev_info_ptr. */
int bsofi_dev_bsoftri(int n, int L, double *dA, int ldd, double *dtau, void *dws,
                      void *stream);
/* BSOF only / BSTRI only (split phases). */
int bsofi_dev_bsof(int n, int L, double *dA, int ldd, double *dtau, void *dws, void *stream);
int bsofi_dev_bstri(int n, int L, double *dA, int ldd, void *dws, void *stream);
/* BSOF + BSTRI + BSOI in one sequence; the factorization also forms the
 * explicit Q_k^T that BSOI consumes, off its critical chain. */
int bsofi_dev_invert(int n, int L, double *dA, int ldd, double *dtau, void *dws, void *stream);
/* Same with an explicit number of BSOF worker CTAs (0 = default). */
int bsofi_dev_invert_ex(int n, int L, double *dA, int ldd, double *dtau, void *dws, void *stream,
                        int workers);

/* The same inversion with BSOI's products on the int8 tensor cores (Ozaki
 * scheme, `slices` 3..8 slices per operand; 2n <= 1536).  dws holds
 * bsofi_dev_ws_bytes_mixed bytes: the FP64 workspace followed by the
 * product's scratch. */
size_t bsofi_dev_ws_bytes_mixed(int n, int L, int ldd, int slices);
int bsofi_dev_invert_mixed(int n, int L, double *dA, int ldd, double *dtau, void *dws,
                           void *stream, int workers, int slices);
/* One product C = A B (M x K times K x N, column-major) on the int8 tensor
 * cores, for tests; scratch of bsofi_dev_ozaki_scratch_bytes, derr a device
 * int set to 1 if a bounded wait gave up. */
size_t bsofi_dev_ozaki_scratch_bytes(int M, int N, int K, int slices);
int bsofi_dev_selftest_ozaki(int M, int N, int K, const double *dA, int lda, const double *dB,
                             int ldb, double *dC, int ldc, int slices, void *scratch, int *derr,
                             void *stream);

/* BSOI of a whole batch in one persistent launch per tile shape (per 256
 * instances).  bsoftri_q_ex: BSOF (forming every Q_k^T) + BSTRI with `workers`
 * BSOF worker CTAs and no side streams; group_prepare: the instance's first
 * carry and zeroed BSOI counters; group_run: the grouped launches (64 x 64
 * tiles on stream_small, 128 x 128 on stream_large), gws holding
 * bsofi_dev_bsoi_group_bytes(count) device bytes; group_finish: the
 * instance's column block 0 and its info word. */
int bsofi_dev_bsoftri_q_ex(int n, int L, double *dA, int ldd, double *dtau, void *dws,
                           void *stream, int workers);
int bsofi_dev_bsoi_group_prepare(int n, int L, double *dA, int ldd, void *dws, void *stream);
size_t bsofi_dev_bsoi_group_bytes(int count);
int bsofi_dev_bsoi_group_run(int count, const int *n, const int *L, double *const *dA,
                             const int *ldd, void *const *dws, void *gws, void *stream_small,
                             void *stream_large);
int bsofi_dev_bsoi_group_finish(int n, int L, double *dA, int ldd, void *dws, void *stream);

/* BSOI: A (reflectors + R^{-1}) <- M^{-1}. */
int bsofi_dev_bsoi(int n, int L, double *dA, int ldd, const double *dtau, void *dws,
                   void *stream);

/* BSOF (also forming every G_k = Q_k^T in the workspace, off the critical
 * chain) + BSTRI; and BSOI that skips Q formation when q_ready (the
 * workspace's G_k belong to the state in dA and dtau). */
int bsofi_dev_bsoftri_q(int n, int L, double *dA, int ldd, double *dtau, void *dws,
                        void *stream);
int bsofi_dev_bsoi_ex(int n, int L, double *dA, int ldd, const double *dtau, void *dws,
                      void *stream, int q_ready);

/* BSOI of the rows [row0, row1) of M^{-1} only (row0 a multiple of 128, row1
 * too unless it is N): the other rows of A are left as they were. */
int bsofi_dev_bsoi_rows(int n, int L, double *dA, int ldd, const double *dtau, void *dws,
                        void *stream, int row0, int row1);

/* One inversion (FP64 when slices = 0, else the mixed path with that many
 * slices) whose factorization chain is gated: the stream waits for wait_ev
 * (optional) before BSOF and records done_ev (optional) right after it, so
 * that a batch can bound how many chains run at once.  Ordered phases, every
 * Q_k^T formed by the BSOF workers; workers as for bsofi_dev_invert_ex. */
int bsofi_dev_invert_gated(int n, int L, double *dA, int ldd, double *dtau, void *dws,
                           void *stream, int workers, int slices, void *wait_ev, void *done_ev);

/* One inversion split over two streams: BSOF (every Q_k^T formed) on
 * chain_stream, then `handoff` recorded there and waited for on gemm_stream,
 * which runs BSTRI and BSOI (FP64, or the mixed path when slices != 0). */
int bsofi_dev_invert_two_streams(int n, int L, double *dA, int ldd, double *dtau, void *dws,
                                 void *chain_stream, void *gemm_stream, void *handoff,
                                 int workers, int slices);
/* Launch plans of the calling thread without persistent GEMM kernels (BSOI
 * and the BSTRI recurrence as per-step launches) while on != 0. */
void bsofi_dev_set_nonpersistent(int on);
/* batch.c: whether batches (and the server's requests) run pipelined, and
 * the BSOF worker count of an instance of block size n. */
int bsofi_batch_pipelined_now(void);
int bsofi_batch_workers_for(int n);
/* FP64 tile engine steps: mma.sync m16n8k8 (0) or m16n8k16 (1). */
void bsofi_dev_set_gemm_k16(int on);
/* Persistent BSOI with TMA-loaded clean 128 x 128 tiles (1) or cp.async (0). */
void bsofi_dev_set_bsoi_tma(int on);

/* Storage-sharded inversion (one inversion over several GPUs, none holding M
 * or M^{-1} whole).  The state (bsofi_dev_shard_state_bytes) holds the
 * compact factorization: block columns 0..L-2 with leading dimension 3n, the
 * last block column as an N x n array, tau, and the pipeline workspace.
 * shard_factor: compact input (packed blocks, or Hubbard when dExpK is set)
 * -> BSOF with every Q_k^T, the diagonal inverses, Z_i and W_i.
 * shard_bstri_columns: block columns [c0, c1) of X = R^{-1}, rows 0..c1 n - 1,
 * into dX (leading dimension ldx >= c1 n).
 * shard_bsoi_rows: dB holds rows [r0, r1) of X in all N columns (leading
 * dimension ldb >= r1 - r0) and receives the same rows of M^{-1}; r0 a
 * multiple of 128, r1 too unless it is N. */
size_t bsofi_dev_shard_state_bytes(int n, int L);
int bsofi_dev_shard_factor(int n, int L, const double *dD, const double *dS,
                           const double *dExpK, const double *dh, double lambda, void *dstate,
                           void *stream);
int bsofi_dev_shard_bstri_columns(int n, int L, int c0, int c1, double *dX, long long ldx,
                                  void *dstate, void *stream);
int bsofi_dev_shard_bsoi_rows(int n, int L, int r0, int r1, double *dB, long long ldb,
                              void *dstate, void *stream);
/* Sign and log|det M| (dout[0], dout[1]) from the state of shard_factor. */
int bsofi_dev_shard_logdet(int n, int L, const void *dstate, double *dout, void *stream);
const double *bsofi_dev_shard_tau(const void *dstate, int n, int L);
/* Compact assembly and log-determinant (kernels_dqmc.cu). */
int bsofi_dev_assemble_compact(int n, int L, const double *dD, const double *dS,
                               const double *dExpK, const double *dh, double lambda,
                               double *band, size_t band_doubles, double *last, void *stream);
int bsofi_dev_logdet_compact(int n, int L, const double *band, const double *last,
                             const double *tau, int inverted, double *out, void *stream);

/* The reflector rows of every block column and tau (what Q formation reads):
 * mode 0 packs them into ref (bsofi_dev_state_ref_doubles doubles), mode 1
 * compares them with ref and sets the device int *dflag to 1 on a difference. */
size_t bsofi_dev_state_ref_doubles(int n, int L);
int bsofi_dev_state_ref(int n, int L, const double *dA, int ldd, const double *dtau, double *ref,
                        int mode, int *dflag, void *stream);

/* BSOI in pieces, for callers that overlap it with host copies:
 * form_q builds every G_k = Q_k^T (needs the reflectors and tau);
 * carry seeds the first step (needs column block L-1);
 * step k needs column block k and leaves column block k+1 final;
 * finish writes column block 0 and folds the wait errors into the info word. */
int bsofi_dev_bsoi_form_q(int n, int L, double *dA, int ldd, const double *dtau, void *dws,
                          void *stream);
int bsofi_dev_bsoi_carry(int n, int L, double *dA, int ldd, void *dws, void *stream);
int bsofi_dev_bsoi_step(int n, int L, int k, double *dA, int ldd, void *dws, void *stream);
int bsofi_dev_bsoi_finish(int n, int L, double *dA, int ldd, void *dws, void *stream);

/* FP32 <-> FP64 copies for the single-precision API: region 0 the whole
 * N x N matrix, 1 the BSOF/BSTRI state (rows [0, min((k+2)n, N)) of block
 * column k), 2 the p-cyclic input blocks.  to_float 0 widens f (pitch ldf)
 * into d (pitch ldd), 1 rounds d into f. */
int bsofi_dev_convert(int n, int L, float *f, int ldf, double *d, int ldd, int region,
                      int to_float, void *stream);
int bsofi_dev_convert_vec(float *f, double *d, int len, int to_float, void *stream);

/* Device address of the int info words inside the workspace: [0] BSTRI info
 * (values >= 0x7f7f7f7f mean 0; i > 0: R(i,i) exactly zero, 1-based global
 * index), [1] BSOF, [2] BSOI, [3] BSTRI wait timeout (nonzero = error). */
int *bsofi_dev_info_ptr(void *dws);

/* Launch plans per (n, L): plan[0] BSOI mode (0 persistent, 1 per-step by
 * tile count, 2/3/4 per-step 64x64 / 128x128 K-stage 32 / 128x128 K-stage 16
 * tiles), plan[1] BSTRI recurrence (launch_gemm cfg per step, or 4 for the
 * persistent recurrence kernel), plan[2]
 * BSOF worker CTAs, plan[3] the BSTRI row group (0 one block row per step,
 * 2..8 block rows per step of the blocked recurrence); plan[0] = 5: persistent BSOI with
 * 64x64 tiles.  get returns 1 for a tuned plan, 0 for
 * the default (plan still filled); set returns -1 for an invalid plan. */
int bsofi_dev_plan_get(int n, int L, int *plan);
int bsofi_dev_plan_set(int n, int L, const int *plan);
void bsofi_dev_plan_clear(void);
void bsofi_dev_plan_clear_one(int n, int L);

/* Number of kernels the last bsofi_dev_* call on this thread launched. */
long long bsofi_dev_launch_count(void);
void bsofi_dev_add_launches(long long c);

/* Event timing of the BSOI step GEMM launches (on/off resets the record);
 * read returns the summed duration (ms) and the number of timed launches. */
void bsofi_dev_timing(int on);
int bsofi_dev_timing_read(double *ms, long long *launches);

/* Device address of the BSOF timeline (4 globaltimer stamps per leaf: loop
 * start, tile ready, leaf published, next-tile update start); returns the
 * number of leaves. */
int bsofi_dev_bsof_timeline(int n, int L, int ldd, void *dws, unsigned long long **ptr);
void bsofi_dev_set_bsof_workers(int w);
/* Factor warps of 16-wide BSOF leaves: 4 (default, the other 4 stage the next
 * tile meanwhile) or 8; process-wide. */
void bsofi_dev_set_bsof_factor_warps(int w);
/* Diagnostics: persistent BSOI launches of this thread poll a word that
 * nothing writes in every step wait (short limit), so the waits give up. */
void bsofi_dev_set_wait_test(int on);
/* Overlap of BSTRI's leading rows with the end of BSOF in single inversions
 * (1, the default) or the two phases in order (0); process-wide. */
void bsofi_dev_set_bstri_overlap(int on);

/* One call of the FP64 tile engine (diagnostics). */
int bsofi_dev_selftest_gemm(int M, int N, int K, double alpha, const double *dA, int lda,
                            int upper_a, const double *dB, int ldb, int upper_b, double beta,
                            double *dC, int ldc, int tile, void *stream);

#ifdef __cplusplus
}
#endif
#endif
