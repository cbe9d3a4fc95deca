/*
 * bsofi_b200_fp32.h -- C ABI of the single-precision library
 * (libbsofi_b200_fp32.so).
 *
 * The reference builds a single-precision variant from the same sources
 * with __SINGLE_PREC__ (scalar_t = float, config.h:132-136; LAPACK calls go
 * to the s* routines, src/bsofi_lapack.c:17-21).  That variant keeps every
 * symbol name and argument list and only changes the scalar type, so a
 * caller switches precision by linking the other library.  This header is
 * that variant's interface: the same names as bsofi_b200.h with float
 * arrays.  A process links one of the two libraries, as with the reference.
 *
 * Arithmetic: the caller's float arrays are widened on the GPU into an FP64
 * working matrix, the FP64 pipeline of libbsofi_b200.so runs on it, and the
 * results are rounded to float on the GPU before they are copied back.  The
 * results are therefore the FP64 results rounded once to float (more
 * accurate than the reference's FP32 LAPACK path, within its FP32 error
 * bound), and host <-> device traffic is half the FP64 library's.  On the
 * B200 the FP64 tensor pipe (DMMA) is the fastest path that keeps FP32
 * accuracy without error-compensated products, and the panel chain is
 * latency-bound whatever the precision.
 *
 * Storage contract, error codes and threading: as bsofi_b200.h (reference
 * src/bsofi_cpu.c:58-85).  work / lwork follow the reference's protocol:
 * lwork = -1 -> work[0] = host workspace length (1), lwork = -2 ->
 * work[0] = device workspace length in floats.
 */
#ifndef BSOFI_B200_FP32_H
#define BSOFI_B200_FP32_H

#ifdef __cplusplus
extern "C" {
#endif

#ifndef BSOFI_INFO_CUDA
#define BSOFI_INFO_CUDA (-1000)
#endif
#ifndef BSOFI_MAX_BLOCK
#define BSOFI_MAX_BLOCK 768
#endif

/* Handle API: cb_hybridXinitH / XbsofiLWorkH / XbsoftriH / XbsoiH /
 * XfinalizeH, src/bsofi_callback.c:101-180 (bsofi.h:282-290). */
int hybridxinith_(int *handle, int *n, int *L, int *lda);
int hybridxbsofilworkh_(int *handle, int *n, int *L, int *lda);
int hybridxbsoftrih_(int *handle, int *n, int *L, float *A, int *lda, float *tau, float *work,
                     int *lwork, int *info);
int hybridxbsoih_(int *handle, int *n, int *L, float *A, int *lda, float *tau, float *work,
                  int *lwork, int *info);
int hybridxfinalizeh_(int *handle);

/* Timer callbacks, src/bsofi_callback.c:189-218 (double in both builds). */
void fgetwalltime_(double tv[2]);
double felapsed_(double t1[2], double t0[2]);

/* lapackX* C names, src/bsofi_cpu.c:31-333 (include/bsofi_cpu.h:24-41). */
int lapackXbsofiLWork(int n, int L, int lda);
int lapackXbsof(int n, int L, float A[], int lda, float tau[], float work[], int lwork,
                int *info);
int lapackXbstri(int n, int L, float A[], int lda, int *info);
int lapackXbsoi_ormqr(int n, int L, float A[], int lda, float tau[], float work[], int lwork,
                      int *info);
int lapackXbsoi_orgqr(int n, int L, float A[], int lda, float tau[], float work[], int lwork,
                      int *info);

/* Fortran twins, include/bsofi_cpu.h:48-72 (src/bsofi_callback.c:24-56). */
int lapackxbsofilwork_(int *n, int *L, int *lda);
int lapackxbsof_(int *n, int *L, float A[], int *lda, float tau[], float work[], int *lwork,
                 int *info);
int lapackxbstri_(int *n, int *L, float A[], int *lda, int *info);
int lapackxbsoi_ormqr_(int *n, int *L, float A[], int *lda, float tau[], float work[],
                       int *lwork, int *info);
int lapackxbsoi_orgqr_(int *n, int *L, float A[], int *lda, float tau[], float work[],
                       int *lwork, int *info);

/* hybridX* names, src/bsofi_hybrid_adaptive.c:43-403
 * (include/bsofi_hybrid.h:110-130); handle, dwork and ldwork are ignored. */
int hybridXbsofiLWork(int n, int L, int lda, int lworkHostDevice);
int hybridXbsoftri(int handle, int n, int L, float A[], int lda, float tau[], float work[],
                   int lwork, float dwork[], int ldwork, int *info);
int hybridXbsoi(int handle, int n, int L, float A[], int lda, float tau[], float work[],
                int lwork, float dwork[], int ldwork, int *info);
/* Fortran twins of the three names above: cb_hybridXbsofiLWork,
 * cb_hybridXbsoftri, cb_hybridXbsoi, src/bsofi_callback.c:62-87
 * (include/bsofi_hybrid.h:57-69).  Every argument by pointer, no cuBLAS
 * handle; a NULL argument gives info = -(its position). */
int hybridxbsofilwork_(int *n, int *L, int *lda, int *lworkHostDevice);
int hybridxbsoftri_(int *n, int *L, float A[], int *lda, float tau[], float work[], int *lwork,
                    float dwork[], int *ldwork, int *info);
int hybridxbsoi_(int *n, int *L, float A[], int *lda, float tau[], float work[], int *lwork,
                 float dwork[], int *ldwork, int *info);

/* Device-pointer names, include/bsofi_gpu.h:34-62 (src/bsofi_gpu.c:74-414):
 * dA is device memory (float, ldda >= n*L), tau HOST memory.  Synchronous. */
int gpuXbsof(int n, int L, float dA[], int ldda, float tau[], float work[], int lwork, float *dT,
             int *info);
int gpuXbstri_rseq(int n, int L, float dA[], int ldda, float dwork[], int ldwork, int *info);
int gpuXbstri_rbatched(int n, int L, float dA[], int ldda, float dwork[], int ldwork, int *info);
int gpuXbsoi_ormqr(int n, int L, float dA[], int ldda, float tau[], float work[], int lwork,
                   float *dT, float dwork[], int ldwork, int *info);
int gpuXbsoi_orgqr(int n, int L, float dA[], int ldda, float tau[], float work[], int lwork,
                   float *dT, float dwork[], int ldwork, int *info);
int gpuXbsoi_batched(int n, int L, float dA[], int ldda, float tau[], float work[], int lwork,
                     float *dT, float dwork[], int ldwork, int *info);

/* Number of kernels the last call on this thread launched (diagnostics). */
long long bsofi_fp32_last_launches(void);

#ifdef __cplusplus
}
#endif
#endif
