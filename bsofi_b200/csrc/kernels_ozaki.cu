// FP64 products on the int8 tensor cores (tcgen05 kind::i8): the Ozaki
// splitting scheme.
//
// Method (Ozaki, Ogita, Oishi, Rump, "Error-free transformations of matrix
// multiplication by using fast routines of matrix multiplication and its
// applications", Numer. Algorithms 59, 2012; its integer form, Ootomo,
// Ozaki, Yokota, "DGEMM on integer matrix multiplication unit", IJHPCA 2024):
// every row i of A is scaled by a power of two 2^-e_i so that its largest
// entry lies in [1/2, 1), and cut into S signed 7-bit integer slices,
//   A(i,k) = 2^e_i * sum_s a_s(i,k) 2^-7(s+1) + r(i,k),  |r| < 2^(e_i - 7S);
// every column j of B likewise with 2^f_j and slices b_t.  Products of
// slices are exact in int32 (|a_s|, |b_t| <= 127, K <= 1536, at most 8
// products per sum), and the S diagonals
//   D_d = sum_{s+t=d} a_s b_t,  d = 0 .. S-1
// accumulate in tensor memory; the terms with s+t >= S are below the
// slices' resolution and dropped.  The epilogue forms, in FP64,
//   C(i,j) = 2^(e_i+f_j) * sum_{d=S-1..0} D_d(i,j) 2^-7(d+2),
// adding the diagonals from the smallest up.  Everything but that final sum
// is exact, so the result is reproducible bit for bit (a numpy restatement
// of the same arithmetic matches exactly).  With S = 8 the inverse's
// residual matches the FP64 path's order; S = 7 reaches about 1e-12.
//
// Kernels: ozaki_rowmax_kernel finds A's row maxima, ozaki_split_kernel
// writes the slices and exponents of both operands; ozaki_gemm_kernel is a
// warp-specialised tcgen05
// kernel: warp 0 issues TMA tile loads (32-byte swizzle, K-major) into a
// 4-stage mbarrier ring, each stage holding all S slices of A and B for 32 K
// bytes; warp 1 issues the S(S+1)/2 MMAs of each 32-deep K step into S int32
// accumulators of 128 x 64 in tensor memory; warps 2-5 read the accumulators
// back (tcgen05.ld) and write the FP64 tile.  (A variant with 128-byte
// swizzled rows, one A slice per stage, measured 45% slower: less data in
// flight.)  The tensor maps cover this GPU's memory only and no load uses
// cluster multicast.
#include <cuda.h>
#include <climits>
#include <mutex>

#include "bsofi_common.cuh"
#include "bsofi_kernels.h"
#include "tcgen05.cuh"

namespace bsofi {

constexpr int OZ_BM = 128, OZ_BN = 64, OZ_BK = 32, OZ_STAGES = 4;
constexpr int OZ_THREADS = 192;
constexpr int OZ_EXP_NONFINITE = INT_MIN;  // exponent of a row/column holding Inf or NaN

// ------------------------------------------------------------------ split
struct OzSplitArgs {
  // A: M x K, two K segments (k < ksplit: a0 with the masks rows >= rlim0 and
  // r - roff0 > k zero; else a1), column-major.
  const double* a0;
  const double* a1;
  long long lda0, lda1;
  int ksplit, rlim0, roff0;
  int M, K, Kp;
  int8_t* a_out;       // S slices of M x Kp (row i of slice s at a_out + s*a_slice + i*Kp)
  long long a_slice;
  int* a_exp;          // M
  // Row maxima of |A| as the bits of non-negative doubles (zeroed before
  // the row-max kernel; bits >= those of +Inf flag a non-finite row).
  unsigned long long* a_max;
  // B: K x N column-major; column j becomes row j of the B slices.
  const double* b;
  long long ldb;
  int N;
  int8_t* b_out;
  long long b_slice;
  int* b_exp;          // N
  int S;
  int a_blocks;        // slice kernel: blocks [0, a_blocks) cut A tiles, the rest B columns
  int a_chunks;        // 128-column chunks of Kp per 32-row A block
};

__device__ __forceinline__ double oz_a(const OzSplitArgs& s, int i, int k) {
  if (k < s.ksplit) {
    if (i >= s.rlim0 || i - s.roff0 > k) return 0.0;
    return s.a0[(long long)k * s.lda0 + i];
  }
  return s.a1[(long long)(k - s.ksplit) * s.lda1 + i];
}

// Cut 16 scaled values (|r| < 1) into S slices of 16 bytes; r is consumed.
__device__ __forceinline__ void oz_slices16(double (&r)[16], int S, int8_t* dst, long long stride) {
  for (int s = 0; s < S; s++) {
    uint32_t w[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      uint32_t word = 0;
#pragma unroll
      for (int b = 0; b < 4; b++) {
        const double t = r[4 * q + b] * 128.0;
        const double v = trunc(t);
        r[4 * q + b] = t - v;  // exact
        word |= ((uint32_t)(int)v & 0xffu) << (8 * b);
      }
      w[q] = word;
    }
    *reinterpret_cast<uint4*>(dst + (long long)s * stride) = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

// Scale factor 2^-e as one exact multiplication when 2^-e is a normal
// double; `exact` false means the caller uses ldexp per element.
__device__ __forceinline__ double pow2_neg(int e, bool& exact) {
  exact = e > -1000 && e < 1000;
  return exact ? ldexp(1.0, -e) : 1.0;
}

// A: two kernels over a 2-D grid of 32-row blocks, so that every SM has many
// independent tiles in flight (the operand is read at close to HBM rate).
// Row maxima: a CTA of 256 threads takes 32 rows x 64 columns, warp w the
// columns w, w+8, ... with lane = row (coalesced, eight loads in flight),
// and folds its maxima into a_max[row] with one atomicMax per row (the bits
// of non-negative doubles order as the values; NaN and Inf, whose bits lie
// at or above +Inf's, mark the row non-finite).  Slices: a CTA takes 32 rows
// x 128 columns; the block is staged in shared memory by the same coalesced
// column reads, then warp w cuts rows 4w..4w+3 with lane l on columns
// 4l..4l+3 (two 16-byte shared loads) and writes one packed 4-byte word per
// slice: 128 contiguous bytes per warp.  B columns: one warp per column
// (K contiguous), eight per CTA, maximum and slices in the same warp.
constexpr int OZ_SPLIT_ROWS = 32, OZ_SPLIT_THREADS = 256, OZ_SPLIT_CHUNK = 128;
constexpr int OZ_MAX_COLS = 64;
constexpr int OZ_SPLIT_LD = OZ_SPLIT_CHUNK + 2;  // row stride of the staged block (16-byte rows)
constexpr unsigned long long OZ_INF_BITS = 0x7ff0000000000000ull;

__global__ void __launch_bounds__(OZ_SPLIT_THREADS) ozaki_rowmax_kernel(OzSplitArgs s) {
  __shared__ unsigned long long s_max[8][OZ_SPLIT_ROWS];
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int r0 = blockIdx.x * OZ_SPLIT_ROWS, k0 = blockIdx.y * OZ_MAX_COLS;
  const int i = r0 + lane;
  unsigned long long mx = 0;
  if (i < s.M) {
    double v[OZ_MAX_COLS / 8];
#pragma unroll
    for (int j = 0; j < OZ_MAX_COLS / 8; j++) {
      const int k = k0 + warp + 8 * j;
      v[j] = k < s.K ? oz_a(s, i, k) : 0.0;
    }
#pragma unroll
    for (int j = 0; j < OZ_MAX_COLS / 8; j++) {
      const unsigned long long b = (unsigned long long)__double_as_longlong(fabs(v[j]));
      mx = b > mx ? b : mx;
    }
  }
  s_max[warp][lane] = mx;
  __syncthreads();
  if (threadIdx.x < OZ_SPLIT_ROWS && r0 + (int)threadIdx.x < s.M) {
    unsigned long long m = 0;
#pragma unroll
    for (int w = 0; w < 8; w++) m = s_max[w][threadIdx.x] > m ? s_max[w][threadIdx.x] : m;
    if (m != 0) atomicMax(s.a_max + r0 + threadIdx.x, m);
  }
}

__global__ void __launch_bounds__(OZ_SPLIT_THREADS) ozaki_split_kernel(OzSplitArgs s) {
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  if ((int)blockIdx.x < s.a_blocks) {
    __shared__ __align__(16) double s_blk[OZ_SPLIT_ROWS][OZ_SPLIT_LD];
    __shared__ double s_sc[OZ_SPLIT_ROWS];
    __shared__ int s_e[OZ_SPLIT_ROWS];
    const int r0 = ((int)blockIdx.x / s.a_chunks) * OZ_SPLIT_ROWS;
    const int k0 = ((int)blockIdx.x % s.a_chunks) * OZ_SPLIT_CHUNK;
    if (threadIdx.x < OZ_SPLIT_ROWS) {
      const int lr = threadIdx.x, i = r0 + lr;
      const unsigned long long bits = i < s.M ? s.a_max[i] : 0ull;
      const bool bad = bits >= OZ_INF_BITS;
      const double mx = bad ? 0.0 : __longlong_as_double((long long)bits);
      int e = 0;
      if (!bad) frexp(mx, &e);
      // Scale 0 makes every slice of a zero or non-finite row zero.
      bool exact;
      const double sc = pow2_neg(e, exact);
      s_sc[lr] = (bad || !(mx > 0.0)) ? 0.0 : (exact ? sc : -1.0);  // -1: ldexp per element
      s_e[lr] = e;
      if (k0 == 0 && i < s.M) s.a_exp[i] = bad ? OZ_EXP_NONFINITE : e;
    }
    {
      const int i = r0 + lane;
      double v[OZ_SPLIT_CHUNK / 8];  // all 16 loads of this warp in flight at once
#pragma unroll
      for (int j = 0; j < OZ_SPLIT_CHUNK / 8; j++) {
        const int k = k0 + warp + 8 * j;
        v[j] = (i < s.M && k < s.K) ? oz_a(s, i, k) : 0.0;
      }
#pragma unroll
      for (int j = 0; j < OZ_SPLIT_CHUNK / 8; j++) s_blk[lane][warp + 8 * j] = v[j];
    }
    __syncthreads();
#pragma unroll 1
    for (int rr = 0; rr < 4; rr++) {
      const int lr = 4 * warp + rr, i = r0 + lr;
      if (i >= s.M) break;  // warp-uniform
      // Kp is a multiple of 32 (4-column groups never straddle it); the last
      // chunk may end before 128 columns.
      if (k0 + 4 * lane >= s.Kp) continue;
      const double sc = s_sc[lr];
      const double2 p0 = *reinterpret_cast<const double2*>(&s_blk[lr][4 * lane]);
      const double2 p1 = *reinterpret_cast<const double2*>(&s_blk[lr][4 * lane + 2]);
      double r[4] = {p0.x, p0.y, p1.x, p1.y};
#pragma unroll
      for (int q = 0; q < 4; q++)
        r[q] = sc == 0.0 ? 0.0 : (sc > 0.0 ? r[q] * sc : ldexp(r[q], -s_e[lr]));
      int8_t* dst = s.a_out + (long long)i * s.Kp + k0 + 4 * lane;
      for (int sl = 0; sl < s.S; sl++) {
        uint32_t word = 0;
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const double t = r[q] * 128.0;
          const double v = trunc(t);
          r[q] = t - v;  // exact
          word |= ((uint32_t)(int)v & 0xffu) << (8 * q);
        }
        *reinterpret_cast<uint32_t*>(dst + (long long)sl * s.a_slice) = word;
      }
    }
    return;
  }
  const int j = ((int)blockIdx.x - s.a_blocks) * 8 + warp;
  if (j >= s.N) return;
  const double* col = s.b + (long long)j * s.ldb;
  double mx = 0.0;
  bool bad = false;
  for (int k = lane; k < s.K; k += 32) {
    bad |= !isfinite(col[k]);
    mx = fmax(mx, fabs(col[k]));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  bad = __any_sync(0xffffffffu, bad);
  int e = 0;
  if (bad) mx = 0.0;
  else frexp(mx, &e);
  if (lane == 0) s.b_exp[j] = bad ? OZ_EXP_NONFINITE : e;
  bool exact;
  const double sc = pow2_neg(e, exact);
  int8_t* row = s.b_out + (long long)j * s.Kp;
  for (int k0 = lane * 16; k0 < s.Kp; k0 += 32 * 16) {
    double r[16];
#pragma unroll
    for (int q = 0; q < 16; q++) {
      const int k = k0 + q;
      const double v = (mx > 0.0 && k < s.K) ? col[k] : 0.0;
      r[q] = exact ? v * sc : ldexp(v, -e);
    }
    oz_slices16(r, s.S, row + k0, s.b_slice);
  }
}

// ------------------------------------------------------------------ GEMM
struct OzGemmArgs {
  int M, N, Kp;
  const int* a_exp;
  const int* b_exp;
  // Output segments: column j < nsplit -> c0 + j*ldc0, else c1 + (j-nsplit)*ldc1.
  double* c0;
  double* c1;
  long long ldc0, ldc1;
  int nsplit;
  int* err;
  long long spin_limit;
};

template <int S>
struct OzCfg {
  static constexpr int A_TILE = OZ_BM * OZ_BK;  // bytes of one A slice tile
  static constexpr int B_TILE = OZ_BN * OZ_BK;
  static constexpr int STAGE = S * (A_TILE + B_TILE);
  // + alignment slack; at least 120 KB so that one CTA holds an SM alone and
  // its tensor-memory allocation never waits for another CTA's.
  static constexpr size_t NEED = (size_t)OZ_STAGES * STAGE + 1024;
  static constexpr size_t SMEM = NEED > 120 * 1024 ? NEED : 120 * 1024;
  static constexpr uint32_t TMEM_COLS = S * OZ_BN <= 256 ? 256 : 512;
  static_assert(S * OZ_BN <= 512, "accumulators exceed tensor memory");
};

template <int S>
__global__ void __launch_bounds__(OZ_THREADS, 1)
    ozaki_gemm_kernel(const __grid_constant__ CUtensorMap tma_a,
                      const __grid_constant__ CUtensorMap tma_b, OzGemmArgs g) {
  using C = OzCfg<S>;
  extern __shared__ uint8_t oz_smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(((uintptr_t)oz_smem_raw + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) uint64_t full[OZ_STAGES];
  __shared__ __align__(8) uint64_t empty[OZ_STAGES];
  __shared__ __align__(8) uint64_t acc_full;
  __shared__ uint32_t tmem_base;
  __shared__ int abort_flag;
  __shared__ int no_abort;  // never set: waits that must not give up on an abort
  volatile int* abort_v = &abort_flag;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int m0 = blockIdx.x * OZ_BM, n0 = blockIdx.y * OZ_BN;
  const int nk = g.Kp / OZ_BK;
  constexpr uint32_t IDESC = tc::idesc_i8(OZ_BM, OZ_BN);

  if (threadIdx.x == 0) {
    for (int i = 0; i < OZ_STAGES; i++) {
      tc::mbar_init(&full[i], 1);
      tc::mbar_init(&empty[i], 1);
    }
    tc::mbar_init(&acc_full, 1);
    abort_flag = 0;
    no_abort = 0;
    tc::fence_barrier_init();
  }
  if (warp == 0) {
    tc::tmem_alloc(&tmem_base, C::TMEM_COLS);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tbase = tmem_base;
  int issued = 0;  // K steps whose loads warp 0 issued

  if (warp == 0 && lane == 0) {
    // TMA producer.
    tc::prefetch_tmap(&tma_a);
    tc::prefetch_tmap(&tma_b);
    for (int kc = 0; kc < nk; kc++) {
      const int st = kc % OZ_STAGES;
      if (kc >= OZ_STAGES &&
          !tc::mbar_wait(&empty[st], ((kc / OZ_STAGES) - 1) & 1, g.spin_limit, abort_v)) {
        abort_flag = 1;
        atomicExch(g.err, 1);
        break;
      }
      tc::mbar_arrive_expect_tx(&full[st], C::STAGE);
      uint8_t* sa = smem + (size_t)st * C::STAGE;
      uint8_t* sb = sa + S * C::A_TILE;
      for (int s = 0; s < S; s++) tc::tma_load_3d(sa + s * C::A_TILE, &tma_a, &full[st], kc * OZ_BK, m0, s);
      for (int t = 0; t < S; t++) tc::tma_load_3d(sb + t * C::B_TILE, &tma_b, &full[st], kc * OZ_BK, n0, t);
      issued = kc + 1;
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer: accumulator d (columns d*64 .. d*64+63) collects s + t = d.
    for (int kc = 0; kc < nk; kc++) {
      const int st = kc % OZ_STAGES;
      if (!tc::mbar_wait(&full[st], (kc / OZ_STAGES) & 1, g.spin_limit, abort_v)) {
        abort_flag = 1;
        atomicExch(g.err, 1);
        break;
      }
      tc::tc_fence_after();
      const uint8_t* sa = smem + (size_t)st * C::STAGE;
      const uint8_t* sb = sa + S * C::A_TILE;
#pragma unroll
      for (int s = 0; s < S; s++) {
        const uint64_t da = tc::desc_k_sw32(sa + s * C::A_TILE);
#pragma unroll
        for (int t = 0; s + t < S; t++)
          tc::mma_i8(tbase + (uint32_t)((s + t) * OZ_BN), da, tc::desc_k_sw32(sb + t * C::B_TILE),
                     IDESC, (kc > 0 || s > 0) ? 1u : 0u);
      }
      tc::mma_commit(&empty[st]);  // the stage is free once these MMAs have read it
    }
    tc::mma_commit(&acc_full);  // every MMA issued above is complete
  } else if (warp >= 2) {
    // Epilogue: warp w reads tensor-memory lanes 32 (w % 4) .. +31.
    const int q = warp % 4;
    // tcgen05.ld is warp-collective: the whole warp goes on or none of it.
    const bool got = tc::mbar_wait(&acc_full, 0, g.spin_limit, abort_v) && !*abort_v;
    if (__all_sync(0xffffffffu, got)) {
      tc::tc_fence_after();
      const int row = m0 + 32 * q + lane;
      const int er = row < g.M ? g.a_exp[row] : 0;
      const uint32_t lane_addr = tbase + ((uint32_t)(32 * q) << 16);
      for (int c0 = 0; c0 < OZ_BN; c0 += 16) {
        double acc[16];
#pragma unroll
        for (int j = 0; j < 16; j++) acc[j] = 0.0;
#pragma unroll
        for (int d = S - 1; d >= 0; d--) {
          uint32_t v[16];
          tc::tmem_ld16(lane_addr + (uint32_t)(d * OZ_BN + c0), v);
          tc::tmem_ld_wait();
          const double sc = ldexp(1.0, -7 * (d + 2));
#pragma unroll
          for (int j = 0; j < 16; j++) acc[j] += (double)(int)v[j] * sc;
        }
        if (row < g.M) {
#pragma unroll
          for (int j = 0; j < 16; j++) {
            const int col = n0 + c0 + j;
            if (col < g.N) {
              const int ec = g.b_exp[col];
              double out;
              if (er == OZ_EXP_NONFINITE || ec == OZ_EXP_NONFINITE) out = __longlong_as_double(0x7ff8000000000000ll);
              else out = ldexp(acc[j], er + ec);
              double* p = col < g.nsplit ? g.c0 + (long long)col * g.ldc0
                                         : g.c1 + (long long)(col - g.nsplit) * g.ldc1;
              p[row] = out;
            }
          }
        }
      }
    } else {
      abort_flag = 1;
      atomicExch(g.err, 1);
    }
  }

  // Teardown: no TMA write or MMA may still be in flight when the CTA's shared
  // and tensor memory are released (on the normal path these waits return at
  // once; after an abort they wait, bounded, for copies and MMAs in flight).
  if (warp == 0 && lane == 0) {
    const int from = issued > OZ_STAGES ? issued - OZ_STAGES : 0;
    for (int kc = from; kc < issued; kc++)
      tc::mbar_wait(&full[kc % OZ_STAGES], (kc / OZ_STAGES) & 1, g.spin_limit, &no_abort);
  }
  if (warp == 1 && lane == 0) tc::mbar_wait(&acc_full, 0, g.spin_limit, &no_abort);
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tbase, C::TMEM_COLS);
  }
}

// ------------------------------------------------------------------ host
namespace {

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                 const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                 const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled from the driver, found once through the runtime.
EncodeTiled encode_tiled() {
  static std::once_flag once;
  static EncodeTiled fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
  });
  return fn;
}

// Tensor map of `slices` int8 matrices of rows x Kp (K contiguous), read in
// boxes of 32 (K) x box_rows x 1 with the 32-byte swizzle.
cudaError_t slice_map(CUtensorMap* m, const int8_t* base, int Kp, int rows, int slices,
                      int box_rows) {
  EncodeTiled f = encode_tiled();
  if (!f) return cudaErrorNotSupported;
  const cuuint64_t dims[3] = {(cuuint64_t)Kp, (cuuint64_t)rows, (cuuint64_t)slices};
  const cuuint64_t strides[2] = {(cuuint64_t)Kp, (cuuint64_t)Kp * (cuuint64_t)rows};
  const cuuint32_t box[3] = {(cuuint32_t)OZ_BK, (cuuint32_t)box_rows, 1};
  const cuuint32_t es[3] = {1, 1, 1};
  const CUresult r = f(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<int8_t*>(base), dims,
                       strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B,
                       CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }
int kpad(int K) { return (K + OZ_BK - 1) / OZ_BK * OZ_BK; }

struct OzScratch {
  int8_t* a;
  int8_t* b;
  int* ea;
  int* eb;
  unsigned long long* amax;
};

OzScratch carve(void* base, int M, int N, int K, int S) {
  const size_t Kp = (size_t)kpad(K);
  char* p = static_cast<char*>(base);
  OzScratch o;
  o.a = reinterpret_cast<int8_t*>(p);
  p += al256((size_t)S * M * Kp);
  o.b = reinterpret_cast<int8_t*>(p);
  p += al256((size_t)S * N * Kp);
  o.ea = reinterpret_cast<int*>(p);
  p += al256(sizeof(int) * (size_t)M);
  o.eb = reinterpret_cast<int*>(p);
  p += al256(sizeof(int) * (size_t)N);
  o.amax = reinterpret_cast<unsigned long long*>(p);
  return o;
}

template <int S>
cudaError_t gemm_s(const CUtensorMap& ma, const CUtensorMap& mb, const OzGemmArgs& g,
                   cudaStream_t st) {
  static PerDevice once;
  const int pend = once.pending();
  if (pend >= 0) {
    cudaError_t e = cudaFuncSetAttribute(ozaki_gemm_kernel<S>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)OzCfg<S>::SMEM);
    if (e != cudaSuccess) return e;
    once.mark(pend);
  }
  const dim3 grid((g.M + OZ_BM - 1) / OZ_BM, (g.N + OZ_BN - 1) / OZ_BN);
  ozaki_gemm_kernel<S><<<grid, OZ_THREADS, OzCfg<S>::SMEM, st>>>(ma, mb, g);
  return cudaGetLastError();
}

}  // namespace

size_t ozaki_scratch_bytes(int M, int N, int K, int S) {
  const size_t Kp = (size_t)kpad(K);
  return al256((size_t)S * M * Kp) + al256((size_t)S * N * Kp) + al256(sizeof(int) * (size_t)M) +
         al256(sizeof(int) * (size_t)N) + al256(sizeof(unsigned long long) * (size_t)M);
}

cudaError_t launch_ozaki_product(const OzProduct& p, cudaStream_t st) {
  if (p.M <= 0 || p.N <= 0 || p.K <= 0) return cudaSuccess;
  if (p.S < kOzakiMinSlices || p.S > kOzakiMaxSlices || p.K > kOzakiMaxK) return cudaErrorInvalidValue;
  if (((uintptr_t)p.scratch & 255) != 0) return cudaErrorInvalidValue;
  const int Kp = kpad(p.K);
  OzScratch o = carve(p.scratch, p.M, p.N, p.K, p.S);
  OzSplitArgs sa;
  sa.a0 = p.a0;
  sa.a1 = p.a1;
  sa.lda0 = p.lda0;
  sa.lda1 = p.lda1;
  sa.ksplit = p.ksplit;
  sa.rlim0 = p.rlim0;
  sa.roff0 = p.roff0;
  sa.M = p.M;
  sa.K = p.K;
  sa.Kp = Kp;
  sa.a_out = o.a;
  sa.a_slice = (long long)p.M * Kp;
  sa.a_exp = o.ea;
  sa.b = p.b;
  sa.ldb = p.ldb;
  sa.N = p.N;
  sa.b_out = o.b;
  sa.b_slice = (long long)p.N * Kp;
  sa.b_exp = o.eb;
  sa.S = p.S;
  sa.a_max = o.amax;
  const int row_blocks = (p.M + OZ_SPLIT_ROWS - 1) / OZ_SPLIT_ROWS;
  sa.a_chunks = (Kp + OZ_SPLIT_CHUNK - 1) / OZ_SPLIT_CHUNK;
  sa.a_blocks = row_blocks * sa.a_chunks;
  const int b_blocks = (p.N + 7) / 8;
  cudaError_t e = cudaMemsetAsync(o.amax, 0, sizeof(unsigned long long) * (size_t)p.M, st);
  if (e != cudaSuccess) return e;
  ozaki_rowmax_kernel<<<dim3(row_blocks, (p.K + OZ_MAX_COLS - 1) / OZ_MAX_COLS), OZ_SPLIT_THREADS,
                        0, st>>>(sa);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  ozaki_split_kernel<<<sa.a_blocks + b_blocks, OZ_SPLIT_THREADS, 0, st>>>(sa);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  CUtensorMap ma, mb;
  if ((e = slice_map(&ma, o.a, Kp, p.M, p.S, OZ_BM)) != cudaSuccess) return e;
  if ((e = slice_map(&mb, o.b, Kp, p.N, p.S, OZ_BN)) != cudaSuccess) return e;
  OzGemmArgs g;
  g.M = p.M;
  g.N = p.N;
  g.Kp = Kp;
  g.a_exp = o.ea;
  g.b_exp = o.eb;
  g.c0 = p.c0;
  g.c1 = p.c1;
  g.ldc0 = p.ldc0;
  g.ldc1 = p.ldc1;
  g.nsplit = p.nsplit;
  g.err = p.err;
  g.spin_limit = 1ll << 20;  // polls of mbarrier.try_wait: about a second at most
  switch (p.S) {
    case 3: return gemm_s<3>(ma, mb, g, st);
    case 4: return gemm_s<4>(ma, mb, g, st);
    case 5: return gemm_s<5>(ma, mb, g, st);
    case 6: return gemm_s<6>(ma, mb, g, st);
    case 7: return gemm_s<7>(ma, mb, g, st);
    default: return gemm_s<8>(ma, mb, g, st);
  }
}

cudaError_t preload_ozaki(size_t* local) {
  cudaError_t e;
  if ((e = preload_one(ozaki_rowmax_kernel, local)) != cudaSuccess) return e;
  if ((e = preload_one(ozaki_split_kernel, local)) != cudaSuccess) return e;
  if ((e = preload_one(ozaki_gemm_kernel<3>, local)) != cudaSuccess) return e;
  if ((e = preload_one(ozaki_gemm_kernel<4>, local)) != cudaSuccess) return e;
  if ((e = preload_one(ozaki_gemm_kernel<5>, local)) != cudaSuccess) return e;
  if ((e = preload_one(ozaki_gemm_kernel<6>, local)) != cudaSuccess) return e;
  if ((e = preload_one(ozaki_gemm_kernel<7>, local)) != cudaSuccess) return e;
  return preload_one(ozaki_gemm_kernel<8>, local);
}

}  // namespace bsofi
