// Complex-FP32 GEMM on the 5th-generation tensor cores (tcgen05, kind::tf32)
// for the precision form of the LU: C <- C - A*B with A (M x K), B (K x N),
// C (M x N) complex64, column-major, interleaved (re, im).
//
// Real embedding: with A~ the 2M x 2K real matrix of 2x2 blocks
// [[ar, -ai], [ai, ar]], B~ = B's interleaved storage read as a real
// 2K x N column-major matrix and C~ likewise for C, C~ -= A~ B~ is exactly the
// complex update.  So B and C are used in place; only A is expanded once
// into a K-major (row-major 2M x 2K) copy by k_expand_a.
//
// Kernel: persistent, one CTA per SM, tiles of 128 rows x BN (64, 128 or
// 256: the widest that gives every SM a tile) columns of C~, taken in a grouped raster (TC_GROUP row blocks at a time,
// all column blocks of the group, rows fastest) so that the tiles running at
// once share their A rows and B columns in L2.  Warp roles:
//   warp 0, one lane: TMA producer -- 128B-swizzled boxes of 32 fp32 of K
//     for A~ (128 rows) and B (BN rows), a TC_STAGES-deep ring of shared
//     memory guarded by full/empty mbarriers;
//   warp 1, one lane: MMA issuer -- tcgen05.mma kind::tf32 (M = 128,
//     N = BN, K = 8 per instruction) into one of two TMEM accumulators
//     (2 x BN of the 512 columns), tcgen05.commit releasing ring slots and,
//     after a tile's last K block, signalling its accumulator full;
//   warps 2-5: epilogue -- tcgen05.ld of the accumulator (TMEM lane = row;
//     warp w reads lanes 32 (w % 4)...), C -= acc in place, then the
//     accumulator is released, so a tile's epilogue overlaps the next
//     tile's main loop.
// Every mbarrier wait is bounded; on timeout the kernel records an error
// code, every role leaves its loop, outstanding copies are drained and the
// TMEM is freed before returning.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>

#include "internal.h"

namespace bg {

#define TC_BM 128            // rows of C~ per tile (= 64 complex rows)
#define TC_BK 32             // fp32 of K per stage (one 128-byte swizzle row)
#define TC_STAGES 4
#define TC_GROUP 16          // row blocks per raster group
#define TC_THREADS 192       // producer warp, MMA warp, 4 epilogue warps
#define TC_A_BYTES (TC_BM * TC_BK * 4)
#define TC_SPIN_LIMIT (1u << 26)

template <int BN>
struct TcCfg {
  static constexpr int B_BYTES = BN * TC_BK * 4;
  static constexpr int STAGE_BYTES = TC_A_BYTES + B_BYTES;
  static constexpr int SMEM = TC_STAGES * STAGE_BYTES + 1024 + 256;
  static constexpr int TMEM_COLS = 2 * BN;     // two accumulators
};

struct TcArgs {
  int M2, N, K2;         // C~ rows (2M), columns, reduction length (2K)
  float *C;              // interleaved complex64 storage of C (column-major, ldc complex)
  size_t ldc;            // in complex elements
  int *err;              // device error flag
  int ntm, ntn;          // row and column blocks
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes));
}
// bounded wait on phase parity; returns false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  uint32_t addr = smem_u32(bar);
  for (uint32_t it = 0; it < TC_SPIN_LIMIT; it++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity));
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(smem_u32(dst)), "l"((uint64_t)map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// K-major, 128-byte swizzle shared-memory matrix descriptor (sm_100 UMMA):
// start>>4 in [0,14), LBO (unused for swizzled K-major) = 1 in [16,30),
// SBO = 1024 B (one 8-row swizzle atom) >> 4 in [32,46), version 1 in [46,48),
// layout SWIZZLE_128B = 2 in [61,64).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// instruction descriptor, kind::tf32: D f32 (bits 4-5 = 1), A/B tf32 (2 at
// bits 7-9 and 10-12), both K-major, N>>3 at 17-22, M>>4 at 24-28
__host__ __device__ constexpr uint32_t tf32_idesc(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// tile t of the grouped raster -> (row block, column block)
__device__ __forceinline__ void tc_tile(const TcArgs &P, int t, int &tm, int &tn) {
  const int per = TC_GROUP * P.ntn;
  const int g = t / per, w = t - g * per;
  const int gm = min(TC_GROUP, P.ntm - g * TC_GROUP);
  tn = w / gm;
  tm = g * TC_GROUP + (w - tn * gm);
}

template <int BN>
__global__ void __launch_bounds__(TC_THREADS, 1)
    k_cgemm_tf32(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, TcArgs P) {
  typedef TcCfg<BN> Cfg;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-byte aligned ring (the 128B swizzle pattern repeats every 1024 bytes)
  unsigned char *ring = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t *full = (uint64_t *)(ring + TC_STAGES * Cfg::STAGE_BYTES);
  uint64_t *empty = full + TC_STAGES;
  uint64_t *acc_full = empty + TC_STAGES;     // [2]
  uint64_t *acc_empty = acc_full + 2;         // [2]
  uint64_t *mma_done = acc_empty + 2;         // every MMA of this CTA has finished
  uint32_t *tmem_slot = (uint32_t *)(mma_done + 1);
  __shared__ volatile int s_fail;
  __shared__ int s_issued, s_consumed;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nk = (P.K2 + TC_BK - 1) / TC_BK;
  const int ntiles = P.ntm * P.ntn;

  if (threadIdx.x == 0) {
    for (int s = 0; s < TC_STAGES; s++) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
    for (int b = 0; b < 2; b++) { mbar_init(&acc_full[b], 1); mbar_init(&acc_empty[b], 4); }
    mbar_init(mma_done, 1);
    s_fail = 0;
    s_issued = 0;
    s_consumed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(Cfg::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      // producer: TMA into the ring; kc counts K blocks over all tiles of this CTA
      int kc = 0;
      for (int t = blockIdx.x; t < ntiles && !s_fail; t += gridDim.x) {
        int tm, tn;
        tc_tile(P, t, tm, tn);
        for (int kb = 0; kb < nk; kb++, kc++) {
          const int s = kc % TC_STAGES;
          if (kc >= TC_STAGES && !mbar_wait(&empty[s], ((kc / TC_STAGES) - 1) & 1)) { s_fail = 1; break; }
          unsigned char *sa = ring + s * Cfg::STAGE_BYTES;
          mbar_expect_tx(&full[s], Cfg::STAGE_BYTES);
          tma_load_2d(sa, &mapA, kb * TC_BK, tm * TC_BM, &full[s]);
          tma_load_2d(sa + TC_A_BYTES, &mapB, kb * TC_BK, tn * BN, &full[s]);
          s_issued = kc + 1;
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // MMA issuer: tile i of this CTA accumulates in TMEM columns (i & 1) * BN
      const uint32_t idesc = tf32_idesc(TC_BM, BN);
      int kc = 0, i = 0;
      for (int t = blockIdx.x; t < ntiles && !s_fail; t += gridDim.x, i++) {
        const int b = i & 1;
        if (i >= 2 && !mbar_wait(&acc_empty[b], ((i >> 1) - 1) & 1)) { s_fail = 4; break; }
        asm volatile("tcgen05.fence::after_thread_sync;");
        const uint32_t dt = tmem + (uint32_t)(b * BN);
        for (int kb = 0; kb < nk; kb++, kc++) {
          const int s = kc % TC_STAGES;
          if (!mbar_wait(&full[s], (kc / TC_STAGES) & 1)) { s_fail = 2; break; }
          asm volatile("tcgen05.fence::after_thread_sync;");
          const uint32_t sa = smem_u32(ring + s * Cfg::STAGE_BYTES), sb = sa + TC_A_BYTES;
#pragma unroll
          for (int k = 0; k < TC_BK / 8; k++) {
            uint64_t da = sw128_desc(sa + k * 32), db = sw128_desc(sb + k * 32);
            uint32_t acc = (kb > 0 || k > 0) ? 1u : 0u;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
                ::"r"(dt), "l"(da), "l"(db), "r"(idesc), "r"(acc));
          }
          // release the slot once these MMAs have read it
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              smem_u32(&empty[s])));
          s_consumed = kc + 1;
        }
        if (s_fail) break;
        // accumulator b is complete when every MMA issued so far has finished
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            smem_u32(&acc_full[b])));
      }
      // no MMA may still run when the TMEM is freed, whichever way the loop ended
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(mma_done)));
      if (!mbar_wait(mma_done, 0) && !s_fail) s_fail = 5;
    }
  } else {
    // epilogue warps 2..5: TMEM lanes 32 (warp % 4) .. + 31
    const int q = warp & 3;
    const size_t ldr = 2 * P.ldc;    // real leading dimension of C~
    int i = 0;
    for (int t = blockIdx.x; t < ntiles && !s_fail; t += gridDim.x, i++) {
      const int b = i & 1;
      int tm, tn;
      tc_tile(P, t, tm, tn);
      if (!mbar_wait(&acc_full[b], (i >> 1) & 1)) { s_fail = 3; break; }
      asm volatile("tcgen05.fence::after_thread_sync;");
      const int row = tm * TC_BM + q * 32 + lane;   // row of C~ (2 x complex row + component)
#pragma unroll 1
      for (int c0 = 0; c0 < BN; c0 += 32) {
        // the 32 loads of C are issued together, before the TMEM read, so
        // that their latencies overlap (a load-subtract-store per column
        // would wait for the previous column's store: C's columns may alias
        // as far as the compiler knows)
        const int col0 = tn * BN + c0;
        float *pc = P.C + (size_t)col0 * ldr + row;
        float cv[32];
        if (row < P.M2) {
#pragma unroll
          for (int j = 0; j < 32; j++) cv[j] = col0 + j < P.N ? pc[(size_t)j * ldr] : 0.f;
        }
        uint32_t r[32];
        const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * BN + c0);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
              "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
              "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
              "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;");
        if (row < P.M2) {
#pragma unroll
          for (int j = 0; j < 32; j++)
            if (col0 + j < P.N) pc[(size_t)j * ldr] = cv[j] - __uint_as_float(r[j]);
        }
      }
      // this warp has read accumulator b: hand it back to the MMA issuer
      asm volatile("tcgen05.fence::before_thread_sync;");
      __syncwarp();
      if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&acc_empty[b])) : "memory");
    }
  }
  __syncthreads();
  if (s_fail && threadIdx.x == 0) {
    atomicExch(P.err, s_fail);
    // drain: wait (bounded) for TMA copies issued but never consumed
    for (int c = s_consumed; c < s_issued; c++) mbar_wait(&full[c % TC_STAGES], (c / TC_STAGES) & 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Cfg::TMEM_COLS));
}

// A~ (row-major 2M x 2K, leading dimension lda2 floats) from complex A (M x K
// column-major, lda complex): rows 2m, 2m+1 and columns 2k, 2k+1 hold
// [[ar, -ai], [ai, ar]].  32 x 32 tiles through shared memory: reads
// coalesced along m (A's columns), writes coalesced along k (A~'s rows).
__global__ void __launch_bounds__(256) k_expand_a(int M, int K, const float2 *A, size_t lda, float *At, size_t lda2) {
  __shared__ float2 tile[32][33];
  const int m0 = blockIdx.x * 32, k0 = blockIdx.y * 32, tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int k = k0 + ty + 8 * q, m = m0 + tx;
    if (k < K && m < M) tile[ty + 8 * q][tx] = A[(size_t)k * lda + m];
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int m = m0 + ty + 8 * q, k = k0 + tx;
    if (k < K && m < M) {
      const float2 a = tile[tx][ty + 8 * q];
      *(float2 *)(At + (size_t)(2 * m) * lda2 + 2 * k) = make_float2(a.x, -a.y);
      *(float2 *)(At + (size_t)(2 * m + 1) * lda2 + 2 * k) = make_float2(a.y, a.x);
    }
  }
}

// ------------------------------------------------------------------ host side
typedef CUresult (*PFN_encodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                    const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                    CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static PFN_encodeTiled get_encode() {
  static PFN_encodeTiled fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_encodeTiled)p;
  }
  return fn;
}

// 2D fp32 tensor map over a row-major (rows x cols) array with leading
// dimension ld floats; box = 32 floats (128 B, swizzled) x box_rows (<= 256)
static int make_map(CUtensorMap *map, const float *base, uint64_t cols, uint64_t rows, uint64_t ld, uint32_t box_rows) {
  PFN_encodeTiled enc = get_encode();
  if (!enc) { set_error("cuTensorMapEncodeTiled unavailable"); return BG_ERR_CUDA; }
  if (((uintptr_t)base & 15) || ((ld * 4) & 15)) { set_error("TMA base/stride not 16-byte aligned"); return BG_ERR_ARG; }
  cuuint64_t dims[2] = {cols, rows};
  cuuint64_t strides[1] = {ld * 4};
  cuuint32_t box[2] = {TC_BK, box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void *)base, dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) { set_error("cuTensorMapEncodeTiled failed (%d)", (int)r); return BG_ERR_CUDA; }
  return BG_OK;
}

template <int BN>
static int launch_tf32(const CUtensorMap &mA, const CUtensorMap &mB, TcArgs P) {
  typedef TcCfg<BN> Cfg;
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    BG_CUDA_TRY(cudaGetDevice(&dev));
    BG_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    BG_CUDA_TRY(cudaFuncSetAttribute(k_cgemm_tf32<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM));
  }
  P.ntm = (P.M2 + TC_BM - 1) / TC_BM;
  P.ntn = (P.N + BN - 1) / BN;
  const int ntiles = P.ntm * P.ntn;
  k_cgemm_tf32<BN><<<std::min(ntiles, sms), TC_THREADS, Cfg::SMEM, stream()>>>(mA, mB, P);
  BG_LAUNCHED();
  return BG_OK;
}

// C -= A*B, complex64 column-major interleaved; At is a device scratch of at
// least 2M x round_up(2K, 32) floats; err a device int (0 on entry).
int cgemm_sub_tf32(int M, int N, int K, const void *A, size_t lda, const void *B, size_t ldb, void *C, size_t ldc,
                   float *At, int *err) {
  if (M <= 0 || N <= 0 || K <= 0) return BG_OK;
  size_t lda2 = ((size_t)2 * K + 31) / 32 * 32;
  dim3 eg((M + 31) / 32, (K + 31) / 32);
  k_expand_a<<<eg, 256, 0, stream()>>>(M, K, (const float2 *)A, lda, At, lda2);
  BG_LAUNCHED();
  // widest tile that still gives every SM a tile (skinny updates of the
  // triangular solves have one row block and few column blocks)
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    BG_CUDA_TRY(cudaGetDevice(&dev));
    BG_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  }
  const long ntm = (2L * M + TC_BM - 1) / TC_BM;
  int BN = N > 128 ? 256 : (N > 64 ? 128 : 64);
  while (BN > 64 && ntm * ((N + BN - 1) / BN) < sms) BN /= 2;
  CUtensorMap mA, mB;
  int st = make_map(&mA, At, (uint64_t)2 * K, (uint64_t)2 * M, lda2, TC_BM);
  if (!st) st = make_map(&mB, (const float *)B, (uint64_t)2 * K, (uint64_t)N, 2 * ldb, BN);
  if (st) return st;
  TcArgs P{2 * M, N, 2 * K, (float *)C, ldc, err, 0, 0};
  prof_start(PROF_GEMM);
  st = BN == 256 ? launch_tf32<256>(mA, mB, P) : (BN == 128 ? launch_tf32<128>(mA, mB, P) : launch_tf32<64>(mA, mB, P));
  prof_stop(PROF_GEMM, 8.0 * M * (double)N * K);
  return st;
}

// One stand-alone GEMM on the library stream with its own scratch (the
// expanded A~ and the error word), synchronised, the pipeline status checked.
int cgemm_sub_device(int M, int N, int K, const void *A, int lda, const void *B, int ldb, void *C, int ldc) {
  if (M <= 0 || N <= 0 || K <= 0) return BG_OK;
  size_t lda2 = ((size_t)2 * K + 31) / 32 * 32;
  float *At = nullptr;
  int *err = nullptr;
  BG_CUDA_TRY(cudaMalloc(&At, sizeof(float) * 2 * (size_t)M * lda2 + 256));
  int *errp = (int *)((char *)At + sizeof(float) * 2 * (size_t)M * lda2);
  err = errp;
  int st = BG_OK;
  cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int), stream());
  if (e != cudaSuccess) { set_error("cudaMemsetAsync: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
  if (!st) st = cgemm_sub_tf32(M, N, K, A, (size_t)lda, B, (size_t)ldb, C, (size_t)ldc, At, err);
  int h = 0;
  if (!st) {
    e = cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, stream());
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream());
    if (e != cudaSuccess) { set_error("complex64 GEMM: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
    else if (h) { set_error("tensor-core GEMM reported a pipeline timeout (code %d)", h); st = BG_ERR_CUDA; }
  } else {
    cudaStreamSynchronize(stream());
  }
  cudaFree(At);
  return st;
}

}  // namespace bg
