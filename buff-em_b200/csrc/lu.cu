// Dense complex128 LU with partial pivoting and the triangular solves on
// sm_100a: replaces HMatrix::LUFactorize / LUSolve (LAPACK zgetrf / zgetrs,
// call sites buff-scatter.cc:285,314).
//
// Factorisation: recursive right-looking LU over column halves.  Leaves of
// width <= 32 are factored by one cooperative kernel (all CTAs own a slice of
// the panel rows in shared memory; one grid barrier per column: pivot
// candidates of every CTA -> global winner -> swap, scale, rank-1 update).
// Row interchanges are then applied to every other column (LAPACK ipiv
// semantics: ipiv[i] is the 1-based row swapped with row i, applied in
// order).  Off-diagonal blocks use a unit-lower TRSM (leaf kernel + GEMM
// recursion) and the Schur complements use a complex GEMM on the FP64 tensor
// cores (mma.sync m8n8k4 f64; tcgen05 has no f64 kind), 4M complex product,
// three-stage cp.async pipeline.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <mutex>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "internal.h"

namespace cg = cooperative_groups;

namespace bg {

struct cdl { double r, i; };
struct cfl { float r, i; };
template <class C> struct CxT;
template <> struct CxT<cdl> { typedef double R; };
template <> struct CxT<cfl> { typedef float R; };

// tensor-core complex-FP32 GEMM (gemm_tc.cu)
int cgemm_sub_tf32(int M, int N, int K, const void *A, size_t lda, const void *B, size_t ldb, void *C, size_t ldc,
                   float *At, int *err);

// =========================================================================
// complex GEMM  C(MxN) -= A(MxK) * B(KxN), column-major, complex128, on the
// FP64 tensor cores with mma.sync m16n8k16 f64 (the sm_90+/sm_100 DMMA shape:
// 2048 FMAs per instruction).  Warp tile 32x32 complex (2 x m16, 4 x n8),
// CTA tile BM x BN, K chunk BK, STAGES-deep cp.async pipeline.  Shared tiles
// are complex-interleaved (one 16-byte load gives re and im); row strides are
// padded so every fragment load phase hits 32 distinct banks.
//   Cr += Ar Br + Ai (-Bi),   Ci += Ar Bi + Ai Br        (4M product)
// Fragment layouts (m16n8k16, lane = 4*t1 + t0):
//   A: a[v] = A[t1 + 8(v&1)][t0 + 4(v>>1)], v = 0..7
//   B: b[v] = B[t0 + 4v][t1],               v = 0..3
//   C: c[v] = C[t1 + 8(v>>1)][2 t0 + (v&1)]
// =========================================================================
__device__ __forceinline__ void dmma16(double (&d)[4], const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
      "{%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]),
        "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

__device__ __forceinline__ void cp16(void *smem, const void *gmem, bool pred) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int n = pred ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <int BM, int BN, int BK, int STAGES>
struct GemmCfg {
  static constexpr int WM = BM / 32, WN = BN / 32, THREADS = WM * WN * 32;
  static constexpr int AP = BM + 2;   // As[k][m] stride (complex), = 2 mod 8
  static constexpr int BP = BK + 4;   // Bs[n][k] stride (complex), = 4 mod 8
  static constexpr int SMEM = STAGES * (BK * AP + BN * BP) * 16;
};

template <int BM, int BN, int BK, int STAGES>
__global__ void __launch_bounds__(GemmCfg<BM, BN, BK, STAGES>::THREADS)
    k_zgemm_sub(int M, int N, int K, const cdl *__restrict__ A, size_t lda, const cdl *__restrict__ B, size_t ldb,
                cdl *C, size_t ldc) {
  using Cfg = GemmCfg<BM, BN, BK, STAGES>;
  constexpr int T = Cfg::THREADS, AP = Cfg::AP, BP = Cfg::BP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cdl *As = (cdl *)smem_raw;              // [STAGES][BK][AP]
  cdl *Bs = As + STAGES * BK * AP;        // [STAGES][BN][BP]
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp % Cfg::WM, wn = warp / Cfg::WM;
  const int t0 = lane & 3, t1 = lane >> 2;
  double cr[2][4][4], ci[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int v = 0; v < 4; v++) cr[i][j][v] = ci[i][j][v] = 0.0;
  const int nchunks = (K + BK - 1) / BK;
  auto load_chunk = [&](int chunk, int stage) {
    const int k0 = chunk * BK;
    cdl *as = As + stage * BK * AP;
    cdl *bs = Bs + stage * BN * BP;
#pragma unroll
    for (int it = 0; it < (BM * BK) / T; it++) {
      int e = tid + it * T;
      int r = e % BM, kk = e / BM;
      int gr = m0 + r, gk = k0 + kk;
      bool ok = gr < M && gk < K;
      cp16(as + kk * AP + r, ok ? A + (size_t)gk * lda + gr : A, ok);
    }
#pragma unroll
    for (int it = 0; it < (BK * BN) / T; it++) {
      int e = tid + it * T;
      int kb = e % BK, nb = e / BK;
      int gk = k0 + kb, gn = n0 + nb;
      bool ok = gk < K && gn < N;
      cp16(bs + nb * BP + kb, ok ? B + (size_t)gn * ldb + gk : B, ok);
    }
  };
#pragma unroll
  for (int s = 0; s < STAGES - 1; s++) {
    if (s < nchunks) load_chunk(s, s);
    cp_commit();
  }
  for (int chunk = 0; chunk < nchunks; chunk++) {
    cp_wait<STAGES - 2>();
    __syncthreads();
    int nxt = chunk + STAGES - 1;
    if (nxt < nchunks) load_chunk(nxt, nxt % STAGES);
    cp_commit();
    const cdl *as = As + (chunk % STAGES) * BK * AP + wm * 32 + t1;
    const cdl *bs = Bs + (chunk % STAGES) * BN * BP + (wn * 32 + t1) * BP + t0;
#pragma unroll
    for (int ks = 0; ks < BK / 16; ks++) {
      double ar[2][8], ai[2][8];
#pragma unroll
      for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int v = 0; v < 8; v++) {
          cdl x = as[(ks * 16 + t0 + 4 * (v >> 1)) * AP + mt * 16 + 8 * (v & 1)];
          ar[mt][v] = x.r;
          ai[mt][v] = x.i;
        }
#pragma unroll
      for (int nt = 0; nt < 4; nt++) {
        double br[4], bi[4], nbi[4];
#pragma unroll
        for (int v = 0; v < 4; v++) {
          cdl x = bs[nt * 8 * BP + ks * 16 + 4 * v];
          br[v] = x.r;
          bi[v] = x.i;
          nbi[v] = -x.i;
        }
#pragma unroll
        for (int mt = 0; mt < 2; mt++) {
          dmma16(cr[mt][nt], ar[mt], br);
          dmma16(cr[mt][nt], ai[mt], nbi);
          dmma16(ci[mt][nt], ar[mt], bi);
          dmma16(ci[mt][nt], ai[mt], br);
        }
      }
    }
  }
  cp_wait<0>();
  // C -= accumulators, eight entries at a time: the loads of a group are
  // issued together before its stores (one memory round trip per group
  // instead of one per entry)
#pragma unroll
  for (int nt = 0; nt < 4; nt++) {
    cdl x[2][4];
#pragma unroll
    for (int mt = 0; mt < 2; mt++)
#pragma unroll
      for (int v = 0; v < 4; v++) {
        const int row = m0 + wm * 32 + mt * 16 + t1 + 8 * (v >> 1);
        const int col = n0 + wn * 32 + nt * 8 + 2 * t0 + (v & 1);
        x[mt][v] = (row < M && col < N) ? C[(size_t)col * ldc + row] : cdl{0.0, 0.0};
      }
#pragma unroll
    for (int mt = 0; mt < 2; mt++)
#pragma unroll
      for (int v = 0; v < 4; v++) {
        const int row = m0 + wm * 32 + mt * 16 + t1 + 8 * (v >> 1);
        const int col = n0 + wn * 32 + nt * 8 + 2 * t0 + (v & 1);
        if (row < M && col < N) {
          cdl y = x[mt][v];
          y.r -= cr[mt][nt][v];
          y.i -= ci[mt][nt][v];
          C[(size_t)col * ldc + row] = y;
        }
      }
  }
}

// CTA tile of the complex128 GEMM, chosen at run time (the batching form's
// autotuner times them per size class): 0 = 64 x 64, 1 = 128 x 64,
// 2 = 64 x 128 complex outputs; warps always own 32 x 32.
static int zg_tile = 0;
void lu_set_gemm_tile(int t) { zg_tile = (t >= 0 && t <= 2) ? t : 0; }
int lu_get_gemm_tile() { return zg_tile; }

template <int BM, int BN>
static int zgemm_launch(int M, int N, int K, const cdl *A, size_t lda, const cdl *B, size_t ldb, cdl *C, size_t ldc) {
  using Cfg = GemmCfg<BM, BN, 16, 3>;
  auto kern = k_zgemm_sub<BM, BN, 16, 3>;
  static bool attr = false;
  if (!attr) {
    BG_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM));
    attr = true;
  }
  dim3 grid((M + BM - 1) / BM, (N + BN - 1) / BN);
  if (grid.y > 65535) { set_error("zgemm: N too large"); return BG_ERR_ARG; }
  kern<<<grid, Cfg::THREADS, Cfg::SMEM, stream()>>>(M, N, K, A, lda, B, ldb, C, ldc);
  BG_LAUNCHED();
  return BG_OK;
}

static int zgemm_sub(int M, int N, int K, const cdl *A, size_t lda, const cdl *B, size_t ldb, cdl *C, size_t ldc) {
  if (M <= 0 || N <= 0 || K <= 0) return BG_OK;
  prof_start(PROF_GEMM);
  int st = zg_tile == 1 ? zgemm_launch<128, 64>(M, N, K, A, lda, B, ldb, C, ldc)
         : zg_tile == 2 ? zgemm_launch<64, 128>(M, N, K, A, lda, B, ldb, C, ldc)
                        : zgemm_launch<64, 64>(M, N, K, A, lda, B, ldb, C, ldc);
  prof_stop(PROF_GEMM, 8.0 * M * (double)N * K);
  return st;
}

// =========================================================================
// leaf triangular solves (n <= 64 rows).  The triangle is staged in shared
// memory once per CTA; each warp then solves TRS_CPW right-hand-side columns
// together: lane l holds rows l and l+32 of each of its columns in registers,
// the solved entries of step i are broadcast with warp shuffles, and every
// lane updates its two rows of every column with the one triangle entry it
// read -- TRS_CPW independent recurrences per step, no block barriers inside
// the substitution.
// =========================================================================
#define TRS_WARPS 8
#define TRS_CPW 4                         // columns per warp per CTA
#define TRS_COLS (TRS_WARPS * TRS_CPW)
template <class C>
__device__ __forceinline__ C cshfl(C v, int src) {
  return C{__shfl_sync(0xffffffffu, v.r, src), __shfl_sync(0xffffffffu, v.i, src)};
}
template <class C>
__global__ void __launch_bounds__(TRS_WARPS * 32) k_trsm_leaf(int n, int m, const C *T, size_t ldt, C *B,
                                                              size_t ldb, int upper) {
  typedef typename CxT<C>::R R;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C(*Ts)[65] = (C(*)[65])smem_raw;   // Ts[r][c]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // staged eight loads per thread at a time (their latencies overlap)
  for (int e0 = 0; e0 < n * n; e0 += 8 * TRS_WARPS * 32) {
    C v[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int e = e0 + u * TRS_WARPS * 32 + tid;
      v[u] = e < n * n ? T[(size_t)(e / n) * ldt + e % n] : C{0, 0};
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int e = e0 + u * TRS_WARPS * 32 + tid;
      if (e < n * n) Ts[e % n][e / n] = v[u];
    }
  }
  __syncthreads();
  const int r0 = lane, r1 = lane + 32;
  const int cbase = blockIdx.x * TRS_COLS + warp * TRS_CPW;
  if (cbase >= m) return;
  C b0[TRS_CPW], b1[TRS_CPW];
#pragma unroll
  for (int j = 0; j < TRS_CPW; j++) {
    const int col = cbase + j;
    const C *bc = B + (size_t)col * ldb;
    b0[j] = (col < m && r0 < n) ? bc[r0] : C{0, 0};
    b1[j] = (col < m && r1 < n) ? bc[r1] : C{0, 0};
  }
  if (!upper) {
    for (int i = 0; i < n; i++) {
      const bool u0 = r0 > i && r0 < n, u1 = r1 > i && r1 < n;
      const C l0 = u0 ? Ts[r0][i] : C{0, 0}, l1 = u1 ? Ts[r1][i] : C{0, 0};
#pragma unroll
      for (int j = 0; j < TRS_CPW; j++) {
        const C x = cshfl(i < 32 ? b0[j] : b1[j], i & 31);
        if (u0) { b0[j].r -= l0.r * x.r - l0.i * x.i; b0[j].i -= l0.r * x.i + l0.i * x.r; }
        if (u1) { b1[j].r -= l1.r * x.r - l1.i * x.i; b1[j].i -= l1.r * x.i + l1.i * x.r; }
      }
    }
  } else {
    for (int i = n - 1; i >= 0; i--) {
      const C u = Ts[i][i];
      const R d = u.r * u.r + u.i * u.i;
      const bool u0 = r0 < i, u1 = r1 < i;
      const C t0 = u0 ? Ts[r0][i] : C{0, 0}, t1 = u1 ? Ts[r1][i] : C{0, 0};
#pragma unroll
      for (int j = 0; j < TRS_CPW; j++) {
        const C v = cshfl(i < 32 ? b0[j] : b1[j], i & 31);
        const C x{(v.r * u.r + v.i * u.i) / d, (v.i * u.r - v.r * u.i) / d};
        if (r0 == i) b0[j] = x;
        if (r1 == i) b1[j] = x;
        if (u0) { b0[j].r -= t0.r * x.r - t0.i * x.i; b0[j].i -= t0.r * x.i + t0.i * x.r; }
        if (u1) { b1[j].r -= t1.r * x.r - t1.i * x.i; b1[j].i -= t1.r * x.i + t1.i * x.r; }
      }
    }
  }
#pragma unroll
  for (int j = 0; j < TRS_CPW; j++) {
    const int col = cbase + j;
    if (col >= m) break;
    C *bc = B + (size_t)col * ldb;
    if (r0 < n) bc[r0] = b0[j];
    if (r1 < n) bc[r1] = b1[j];
  }
}

// small-N complex64 GEMM (C -= A B, N <= 16): one thread per row, used where
// a tensor-core tile would be mostly padding (few right-hand sides)
__global__ void k_cgemm_small(int M, int N, int K, const cfl *A, size_t lda, const cfl *B, size_t ldb, cfl *Cm,
                              size_t ldc) {
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= M) return;
  float ar[16], ai[16];
  for (int n = 0; n < N; n++) ar[n] = ai[n] = 0.f;
  for (int k = 0; k < K; k++) {
    cfl a = A[(size_t)k * lda + m];
#pragma unroll 4
    for (int n = 0; n < N; n++) {
      cfl b = B[(size_t)n * ldb + k];
      ar[n] += a.r * b.r - a.i * b.i;
      ai[n] += a.r * b.i + a.i * b.r;
    }
  }
  for (int n = 0; n < N; n++) {
    cfl *p = Cm + (size_t)n * ldc + m;
    p->r -= ar[n];
    p->i -= ai[n];
  }
}

// per-matrix scratch for the tensor-core path
struct TcScratch {
  float *At = nullptr;
  size_t at_floats = 0;
  int *err = nullptr;
};
static thread_local TcScratch *t_tc = nullptr;
#define TC_MCHUNK 8192

static int gemm_sub(int M, int N, int K, const cdl *A, size_t lda, const cdl *B, size_t ldb, cdl *C, size_t ldc) {
  return zgemm_sub(M, N, K, A, lda, B, ldb, C, ldc);
}
static int gemm_sub(int M, int N, int K, const cfl *A, size_t lda, const cfl *B, size_t ldb, cfl *C, size_t ldc) {
  if (M <= 0 || N <= 0 || K <= 0) return BG_OK;
  if (N <= 16 || !t_tc) {
    if (N > 16) { set_error("complex64 GEMM needs the tensor-core scratch"); return BG_ERR_STATE; }
    k_cgemm_small<<<(M + 127) / 128, 128, 0, stream()>>>(M, N, K, A, lda, B, ldb, C, ldc);
    BG_LAUNCHED();
    return BG_OK;
  }
  size_t lda2 = ((size_t)2 * K + 31) / 32 * 32;
  size_t cap = std::min<size_t>(t_tc->at_floats / (2 * lda2), TC_MCHUNK);
  int mch = (int)std::min<size_t>((size_t)M, cap);
  if (mch < M) mch = mch / 64 * 64;   // chunked: whole 64-row tiles per chunk
  if (mch <= 0) { set_error("tensor-core scratch too small"); return BG_ERR_STATE; }
  for (int m0 = 0; m0 < M; m0 += mch) {
    int mm = std::min(mch, M - m0);
    int st = cgemm_sub_tf32(mm, N, K, A + m0, lda, B, ldb, C + m0, ldc, t_tc->At, t_tc->err);
    if (st) return st;
  }
  return BG_OK;
}

// X = L^{-1} B (unit lower, upper=0) or U^{-1} B (upper=1), L/U n x n at T
template <class C>
static int trsm(int n, int m, const C *T, size_t ldt, C *B, size_t ldb, int upper) {
  if (n <= 0 || m <= 0) return BG_OK;
  if (n <= 64) {
    const int smem = 64 * 65 * (int)sizeof(C);
    static bool attr = false;
    if (!attr) {
      BG_CUDA_TRY(cudaFuncSetAttribute(k_trsm_leaf<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      attr = true;
    }
    int blocks = (m + TRS_COLS - 1) / TRS_COLS;
    prof_start(PROF_TRSM);
    k_trsm_leaf<C><<<blocks, TRS_WARPS * 32, smem, stream()>>>(n, m, T, ldt, B, ldb, upper);
    BG_LAUNCHED();
    prof_stop(PROF_TRSM, 4.0 * n * (double)n * m);
    return BG_OK;
  }
  int n1 = (n / 2 + 31) / 32 * 32;
  if (n1 >= n) n1 = n / 2;
  int n2 = n - n1;
  int st;
  if (!upper) {
    if ((st = trsm(n1, m, T, ldt, B, ldb, 0))) return st;
    if ((st = gemm_sub(n2, m, n1, T + n1, ldt, B, ldb, B + n1, ldb))) return st;
    return trsm(n2, m, T + n1 + (size_t)n1 * ldt, ldt, B + n1, ldb, 0);
  }
  if ((st = trsm(n2, m, T + n1 + (size_t)n1 * ldt, ldt, B + n1, ldb, 1))) return st;
  if ((st = gemm_sub(n1, m, n2, T + (size_t)n1 * ldt, ldt, B + n1, ldb, B, ldb))) return st;
  return trsm(n1, m, T, ldt, B, ldb, 1);
}

// =========================================================================
// cooperative panel factorisation of A[k0:Nr, k0:k0+w] (w <= 32).  Each CTA
// holds a slice of rows_per rows in shared memory, column-major (column c at
// S + c * rows_per): the pivot scan and the rank-1 update walk a column with
// consecutive threads on consecutive rows, free of bank conflicts.  One grid
// barrier per column exchanges the CTAs' pivot candidates.
// =========================================================================
template <class C>
struct PanelArgs {
  C *A;
  size_t ld;
  int Nr;          // number of rows of the full matrix
  int k0, w;
  int rows_per;    // rows owned per CTA
  int *ipiv;       // global, 1-based
  int *info;       // device int (0 = ok)
  double *cval;    // [2][grid] candidate |re|+|im|
  int *cidx;       // [2][grid] candidate row
  C *crow;         // [2][grid][32] candidate row values
  C *jrow;         // [2][32] values of row k0+j before the swap
};

__device__ __forceinline__ bool better(double v, int i, double bv, int bi) {
  return v > bv || (v == bv && i < bi);
}

template <class C>
__global__ void __launch_bounds__(256) k_panel(PanelArgs<C> P) {
  typedef typename CxT<C>::R R;
  cg::grid_group grid = cg::this_grid();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *S = (C *)smem_raw;                     // [w][rows_per]: column c at S + c * rows_per
  __shared__ double rv[8];
  __shared__ int ri[8];
  __shared__ int s_piv;
  __shared__ C prow[32];
  const int w = P.w, G = gridDim.x, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int r0 = P.k0 + blockIdx.x * P.rows_per;
  const int r1 = min(P.Nr, r0 + P.rows_per);
  const int nr = max(0, r1 - r0), lds = P.rows_per;
  // slice staged with eight loads per thread in flight
  for (int e0 = 0; e0 < nr * w; e0 += 8 * 256) {
    C v[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int e = e0 + u * 256 + tid;
      v[u] = e < nr * w ? P.A[(size_t)(P.k0 + e / nr) * P.ld + r0 + e % nr] : C{0, 0};
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int e = e0 + u * 256 + tid;
      if (e < nr * w) S[(e / nr) * lds + e % nr] = v[u];
    }
  }
  __syncthreads();
  for (int j = 0; j < w; j++) {
    const int gj = P.k0 + j, buf = j & 1;
    // 1. local pivot candidate (i[cz]amax: max |re|+|im|, first index on ties)
    double bv = -1.0;
    int bi = 0x7fffffff;
    for (int r = tid; r < nr; r += 256) {
      int gr = r0 + r;
      if (gr < gj) continue;
      C v = S[j * lds + r];
      double a = (double)(fabs(v.r) + fabs(v.i));
      if (better(a, gr, bv, bi)) { bv = a; bi = gr; }
    }
    for (int o = 16; o > 0; o >>= 1) {
      double ov = __shfl_xor_sync(0xffffffffu, bv, o);
      int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (better(ov, oi, bv, bi)) { bv = ov; bi = oi; }
    }
    if (lane == 0) { rv[wid] = bv; ri[wid] = bi; }
    __syncthreads();
    if (tid == 0) {
      for (int k = 1; k < 8; k++)
        if (better(rv[k], ri[k], rv[0], ri[0])) { rv[0] = rv[k]; ri[0] = ri[k]; }
      P.cval[buf * G + blockIdx.x] = rv[0];
      P.cidx[buf * G + blockIdx.x] = ri[0];
    }
    __syncthreads();
    int myc = ri[0];
    if (rv[0] >= 0.0 && tid < w) P.crow[((size_t)buf * G + blockIdx.x) * 32 + tid] = S[tid * lds + myc - r0];
    if (gj >= r0 && gj < r1 && tid < w) P.jrow[buf * 32 + tid] = S[tid * lds + gj - r0];
    grid.sync();
    // 2. global pivot
    if (tid < 32) {
      double v = -1.0;
      int i = 0x7fffffff, b = 0;
      for (int k = lane; k < G; k += 32) {
        double cv = P.cval[buf * G + k];
        int ci = P.cidx[buf * G + k];
        if (better(cv, ci, v, i)) { v = cv; i = ci; b = k; }
      }
      for (int o = 16; o > 0; o >>= 1) {
        double ov = __shfl_xor_sync(0xffffffffu, v, o);
        int oi = __shfl_xor_sync(0xffffffffu, i, o);
        int ob = __shfl_xor_sync(0xffffffffu, b, o);
        if (better(ov, oi, v, i)) { v = ov; i = oi; b = ob; }
      }
      if (lane < w) prow[lane] = P.crow[((size_t)buf * G + b) * 32 + lane];
      if (lane == 0) s_piv = i;
    }
    __syncthreads();
    const int piv = s_piv;
    if (blockIdx.x == 0 && tid == 0) P.ipiv[gj] = piv + 1;
    // 3. swap rows gj and piv inside the panel
    if (piv != gj) {
      if (piv >= r0 && piv < r1 && tid < w) S[tid * lds + piv - r0] = P.jrow[buf * 32 + tid];
      if (gj >= r0 && gj < r1 && tid < w) S[tid * lds + gj - r0] = prow[tid];
    }
    __syncthreads();
    // 4. scale the column below the pivot and update the rest of the panel
    C p = prow[j];
    R d = p.r * p.r + p.i * p.i;
    if (d == (R)0) {
      if (blockIdx.x == 0 && tid == 0) atomicCAS(P.info, 0, gj + 1);
    } else {
      C inv{p.r / d, -p.i / d};
      int ncol = w - j - 1;
      for (int r = tid; r < nr; r += 256) {
        int gr = r0 + r;
        if (gr <= gj) continue;
        C v = S[j * lds + r];
        C l{v.r * inv.r - v.i * inv.i, v.r * inv.i + v.i * inv.r};
        S[j * lds + r] = l;
        for (int c = 1; c <= ncol; c++) {
          C u = prow[j + c];
          C &t = S[(j + c) * lds + r];
          t.r -= l.r * u.r - l.i * u.i;
          t.i -= l.r * u.i + l.i * u.r;
        }
      }
    }
    __syncthreads();
  }
  for (int e = tid; e < nr * w; e += 256) {
    const int r = e % nr, c = e / nr;
    P.A[(size_t)(P.k0 + c) * P.ld + r0 + r] = S[c * lds + r];
  }
}

template <class C>
__device__ __forceinline__ C ldcg_c(const C *p);
template <>
__device__ __forceinline__ cdl ldcg_c<cdl>(const cdl *p) {
  double2 v = __ldcg((const double2 *)p);
  return cdl{v.x, v.y};
}
template <>
__device__ __forceinline__ cfl ldcg_c<cfl>(const cfl *p) {
  float2 v = __ldcg((const float2 *)p);
  return cfl{v.x, v.y};
}

// The same panel on one thread-block cluster (up to 16 CTAs, the slices in
// their shared memory): when the panel fits, the per-column grid barrier
// becomes a cluster barrier and the candidate exchange reads the other CTAs'
// shared memory directly (distributed shared memory) instead of global
// memory.  Pivot choice, interchanges and arithmetic are those of k_panel.
// Candidate slots are double-buffered by column parity: a CTA writing the
// slots of column j + 2 has passed the barrier of column j + 1, which every
// CTA reaches only after reading column j's slots.  The last barrier keeps
// every CTA's shared memory alive until all remote reads are done.
#define PCL_THREADS 512     // threads per CTA of the cluster panel (about one row each)
template <class C>
__global__ void __launch_bounds__(PCL_THREADS) k_panel_cl(PanelArgs<C> P) {
  typedef typename CxT<C>::R R;
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *S = (C *)smem_raw;                     // [w][rows_per]: column c at S + c * rows_per
  __shared__ double rv[PCL_THREADS / 32];
  __shared__ int ri[PCL_THREADS / 32];
  __shared__ double cval[2];                // this CTA's candidate, per column parity
  __shared__ int cidx[2];
  __shared__ C crow[2][32];                 // its candidate row
  __shared__ C jrow[2][32];                 // row k0 + j before the swap (CTA holding it)
  __shared__ int s_piv;
  __shared__ C prow[32], jr[32];
  const int w = P.w, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int rank = (int)cl.block_rank(), G = (int)cl.num_blocks();
  const int r0 = P.k0 + rank * P.rows_per;
  const int r1 = min(P.Nr, r0 + P.rows_per);
  const int nr = max(0, r1 - r0), lds = P.rows_per;
  for (int e0 = 0; e0 < nr * w; e0 += 8 * PCL_THREADS) {
    C v[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int e = e0 + u * PCL_THREADS + tid;
      v[u] = e < nr * w ? P.A[(size_t)(P.k0 + e / nr) * P.ld + r0 + e % nr] : C{0, 0};
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int e = e0 + u * PCL_THREADS + tid;
      if (e < nr * w) S[(e / nr) * lds + e % nr] = v[u];
    }
  }
  __syncthreads();
  for (int j = 0; j < w; j++) {
    const int gj = P.k0 + j, buf = j & 1;
    // 1. local pivot candidate (i[cz]amax: max |re|+|im|, first index on ties)
    double bv = -1.0;
    int bi = 0x7fffffff;
    for (int r = tid; r < nr; r += PCL_THREADS) {
      int gr = r0 + r;
      if (gr < gj) continue;
      C v = S[j * lds + r];
      double a = (double)(fabs(v.r) + fabs(v.i));
      if (better(a, gr, bv, bi)) { bv = a; bi = gr; }
    }
    for (int o = 16; o > 0; o >>= 1) {
      double ov = __shfl_xor_sync(0xffffffffu, bv, o);
      int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (better(ov, oi, bv, bi)) { bv = ov; bi = oi; }
    }
    if (lane == 0) { rv[wid] = bv; ri[wid] = bi; }
    __syncthreads();
    if (tid == 0) {
      for (int k = 1; k < PCL_THREADS / 32; k++)
        if (better(rv[k], ri[k], rv[0], ri[0])) { rv[0] = rv[k]; ri[0] = ri[k]; }
      cval[buf] = rv[0];
      cidx[buf] = ri[0];
    }
    __syncthreads();
    const int myc = ri[0];
    if (rv[0] >= 0.0 && tid < w) crow[buf][tid] = S[tid * lds + myc - r0];
    if (gj >= r0 && gj < r1 && tid < w) jrow[buf][tid] = S[tid * lds + gj - r0];
    cl.sync();   // every CTA's candidate is visible in the cluster
    // 2. global pivot: lane k reads CTA k's candidate
    if (tid < 32) {
      double v = -1.0;
      int i = 0x7fffffff, b = 0;
      if (lane < G) {
        v = *cl.map_shared_rank(&cval[buf], lane);
        i = *cl.map_shared_rank(&cidx[buf], lane);
        b = lane;
      }
      for (int o = 16; o > 0; o >>= 1) {
        double ov = __shfl_xor_sync(0xffffffffu, v, o);
        int oi = __shfl_xor_sync(0xffffffffu, i, o);
        int ob = __shfl_xor_sync(0xffffffffu, b, o);
        if (better(ov, oi, v, i)) { v = ov; i = oi; b = ob; }
      }
      const int owner = (gj - P.k0) / P.rows_per;   // CTA holding row gj
      if (lane < w) {
        prow[lane] = *cl.map_shared_rank(&crow[buf][lane], b);
        jr[lane] = *cl.map_shared_rank(&jrow[buf][lane], owner);
      }
      if (lane == 0) s_piv = i;
    }
    __syncthreads();
    const int piv = s_piv;
    if (rank == 0 && tid == 0) P.ipiv[gj] = piv + 1;
    // 3. swap rows gj and piv inside the panel
    if (piv != gj) {
      if (piv >= r0 && piv < r1 && tid < w) S[tid * lds + piv - r0] = jr[tid];
      if (gj >= r0 && gj < r1 && tid < w) S[tid * lds + gj - r0] = prow[tid];
    }
    __syncthreads();
    // 4. scale the column below the pivot and update the rest of the panel
    C p = prow[j];
    R d = p.r * p.r + p.i * p.i;
    if (d == (R)0) {
      if (rank == 0 && tid == 0) atomicCAS(P.info, 0, gj + 1);
    } else {
      C inv{p.r / d, -p.i / d};
      int ncol = w - j - 1;
      for (int r = tid; r < nr; r += PCL_THREADS) {
        int gr = r0 + r;
        if (gr <= gj) continue;
        C v = S[j * lds + r];
        C l{v.r * inv.r - v.i * inv.i, v.r * inv.i + v.i * inv.r};
        S[j * lds + r] = l;
        for (int c = 1; c <= ncol; c++) {
          C u = prow[j + c];
          C &t = S[(j + c) * lds + r];
          t.r -= l.r * u.r - l.i * u.i;
          t.i -= l.r * u.i + l.i * u.r;
        }
      }
    }
    __syncthreads();
  }
  for (int e = tid; e < nr * w; e += PCL_THREADS) {
    const int r = e % nr, c = e / nr;
    P.A[(size_t)(P.k0 + c) * P.ld + r0 + r] = S[c * lds + r];
  }
  cl.sync();   // no CTA leaves while another may still read its shared memory
}

// apply the interchanges ipiv[k0..k0+w) to columns [c0, c1) of A
template <class C>
__global__ void k_laswp(C *A, size_t ld, const int *ipiv, int k0, int w, int c0, int c1, int skip0, int skip1) {
  int col = c0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= c1 || (col >= skip0 && col < skip1)) return;
  C *cp = A + (size_t)col * ld;
  for (int i = 0; i < w; i++) {
    int p = ipiv[k0 + i] - 1;
    if (p != k0 + i) {
      C t = cp[k0 + i];
      cp[k0 + i] = cp[p];
      cp[p] = t;
    }
  }
}

struct LUWork {
  double *cval;
  int *cidx;
  void *crow, *jrow;
  int *info;
};

static int panel_grid = 0, panel_smem_max = 0, panel_rows_target = 32;

// cluster size of k_panel_cl<C> on this device (0: no cluster path), found
// once: the largest of 16 and 8 that the occupancy query allows with a full
// slice of shared memory per CTA
static int panel_cl_smem_max = 0;
template <class C>
static int panel_cluster_size() {
  static int cs = -1;
  if (cs >= 0) return cs;
  cs = 0;
  int dev = 0, smemopt = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&smemopt, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
    return cs;
  panel_cl_smem_max = smemopt - 6 * 1024;   // room for the kernel's static shared memory
  if (cudaFuncSetAttribute(k_panel_cl<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, panel_cl_smem_max) != cudaSuccess ||
      cudaFuncSetAttribute(k_panel_cl<C>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
    cudaGetLastError();
    return cs;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(16);
  cfg.blockDim = dim3(PCL_THREADS);
  cfg.dynamicSmemBytes = panel_cl_smem_max;
  int best = 0;
  if (cudaOccupancyMaxPotentialClusterSize(&best, (void *)k_panel_cl<C>, &cfg) != cudaSuccess) best = 0;
  int want = best >= 16 ? 16 : (best >= 8 ? 8 : 0);
  if (want) {
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = want;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(want);
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, (void *)k_panel_cl<C>, &cfg) != cudaSuccess || nclusters < 1) want = 0;
  }
  cudaGetLastError();
  cs = want;
  return cs;
}

template <class C>
static int panel_leaf(bg_matrix *m, const LUWork &W, int k0, int w) {
  int N = m->N;
  int Mp = N - k0;
  // the whole panel in one cluster's shared memory: cluster barriers and
  // distributed shared memory instead of a grid barrier per column
  const int CS = panel_cluster_size<C>();
  if (CS) {
    const int G = std::min(CS, std::max(1, (Mp + panel_rows_target - 1) / panel_rows_target));
    const int rows = (Mp + G - 1) / G;
    const size_t smem = (size_t)rows * w * sizeof(C);
    // past ~512 rows per CTA the row updates of 16 CTAs cost more than the
    // grid barrier they save (148 CTAs share them in the grid form)
    if (rows <= 512 && smem <= (size_t)panel_cl_smem_max) {
      PanelArgs<C> P{(C *)m->d, m->ld, N, k0, w, rows, m->d_ipiv, W.info, W.cval, W.cidx, (C *)W.crow, (C *)W.jrow};
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(G);
      cfg.blockDim = dim3(PCL_THREADS);
      cfg.dynamicSmemBytes = smem;
      cfg.stream = stream();
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = G;
      at[0].val.clusterDim.y = 1;
      at[0].val.clusterDim.z = 1;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      prof_start(PROF_PANEL);
      BG_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_panel_cl<C>, P));
      BG_LAUNCHED();
      prof_stop(PROF_PANEL, 8.0 * Mp * (double)w * w / 2);
      prof_start(PROF_LASWP);
      k_laswp<C><<<(N + 255) / 256, 256, 0, stream()>>>((C *)m->d, m->ld, m->d_ipiv, k0, w, 0, N, k0, k0 + w);
      BG_LAUNCHED();
      prof_stop(PROF_LASWP, 0.0);
      return BG_OK;
    }
  }
  int G = std::min(panel_grid, std::max(1, (Mp + panel_rows_target - 1) / panel_rows_target));
  while (G < panel_grid && (size_t)((Mp + G - 1) / G) * w * sizeof(C) > (size_t)panel_smem_max) G++;
  int rows = (Mp + G - 1) / G;
  size_t smem = (size_t)rows * w * sizeof(C);
  if ((int)smem > panel_smem_max) {
    set_error("panel slice of %zu bytes exceeds shared memory (N=%d too large for this build)", smem, N);
    return BG_ERR_ARG;
  }
  static bool attr = false;
  if (!attr) {
    BG_CUDA_TRY(cudaFuncSetAttribute(k_panel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, panel_smem_max));
    attr = true;
  }
  PanelArgs<C> P{(C *)m->d, m->ld, N, k0, w, rows, m->d_ipiv, W.info, W.cval, W.cidx, (C *)W.crow, (C *)W.jrow};
  void *args[] = {&P};
  prof_start(PROF_PANEL);
  BG_CUDA_TRY(cudaLaunchCooperativeKernel((void *)k_panel<C>, dim3(G), dim3(256), args, smem, stream()));
  BG_LAUNCHED();
  prof_stop(PROF_PANEL, 8.0 * Mp * (double)w * w / 2);
  int threads = 256;
  int blocks = (N + threads - 1) / threads;
  prof_start(PROF_LASWP);
  k_laswp<C><<<blocks, threads, 0, stream()>>>((C *)m->d, m->ld, m->d_ipiv, k0, w, 0, N, k0, k0 + w);
  BG_LAUNCHED();
  prof_stop(PROF_LASWP, 0.0);
  return BG_OK;
}

// factor columns [k0, k0+n) (rows k0..N-1); interchanges applied to all columns
template <class C>
static int getrf_rec(bg_matrix *m, const LUWork &W, int k0, int n) {
  if (n <= 32) return panel_leaf<C>(m, W, k0, n);
  int n1 = (n / 2 + 31) / 32 * 32;
  if (n1 >= n) n1 = 32;
  int n2 = n - n1;
  int st;
  C *A = (C *)m->d;
  size_t ld = m->ld;
  int N = m->N;
  if ((st = getrf_rec<C>(m, W, k0, n1))) return st;
  C *A11 = A + k0 + (size_t)k0 * ld;
  C *A12 = A + k0 + (size_t)(k0 + n1) * ld;
  C *A21 = A + (k0 + n1) + (size_t)k0 * ld;
  C *A22 = A + (k0 + n1) + (size_t)(k0 + n1) * ld;
  if ((st = trsm<C>(n1, n2, A11, ld, A12, ld, 0))) return st;
  if ((st = gemm_sub(N - k0 - n1, n2, n1, A21, ld, A12, ld, A22, ld))) return st;
  return getrf_rec<C>(m, W, k0 + n1, n2);
}

static int build_perm(bg_matrix *m);

static int panel_init() {
  if (panel_grid) return BG_OK;
  int dev = 0, sms = 0, smemopt = 0;
  BG_CUDA_TRY(cudaGetDevice(&dev));
  BG_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  BG_CUDA_TRY(cudaDeviceGetAttribute(&smemopt, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  panel_smem_max = smemopt - 2048;
  panel_grid = sms;  // at most one CTA per SM (cooperative residency)
  if (const char *e = std::getenv("BG_PANEL_ROWS")) panel_rows_target = std::max(8, std::atoi(e));
  return BG_OK;
}

int lu_factor(bg_matrix *m) {
  int st = ensure_device();
  if (!st) st = panel_init();
  if (st) return st;
  int N = m->N;
  const size_t csz = m->precision == BG_C128 ? sizeof(cdl) : sizeof(cfl);
  // workspace: candidate rows, j-rows, candidate values/indices, info, error
  // flag, and (complex64) the expanded-A scratch of the tensor-core GEMM
  size_t at_floats = 0;
  if (m->precision == BG_C64) at_floats = (size_t)2 * TC_MCHUNK * (((size_t)2 * N + 31) / 32 * 32);
  size_t need = csz * 2 * panel_grid * 32 + csz * 64 + sizeof(double) * 2 * panel_grid + sizeof(int) * 2 * panel_grid +
                256 + sizeof(float) * at_floats;
  if (m->work_bytes < need) {
    if (m->d_work) cudaFree(m->d_work);
    m->d_work = nullptr;
    m->work_bytes = 0;
    BG_CUDA_TRY(cudaMalloc(&m->d_work, need));
    m->work_bytes = need;
  }
  char *w = (char *)m->d_work;
  LUWork W;
  W.crow = (void *)w; w += csz * 2 * panel_grid * 32;
  W.jrow = (void *)w; w += csz * 64;
  W.cval = (double *)w; w += sizeof(double) * 2 * panel_grid;
  W.cidx = (int *)w; w += sizeof(int) * 2 * panel_grid;
  W.info = (int *)w;
  int *tcerr = W.info + 1;
  w += 256;
  BG_CUDA_TRY(cudaMemsetAsync(W.info, 0, 2 * sizeof(int), stream()));
  if (m->precision == BG_C128) {
    if ((st = getrf_rec<cdl>(m, W, 0, N))) return st;
  } else {
    TcScratch sc;
    sc.At = (float *)w;
    sc.at_floats = at_floats;
    sc.err = tcerr;
    t_tc = &sc;
    st = getrf_rec<cfl>(m, W, 0, N);
    t_tc = nullptr;
    if (st) return st;
  }
  int info[2] = {0, 0};
  BG_CUDA_TRY(cudaMemcpyAsync(info, W.info, 2 * sizeof(int), cudaMemcpyDeviceToHost, stream()));
  BG_CUDA_TRY(cudaStreamSynchronize(stream()));
  if (info[1]) {
    set_error("tensor-core GEMM reported a pipeline timeout (code %d)", info[1]);
    return BG_ERR_CUDA;
  }
  if ((st = build_perm(m))) return st;
  return info[0];
}

int zgemm_sub_device(int M, int N, int K, const void *A, int lda, const void *B, int ldb, void *C, int ldc) {
  int st = ensure_device();
  if (st) return st;
  return zgemm_sub(M, N, K, (const cdl *)A, (size_t)lda, (const cdl *)B, (size_t)ldb, (cdl *)C, (size_t)ldc);
}

// =========================================================================
// few-right-hand-side solves: B <- U^{-1} L^{-1} P B in one gather and two
// single-pass triangular sweeps.  In a sweep each CTA takes the next 64-row
// block in dependency order from a ticket counter, accumulates the products
// with already-solved blocks as their ready flags appear (flag == epoch),
// solves its diagonal block with warp shuffles (one warp per right-hand
// side), publishes the block and raises its flag.  A CTA only ever waits on
// blocks with smaller tickets, which are already running, so the sweep
// always makes progress; every wait is bounded and a timeout is recorded in
// the error word, which also makes the other CTAs give up early.
// =========================================================================
#define TV_B 64
#define TV_MAXRHS 4
#define TV_SPIN (1 << 22)

template <class C>
__global__ void k_gather_rows(int N, int nrhs, const int *perm, const C *src, size_t lds, C *dst, size_t ldd) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y;
  if (i < N && j < nrhs) dst[(size_t)j * ldd + i] = src[(size_t)j * lds + perm[i]];
}

template <class C>
constexpr int trsv_smem() {
  return TV_B * (TV_B + 1) * (int)sizeof(C) + 2 * TV_B * TV_MAXRHS * (int)sizeof(C);
}

template <class C, bool UPPER>
__global__ void __launch_bounds__(128) k_trsv(int N, const C *A, size_t ld, C *X, size_t ldx, int nrhs, int *flags,
                                              int epoch, int *ticket, int *err) {
  typedef typename CxT<C>::R R;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C(*D)[TV_B + 1] = (C(*)[TV_B + 1])smem_raw;                    // diagonal block
  C(*part)[TV_MAXRHS] = (C(*)[TV_MAXRHS])(smem_raw + TV_B * (TV_B + 1) * sizeof(C));   // part[row][rhs]
  C(*xs)[TV_MAXRHS] = part + TV_B;                                                    // solved block x[col][rhs]
  __shared__ int s_blk, s_abort;
  __shared__ C dinv[TV_B];   // upper sweep: 1 / u_ii of the diagonal block
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nb = (N + TV_B - 1) / TV_B;
  if (tid == 0) { s_blk = atomicAdd(ticket, 1); s_abort = 0; }
  __syncthreads();
  const int lb = s_blk;
  const int bi = UPPER ? nb - 1 - lb : lb;
  const int r0 = bi * TV_B, rows = min(TV_B, N - r0);
  const int row = tid & (TV_B - 1), half = tid >> 6;
  // this block's right-hand-side rows (written by no other CTA), read now
  // so that the final combine does not wait for memory
  C bx[TV_MAXRHS];
#pragma unroll
  for (int j = 0; j < TV_MAXRHS; j++)
    bx[j] = (half == 0 && row < rows && j < nrhs) ? X[(size_t)j * ldx + r0 + row] : C{0, 0};
  // stage the diagonal block, eight loads per thread in flight
  for (int e0 = 0; e0 < rows * rows; e0 += 8 * 128) {
    C v[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int e = e0 + u * 128 + tid;
      v[u] = e < rows * rows ? A[(size_t)(r0 + e / rows) * ld + r0 + e % rows] : C{0, 0};
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int e = e0 + u * 128 + tid;
      if (e < rows * rows) D[e % rows][e / rows] = v[u];
    }
  }
  if (UPPER) {
    // reciprocals of the diagonal, conj(u) / |u|^2, computed before this
    // block waits for anything (the solve below multiplies instead of
    // dividing on its sequential path); barriers of the loop or of the
    // combine below order them before their use
    if (tid < rows) {
      const int e = tid * rows + tid;
      const C u = A[(size_t)(r0 + e / rows) * ld + r0 + e % rows];
      const R d = u.r * u.r + u.i * u.i;
      dinv[tid] = C{u.r / d, -u.i / d};
    }
  }
  C acc[TV_MAXRHS];
#pragma unroll
  for (int j = 0; j < TV_MAXRHS; j++) acc[j] = C{0, 0};
  for (int q = 0; q < lb; q++) {
    const int bj = UPPER ? nb - 1 - q : q;
    const int c0 = bj * TV_B, cols = min(TV_B, N - c0);
    // this thread's row of block (bi, bj) over its half of the columns:
    // A does not depend on x, so it is read before waiting for block bj
    C a[32];
    {
      const C *ap = A + (size_t)(c0 + half * 32) * ld + r0 + row;
#pragma unroll
      for (int u = 0; u < 32; u++)
        a[u] = (row < rows && half * 32 + u < cols) ? ap[(size_t)u * ld] : C{0, 0};
    }
    if (tid == 0) {
      volatile int *f = flags + bj;
      int it = 0;
      while (*f != epoch) {
        if (*(volatile int *)err || ++it > TV_SPIN) {
          if (it > TV_SPIN) atomicCAS(err, 0, 100 + (UPPER ? 1 : 0));
          s_abort = 1;
          break;
        }
        __nanosleep(64);
      }
      __threadfence();
    }
    __syncthreads();
    if (s_abort) return;
    // the solved block's x, once per CTA (at most 2 per thread)
    {
      C v[2];
#pragma unroll
      for (int u = 0; u < 2; u++) {
        const int e = u * 128 + tid;
        v[u] = e < cols * nrhs ? ldcg_c(X + (size_t)(e / cols) * ldx + c0 + e % cols) : C{0, 0};
      }
#pragma unroll
      for (int u = 0; u < 2; u++) {
        const int e = u * 128 + tid;
        if (e < cols * nrhs) xs[e % cols][e / cols] = v[u];
      }
    }
    __syncthreads();
    if (row < rows) {
#pragma unroll
      for (int u = 0; u < 32; u++) {
        if (half * 32 + u >= cols) break;
#pragma unroll
        for (int j = 0; j < TV_MAXRHS; j++) {
          if (j < nrhs) {
            const C x = xs[half * 32 + u][j];
            acc[j].r += a[u].r * x.r - a[u].i * x.i;
            acc[j].i += a[u].r * x.i + a[u].i * x.r;
          }
        }
      }
    }
    __syncthreads();   // xs is rewritten for the next block
  }
  if (half == 1 && row < rows)
#pragma unroll
    for (int j = 0; j < TV_MAXRHS; j++)
      if (j < nrhs) part[row][j] = acc[j];
  __syncthreads();
  if (half == 0 && row < rows)
#pragma unroll
    for (int j = 0; j < TV_MAXRHS; j++)
      if (j < nrhs) {
        const C b = bx[j];
        C p = part[row][j];
        part[row][j] = C{b.r - acc[j].r - p.r, b.i - acc[j].i - p.i};
      }
  __syncthreads();
  // diagonal solve: warp j handles right-hand side j, lanes hold rows l, l+32
  if (warp < nrhs) {
    const int j = warp, q0 = lane, q1 = lane + 32;
    C b0 = q0 < rows ? part[q0][j] : C{0, 0};
    C b1 = q1 < rows ? part[q1][j] : C{0, 0};
    if (!UPPER) {
      for (int i = 0; i < rows; i++) {
        C x = cshfl(i < 32 ? b0 : b1, i & 31);
        if (q0 > i && q0 < rows) { C l = D[q0][i]; b0.r -= l.r * x.r - l.i * x.i; b0.i -= l.r * x.i + l.i * x.r; }
        if (q1 > i && q1 < rows) { C l = D[q1][i]; b1.r -= l.r * x.r - l.i * x.i; b1.i -= l.r * x.i + l.i * x.r; }
      }
    } else {
      for (int i = rows - 1; i >= 0; i--) {
        C v = cshfl(i < 32 ? b0 : b1, i & 31);
        const C iu = dinv[i];
        C x{v.r * iu.r - v.i * iu.i, v.r * iu.i + v.i * iu.r};
        if (q0 == i) b0 = x;
        if (q1 == i) b1 = x;
        if (q0 < i) { C t = D[q0][i]; b0.r -= t.r * x.r - t.i * x.i; b0.i -= t.r * x.i + t.i * x.r; }
        if (q1 < i) { C t = D[q1][i]; b1.r -= t.r * x.r - t.i * x.i; b1.i -= t.r * x.i + t.i * x.r; }
      }
    }
    if (q0 < rows) X[(size_t)j * ldx + r0 + q0] = b0;
    if (q1 < rows) X[(size_t)j * ldx + r0 + q1] = b1;
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) atomicExch(flags + bi, epoch);
}

// host: permutation from LAPACK interchanges, kept beside the factors
static int build_perm(bg_matrix *m) {
  int N = m->N;
  std::vector<int> ipiv(N), perm(N);
  BG_CUDA_TRY(cudaMemcpyAsync(ipiv.data(), m->d_ipiv, sizeof(int) * N, cudaMemcpyDeviceToHost, stream()));
  BG_CUDA_TRY(cudaStreamSynchronize(stream()));
  for (int i = 0; i < N; i++) perm[i] = i;
  for (int i = 0; i < N; i++) std::swap(perm[i], perm[ipiv[i] - 1]);
  if (!m->d_perm) BG_CUDA_TRY(cudaMalloc(&m->d_perm, sizeof(int) * (N + 2 * ((N + TV_B - 1) / TV_B) + 8)));
  BG_CUDA_TRY(cudaMemcpyAsync(m->d_perm, perm.data(), sizeof(int) * N, cudaMemcpyHostToDevice, stream()));
  // ready flags of both sweeps + tickets + error word, zeroed once
  BG_CUDA_TRY(cudaMemsetAsync(m->d_perm + N, 0, sizeof(int) * (2 * ((N + TV_B - 1) / TV_B) + 8), stream()));
  BG_CUDA_TRY(cudaStreamSynchronize(stream()));
  return BG_OK;
}

template <class C>
static int getrs(bg_matrix *m, C *B, size_t ldb, int nrhs) {
  int N = m->N;
  const C *A = (const C *)m->d;
  const int nb = (N + TV_B - 1) / TV_B;
  int *flagsL = m->d_perm + N, *flagsU = flagsL + nb, *tick = flagsU + nb, *err = tick + 2;
  const int smem = trsv_smem<C>();
  static bool attr = false;
  if (!attr) {
    BG_CUDA_TRY(cudaFuncSetAttribute(k_trsv<C, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    BG_CUDA_TRY(cudaFuncSetAttribute(k_trsv<C, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr = true;
  }
  for (int r0 = 0; r0 < nrhs; r0 += TV_MAXRHS) {
    int nr = std::min(TV_MAXRHS, nrhs - r0);
    C *Bp = B + (size_t)r0 * ldb;
    C *T = nullptr;
    BG_CUDA_TRY(cudaMallocAsync((void **)&T, sizeof(C) * (size_t)N * nr, stream()));
    k_gather_rows<C><<<dim3((N + 255) / 256, nr), 256, 0, stream()>>>(N, nr, m->d_perm, Bp, ldb, T, N);
    BG_LAUNCHED();
    int epoch = ++m->solve_epoch;
    BG_CUDA_TRY(cudaMemsetAsync(tick, 0, 2 * sizeof(int), stream()));
    prof_start(PROF_TRSV);
    k_trsv<C, false><<<nb, 128, smem, stream()>>>(N, A, m->ld, T, N, nr, flagsL, epoch, tick, err);
    BG_LAUNCHED();
    k_trsv<C, true><<<nb, 128, smem, stream()>>>(N, A, m->ld, T, N, nr, flagsU, epoch, tick + 1, err);
    BG_LAUNCHED();
    // bytes of the two triangles read once
    prof_stop(PROF_TRSV, (double)sizeof(C) * (double)N * N);
    BG_CUDA_TRY(cudaMemcpy2DAsync(Bp, sizeof(C) * ldb, T, sizeof(C) * N, sizeof(C) * N, nr, cudaMemcpyDeviceToDevice,
                                  stream()));
    BG_CUDA_TRY(cudaFreeAsync(T, stream()));
  }
  return BG_OK;
}

// Many right-hand sides (N-column blocks of the buff-neq chain): one row
// gather by the factor permutation, then the recursive GEMM-based triangular
// solves used inside the factorisation (unit L, then U), in column chunks so
// the scratch stays bounded.
int lu_solve_many(bg_matrix *m, void *dB, size_t ldb, int nrhs) {
  if (!m->d_perm) { set_error("solve: factorization state missing"); return BG_ERR_STATE; }
  if (m->precision != BG_C128) { set_error("lu_solve_many: complex128 only"); return BG_ERR_ARG; }
  int N = m->N;
  const cdl *A = (const cdl *)m->d;
  cdl *B = (cdl *)dB;
  const int chunk = 4096;
  cdl *T = nullptr;
  int w = std::min(chunk, nrhs);
  if (w <= 0) return BG_OK;
  BG_CUDA_TRY(cudaMallocAsync((void **)&T, sizeof(cdl) * (size_t)N * w, stream()));
  int st = BG_OK;
  for (int r0 = 0; r0 < nrhs && !st; r0 += chunk) {
    int nr = std::min(chunk, nrhs - r0);
    cdl *Bp = B + (size_t)r0 * ldb;
    k_gather_rows<cdl><<<dim3((N + 255) / 256, nr), 256, 0, stream()>>>(N, nr, m->d_perm, Bp, ldb, T, N);
    BG_LAUNCHED();
    if ((st = trsm<cdl>(N, nr, A, m->ld, T, N, 0))) break;
    if ((st = trsm<cdl>(N, nr, A, m->ld, T, N, 1))) break;
    cudaError_t e = cudaMemcpy2DAsync(Bp, sizeof(cdl) * ldb, T, sizeof(cdl) * N, sizeof(cdl) * N, nr,
                                      cudaMemcpyDeviceToDevice, stream());
    if (e != cudaSuccess) { set_error("lu_solve_many: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
  }
  cudaFreeAsync(T, stream());
  return st;
}

int lu_solve(bg_matrix *m, void *dB, int ldb, int nrhs) {
  if (!m->d_perm) { set_error("solve: factorization state missing"); return BG_ERR_STATE; }
  if (m->precision == BG_C128) return getrs<cdl>(m, (cdl *)dB, (size_t)ldb, nrhs);
  return getrs<cfl>(m, (cfl *)dB, (size_t)ldb, nrhs);
}

// error word of the triangular sweeps (0 = ok)
int lu_solve_status(bg_matrix *m) {
  if (!m->d_perm) return BG_OK;
  int N = m->N, nb = (N + TV_B - 1) / TV_B, e = 0;
  BG_CUDA_TRY(cudaMemcpyAsync(&e, m->d_perm + N + 2 * nb + 2, sizeof(int), cudaMemcpyDeviceToHost, stream()));
  BG_CUDA_TRY(cudaStreamSynchronize(stream()));
  if (e) { set_error("triangular solve timed out waiting for a block (code %d)", e); return BG_ERR_CUDA; }
  return BG_OK;
}


// =========================================================================
// Allocation-free variant of the device solve.
//
// Some callers cannot allocate GPU memory at solve time: a host application
// whose framework has already reserved the device memory for its own pool,
// or a time-critical loop that cannot accept an allocation's possible failure
// or implicit synchronisation.  For them the gather buffer of the solve lives
// in this fixed device array instead of a stream-ordered allocation.  The
// array (NOALLOC_BYTES) is held by every GPU that loads the library until the
// process exits.  All calls share it: it keeps the last call's contents, and
// two calls whose work overlaps on the GPU would race on it (calls through
// this library are ordered on its single stream).  The gather overwrites the
// part of the array a call uses before it is read, so nothing in it has to
// start at zero; the sweep tickets that must start at zero live beside the
// factors and are cleared by every call.
// =========================================================================
#define NOALLOC_BYTES (4u << 20)
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];
static void *s_noalloc_ptr[64];
static std::mutex s_noalloc_mu;

// once per device, with that device current: the array's device address (the
// host-side symbol is only a stand-in and must never be passed to a kernel)
static int noalloc_setup(void **ptr) {
  int dev = 0;
  BG_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) { set_error("device ordinal %d out of range", dev); return BG_ERR_CUDA; }
  std::lock_guard<std::mutex> lock(s_noalloc_mu);
  if (!s_noalloc_ptr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      set_error("cudaGetSymbolAddress of the solve scratch failed: %s", cudaGetErrorString(e));
      return BG_ERR_CUDA;
    }
    s_noalloc_ptr[dev] = p;
  }
  *ptr = s_noalloc_ptr[dev];
  return BG_OK;
}

template <class C>
static int getrs_noalloc(bg_matrix *m, C *B, size_t ldb, int nrhs, void *scratch) {
  int N = m->N;
  const C *A = (const C *)m->d;
  const int nb = (N + TV_B - 1) / TV_B;
  int *flagsL = m->d_perm + N, *flagsU = flagsL + nb, *tick = flagsU + nb, *err = tick + 2;
  const int smem = trsv_smem<C>();
  BG_CUDA_TRY(cudaFuncSetAttribute(k_trsv<C, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  BG_CUDA_TRY(cudaFuncSetAttribute(k_trsv<C, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  C *T = (C *)scratch;
  k_gather_rows<C><<<dim3((N + 255) / 256, nrhs), 256, 0, stream()>>>(N, nrhs, m->d_perm, B, ldb, T, N);
  BG_LAUNCHED();
  int epoch = ++m->solve_epoch;
  BG_CUDA_TRY(cudaMemsetAsync(tick, 0, 2 * sizeof(int), stream()));
  k_trsv<C, false><<<nb, 128, smem, stream()>>>(N, A, m->ld, T, N, nrhs, flagsL, epoch, tick, err);
  BG_LAUNCHED();
  k_trsv<C, true><<<nb, 128, smem, stream()>>>(N, A, m->ld, T, N, nrhs, flagsU, epoch, tick + 1, err);
  BG_LAUNCHED();
  BG_CUDA_TRY(cudaMemcpy2DAsync(B, sizeof(C) * ldb, T, sizeof(C) * N, sizeof(C) * N, nrhs, cudaMemcpyDeviceToDevice,
                                stream()));
  return BG_OK;
}

int lu_noalloc_check(const bg_matrix *m, int nrhs) {
  size_t esz = m->precision == BG_C128 ? sizeof(cdl) : sizeof(cfl);
  if (nrhs > TV_MAXRHS) {
    set_error("allocation-free solve: at most %d right-hand sides per call (got %d)", TV_MAXRHS, nrhs);
    return BG_ERR_ARG;
  }
  if ((size_t)m->N * nrhs * esz > NOALLOC_BYTES) {
    set_error("allocation-free solve: N*nrhs*%zu = %zu bytes exceeds its fixed %u-byte scratch", esz,
              (size_t)m->N * nrhs * esz, NOALLOC_BYTES);
    return BG_ERR_ARG;
  }
  return BG_OK;
}

int lu_solve_noalloc(bg_matrix *m, void *dB, int ldb, int nrhs) {
  int st0 = lu_noalloc_check(m, nrhs);
  if (st0) return st0;
  if (!m->d_perm) { set_error("solve: factorization state missing"); return BG_ERR_STATE; }
  void *scratch = nullptr;
  int st = noalloc_setup(&scratch);
  if (st) return st;
  if (m->precision == BG_C128) st = getrs_noalloc<cdl>(m, (cdl *)dB, (size_t)ldb, nrhs, scratch);
  else st = getrs_noalloc<cfl>(m, (cfl *)dB, (size_t)ldb, nrhs, scratch);
  if (!st) st = lu_solve_status(m);
  return st;
}

// =========================================================================
// Capture-safe factor and solve for the batched frequency sweeps: no host
// synchronisation and no allocation between lu_capture_prepare() and the
// end of the solve, so the whole sequence can be recorded into a CUDA graph
// and replayed.  The pivot permutation is built on the device, the
// factorisation status stays in the workspace (lu_capture_info), and the
// solve clears its ready flags itself on every replay (epoch 1).
// =========================================================================

// perm = composition of the interchanges ipiv (1-based), one block; the
// sequential swaps run in shared memory when 8 N bytes fit, else in global
__global__ void k_build_perm(int N, const int *ipiv, int *perm, int use_smem) {
  extern __shared__ int sp[];
  int *p = use_smem ? sp : perm;
  const int *iv = ipiv;
  int *ivs = use_smem ? sp + N : nullptr;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    p[i] = i;
    if (use_smem) ivs[i] = ipiv[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int *q = use_smem ? ivs : iv;
    for (int i = 0; i < N; i++) {
      int j = q[i] - 1, t = p[i];
      p[i] = p[j];
      p[j] = t;
    }
  }
  __syncthreads();
  if (use_smem)
    for (int i = threadIdx.x; i < N; i += blockDim.x) perm[i] = p[i];
}

static size_t lu_work_bytes(bg_matrix *m) {
  const size_t csz = m->precision == BG_C128 ? sizeof(cdl) : sizeof(cfl);
  return csz * 2 * panel_grid * 32 + csz * 64 + sizeof(double) * 2 * panel_grid + sizeof(int) * 2 * panel_grid + 256;
}

// allocates everything the captured factor/solve touch (complex128 only)
int lu_capture_prepare(bg_matrix *m) {
  int st = ensure_device();
  if (!st) st = panel_init();
  if (st) return st;
  if (m->precision != BG_C128) { set_error("batched sweeps factor complex128 matrices"); return BG_ERR_ARG; }
  size_t need = lu_work_bytes(m);
  if (m->work_bytes < need) {
    if (m->d_work) cudaFree(m->d_work);
    m->d_work = nullptr;
    m->work_bytes = 0;
    BG_CUDA_TRY(cudaMalloc(&m->d_work, need));
    m->work_bytes = need;
  }
  int N = m->N;
  if (!m->d_perm) BG_CUDA_TRY(cudaMalloc(&m->d_perm, sizeof(int) * (N + 2 * ((N + TV_B - 1) / TV_B) + 8)));
  BG_CUDA_TRY(cudaMemsetAsync(m->d_perm + N, 0, sizeof(int) * (2 * ((N + TV_B - 1) / TV_B) + 8), stream()));
  BG_CUDA_TRY(cudaStreamSynchronize(stream()));
  static bool attr = false;
  if (!attr) {
    BG_CUDA_TRY(cudaFuncSetAttribute(k_build_perm, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    attr = true;
  }
  return BG_OK;
}

void lu_set_panel_rows(int rows) { panel_rows_target = std::max(8, rows); }
int lu_get_panel_rows() { return panel_rows_target; }

int lu_factor_enqueue(bg_matrix *m) {
  int N = m->N;
  char *w = (char *)m->d_work;
  LUWork W;
  W.crow = (void *)w; w += sizeof(cdl) * 2 * panel_grid * 32;
  W.jrow = (void *)w; w += sizeof(cdl) * 64;
  W.cval = (double *)w; w += sizeof(double) * 2 * panel_grid;
  W.cidx = (int *)w; w += sizeof(int) * 2 * panel_grid;
  W.info = (int *)w;
  BG_CUDA_TRY(cudaMemsetAsync(W.info, 0, 2 * sizeof(int), stream()));
  int st = getrf_rec<cdl>(m, W, 0, N);
  if (st) return st;
  int use_smem = (size_t)8 * N <= 200 * 1024;
  k_build_perm<<<1, 1024, use_smem ? 8 * (size_t)N : 0, stream()>>>(N, m->d_ipiv, m->d_perm, use_smem);
  BG_LAUNCHED();
  m->factored = true;
  return BG_OK;
}

// device address of the factorisation status of the last captured factor
// (LAPACK info; 0 = ok) and of the triangular sweeps' sticky error word
int *lu_capture_info_ptr(bg_matrix *m) {
  char *w = (char *)m->d_work + sizeof(cdl) * 2 * panel_grid * 32 + sizeof(cdl) * 64 +
            sizeof(double) * 2 * panel_grid + sizeof(int) * 2 * panel_grid;
  return (int *)w;
}
int *lu_capture_solve_err_ptr(bg_matrix *m) {
  int nb = (m->N + TV_B - 1) / TV_B;
  return m->d_perm + m->N + 2 * nb + 2;
}

// B (N x nrhs, nrhs <= TV_MAXRHS) <- A^{-1} B with T an N x nrhs device scratch
int lu_solve_enqueue(bg_matrix *m, void *dB, int ldb, int nrhs, void *dT) {
  int N = m->N;
  if (nrhs > TV_MAXRHS) { set_error("captured solve: at most %d right-hand sides", TV_MAXRHS); return BG_ERR_ARG; }
  const cdl *A = (const cdl *)m->d;
  cdl *B = (cdl *)dB, *T = (cdl *)dT;
  const int nb = (N + TV_B - 1) / TV_B;
  int *flagsL = m->d_perm + N, *flagsU = flagsL + nb, *tick = flagsU + nb, *err = tick + 2;
  const int smem = trsv_smem<cdl>();
  static bool attr = false;
  if (!attr) {
    BG_CUDA_TRY(cudaFuncSetAttribute(k_trsv<cdl, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    BG_CUDA_TRY(cudaFuncSetAttribute(k_trsv<cdl, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr = true;
  }
  BG_CUDA_TRY(cudaMemsetAsync(flagsL, 0, sizeof(int) * (2 * nb + 2), stream()));
  k_gather_rows<cdl><<<dim3((N + 255) / 256, nrhs), 256, 0, stream()>>>(N, nrhs, m->d_perm, B, ldb, T, N);
  BG_LAUNCHED();
  k_trsv<cdl, false><<<nb, 128, smem, stream()>>>(N, A, m->ld, T, N, nrhs, flagsL, 1, tick, err);
  BG_LAUNCHED();
  k_trsv<cdl, true><<<nb, 128, smem, stream()>>>(N, A, m->ld, T, N, nrhs, flagsU, 1, tick + 1, err);
  BG_LAUNCHED();
  BG_CUDA_TRY(cudaMemcpy2DAsync(B, sizeof(cdl) * ldb, T, sizeof(cdl) * N, sizeof(cdl) * N, nrhs,
                                cudaMemcpyDeviceToDevice, stream()));
  return BG_OK;
}

}  // namespace bg
