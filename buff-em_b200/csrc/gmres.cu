// Learned form, solver side: restarted GMRES(m) in FP64 on the device with a
// sparse right preconditioner on the near-field pattern (diagonal Jacobi or
// the near-field sparse approximate inverse predicted by the graph network of
// gnn.cu).  Up to four right-hand sides run in lockstep so that every Arnoldi
// step costs one pass over the dense complex128 matrix (HBM-bound, 16 N^2
// bytes); classical Gram-Schmidt with one re-orthogonalisation; Givens
// rotations on the host from the per-step coefficients.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <vector>

#include "internal.h"

namespace bg {

struct z2 { double r, i; };
typedef std::complex<double> zc;

#define GM_MAXRHS 4
#define GV_ROWS 128
#define GV_COLS 256

// Y[:, j] = A X[:, j] for the dense complex128 matrix: partial sums per
// 256-column chunk (summed in a fixed order by k_gm_matvec_sum); columns are
// read four at a time so each thread keeps four 16-byte loads in flight.
__global__ void __launch_bounds__(GV_ROWS) k_gm_matvec_part(int N, const z2 *A, size_t lda, const z2 *X, size_t ldx,
                                                            int nrhs, z2 *partial) {
  __shared__ z2 xs[GV_COLS][GM_MAXRHS];
  int row = blockIdx.x * GV_ROWS + threadIdx.x;
  int c0 = blockIdx.y * GV_COLS;
  int nc = min(GV_COLS, N - c0);
  for (int e = threadIdx.x; e < nc * nrhs; e += GV_ROWS) {
    int c = e / nrhs, j = e % nrhs;
    xs[c][j] = X[(size_t)j * ldx + c0 + c];
  }
  __syncthreads();
  if (row >= N) return;
  double ar[GM_MAXRHS] = {0, 0, 0, 0}, ai[GM_MAXRHS] = {0, 0, 0, 0};
  const z2 *ap = A + (size_t)c0 * lda + row;
  int c = 0;
  for (; c + 4 <= nc; c += 4) {
    z2 a[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      double2 t = __ldcs(reinterpret_cast<const double2 *>(ap + (size_t)(c + u) * lda));
      a[u] = z2{t.x, t.y};
    }
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
      for (int j = 0; j < GM_MAXRHS; j++)
        if (j < nrhs) {
          z2 x = xs[c + u][j];
          ar[j] += a[u].r * x.r - a[u].i * x.i;
          ai[j] += a[u].r * x.i + a[u].i * x.r;
        }
  }
  for (; c < nc; c++) {
    z2 a = ap[(size_t)c * lda];
#pragma unroll
    for (int j = 0; j < GM_MAXRHS; j++)
      if (j < nrhs) {
        z2 x = xs[c][j];
        ar[j] += a.r * x.r - a.i * x.i;
        ai[j] += a.r * x.i + a.i * x.r;
      }
  }
  for (int j = 0; j < nrhs; j++) partial[((size_t)blockIdx.y * nrhs + j) * N + row] = z2{ar[j], ai[j]};
}

// Same for the complex64 copy of the matrix: each thread takes two adjacent
// rows (one 16-byte load per column), FP32 accumulation within a chunk,
// complex64 partials summed in FP64 across chunks.  Reads row N when N is odd: complex64 matrices
// are stored with a leading dimension padded to a multiple of 32 (> N then).
__global__ void __launch_bounds__(GV_ROWS) k_gm_matvec_part_c64(int N, const float4 *A, size_t lda2, const z2 *X,
                                                                size_t ldx, int nrhs, float2 *partial) {
  __shared__ float2 xs[GV_COLS][GM_MAXRHS];
  int row = 2 * (blockIdx.x * GV_ROWS + threadIdx.x);
  int c0 = blockIdx.y * GV_COLS;
  int nc = min(GV_COLS, N - c0);
  for (int e = threadIdx.x; e < nc * nrhs; e += GV_ROWS) {
    int c = e / nrhs, j = e % nrhs;
    z2 x = X[(size_t)j * ldx + c0 + c];
    xs[c][j] = make_float2((float)x.r, (float)x.i);
  }
  __syncthreads();
  if (row >= N) return;
  float ar0[GM_MAXRHS] = {0, 0, 0, 0}, ai0[GM_MAXRHS] = {0, 0, 0, 0};
  float ar1[GM_MAXRHS] = {0, 0, 0, 0}, ai1[GM_MAXRHS] = {0, 0, 0, 0};
  const float4 *ap = A + (size_t)c0 * lda2 + (row >> 1);
  int c = 0;
  for (; c + 4 <= nc; c += 4) {
    float4 a[4];
#pragma unroll
    for (int u = 0; u < 4; u++) a[u] = __ldcs(ap + (size_t)(c + u) * lda2);
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
      for (int j = 0; j < GM_MAXRHS; j++)
        if (j < nrhs) {
          float2 x = xs[c + u][j];
          ar0[j] += a[u].x * x.x - a[u].y * x.y;
          ai0[j] += a[u].x * x.y + a[u].y * x.x;
          ar1[j] += a[u].z * x.x - a[u].w * x.y;
          ai1[j] += a[u].z * x.y + a[u].w * x.x;
        }
  }
  for (; c < nc; c++) {
    float4 a = ap[(size_t)c * lda2];
#pragma unroll
    for (int j = 0; j < GM_MAXRHS; j++)
      if (j < nrhs) {
        float2 x = xs[c][j];
        ar0[j] += a.x * x.x - a.y * x.y;
        ai0[j] += a.x * x.y + a.y * x.x;
        ar1[j] += a.z * x.x - a.w * x.y;
        ai1[j] += a.z * x.y + a.w * x.x;
      }
  }
  for (int j = 0; j < nrhs; j++) {
    partial[((size_t)blockIdx.y * nrhs + j) * N + row] = make_float2(ar0[j], ai0[j]);
    if (row + 1 < N) partial[((size_t)blockIdx.y * nrhs + j) * N + row + 1] = make_float2(ar1[j], ai1[j]);
  }
}

// Same product for a complex64 matrix known to be symmetric (M = M^T, as
// every assembled VIE matrix is): only the 256 x 256 tiles (I, J) with I <= J
// are read, half the bytes of the full product.  Tile (I, J) gives the
// chunk-J partial of rows I (A_IJ x_J) and, for I < J, the chunk-I partial of
// rows J (A_IJ^T x_I, which is A_JI x_I by symmetry), so every partial slot
// of k_gm_matvec_sum is still written exactly once.  A warp owns 64 columns
// of the tile and all 256 rows (8 per lane, two 8-byte complex entries per
// 16-byte read, four columns per step) and streams them into shared memory
// with one bulk copy per column segment (2 KB, issued by one lane, counted on
// an mbarrier per stage), two stages deep, so the next step's copies are in
// flight while a step is computed; the transposed products of four columns
// are reduce-scattered across the warp's lanes, the direct ones summed over
// the four warps through shared memory.  FP32
// accumulation within a tile, complex64 partials summed in FP64, as in
// k_gm_matvec_part_c64.
// The last tile's segments are N's rows rounded up to an even count: the
// padding rows of a complex64 matrix are zero from its allocation.
// 16-byte asynchronous global-to-shared copy; src_bytes < 16 zero-fills the rest
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int src_bytes) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int K>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(K) : "memory"); }

// Bulk copies of the symmetric product: one cp.async.bulk per column segment
// (global -> this CTA's shared memory, completion counted in bytes on an
// mbarrier), every wait bounded.  A wait that runs out sets g_mv_timeout,
// which the solve reads back and reports.
#define SY_SPIN (1u << 24)
__device__ int g_mv_timeout;
__device__ __forceinline__ unsigned sy_saddr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void sy_mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sy_saddr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void sy_mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sy_saddr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool sy_mbar_wait(unsigned long long *bar, unsigned parity) {
  const unsigned a = sy_saddr(bar);
  for (unsigned it = 0; it < SY_SPIN; it++) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void sy_bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   sy_saddr(dst)),
               "l"(src), "r"(bytes), "r"(sy_saddr(bar))
               : "memory");
}

#define SY_STAGES 2
// shared memory: per warp SY_STAGES stages of 4 columns x 256 rows (as 4 x 128
// float4), then x of the tile's columns.  x of the tile's rows is staged in
// the stage buffers (read into registers before the first copy is issued)
// and the direct sums of the four warps reuse them after the loop, so a
// block needs 72 KB for 3 right-hand sides and three blocks fit on an SM.
template <int NR>
constexpr size_t sym_smem_bytes() {
  return sizeof(float4) * 4 * SY_STAGES * 4 * 128 + sizeof(float2) * 256 * NR;
}

template <int NR>
__global__ void __launch_bounds__(128, 3) k_gm_matvec_sym_c64(int N, const float4 *A, size_t lda2, const z2 *X,
                                                           size_t ldx, float2 *partial) {
  const int I = blockIdx.x, J = blockIdx.y;
  if (I > J) return;
  const int r0 = I * 256, c0 = J * 256;
  const int nr = min(256, N - r0), nc = min(256, N - c0);
  extern __shared__ __align__(16) unsigned char sym_smem[];
  __shared__ __align__(8) unsigned long long sy_bar[4][SY_STAGES];            // per warp and stage
  float4 *stage = reinterpret_cast<float4 *>(sym_smem);                        // [4 warps][STAGES][4][128]
  float2 (*xr)[NR] = reinterpret_cast<float2 (*)[NR]>(sym_smem);              // in the stage buffers, until loaded
  float2 (*xc)[NR] = reinterpret_cast<float2 (*)[NR]>(stage + 4 * SY_STAGES * 4 * 128);
  float2 (*dacc)[256][NR] = reinterpret_cast<float2 (*)[256][NR]>(sym_smem);  // [4][256][NR], after the loop
  for (int e = threadIdx.x; e < 256 * NR; e += 128) {
    int i = e / NR, j = e % NR;
    z2 a = i < nr ? X[(size_t)j * ldx + r0 + i] : z2{0.0, 0.0};
    z2 b = i < nc ? X[(size_t)j * ldx + c0 + i] : z2{0.0, 0.0};
    xr[i][j] = make_float2((float)a.r, (float)a.i);
    xc[i][j] = make_float2((float)b.r, (float)b.i);
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const bool trans = I < J;
  // packed FP32 pairs: D = (re, im) accumulators of this lane's 8 rows; the
  // transposed products use this lane's x_I values as broadcast pairs
  // (xr, xr) and (xi, xi), so a complex multiply-accumulate is two __ffma2_rn:
  //   (re, im) += (ar, ai) * (yr, yr) + (-ai, ar) * (yi, yi)
  float2 D[8][NR], Yr[8][NR], Yi[8][NR];
#pragma unroll
  for (int q = 0; q < 8; q++)
#pragma unroll
    for (int j = 0; j < NR; j++) {
      D[q][j] = make_float2(0.f, 0.f);
      float2 y = xr[64 * (q >> 1) + 2 * lane + (q & 1)][j];
      Yr[q][j] = make_float2(y.x, y.x);
      Yi[q][j] = make_float2(y.y, y.y);
    }
  __syncthreads();   // x of the rows is in registers: the stage buffers are free
  // column segments of this tile: rows r0 .. r0 + nr rounded up to an even
  // count (16-byte copies; the padding rows of a complex64 matrix are zero)
  const float4 *colbase = A + (size_t)c0 * lda2 + (r0 >> 1);
  const unsigned segbytes = (unsigned)((nr + 1) >> 1) * 16u;
  const int cbeg = 64 * w, cend = min(nc, 64 * w + 64);
  const int nsteps = cend > cbeg ? (cend - cbeg + 3) / 4 : 0;
  float4 *my = stage + (size_t)w * SY_STAGES * 4 * 128;
  unsigned long long *bar = sy_bar[w];
  // The warp's stage buffers start at zero: rows past the copied segment and
  // columns past the tile's last are never written, and enter the products
  // only with zero factors (x of those rows and columns is zero).
  for (int e = lane; e < SY_STAGES * 4 * 128; e += 32) my[e] = make_float4(0.f, 0.f, 0.f, 0.f);
  if (lane == 0)
    for (int q = 0; q < SY_STAGES; q++) sy_mbar_init(&bar[q], 1);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // the zeros before any bulk copy
  if (lane == 0) asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  __syncwarp();
  // lane 0 issues step g's copies: one per column of the step
  auto issue = [&](int g) {
    if (g < nsteps && lane == 0) {
      const int cb = cbeg + 4 * g, ncol = min(4, cend - cb);
      float4 *buf = my + (g % SY_STAGES) * 4 * 128;
      unsigned long long *b = &bar[g % SY_STAGES];
      sy_mbar_expect_tx(b, (unsigned)ncol * segbytes);
      for (int u = 0; u < ncol; u++) sy_bulk_g2s(buf + u * 128, colbase + (size_t)(cb + u) * lda2, segbytes, b);
    }
  };
  const int hi = (lane >> 4) & 1, b3 = (lane >> 3) & 1;
  int fail = 0, waited = 0;
  issue(0);
  for (int g = 0; g < nsteps; g++) {
    __syncwarp();          // every lane has read the buffer that step g + 1 refills
    issue(g + 1);
    const bool ok = sy_mbar_wait(&bar[g % SY_STAGES], (unsigned)(g / SY_STAGES) & 1u);
    waited = g + 1;
    if (__any_sync(0xffffffffu, !ok)) {
      fail = 1;
      break;
    }
    const float4 *buf = my + (g % SY_STAGES) * 4 * 128;
    const int c = cbeg + 4 * g;
    float t[4][2 * NR];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      // transposed sums in two independent chains (even and odd rows)
      float2 T0[NR], T1[NR];
#pragma unroll
      for (int jj = 0; jj < NR; jj++) T0[jj] = T1[jj] = make_float2(0.f, 0.f);
#pragma unroll
      for (int k = 0; k < 4; k++) {
        float4 v = buf[u * 128 + lane + 32 * k];
        float2 e0 = make_float2(v.x, v.y), e1 = make_float2(v.z, v.w);
        float2 s0 = make_float2(-v.y, v.x), s1 = make_float2(-v.w, v.z);
#pragma unroll
        for (int jj = 0; jj < NR; jj++) {
          float2 x = xc[c + u][jj];          // zero past nc
          float2 xrr = make_float2(x.x, x.x), xii = make_float2(x.y, x.y);
          D[2 * k][jj] = __ffma2_rn(e0, xrr, D[2 * k][jj]);
          D[2 * k][jj] = __ffma2_rn(s0, xii, D[2 * k][jj]);
          D[2 * k + 1][jj] = __ffma2_rn(e1, xrr, D[2 * k + 1][jj]);
          D[2 * k + 1][jj] = __ffma2_rn(s1, xii, D[2 * k + 1][jj]);
          T0[jj] = __ffma2_rn(e0, Yr[2 * k][jj], T0[jj]);
          T0[jj] = __ffma2_rn(s0, Yi[2 * k][jj], T0[jj]);
          T1[jj] = __ffma2_rn(e1, Yr[2 * k + 1][jj], T1[jj]);
          T1[jj] = __ffma2_rn(s1, Yi[2 * k + 1][jj], T1[jj]);
        }
      }
#pragma unroll
      for (int jj = 0; jj < NR; jj++) {
        t[u][2 * jj] = T0[jj].x + T1[jj].x;
        t[u][2 * jj + 1] = T0[jj].y + T1[jj].y;
      }
    }
    if (trans) {
      // reduce-scatter of the four columns over the warp: halves exchanged
      // across lane bit 4, then bit 3, then full sums over bits 0-2
      float k2[2][2 * NR];
#pragma unroll
      for (int m = 0; m < 2; m++)
#pragma unroll
        for (int e = 0; e < 2 * NR; e++) {
          float keep = hi ? t[2 + m][e] : t[m][e];
          float send = hi ? t[m][e] : t[2 + m][e];
          k2[m][e] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
        }
      float f[2 * NR];
#pragma unroll
      for (int e = 0; e < 2 * NR; e++) {
        float keep = b3 ? k2[1][e] : k2[0][e];
        float send = b3 ? k2[0][e] : k2[1][e];
        f[e] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
      }
#pragma unroll
      for (int o = 4; o > 0; o >>= 1)
#pragma unroll
        for (int e = 0; e < 2 * NR; e++) f[e] += __shfl_xor_sync(0xffffffffu, f[e], o);
      int cc = c + 2 * hi + b3;
      if ((lane & 7) == 0 && cc < cend) {
#pragma unroll
        for (int j = 0; j < NR; j++) partial[((size_t)I * NR + j) * N + c0 + cc] = make_float2(f[2 * j], f[2 * j + 1]);
      }
    }
  }
  if (fail) {
    if (lane == 0) atomicExch(&g_mv_timeout, 1);
    // copies still in flight land before the buffers are reused (bounded)
    // (the step whose wait ran out and the one issued after it)
    for (int g = waited - 1; g <= min(nsteps - 1, waited); g++)
      sy_mbar_wait(&bar[g % SY_STAGES], (unsigned)(g / SY_STAGES) & 1u);
  }
  __syncthreads();          // every warp is done with its stage buffers
#pragma unroll
  for (int k = 0; k < 4; k++)
#pragma unroll
    for (int j = 0; j < NR; j++) {
      dacc[w][64 * k + 2 * lane][j] = D[2 * k][j];
      dacc[w][64 * k + 2 * lane + 1][j] = D[2 * k + 1][j];
    }
  __syncthreads();
  for (int e = threadIdx.x; e < nr * NR; e += 128) {
    int i = e / NR, j = e % NR;
    float sr = 0.f, si = 0.f;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      float2 v = dacc[q][i][j];
      sr += v.x;
      si += v.y;
    }
    partial[((size_t)J * NR + j) * N + r0 + i] = make_float2(sr, si);
  }
}

// the complex64 kernels' partials are FP32 sums already: stored as complex64
// (half the bytes of the partial buffer) and added up in FP64 here
__global__ void k_gm_matvec_sum_f(int N, int nchunk, int nrhs, const float2 *partial, z2 *Y, size_t ldy) {
  int row = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y;
  if (row >= N || j >= nrhs) return;
  // four chunks per round keep four loads in flight; the sum order is fixed
  double sr = 0, si = 0;
  const size_t stride = (size_t)nrhs * N;
  const float2 *p = partial + (size_t)j * N + row;
  int k = 0;
  for (; k + 4 <= nchunk; k += 4) {
    float2 a = p[(size_t)k * stride], b = p[(size_t)(k + 1) * stride], c = p[(size_t)(k + 2) * stride],
           d = p[(size_t)(k + 3) * stride];
    sr += a.x; si += a.y;
    sr += b.x; si += b.y;
    sr += c.x; si += c.y;
    sr += d.x; si += d.y;
  }
  for (; k < nchunk; k++) {
    float2 a = p[(size_t)k * stride];
    sr += a.x;
    si += a.y;
  }
  Y[(size_t)j * ldy + row] = z2{sr, si};
}

__global__ void k_gm_matvec_sum(int N, int nchunk, int nrhs, const z2 *partial, z2 *Y, size_t ldy) {
  int row = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y;
  if (row >= N || j >= nrhs) return;
  double sr = 0, si = 0;
  for (int k = 0; k < nchunk; k++) {
    z2 p = partial[((size_t)k * nrhs + j) * N + row];
    sr += p.r;
    si += p.i;
  }
  Y[(size_t)j * ldy + row] = z2{sr, si};
}

// Y = M X for the sparse preconditioner, eight lanes per row (the row's
// entries are contiguous, so a warp's loads cover four rows' lists in
// order) and every right-hand side per read of the matrix; the lanes'
// partial sums are combined by a fixed butterfly (deterministic)
__global__ void k_gm_spmv8(int N, const int *rowptr, const int *col, const z2 *val, const z2 *X, size_t ldx, int nrhs,
                           z2 *Y, size_t ldy) {
  int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 3, sub = threadIdx.x & 7;
  double sr[GM_MAXRHS] = {0, 0, 0, 0}, si[GM_MAXRHS] = {0, 0, 0, 0};
  if (row < N) {
    int p1 = rowptr[row + 1];
    for (int p = rowptr[row] + sub; p < p1; p += 8) {
      z2 m = val[p];
      int c = col[p];
#pragma unroll
      for (int j = 0; j < GM_MAXRHS; j++)
        if (j < nrhs) {
          z2 x = X[(size_t)j * ldx + c];
          sr[j] += m.r * x.r - m.i * x.i;
          si[j] += m.r * x.i + m.i * x.r;
        }
    }
  }
#pragma unroll
  for (int o = 4; o > 0; o >>= 1)
#pragma unroll
    for (int j = 0; j < GM_MAXRHS; j++) {
      sr[j] += __shfl_xor_sync(0xffffffffu, sr[j], o);
      si[j] += __shfl_xor_sync(0xffffffffu, si[j], o);
    }
  if (row < N && sub == 0)
    for (int j = 0; j < nrhs; j++) Y[(size_t)j * ldy + row] = z2{sr[j], si[j]};
}

// dots[j*(k) + c] = <V_j[:,c], w_j>  (c < k), block reduction per (c, j)
__global__ void k_gm_dots(int N, int k, const z2 *V, size_t ldv, size_t vstride, const z2 *W, size_t ldw, z2 *dots) {
  int c = blockIdx.x, j = blockIdx.y;
  const z2 *v = V + j * vstride + (size_t)c * ldv;
  const z2 *w = W + (size_t)j * ldw;
  double sr = 0, si = 0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    z2 a = v[i], b = w[i];
    sr += a.r * b.r + a.i * b.i;   // conj(a) b
    si += a.r * b.i - a.i * b.r;
  }
  __shared__ double rs[32], is[32];
  for (int o = 16; o > 0; o >>= 1) {
    sr += __shfl_xor_sync(0xffffffffu, sr, o);
    si += __shfl_xor_sync(0xffffffffu, si, o);
  }
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { rs[wid] = sr; is[wid] = si; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) { a += rs[q]; b += is[q]; }
    dots[(size_t)j * gridDim.x + c] = z2{a, b};
  }
}

// w_j -= V_j[:, 0:k] h_j
__global__ void k_gm_subtract(int N, int k, const z2 *V, size_t ldv, size_t vstride, const z2 *h, size_t ldh, z2 *W,
                              size_t ldw) {
  int row = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y;
  if (row >= N) return;
  const z2 *v = V + j * vstride + row;
  const z2 *hj = h + (size_t)j * ldh;
  double sr = 0, si = 0;
  for (int c = 0; c < k; c++) {
    z2 a = v[(size_t)c * ldv], b = hj[c];
    sr += a.r * b.r - a.i * b.i;
    si += a.r * b.i + a.i * b.r;
  }
  z2 *w = W + (size_t)j * ldw + row;
  w->r -= sr;
  w->i -= si;
}

// V_j[:, c] = s_j * W_j ; X_j += sum_c V_j[:, c] y_j[c] ; etc.
__global__ void k_gm_scale_copy(int N, const z2 *W, size_t ldw, const double *s, z2 *V, size_t ldv_col_stride,
                                size_t vstride) {
  int row = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y;
  if (row >= N) return;
  z2 w = W[(size_t)j * ldw + row];
  double f = s[j];
  V[j * vstride + ldv_col_stride + row] = z2{w.r * f, w.i * f};
}

__global__ void k_gm_combine(int N, int k, const z2 *V, size_t ldv, size_t vstride, const z2 *y, size_t ldy, z2 *Z,
                             size_t ldz) {
  int row = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y;
  if (row >= N) return;
  const z2 *v = V + j * vstride + row;
  double sr = 0, si = 0;
  for (int c = 0; c < k; c++) {
    z2 a = v[(size_t)c * ldv], b = y[(size_t)j * ldy + c];
    sr += a.r * b.r - a.i * b.i;
    si += a.r * b.i + a.i * b.r;
  }
  Z[(size_t)j * ldz + row] = z2{sr, si};
}

__global__ void k_gm_axpy(int N, const z2 *D, size_t ldd, z2 *X, size_t ldx, int sign) {
  int row = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y;
  if (row >= N) return;
  z2 d = D[(size_t)j * ldd + row];
  z2 *x = X + (size_t)j * ldx + row;
  x->r += sign * d.r;
  x->i += sign * d.i;
}

// Gram-Schmidt dot products split over GM_DSPLIT row slices, so that even the
// first steps (one or two basis vectors) keep the GPU busy; slice s of
// <V_j[:,c], w_j> goes to part[(j k + c) GM_DSPLIT + s] and the slices are
// added in a fixed order by the consumer (k_gm_hacc, k_gm_givens)
#define GM_DSPLIT 16
__global__ void k_gm_dots_part(int N, int k, const z2 *V, size_t ldv, size_t vstride, const z2 *W, size_t ldw,
                               z2 *part) {
  int c = blockIdx.x, j = blockIdx.y, sl = blockIdx.z;
  int len = (N + GM_DSPLIT - 1) / GM_DSPLIT, i0 = sl * len, i1 = min(N, i0 + len);
  const z2 *v = V + j * vstride + (size_t)c * ldv;
  const z2 *w = W + (size_t)j * ldw;
  double sr = 0, si = 0;
  for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    z2 a = v[i], b = w[i];
    sr += a.r * b.r + a.i * b.i;   // conj(a) b
    si += a.r * b.i - a.i * b.r;
  }
  __shared__ double rs[32], is[32];
  for (int o = 16; o > 0; o >>= 1) {
    sr += __shfl_xor_sync(0xffffffffu, sr, o);
    si += __shfl_xor_sync(0xffffffffu, si, o);
  }
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { rs[wid] = sr; is[wid] = si; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) { a += rs[q]; b += is[q]; }
    part[((size_t)j * k + c) * GM_DSPLIT + sl] = z2{a, b};
  }
}

// Device-side Arnoldi bookkeeping, so that a restart cycle needs no host
// round trip per step.  H (per right-hand side, (m+1) x m column-major), the
// rotated residual vector g and the rotations (cs, sn) live on the device.
// k_gm_hacc adds one Gram-Schmidt pass's coefficients into column k;
// k_gm_givens finishes column k: subdiagonal = |w|, 1/|w| for the next basis
// vector, the previous rotations applied, a new rotation that zeroes the
// subdiagonal, g updated, |g[k+1]| recorded as the residual estimate.
__global__ void k_gm_hacc(int k, int m, const z2 *part, z2 *dots, z2 *H, int add) {
  int j = blockIdx.x, c = threadIdx.x;
  if (c > k) return;
  const z2 *p = part + ((size_t)j * (k + 1) + c) * GM_DSPLIT;
  z2 d{0.0, 0.0};
  for (int sl = 0; sl < GM_DSPLIT; sl++) { d.r += p[sl].r; d.i += p[sl].i; }
  dots[(size_t)j * (k + 1) + c] = d;   // this pass's coefficients, for k_gm_subtract
  z2 *h = H + (size_t)j * (m + 1) * m + (size_t)k * (m + 1) + c;
  if (add) { h->r += d.r; h->i += d.i; }
  else *h = d;
}

__device__ __forceinline__ z2 zmul2(z2 a, z2 b) { return z2{a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r}; }
__device__ __forceinline__ z2 zconj2(z2 a) { return z2{a.r, -a.i}; }

__global__ void k_gm_givens(int k, int m, int nrhs, const z2 *npart, z2 *H, z2 *g, z2 *cs, z2 *sn, double *sc,
                            double *res) {
  int j = threadIdx.x;
  if (j >= nrhs) return;
  double n2 = 0.0;
  for (int sl = 0; sl < GM_DSPLIT; sl++) n2 += npart[(size_t)j * GM_DSPLIT + sl].r;
  double wn = sqrt(fmax(n2, 0.0));
  sc[j] = wn > 0 ? 1.0 / wn : 0.0;
  z2 *hc = H + (size_t)j * (m + 1) * m + (size_t)k * (m + 1);
  z2 *csj = cs + (size_t)j * m, *snj = sn + (size_t)j * m, *gj = g + (size_t)j * (m + 1);
  hc[k + 1] = z2{wn, 0.0};
  for (int i = 0; i < k; i++) {
    z2 a = zmul2(csj[i], hc[i]), b = zmul2(snj[i], hc[i + 1]);
    z2 t{a.r + b.r, a.i + b.i};
    z2 c = zmul2(z2{-snj[i].r, snj[i].i}, hc[i]), d = zmul2(zconj2(csj[i]), hc[i + 1]);
    hc[i + 1] = z2{c.r + d.r, c.i + d.i};
    hc[i] = t;
  }
  double a = hypot(hc[k].r, hc[k].i), b = hypot(hc[k + 1].r, hc[k + 1].i);
  double r = sqrt(a * a + b * b);
  // unitary [c s; -conj(s) conj(c)] with c = conj(hk)/r, s = conj(hk1)/r maps (hk, hk1) to (r, 0)
  csj[k] = r > 0 ? z2{hc[k].r / r, -hc[k].i / r} : z2{1.0, 0.0};
  snj[k] = r > 0 ? z2{hc[k + 1].r / r, -hc[k + 1].i / r} : z2{0.0, 0.0};
  hc[k] = z2{r, 0.0};
  hc[k + 1] = z2{0.0, 0.0};
  z2 gk = gj[k];
  gj[k] = zmul2(csj[k], gk);
  gj[k + 1] = zmul2(z2{-snj[k].r, snj[k].i}, gk);
  res[(size_t)j * m + k] = hypot(gj[k + 1].r, gj[k + 1].i);
}

// residual estimates are read back every GM_CHECK steps (and at the end of a
// cycle): the steps in between run without host synchronisation
#define GM_CHECK 8

struct GmState {
  int N, nrhs, m;
  z2 *V, *W, *Z, *R, *part, *dots, *h;
  double *sc;
  int nchunk;
};

static int dense_matvec(bg_matrix *A, const z2 *X, z2 *Y, GmState &S) {
  int N = S.N;
  prof_start(PROF_MATVEC);
  float2 *pf = reinterpret_cast<float2 *>(S.part);
  if (A->precision == BG_C64 && A->symmetric) {
    dim3 g1(S.nchunk, S.nchunk);
    const float4 *a4 = (const float4 *)A->d;
    size_t l2 = A->ld / 2;
    static bool attr = false;
    if (!attr) {
      BG_CUDA_TRY(cudaFuncSetAttribute(k_gm_matvec_sym_c64<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sym_smem_bytes<1>()));
      BG_CUDA_TRY(cudaFuncSetAttribute(k_gm_matvec_sym_c64<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sym_smem_bytes<2>()));
      BG_CUDA_TRY(cudaFuncSetAttribute(k_gm_matvec_sym_c64<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sym_smem_bytes<3>()));
      BG_CUDA_TRY(cudaFuncSetAttribute(k_gm_matvec_sym_c64<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sym_smem_bytes<4>()));
      attr = true;
    }
    switch (S.nrhs) {
      case 1: k_gm_matvec_sym_c64<1><<<g1, 128, sym_smem_bytes<1>(), stream()>>>(N, a4, l2, X, N, pf); break;
      case 2: k_gm_matvec_sym_c64<2><<<g1, 128, sym_smem_bytes<2>(), stream()>>>(N, a4, l2, X, N, pf); break;
      case 3: k_gm_matvec_sym_c64<3><<<g1, 128, sym_smem_bytes<3>(), stream()>>>(N, a4, l2, X, N, pf); break;
      default: k_gm_matvec_sym_c64<4><<<g1, 128, sym_smem_bytes<4>(), stream()>>>(N, a4, l2, X, N, pf); break;
    }
  } else if (A->precision == BG_C64) {
    dim3 g1((N + 2 * GV_ROWS - 1) / (2 * GV_ROWS), S.nchunk);
    k_gm_matvec_part_c64<<<g1, GV_ROWS, 0, stream()>>>(N, (const float4 *)A->d, A->ld / 2, X, N, S.nrhs, pf);
  } else {
    dim3 g1((N + GV_ROWS - 1) / GV_ROWS, S.nchunk);
    k_gm_matvec_part<<<g1, GV_ROWS, 0, stream()>>>(N, (const z2 *)A->d, A->ld, X, N, S.nrhs, S.part);
  }
  BG_LAUNCHED();
  if (A->precision == BG_C64)
    k_gm_matvec_sum_f<<<dim3((N + 255) / 256, S.nrhs), 256, 0, stream()>>>(N, S.nchunk, S.nrhs, pf, Y, N);
  else
    k_gm_matvec_sum<<<dim3((N + 255) / 256, S.nrhs), 256, 0, stream()>>>(N, S.nchunk, S.nrhs, S.part, Y, N);
  BG_LAUNCHED();
  // algorithmic bytes of matrix read: the upper-triangle tiles for a
  // symmetric complex64 matrix, the whole matrix otherwise
  double nn = (double)N * N;
  double bytes = A->precision == BG_C64 ? (A->symmetric ? 4.0 * nn + 4.0 * 256.0 * N : 8.0 * nn) : 16.0 * nn;
  prof_stop(PROF_MATVEC, bytes);
  return BG_OK;
}

static int precond(const bg_precond *P, const z2 *X, z2 *Y, GmState &S) {
  int N = S.N;
  if (P) prof_start(PROF_PRECOND);
  if (!P) {
    BG_CUDA_TRY(cudaMemcpyAsync(Y, X, sizeof(z2) * (size_t)N * S.nrhs, cudaMemcpyDeviceToDevice, stream()));
    return BG_OK;
  }
  k_gm_spmv8<<<(unsigned)(((size_t)N * 8 + 255) / 256), 256, 0, stream()>>>(N, P->rowptr, P->col, (const z2 *)P->val,
                                                                             X, N, S.nrhs, Y, N);
  BG_LAUNCHED();
  prof_stop(PROF_PRECOND, 0.0);
  return BG_OK;
}

static int colnorms(const z2 *X, GmState &S, std::vector<double> &out) {
  // reuse k_gm_dots with V = W = X (k = 1 column)
  k_gm_dots<<<dim3(1, S.nrhs), 256, 0, stream()>>>(S.N, 1, X, S.N, (size_t)S.N, X, S.N, S.dots);
  BG_LAUNCHED();
  std::vector<z2> h(S.nrhs);
  BG_CUDA_TRY(cudaMemcpyAsync(h.data(), S.dots, sizeof(z2) * S.nrhs, cudaMemcpyDeviceToHost, stream()));
  BG_CUDA_TRY(cudaStreamSynchronize(stream()));
  out.resize(S.nrhs);
  for (int j = 0; j < S.nrhs; j++) out[j] = std::sqrt(std::max(h[j].r, 0.0));
  return BG_OK;
}

// Restart policy.  A cycle has the requested length (restart); after a cycle
// that gains fewer than GM_SLOW digits of the true residual per step the
// next one is twice as long, up to GM_MAXGROW times the request and at most
// GM_MAXM steps (restarted GMRES stagnates on indefinite problems -- the VIE
// system at high frequency -- where a longer cycle still converges; the
// learned or Jacobi-preconditioned VIE solves at moderate frequency gain
// 0.05-0.08 digits per step and never grow).  With an alternative
// preconditioner Palt, a cycle of full length that gains less than one digit
// switches to Palt for the rest of the solve (right preconditioning: every
// restart solves for a correction, so the switch needs nothing else).  Once
// at full length with nothing left to switch to, the solve stops early,
// unconverged, when the last cycle's rate could not reach tol within the
// remaining steps even at twice that rate, so that a caller with a direct
// fallback does not spend the whole budget first.
#define GM_SLOW 0.025
#define GM_MAXM 200
#define GM_MAXGROW 4

static thread_local GmInfo t_gm_info;
GmInfo gmres_last_info() { return t_gm_info; }

// solve A X = B (device, N x nrhs complex128, in place), right preconditioner P
int gmres_solve(bg_matrix *A, const bg_precond *P, void *dB, int ldb, int nrhs, double tol, int restart, int maxit,
                double *stats, const bg_precond *Palt, int *cycle) {
  const int m0 = std::max(2, std::min(restart, GM_MAXM));
  const int N = A->N, m = std::max(m0, std::min(GM_MAXGROW * m0, GM_MAXM));   // m: allocation and strides
  // current cycle length (a caller's earlier solve of the same system may have grown it)
  int mc = cycle ? std::max(m0, std::min(*cycle, m)) : m0;
  if (nrhs > GM_MAXRHS) { set_error("gmres: at most %d right-hand sides per call", GM_MAXRHS); return BG_ERR_ARG; }
  GmState S{N, nrhs, m};
  S.nchunk = (N + GV_COLS - 1) / GV_COLS;
  size_t nv = (size_t)N * (m + 1) * nrhs;
  size_t nH = (size_t)nrhs * (m + 1) * m, ng = (size_t)nrhs * (m + 1), ncs = (size_t)nrhs * m;
  size_t ndp = (size_t)nrhs * (m + 1) * GM_DSPLIT;
  size_t bytes = sizeof(z2) * (nv + 4 * (size_t)N * nrhs + (size_t)S.nchunk * nrhs * N + 2 * (size_t)(m + 2) * nrhs +
                               nH + ng + 2 * ncs + ndp) +
                 sizeof(double) * (8 + ncs);
  char *w = nullptr;
  BG_CUDA_TRY(cudaMallocAsync((void **)&w, bytes, stream()));
  S.V = (z2 *)w;
  S.W = S.V + nv;
  S.Z = S.W + (size_t)N * nrhs;
  S.R = S.Z + (size_t)N * nrhs;
  z2 *X = S.R + (size_t)N * nrhs;
  S.part = X + (size_t)N * nrhs;
  S.dots = S.part + (size_t)S.nchunk * nrhs * N;
  S.h = S.dots + (size_t)(m + 2) * nrhs;
  z2 *Hd = S.h + (size_t)(m + 2) * nrhs, *gd = Hd + nH, *csd = gd + ng, *snd = csd + ncs, *dpart = snd + ncs;
  S.sc = (double *)(dpart + ndp);
  double *resd = S.sc + 8;
  const size_t vstride = (size_t)N * (m + 1);
  // residual estimates read back to pinned host memory (one buffer per library instance)
  static double *res_host = nullptr;
  static size_t res_cap = 0;
  if (res_cap < ncs) {
    if (res_host) cudaFreeHost(res_host);
    res_host = nullptr;
    BG_CUDA_TRY(cudaMallocHost((void **)&res_host, sizeof(double) * ncs));
    res_cap = ncs;
  }
  int st = BG_OK;
  static const int zero = 0;
  BG_CUDA_TRY(cudaMemcpyToSymbolAsync(g_mv_timeout, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, stream()));
  // X = 0
  BG_CUDA_TRY(cudaMemsetAsync(X, 0, sizeof(z2) * (size_t)N * nrhs, stream()));
  // B contiguous copy in W for norms
  BG_CUDA_TRY(cudaMemcpy2DAsync(S.W, sizeof(z2) * N, dB, sizeof(z2) * ldb, sizeof(z2) * N, nrhs,
                                cudaMemcpyDeviceToDevice, stream()));
  std::vector<double> bn, rn;
  if ((st = colnorms(S.W, S, bn))) { cudaFreeAsync(w, stream()); return st; }
  for (auto &v : bn) v = std::max(v, 1e-300);
  int total = 0, cycles = 0, switched = 0, gave_up = 0, longest = mc;
  double relres = 1.0, first = -1, prev = -1;
  int prev_len = 0;
  dim3 gr((N + 255) / 256, nrhs);
  while (!st && total < maxit) {
    // R = B - A X
    if ((st = dense_matvec(A, X, S.R, S))) break;
    BG_CUDA_TRY(cudaMemcpy2DAsync(S.Z, sizeof(z2) * N, dB, sizeof(z2) * ldb, sizeof(z2) * N, nrhs,
                                  cudaMemcpyDeviceToDevice, stream()));
    k_gm_axpy<<<gr, 256, 0, stream()>>>(N, S.R, N, S.Z, N, -1);   // Z = B - AX
    g_launches++;
    if ((st = colnorms(S.Z, S, rn))) break;
    relres = 0;
    for (int j = 0; j < nrhs; j++) relres = std::max(relres, rn[j] / bn[j]);
    if (first < 0) first = relres;
    if (relres <= tol) break;
    if (prev > 0 && prev_len > 0) {
      const double red = relres / prev;   // reduction over the last cycle
      const bool full = prev_len >= m;    // the last cycle had the longest length
      bool just_switched = false;
      const double digits_per_step = -std::log10(std::max(red, 1e-300)) / prev_len;
      if (!full && digits_per_step < GM_SLOW) {
        mc = std::min(2 * mc, m);
      } else if (full && red > 0.1 && Palt && !switched) {
        P = Palt;              // the given preconditioner stagnates at full length: switch
        switched = 1;
        just_switched = true;
      }
      // early stop, at full length with nothing left to switch to (the rate
      // of a cycle run with the replaced preconditioner does not count): at
      // twice the last cycle's rate per step the target is still out of reach
      if (full && (!Palt || switched) && !just_switched) {
        double rate = std::pow(std::max(red, 1e-300), 1.0 / prev_len);
        double need = std::log(tol / relres) / std::log(std::max(rate * rate, 1e-300));
        if (rate >= 1.0 || (std::isfinite(need) && need > (double)(maxit - total))) {
          gave_up = 1;
          break;
        }
      }
    }
    prev = relres;
    longest = std::max(longest, mc);
    cycles++;
    // V[:,0] = Z / beta
    std::vector<double> inv(nrhs);
    for (int j = 0; j < nrhs; j++) inv[j] = rn[j] > 0 ? 1.0 / rn[j] : 0.0;
    BG_CUDA_TRY(cudaMemcpyAsync(S.sc, inv.data(), sizeof(double) * nrhs, cudaMemcpyHostToDevice, stream()));
    k_gm_scale_copy<<<gr, 256, 0, stream()>>>(N, S.Z, N, S.sc, S.V, 0, vstride);
    g_launches++;
    // Hessenberg, rotations and rotated residual on the device
    {
      std::vector<z2> g0(ng, z2{0.0, 0.0});
      for (int j = 0; j < nrhs; j++) g0[(size_t)j * (m + 1)] = z2{rn[j], 0.0};
      BG_CUDA_TRY(cudaMemcpyAsync(gd, g0.data(), sizeof(z2) * ng, cudaMemcpyHostToDevice, stream()));
    }
    const int total0 = total;
    int k = 0, kconv = -1, checked = 0;
    for (; k < mc && total < maxit; k++, total++) {
      // W = A M V[:,k]
      z2 *vk = S.V + (size_t)k * N;   // rhs j at vk + j*vstride: gather into R contiguous
      for (int j = 0; j < nrhs; j++)
        BG_CUDA_TRY(cudaMemcpyAsync(S.R + (size_t)j * N, vk + j * vstride, sizeof(z2) * N, cudaMemcpyDeviceToDevice,
                                    stream()));
      if ((st = precond(P, S.R, S.Z, S))) break;
      if ((st = dense_matvec(A, S.Z, S.W, S))) break;
      // CGS2: two passes, coefficients summed into column k of H on the device
      prof_start(PROF_ORTHO);
      for (int pass = 0; pass < 2; pass++) {
        k_gm_dots_part<<<dim3(k + 1, nrhs, GM_DSPLIT), 256, 0, stream()>>>(N, k + 1, S.V, N, vstride, S.W, N, dpart);
        g_launches++;
        k_gm_hacc<<<nrhs, 256, 0, stream()>>>(k, m, dpart, S.dots, Hd, pass);
        g_launches++;
        k_gm_subtract<<<gr, 256, 0, stream()>>>(N, k + 1, S.V, N, vstride, S.dots, (size_t)(k + 1), S.W, N);
        g_launches++;
      }
      k_gm_dots_part<<<dim3(1, nrhs, GM_DSPLIT), 256, 0, stream()>>>(N, 1, S.W, N, (size_t)N, S.W, N, dpart);
      g_launches++;
      k_gm_givens<<<1, 32, 0, stream()>>>(k, m, nrhs, dpart, Hd, gd, csd, snd, S.sc, resd);
      g_launches++;
      prof_stop(PROF_ORTHO, 0.0);
      if (k + 1 <= m) {
        k_gm_scale_copy<<<gr, 256, 0, stream()>>>(N, S.W, N, S.sc, S.V, (size_t)(k + 1) * N, vstride);
        g_launches++;
      }
      if ((k + 1) % GM_CHECK == 0 || k + 1 == mc || total + 1 == maxit) {
        // one round trip for the residual estimates of the last few steps
        BG_CUDA_TRY(cudaMemcpy2DAsync(res_host, sizeof(double) * m, resd, sizeof(double) * m,
                                      sizeof(double) * (k + 1), nrhs, cudaMemcpyDeviceToHost, stream()));
        BG_CUDA_TRY(cudaStreamSynchronize(stream()));
        for (int kk = checked; kk <= k && kconv < 0; kk++) {
          double rr = 0;
          for (int j = 0; j < nrhs; j++) rr = std::max(rr, res_host[(size_t)j * m + kk] / bn[j]);
          relres = rr;
          if (rr <= tol) kconv = kk;
        }
        checked = k + 1;
        if (kconv >= 0) { k++; total++; break; }
      }
    }
    if (st) break;
    bool conv = kconv >= 0;
    if (!conv && checked < k) {
      // steps after the last check (the cycle ended on maxit)
      BG_CUDA_TRY(cudaMemcpy2DAsync(res_host, sizeof(double) * m, resd, sizeof(double) * m, sizeof(double) * k, nrhs,
                                    cudaMemcpyDeviceToHost, stream()));
      BG_CUDA_TRY(cudaStreamSynchronize(stream()));
      for (int kk = checked; kk < k && kconv < 0; kk++) {
        double rr = 0;
        for (int j = 0; j < nrhs; j++) rr = std::max(rr, res_host[(size_t)j * m + kk] / bn[j]);
        relres = rr;
        if (rr <= tol) kconv = kk;
      }
      conv = kconv >= 0;
    }
    // the least-squares problem over the first kconv + 1 columns (columns and
    // g entries before a step are final once that step is done)
    if (conv) k = kconv + 1;
    total = total0 + k;
    prev_len = k;
    std::vector<z2> Hh(nH), gh(ng);
    BG_CUDA_TRY(cudaMemcpyAsync(Hh.data(), Hd, sizeof(z2) * nH, cudaMemcpyDeviceToHost, stream()));
    BG_CUDA_TRY(cudaMemcpyAsync(gh.data(), gd, sizeof(z2) * ng, cudaMemcpyDeviceToHost, stream()));
    BG_CUDA_TRY(cudaStreamSynchronize(stream()));
    // back substitution y = H^-1 g, X += M V y
    std::vector<z2> yh((size_t)nrhs * k);
    for (int j = 0; j < nrhs; j++) {
      auto Hj = [&](int r, int c) { z2 v = Hh[(size_t)j * (m + 1) * m + (size_t)c * (m + 1) + r]; return zc(v.r, v.i); };
      std::vector<zc> y(k);
      for (int i = k - 1; i >= 0; i--) {
        zc sum(gh[(size_t)j * (m + 1) + i].r, gh[(size_t)j * (m + 1) + i].i);
        for (int c = i + 1; c < k; c++) sum -= Hj(i, c) * y[c];
        y[i] = sum / Hj(i, i);
      }
      for (int i = 0; i < k; i++) yh[(size_t)j * k + i] = z2{y[i].real(), y[i].imag()};
    }
    BG_CUDA_TRY(cudaMemcpyAsync(S.h, yh.data(), sizeof(z2) * yh.size(), cudaMemcpyHostToDevice, stream()));
    k_gm_combine<<<gr, 256, 0, stream()>>>(N, k, S.V, N, vstride, S.h, (size_t)k, S.R, N);
    g_launches++;
    if ((st = precond(P, S.R, S.Z, S))) break;
    k_gm_axpy<<<gr, 256, 0, stream()>>>(N, S.Z, N, X, N, 1);
    g_launches++;
    if (conv) {
      // confirm with the true residual
      if ((st = dense_matvec(A, X, S.R, S))) break;
      BG_CUDA_TRY(cudaMemcpy2DAsync(S.Z, sizeof(z2) * N, dB, sizeof(z2) * ldb, sizeof(z2) * N, nrhs,
                                    cudaMemcpyDeviceToDevice, stream()));
      k_gm_axpy<<<gr, 256, 0, stream()>>>(N, S.R, N, S.Z, N, -1);
      g_launches++;
      if ((st = colnorms(S.Z, S, rn))) break;
      relres = 0;
      for (int j = 0; j < nrhs; j++) relres = std::max(relres, rn[j] / bn[j]);
      if (relres <= tol * 10) break;
    }
  }
  if (!st) {
    cudaError_t e = cudaMemcpy2DAsync(dB, sizeof(z2) * ldb, X, sizeof(z2) * N, sizeof(z2) * N, nrhs,
                                      cudaMemcpyDeviceToDevice, stream());
    if (e != cudaSuccess) { set_error("gmres: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
  }
  if (!st) {
    // a bounded wait of the symmetric product that ran out (none expected)
    int to = 0;
    cudaError_t e = cudaMemcpyFromSymbolAsync(&to, g_mv_timeout, sizeof(int), 0, cudaMemcpyDeviceToHost, stream());
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream());
    if (e != cudaSuccess) { set_error("gmres: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
    else if (to) { set_error("gmres: a bulk copy of the matrix-vector product timed out"); st = BG_ERR_CUDA; }
  }
  cudaFreeAsync(w, stream());
  if (stats) { stats[0] = total; stats[1] = relres; stats[2] = first; }
  if (cycle) *cycle = mc;
  t_gm_info.switched |= switched;
  t_gm_info.gave_up |= gave_up;
  t_gm_info.longest_cycle = std::max(t_gm_info.longest_cycle, longest);
  return st;
}

// GMRES with FP64 iterative refinement: each Krylov solve runs against the
// complex64 copy F of A (8 N^2 bytes per step instead of 16), corrections
// accumulate in FP64 and the residual b - A x is recomputed with the
// complex128 matrix A between solves, until max_j |b_j - A x_j| / |b_j| <= tol.
// A sweep asks the Krylov solve for inner_tol, or for less once the residual
// is within 1/inner_tol of the target.
int gmres_solve_mixed(bg_matrix *A, bg_matrix *F, const bg_precond *P, void *dB, int ldb, int nrhs, double tol,
                      int restart, int maxit, double inner_tol, double *stats) {
  int N = A->N;
  if (nrhs > GM_MAXRHS) { set_error("gmres: at most %d right-hand sides per call", GM_MAXRHS); return BG_ERR_ARG; }
  GmState S{N, nrhs, 0};
  S.nchunk = (N + GV_COLS - 1) / GV_COLS;
  size_t nn = (size_t)N * nrhs;
  char *w = nullptr;
  BG_CUDA_TRY(cudaMallocAsync((void **)&w, sizeof(z2) * (4 * nn + (size_t)S.nchunk * nn + 4 * nrhs), stream()));
  z2 *B0 = (z2 *)w, *X = B0 + nn, *R = X + nn, *T = R + nn;
  S.part = T + nn;
  S.dots = S.part + (size_t)S.nchunk * nn;
  int st = BG_OK;
  dim3 gr((N + 255) / 256, nrhs);
  std::vector<double> bn, rn;
  BG_CUDA_TRY(cudaMemcpy2DAsync(B0, sizeof(z2) * N, dB, sizeof(z2) * ldb, sizeof(z2) * N, nrhs,
                                cudaMemcpyDeviceToDevice, stream()));
  BG_CUDA_TRY(cudaMemsetAsync(X, 0, sizeof(z2) * nn, stream()));
  BG_CUDA_TRY(cudaMemcpyAsync(R, B0, sizeof(z2) * nn, cudaMemcpyDeviceToDevice, stream()));
  if ((st = colnorms(B0, S, bn))) { cudaFreeAsync(w, stream()); return st; }
  for (auto &v : bn) v = std::max(v, 1e-300);
  int total = 0, sweeps = 0;
  double relres = 1.0;
  t_gm_info = GmInfo{};
  // the diagonal of A: the preconditioner a stagnating P is replaced by
  bg_precond *J = nullptr;
  if (P && !P->jacobi && (st = precond_jacobi(A, &J))) { cudaFreeAsync(w, stream()); return st; }
  const bg_precond *Pcur = P;
  int cycle = restart;   // restart cycle length, carried over the refinement sweeps
  while (!st && relres > tol && total < maxit && sweeps < 40) {
    double ist[3] = {0, 0, 0};
    // R <- approximately F^{-1} R (in place); the last sweeps only need the
    // remaining reduction (with a 0.3 margin), not a full inner_tol
    double itol = std::min(0.5, std::max(inner_tol, 0.3 * tol / relres));
    const int sw0 = t_gm_info.switched;
    if ((st = gmres_solve(F, Pcur, R, N, nrhs, itol, restart, maxit - total, ist, Pcur == P ? J : nullptr, &cycle)))
      break;
    if (t_gm_info.switched && !sw0) Pcur = J;   // later sweeps keep the replacement
    total += (int)ist[0];
    sweeps++;
    if (t_gm_info.gave_up) break;
    k_gm_axpy<<<gr, 256, 0, stream()>>>(N, R, N, X, N, 1);
    g_launches++;
    if ((st = dense_matvec(A, X, T, S))) break;
    BG_CUDA_TRY(cudaMemcpyAsync(R, B0, sizeof(z2) * nn, cudaMemcpyDeviceToDevice, stream()));
    k_gm_axpy<<<gr, 256, 0, stream()>>>(N, T, N, R, N, -1);
    g_launches++;
    if ((st = colnorms(R, S, rn))) break;
    relres = 0;
    for (int j = 0; j < nrhs; j++) relres = std::max(relres, rn[j] / bn[j]);
    if (!std::isfinite(relres)) { set_error("gmres: non-finite residual"); st = BG_ERR_NUMERIC; }
  }
  if (!st) {
    cudaError_t e = cudaMemcpy2DAsync(dB, sizeof(z2) * ldb, X, sizeof(z2) * N, sizeof(z2) * N, nrhs,
                                      cudaMemcpyDeviceToDevice, stream());
    if (e != cudaSuccess) { set_error("gmres: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
  }
  if (J) bg_precond_destroy(J);
  cudaFreeAsync(w, stream());
  if (stats) { stats[0] = total; stats[1] = relres; stats[2] = sweeps; }
  t_gm_info.steps = total;
  t_gm_info.relres = relres;
  t_gm_info.sweeps = sweeps;
  return st;
}

// diagonal (Jacobi) preconditioner from the assembled matrix
__global__ void k_gm_diag_inv(int N, const z2 *A, size_t lda, int *rowptr, int *col, z2 *val) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > N) return;
  rowptr[i] = i;
  if (i == N) return;
  z2 a = A[(size_t)i * lda + i];
  double d = a.r * a.r + a.i * a.i;
  col[i] = i;
  val[i] = z2{a.r / d, -a.i / d};
}

int precond_jacobi(bg_matrix *A, bg_precond **out) {
  bg_precond *P = new bg_precond();
  P->N = A->N;
  P->nnz = A->N;
  P->jacobi = true;
  BG_CUDA_TRY(cudaMallocAsync((void **)&P->rowptr, sizeof(int) * (A->N + 1), stream()));
  BG_CUDA_TRY(cudaMallocAsync((void **)&P->col, sizeof(int) * A->N, stream()));
  BG_CUDA_TRY(cudaMallocAsync((void **)&P->val, sizeof(z2) * A->N, stream()));
  k_gm_diag_inv<<<(A->N + 256) / 256, 256, 0, stream()>>>(A->N, (const z2 *)A->d, A->ld, P->rowptr, P->col,
                                                          (z2 *)P->val);
  BG_LAUNCHED();
  *out = P;
  return BG_OK;
}

}  // namespace bg
