// Precision form: conversion of the complex128 VIE matrix to complex64 for
// the tensor-core LU, and FP64 iterative refinement of the solution against
// the complex128 matrix (the refinement residual is the only FP64 work on the
// solve side).
//
//   x_0 = 0, r_0 = b
//   repeat:  d = (LU_32)^{-1} r  (complex64, tensor-core factors)
//            x += d               (complex128)
//            r  = b - A_64 x      (complex128 matrix-vector product)
//   until max_j |r_j| / |b_j| <= tol (2-norms) or maxit
//
// The matrix-vector product is HBM-bound (16 N^2 bytes per sweep): a 2-D
// grid (row blocks x column chunks) writes partial sums that a second kernel
// reduces in a fixed order (deterministic).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "internal.h"

namespace bg {

struct c2 { double r, i; };
struct c1 { float r, i; };

__global__ void k_c128_to_c64(int N, const c2 *src, size_t lds, c1 *dst, size_t ldd) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  size_t col = blockIdx.y;
  if (i >= (size_t)N) return;
  c2 v = src[col * lds + i];
  dst[col * ldd + i] = c1{(float)v.r, (float)v.i};
}

__global__ void k_vec_to_c64(int n, const c2 *src, c1 *dst) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = c1{(float)src[i].r, (float)src[i].i};
}

__global__ void k_axpy_c64(int n, const c1 *d, c2 *x) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) { x[i].r += (double)d[i].r; x[i].i += (double)d[i].i; }
}

#define MV_ROWS 128
#define MV_COLS 256
#define MV_MAXRHS 4
// partial[chunk][j][row] = sum_{c in chunk} A[row, c] x[c, j]
__global__ void __launch_bounds__(MV_ROWS) k_matvec_part(int N, const c2 *A, size_t lda, const c2 *X, size_t ldx,
                                                         int nrhs, c2 *partial) {
  __shared__ c2 xs[MV_COLS][MV_MAXRHS];
  int row = blockIdx.x * MV_ROWS + threadIdx.x;
  int c0 = blockIdx.y * MV_COLS;
  int nc = min(MV_COLS, N - c0);
  for (int e = threadIdx.x; e < nc * nrhs; e += MV_ROWS) {
    int c = e / nrhs, j = e % nrhs;
    xs[c][j] = X[(size_t)j * ldx + c0 + c];
  }
  __syncthreads();
  if (row >= N) return;
  double ar[MV_MAXRHS] = {0, 0, 0, 0}, ai[MV_MAXRHS] = {0, 0, 0, 0};
  const c2 *ap = A + (size_t)c0 * lda + row;
  int c = 0;
  // eight columns' loads in flight per thread, then their products in order
  for (; c + 8 <= nc; c += 8) {
    c2 a[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      double2 t = __ldcs(reinterpret_cast<const double2 *>(ap + (size_t)(c + u) * lda));
      a[u] = c2{t.x, t.y};
    }
#pragma unroll
    for (int u = 0; u < 8; u++)
#pragma unroll
      for (int j = 0; j < MV_MAXRHS; j++)
        if (j < nrhs) {
          c2 x = xs[c + u][j];
          ar[j] += a[u].r * x.r - a[u].i * x.i;
          ai[j] += a[u].r * x.i + a[u].i * x.r;
        }
  }
  for (; c < nc; c++) {
    c2 a = ap[(size_t)c * lda];
#pragma unroll
    for (int j = 0; j < MV_MAXRHS; j++) {
      if (j < nrhs) {
        c2 x = xs[c][j];
        ar[j] += a.r * x.r - a.i * x.i;
        ai[j] += a.r * x.i + a.i * x.r;
      }
    }
  }
  for (int j = 0; j < nrhs; j++)
    partial[((size_t)blockIdx.y * nrhs + j) * N + row] = c2{ar[j], ai[j]};
}

// R = B - sum over chunks; also per-block squared norms of R for each rhs
__global__ void k_matvec_reduce(int N, int nchunk, int nrhs, const c2 *partial, const c2 *B, size_t ldb, c2 *R,
                                size_t ldr, double *sq) {
  int row = blockIdx.x * blockDim.x + threadIdx.x;
  __shared__ double red[MV_MAXRHS][8];
  double loc[MV_MAXRHS] = {0, 0, 0, 0};
  if (row < N) {
    for (int j = 0; j < nrhs; j++) {
      double sr = 0, si = 0;
      for (int k = 0; k < nchunk; k++) {
        c2 p = partial[((size_t)k * nrhs + j) * N + row];
        sr += p.r;
        si += p.i;
      }
      c2 b = B[(size_t)j * ldb + row];
      c2 r{b.r - sr, b.i - si};
      R[(size_t)j * ldr + row] = r;
      loc[j] = r.r * r.r + r.i * r.i;
    }
  }
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int j = 0; j < nrhs; j++) {
    double v = loc[j];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[j][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < nrhs) {
    double s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[threadIdx.x][w];
    sq[(size_t)blockIdx.x * nrhs + threadIdx.x] = s;
  }
}

__global__ void k_colnorm2(int N, int nrhs, const c2 *B, size_t ldb, double *sq) {
  int row = blockIdx.x * blockDim.x + threadIdx.x;
  __shared__ double red[MV_MAXRHS][8];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int j = 0; j < nrhs; j++) {
    double v = 0;
    if (row < N) { c2 b = B[(size_t)j * ldb + row]; v = b.r * b.r + b.i * b.i; }
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[j][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < nrhs) {
    double s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[threadIdx.x][w];
    sq[(size_t)blockIdx.x * nrhs + threadIdx.x] = s;
  }
}

int matrix_convert(const bg_matrix *src, bg_matrix *dst) {
  if (src->precision != BG_C128 || dst->precision != BG_C64 || src->N != dst->N) {
    set_error("bg_matrix_convert: complex128 source and complex64 destination of equal size required");
    return BG_ERR_ARG;
  }
  dim3 grid((src->N + 255) / 256, src->N);
  k_c128_to_c64<<<grid, 256, 0, stream()>>>(src->N, (const c2 *)src->d, src->ld, (c1 *)dst->d, dst->ld);
  BG_LAUNCHED();
  dst->factored = false;
  dst->symmetric = src->symmetric && !src->factored;
  return BG_OK;
}

static int sum_blocks(const double *dsq, int nblocks, int nrhs, std::vector<double> &out) {
  std::vector<double> h((size_t)nblocks * nrhs);
  BG_CUDA_TRY(cudaMemcpyAsync(h.data(), dsq, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, stream()));
  BG_CUDA_TRY(cudaStreamSynchronize(stream()));
  out.assign(nrhs, 0.0);
  for (int b = 0; b < nblocks; b++)
    for (int j = 0; j < nrhs; j++) out[j] += h[(size_t)b * nrhs + j];
  return BG_OK;
}

// A: complex128 matrix (residuals), F: complex64 LU factors of A.
// B (device, N x nrhs complex128, ldb) is overwritten by X.
int solve_refined(bg_matrix *A, bg_matrix *F, void *dB, int ldb, int nrhs, double tol, int maxit, double *stats) {
  if (nrhs > MV_MAXRHS) { set_error("refined solve: at most %d right-hand sides per call", MV_MAXRHS); return BG_ERR_ARG; }
  int N = A->N;
  int nchunk = (N + MV_COLS - 1) / MV_COLS, nrb = (N + MV_ROWS - 1) / MV_ROWS;
  int nb256 = (N + 255) / 256;
  size_t bytes = sizeof(c2) * (size_t)N * nrhs * 3 + sizeof(c1) * (size_t)N * nrhs +
                 sizeof(c2) * (size_t)nchunk * nrhs * N + sizeof(double) * (size_t)nb256 * nrhs * 2;
  char *w = nullptr;
  BG_CUDA_TRY(cudaMallocAsync((void **)&w, bytes, stream()));
  c2 *B0 = (c2 *)w;                      // copy of b
  c2 *X = B0 + (size_t)N * nrhs;         // solution
  c2 *R = X + (size_t)N * nrhs;          // residual
  c1 *R32 = (c1 *)(R + (size_t)N * nrhs);
  c2 *part = (c2 *)(R32 + (size_t)N * nrhs);
  double *sq = (double *)(part + (size_t)nchunk * nrhs * N);
  int st = BG_OK;
  auto fail = [&](cudaError_t e) { set_error("refined solve: %s", cudaGetErrorString(e)); return BG_ERR_CUDA; };
  cudaError_t e = cudaMemcpy2DAsync(B0, sizeof(c2) * N, dB, sizeof(c2) * ldb, sizeof(c2) * N, nrhs,
                                    cudaMemcpyDeviceToDevice, stream());
  if (e != cudaSuccess) st = fail(e);
  if (!st && (e = cudaMemsetAsync(X, 0, sizeof(c2) * (size_t)N * nrhs, stream())) != cudaSuccess) st = fail(e);
  if (!st && (e = cudaMemcpyAsync(R, B0, sizeof(c2) * (size_t)N * nrhs, cudaMemcpyDeviceToDevice, stream())) !=
                 cudaSuccess)
    st = fail(e);
  std::vector<double> bn, rn;
  if (!st) {
    k_colnorm2<<<nb256, 256, 0, stream()>>>(N, nrhs, B0, N, sq);
    if ((e = cudaGetLastError()) != cudaSuccess) st = fail(e);
    else { g_launches++; st = sum_blocks(sq, nb256, nrhs, bn); }
  }
  int it = 0;
  double first = -1, last = 1;
  for (; !st && it < maxit; it++) {
    k_vec_to_c64<<<(N * nrhs + 255) / 256, 256, 0, stream()>>>(N * nrhs, R, R32);
    g_launches++;
    if ((st = lu_solve(F, R32, N, nrhs))) break;
    k_axpy_c64<<<(N * nrhs + 255) / 256, 256, 0, stream()>>>(N * nrhs, R32, X);
    g_launches++;
    prof_start(PROF_RESID);
    k_matvec_part<<<dim3(nrb, nchunk), MV_ROWS, 0, stream()>>>(N, (const c2 *)A->d, A->ld, X, N, nrhs, part);
    g_launches++;
    k_matvec_reduce<<<nb256, 256, 0, stream()>>>(N, nchunk, nrhs, part, B0, N, R, N, sq);
    g_launches++;
    prof_stop(PROF_RESID, 16.0 * (double)N * N);
    if ((e = cudaGetLastError()) != cudaSuccess) { st = fail(e); break; }
    if ((st = sum_blocks(sq, nb256, nrhs, rn))) break;
    last = 0;
    for (int j = 0; j < nrhs; j++) last = std::max(last, std::sqrt(rn[j] / std::max(bn[j], 1e-300)));
    if (first < 0) first = last;
    if (!std::isfinite(last)) { set_error("refined solve: non-finite residual"); st = BG_ERR_NUMERIC; break; }
    if (last <= tol) { it++; break; }
  }
  if (!st) st = lu_solve_status(F);
  if (!st) {
    e = cudaMemcpy2DAsync(dB, sizeof(c2) * ldb, X, sizeof(c2) * N, sizeof(c2) * N, nrhs, cudaMemcpyDeviceToDevice,
                          stream());
    if (e != cudaSuccess) st = fail(e);
  }
  cudaFreeAsync(w, stream());
  if (stats) { stats[0] = it; stats[1] = last; stats[2] = first; }
  return st;
}

}  // namespace bg
