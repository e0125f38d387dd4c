// buff-neq's per-frequency flux chain (GetFlux, GetFlux.cc:291-436, and
// ComputeDressedRytovMatrix, GetFlux.cc:155-272) for one geometry as it
// stands (no geometrical transforms) at uniform temperature per object:
//
//   W    = (1 + S^-1 V S^-1 G)^-1            (by LU; once per frequency)
//   DR_s = W (S^-1 R_s S^-1) W^H             (per source object s)
//   Flux[s][d][q] = GetPFTMatrix(0, w, {EMT, DR_s})[d][q]
//
// with S the Gram matrix of the basis functions (GetOverlapElements), V and
// R_s the overlap blocks of -w^2 (eps - 1) and 4 w Im(eps) / (pi Z0)
// (GetOverlaps; R only on object s), G the G block of the VIE matrix.
//
// B200 layout: every matrix is dense complex128 in HBM, column-major with
// leading dimension N.  S^-1 is frequency independent and kept for the
// geometry's lifetime.  Products with S^-1 and the two N-column solves run
// on the FP64 tensor-core GEMM (the same recursive kernels as the LU); the
// sparse V and R_s products are gathers of <= 7 entries per row.  S, V and
// R_s couple only basis functions of one object, so S^-1 is block diagonal
// and S^-1 R_s S^-1 lives in the (s, s) block: the chain skips the columns
// and rows that are exactly zero, which leaves every computed entry equal
// to the dense product (the skipped terms are exact zeros).
//
// The reference recomputes W for every source object; it does not depend on
// the source, so it is factored once per frequency here.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <utility>
#include <vector>

#include "internal.h"

namespace bg {
namespace {

struct z { double r, i; };

constexpr int NSLOT = 8;

// dst = 0 (ld x n columns)
__global__ void k_zero(z *A, size_t ld, int rows, int cols) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  size_t n = (size_t)rows * cols;
  if (i >= n) return;
  size_t c = i / rows, r = i % rows;
  A[c * ld + r] = z{0.0, 0.0};
}

// A[r][c] = S[r][c] for the sparse rows (dense Gram matrix)
__global__ void k_scatter_S(int N, const int *idx, const double *S, z *A, size_t ld) {
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= N) return;
  for (int k = 0; k < NSLOT; k++) {
    int b = idx[NSLOT * (size_t)a + k];
    if (b >= 0) A[(size_t)b * ld + a] = z{S[NSLOT * (size_t)a + k], 0.0};
  }
}

__global__ void k_add_identity(z *A, size_t ld, int N, double s) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) A[(size_t)i * ld + i].r += s;
}

// Y[r0:r1, c] = V[r, :] X[:, c] for rows r in [r0, r1) (V sparse by rows, the
// SetEntry of AssembleOverlapBlocks); one thread per (row, column)
__global__ void k_sparse_rows(int r0, int r1, int ncol, const int *idx, const z *V, const z *X, size_t ldx, z *Y,
                              size_t ldy) {
  int r = r0 + blockIdx.x * blockDim.x + threadIdx.x;
  int c = blockIdx.y;
  if (r >= r1 || c >= ncol) return;
  double sr = 0.0, si = 0.0;
  for (int k = 0; k < NSLOT; k++) {
    int b = idx[NSLOT * (size_t)r + k];
    if (b < 0) continue;
    z v = V[NSLOT * (size_t)r + k], x = X[(size_t)c * ldx + b];
    sr += v.r * x.r - v.i * x.i;
    si += v.r * x.i + v.i * x.r;
  }
  Y[(size_t)c * ldy + r] = z{sr, si};
}

// Y[:, c] = X R[:, c] for the columns c of object s.  The sparsity pattern is
// symmetric, so the rows b with an entry in column c are the slots of row c,
// and R[b][c] is the slot of row b that names c.
__global__ void k_sparse_cols(int nrow, int c0, int c1, const int *idx, const double *R, const z *X, size_t ldx, z *Y,
                              size_t ldy) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  int c = c0 + blockIdx.y;
  if (r >= nrow || c >= c1) return;
  double sr = 0.0, si = 0.0;
  for (int k = 0; k < NSLOT; k++) {
    int b = idx[NSLOT * (size_t)c + k];
    if (b < 0) continue;
    double v = 0.0;
    for (int m = 0; m < NSLOT; m++)
      if (idx[NSLOT * (size_t)b + m] == c) v = R[NSLOT * (size_t)b + m];
    z x = X[(size_t)b * ldx + r];
    sr += x.r * v;
    si += x.i * v;
  }
  Y[(size_t)c * ldy + r] = z{sr, si};
}

// B = s * A^H (N x N, 32 x 32 tiles through shared memory)
__global__ void k_adjoint(int N, const z *A, size_t lda, z *B, size_t ldb, double s) {
  __shared__ z t[32][33];
  int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += 8) {
    int r = bx + threadIdx.x, c = by + j;
    if (r < N && c < N) t[j][threadIdx.x] = A[(size_t)c * lda + r];
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += 8) {
    int r = by + threadIdx.x, c = bx + j;   // B[r][c] = conj(A[c][r])
    if (r < N && c < N) {
      z v = t[threadIdx.x][j];
      B[(size_t)c * ldb + r] = z{s * v.r, -s * v.i};
    }
  }
}

}  // namespace
}  // namespace bg

using namespace bg;

struct bg_neq {
  bg_geometry *g = nullptr;
  int N = 0;
  z *Sinv = nullptr;        // N x N
  z *M1 = nullptr, *M2 = nullptr;
  bg_matrix *W = nullptr;   // 1 + S^-1 V S^-1 G, factored
  int *idx = nullptr, *cnt = nullptr;
  double *S = nullptr, *R = nullptr;
  z *V = nullptr;
  double w_ready = 0.0, wi_ready = 0.0;
  bool have_w = false;
};

namespace {

void neq_free(bg_neq *h) {
  if (!h) return;
  cudaFree(h->Sinv); cudaFree(h->M1); cudaFree(h->M2);
  cudaFree(h->idx); cudaFree(h->cnt); cudaFree(h->S); cudaFree(h->R); cudaFree(h->V);
  if (h->W) bg_matrix_destroy(h->W);
  delete h;
}

int launched() {
  BG_LAUNCHED();
  return BG_OK;
}

constexpr int YMAX = 65535;   // grid.y limit: column loops in chunks

int launch_zero(z *A, size_t ld, int rows, int cols) {
  size_t n = (size_t)rows * cols;
  if (!n) return BG_OK;
  k_zero<<<(unsigned)((n + 255) / 256), 256, 0, stream()>>>(A, ld, rows, cols);
  BG_LAUNCHED();
  return BG_OK;
}

// W for omega: overlaps, G, M3 = 1 + S^-1 V S^-1 G, LU
int neq_prepare(bg_neq *h, double wr, double wi) {
  if (h->have_w && h->w_ready == wr && h->wi_ready == wi) return BG_OK;
  h->have_w = false;
  bg_geometry *g = h->g;
  int N = h->N, st;
  size_t ld = N;
  const std::vector<int> &off = g->bfOffset;
  if ((st = neq_overlaps(g, wr, h->idx, h->S, h->V, h->R, h->cnt))) return st;
  // M2 <- G (far + near entries of the VIE matrix, no V^-1 Gram part)
  if ((st = bg_geometry_precompute(g))) return st;
  if ((st = assemble_far(g, wr, wi, h->M2, ld)) || (st = assemble_near(g, wr, wi, h->M2, ld))) return st;
  // M1 <- -S^-1 G   (per object block rows: S^-1 is block diagonal)
  int NO = (int)g->objs.size();
  for (int o = 0; o < NO; o++) {
    int r0 = off[o], n = off[o + 1] - off[o];
    if ((st = launch_zero(h->M1 + r0, ld, n, N))) return st;
    if ((st = zgemm_sub_device(n, N, n, h->Sinv + r0 + (size_t)r0 * ld, N, h->M2 + r0, N, h->M1 + r0, N))) return st;
  }
  // M2 <- V M1 = -V S^-1 G
  for (int c0 = 0; c0 < N; c0 += YMAX) {
    int nc = std::min(YMAX, N - c0);
    k_sparse_rows<<<dim3((N + 127) / 128, nc), 128, 0, stream()>>>(0, N, nc, h->idx, h->V, h->M1 + (size_t)c0 * ld,
                                                                    ld, h->M2 + (size_t)c0 * ld, ld);
    BG_LAUNCHED();
  }
  // W <- 0 - S^-1 M2 = S^-1 V S^-1 G, then + 1
  z *Wd = (z *)h->W->d;
  size_t ldw = h->W->ld;
  for (int o = 0; o < NO; o++) {
    int r0 = off[o], n = off[o + 1] - off[o];
    if ((st = launch_zero(Wd + r0, ldw, n, N))) return st;
    if ((st = zgemm_sub_device(n, N, n, h->Sinv + r0 + (size_t)r0 * ld, N, h->M2 + r0, N, Wd + r0, (int)ldw))) return st;
  }
  k_add_identity<<<(N + 255) / 256, 256, 0, stream()>>>(Wd, ldw, N, 1.0);
  BG_LAUNCHED();
  h->W->factored = false;
  int info = bg_lu_factor(h->W);
  if (info < 0) return info;
  if (info > 0) { set_error("buff-neq: 1 + S^-1 V S^-1 G is singular (pivot %d)", info); return BG_ERR_NUMERIC; }
  h->w_ready = wr;
  h->wi_ready = wi;
  h->have_w = true;
  return BG_OK;
}

// DR of source object s into M1 (device, ld N)
int neq_dr(bg_neq *h, int s) {
  bg_geometry *g = h->g;
  int N = h->N, st;
  size_t ld = N;
  int c0 = g->bfOffset[s], c1 = g->bfOffset[s + 1], ns = c1 - c0;
  // M2[:, s] <- S^-1 R_s (columns of object s; S^-1 rows of object s only)
  if ((st = launch_zero(h->M2, ld, N, N))) return st;
  for (int cc = c0; cc < c1; cc += YMAX) {
    int ce = std::min(c1, cc + YMAX);
    k_sparse_cols<<<dim3((N + 127) / 128, ce - cc), 128, 0, stream()>>>(N, cc, ce, h->idx, h->R, h->Sinv, ld, h->M2, ld);
    BG_LAUNCHED();
  }
  // M1 <- -(S^-1 R_s) S^-1 = -SRS, nonzero in the (s, s) block only
  if ((st = launch_zero(h->M1, ld, N, N))) return st;
  if ((st = zgemm_sub_device(ns, ns, ns, h->M2 + c0 + (size_t)c0 * ld, N, h->Sinv + c0 + (size_t)c0 * ld, N,
                             h->M1 + c0 + (size_t)c0 * ld, N)))
    return st;
  // M1[:, s] <- W^-1 (-SRS)[:, s]; the other columns stay exactly zero
  if ((st = lu_solve_many(h->W, h->M1 + (size_t)c0 * ld, ld, ns))) return st;
  // M2 <- -(M1)^H = (W SRS)^H = SRS W^H
  dim3 tb(32, 8), tg((N + 31) / 32, (N + 31) / 32);
  k_adjoint<<<tg, tb, 0, stream()>>>(N, h->M1, ld, h->M2, ld, -1.0);
  BG_LAUNCHED();
  // M2 <- W^-1 M2 = W SRS W^H
  if ((st = lu_solve_many(h->W, h->M2, ld, N))) return st;
  std::swap(h->M1, h->M2);
  return BG_OK;
}

}  // namespace

extern "C" {

int bg_neq_create(bg_geometry *g, bg_neq **out) {
  if (!g || !out) { set_error("bg_neq_create: bad arguments"); return BG_ERR_ARG; }
  *out = nullptr;
  int st = upload_geometry(g);
  if (st) return st;
  bg_neq *h = new (std::nothrow) bg_neq();
  if (!h) { set_error("out of host memory"); return BG_ERR_NOMEM; }
  h->g = g;
  int N = h->N = g->N;
  size_t nn = (size_t)N * N * sizeof(z);
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = cudaMalloc(&h->Sinv, nn);
  if (e == cudaSuccess) e = cudaMalloc(&h->M1, nn);
  if (e == cudaSuccess) e = cudaMalloc(&h->M2, nn);
  if (e == cudaSuccess) e = cudaMalloc(&h->idx, sizeof(int) * NSLOT * (size_t)N);
  if (e == cudaSuccess) e = cudaMalloc(&h->cnt, sizeof(int) * (size_t)N);
  if (e == cudaSuccess) e = cudaMalloc(&h->S, sizeof(double) * NSLOT * (size_t)N);
  if (e == cudaSuccess) e = cudaMalloc(&h->R, sizeof(double) * NSLOT * (size_t)N);
  if (e == cudaSuccess) e = cudaMalloc(&h->V, sizeof(z) * NSLOT * (size_t)N);
  if (e != cudaSuccess) {
    neq_free(h);
    set_error("bg_neq_create: cannot allocate 3 x %.2f GB on the device: %s", nn / 1e9, cudaGetErrorString(e));
    return BG_ERR_NOMEM;
  }
  if ((st = bg_matrix_create(g, BG_C128, &h->W))) { neq_free(h); return st; }
  // S^-1 (SInverse, CreateBNEQData.cc:122-141): dense S, LU, solve with the
  // identity, per object block
  if ((st = neq_overlaps(g, 1.0, h->idx, h->S, h->V, h->R, h->cnt))) { neq_free(h); return st; }
  z *Sd = (z *)h->W->d;
  size_t ldw = h->W->ld;
  if ((st = launch_zero(Sd, ldw, N, N)) || (st = launch_zero(h->Sinv, N, N, N))) { neq_free(h); return st; }
  k_scatter_S<<<(N + 127) / 128, 128, 0, stream()>>>(N, h->idx, h->S, Sd, ldw);
  if ((st = launched())) { neq_free(h); return st; }
  k_add_identity<<<(N + 255) / 256, 256, 0, stream()>>>(h->Sinv, N, N, 1.0);
  if ((st = launched())) { neq_free(h); return st; }
  int info = bg_lu_factor(h->W);
  if (info != 0) {
    neq_free(h);
    if (info > 0) { set_error("bg_neq_create: Gram matrix is singular (pivot %d)", info); return BG_ERR_NUMERIC; }
    return info;
  }
  if ((st = lu_solve_many(h->W, h->Sinv, N, N))) { neq_free(h); return st; }
  cudaError_t e2 = cudaStreamSynchronize(stream());
  if (e2 != cudaSuccess) { neq_free(h); set_error("bg_neq_create: %s", cudaGetErrorString(e2)); return BG_ERR_CUDA; }
  *out = h;
  return BG_OK;
}

void bg_neq_destroy(bg_neq *h) { neq_free(h); }

int bg_neq_dressed_rytov(bg_neq *h, double omega_re, double omega_im, int src, void *out_host) {
  if (!h || !out_host || src < 0 || src >= (int)h->g->objs.size() || omega_re == 0.0) {
    set_error("bg_neq_dressed_rytov: bad arguments");
    return BG_ERR_ARG;
  }
  int st = neq_prepare(h, omega_re, omega_im);
  if (!st) st = neq_dr(h, src);
  if (!st) {
    cudaError_t e = cudaMemcpyAsync(out_host, h->M1, sizeof(z) * (size_t)h->N * h->N, cudaMemcpyDeviceToHost, stream());
    if (e != cudaSuccess) { set_error("D2H: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
  }
  cudaError_t e2 = cudaStreamSynchronize(stream());
  if (!st && e2 != cudaSuccess) { set_error("bg_neq_dressed_rytov: %s", cudaGetErrorString(e2)); st = BG_ERR_CUDA; }
  return st;
}

int bg_neq_flux(bg_neq *h, double omega_re, double omega_im, double *flux) {
  if (!h || !flux || omega_re == 0.0) { set_error("bg_neq_flux: bad arguments"); return BG_ERR_ARG; }
  int NO = (int)h->g->objs.size();
  int st = neq_prepare(h, omega_re, omega_im);
  for (int s = 0; s < NO && !st; s++) {
    if ((st = neq_dr(h, s))) break;
    st = pft_emt_dr(h->g, omega_re, omega_im, h->M1, h->N, flux + (size_t)s * NO * 8);
  }
  cudaError_t e2 = cudaStreamSynchronize(stream());
  if (!st && e2 != cudaSuccess) { set_error("bg_neq_flux: %s", cudaGetErrorString(e2)); st = BG_ERR_CUDA; }
  return st;
}

int bg_pft_dr_device(bg_geometry *g, double omega_re, double omega_im, const void *DR_dev, int ld, double *out) {
  if (!g || !DR_dev || !out || ld < g->N || omega_re == 0.0) { set_error("bg_pft_dr_device: bad arguments"); return BG_ERR_ARG; }
  int st = upload_geometry(g);
  if (!st) st = pft_emt_dr(g, omega_re, omega_im, DR_dev, (size_t)ld, out);
  cudaError_t e2 = cudaStreamSynchronize(stream());
  if (!st && e2 != cudaSuccess) { set_error("bg_pft_dr_device: %s", cudaGetErrorString(e2)); st = BG_ERR_CUDA; }
  return st;
}

}  // extern "C"
