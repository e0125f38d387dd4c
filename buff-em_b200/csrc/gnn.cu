// Learned form, network side: a graph network over the near-field graph of
// the SWG basis functions (nodes = basis functions, edges = pairs sharing a
// vertex, self pairs included) that predicts the entries of a sparse
// approximate inverse M on that pattern, used as the right preconditioner of
// GMRES (gmres.cu).
//
//   node features f_i (8) and edge features g_e (8) from the assembled
//   matrix (ratios to the diagonal) and the geometry;
//   h^0 = relu(W0 f + b0)                                           (width 64)
//   3 x [ z_e = Wmh h_{j(e)} + Wme g_e + bm         (Wmh h computed per node)
//         agg_i = mean_{e in row i} relu(z_e)
//         h_i <- h_i + relu(Wuh h_i + Wua agg_i + bu) ]
//   edge readout: y_e = relu(Wri h_i + Wrj h_j + Wrg g_e + br)       (64)
//                 o_e = Wo y_e + bo                                 (4)
//                 c = GNN_CMAX (tanh(o0) + i tanh(o1))
//                 s = smax (tanh(o2) + i tanh(o3) / 2)
//   m_ij = [delta_ij + c - [i != j] s A_ij / A_ii] / A_jj
// With s = 1 and c = 0 the off-diagonal term would be the first-order
// Neumann approximation of A^{-1} around its diagonal.  Written D M = I - K
// (D = diag A), M is singular where K has an eigenvalue 1, and a preconditioner
// close to that makes GMRES stall on a few modes that no averaged objective
// sees.  For a constant coefficient K = s K1, K1 the scaled near-field
// off-diagonal part (K1_ij = A_ij / A_jj on the pattern), whose dominant
// eigenvalue is real and positive on these matrices (about 2.2 at N = 8k, 2.6
// at N = 57k); GMRES stalled exactly when s crossed 1 / rho(K1).  So a power
// iteration estimates rho(K1) for the matrix at hand and the coefficient is
// bounded by smax = GNN_SREL / max(GNN_SREL, rho(K1)), with the diagonal
// correction c kept small.  Wo and bo start at zero, so the untrained network
// is the Jacobi (diagonal) inverse.
//
// Training objective (per matrix; p probes z and a right-hand side b with its
// LU solution x):
//   L = |A M Z - Z|_F^2 / (N p) + lambda |M b - x|^2 / |x|^2
// The probes are random, or random vectors pushed k times through the Jacobi
// error map z <- z - A D^{-1} z and rescaled to |z|^2 = 2N: those concentrate
// on the modes where the off-diagonal part dominates, which a Frobenius
// objective over random probes barely sees but which decide how many GMRES
// steps the preconditioned system takes.
// The parameters descend log L (gradient dL / L), which weighs matrices of
// very different conditioning alike.  G = 2 dL/dconj(M) on the pattern,
// hand-written backward kernels, Adam with global gradient-norm clipping.
// FP32 in the network; products with A in FP64.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "internal.h"

namespace bg {

#define GW 64          // width
#define GF 8           // node features
#define GE 8           // edge features
#define GL 3           // message-passing layers
#define GO 4           // outputs per edge
#define GNN_MAXP 16    // probes per training step
#define GNN_CMAX 0.1f  // bound of the diagonal-term correction c
#define GNN_SREL 0.7   // |Re s| < GNN_SREL / rho(K1)
#define GNN_POWER_ITERS 16

// parameter layout (floats); matrices row-major (out x in)
struct GnnLayout {
  int W0, b0, Wmh[GL], Wme[GL], bm[GL], Wuh[GL], Wua[GL], bu[GL], Wri, Wrj, Wrg, br, Wo, bo, total;
  GnnLayout() {
    int o = 0;
    W0 = o; o += GW * GF;
    b0 = o; o += GW;
    for (int l = 0; l < GL; l++) {
      Wmh[l] = o; o += GW * GW;
      Wme[l] = o; o += GW * GE;
      bm[l] = o; o += GW;
      Wuh[l] = o; o += GW * GW;
      Wua[l] = o; o += GW * GW;
      bu[l] = o; o += GW;
    }
    Wri = o; o += GW * GW;
    Wrj = o; o += GW * GW;
    Wrg = o; o += GW * GE;
    br = o; o += GW;
    Wo = o; o += GO * GW;
    bo = o; o += GO;
    total = o;
  }
};
static const GnnLayout LAY;

struct z2g { double r, i; };

__device__ __forceinline__ z2g zmul(z2g a, z2g b) { return z2g{a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r}; }
__device__ __forceinline__ z2g zconj(z2g a) { return z2g{a.r, -a.i}; }
__device__ __forceinline__ z2g zdiv(z2g a, z2g b) {
  double d = b.r * b.r + b.i * b.i;
  return z2g{(a.r * b.r + a.i * b.i) / d, (a.i * b.r - a.r * b.i) / d};
}

// ------------------------------------------------------------------ features
// One thread per row i.  A column-major: A_ij at A[j * lda + i].
// node: 1, Re/Im(A_ii)/|A_ii|, omega h, area/h^2, radius/h, degree/100, log10|A_ii|/10
// edge: Re/Im(A_ij/A_ii), Re/Im(A_ji/A_jj), distance of face centroids / h,
//       common vertices / 5, [i == j], |A_ij/A_ii|
__global__ void k_gnn_features(int N, const int *rowptr, const int *col, const z2g *A, size_t lda, DevGeom g,
                               double omega, double h, float *F, float *Ef, z2g *ratio, z2g *dinv) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  z2g a = A[(size_t)i * lda + i];
  double am = sqrt(a.r * a.r + a.i * a.i);
  dinv[i] = zdiv(z2g{1.0, 0.0}, a);
  float *f = F + (size_t)i * GF;
  int deg = rowptr[i + 1] - rowptr[i];
  f[0] = 1.f;
  f[1] = (float)(a.r / am);
  f[2] = (float)(a.i / am);
  f[3] = (float)(omega * h);
  f[4] = (float)(g.bfArea[i] / (h * h));
  f[5] = (float)(g.bfRadius[i] / h);
  f[6] = (float)(deg / 100.0);
  f[7] = (float)(0.1 * log10(am + 1e-300));
  int4 vi = g.bfV[i];
  int2 qi = g.bfQ[i];
  int Vi[5] = {qi.x, vi.x, vi.y, vi.z, qi.y};
  double ci[3] = {0, 0, 0};
  for (int k = 1; k < 4; k++)
    for (int c = 0; c < 3; c++) ci[c] += g.V4[4 * Vi[k] + c] / 3.0;
  for (int e = rowptr[i]; e < rowptr[i + 1]; e++) {
    int j = col[e];
    z2g r = zdiv(A[(size_t)j * lda + i], a);
    z2g rt = zdiv(A[(size_t)i * lda + j], A[(size_t)j * lda + j]);
    int4 vj = g.bfV[j];
    int2 qj = g.bfQ[j];
    int Vj[5] = {qj.x, vj.x, vj.y, vj.z, qj.y};
    int ncv = 0;
    for (int p = 0; p < 5; p++)
      for (int q = 0; q < 5; q++) ncv += Vi[p] == Vj[q];
    double cj[3] = {0, 0, 0};
    for (int k = 1; k < 4; k++)
      for (int c = 0; c < 3; c++) cj[c] += g.V4[4 * Vj[k] + c] / 3.0;
    double dist = sqrt((ci[0] - cj[0]) * (ci[0] - cj[0]) + (ci[1] - cj[1]) * (ci[1] - cj[1]) +
                       (ci[2] - cj[2]) * (ci[2] - cj[2]));
    float *ge = Ef + (size_t)e * GE;
    ge[0] = (float)r.r;
    ge[1] = (float)r.i;
    ge[2] = (float)rt.r;
    ge[3] = (float)rt.i;
    ge[4] = (float)(dist / h);
    ge[5] = (float)(ncv / 5.0);
    ge[6] = (i == j) ? 1.f : 0.f;
    ge[7] = (float)sqrt(r.r * r.r + r.i * r.i);
    ratio[e] = r;
  }
}

// ------------------------------------------------------------------ node maps
// Y[n][o] (+)= sum_k X[n][k] W[o][k] (+ bias[o]); one block per node
__global__ void k_gnn_linear(int N, int in, int out, const float *X, int ldx, const float *W, const float *bias,
                             float *Y, int ldy, int accumulate) {
  int n = blockIdx.x;
  int o = threadIdx.x;
  if (n >= N || o >= out) return;
  const float *x = X + (size_t)n * ldx;
  const float *w = W + (size_t)o * in;
  float s = bias ? bias[o] : 0.f;
  for (int k = 0; k < in; k++) s += x[k] * w[k];
  float *y = Y + (size_t)n * ldy + o;
  *y = accumulate ? *y + s : s;
}

__global__ void k_gnn_relu(int n, const float *Z, float *H) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) H[i] = fmaxf(Z[i], 0.f);
}

// messages and mean aggregation over row i: Zm[e] = P[j(e)] + Wme g_e + bm
__global__ void k_gnn_msg(int N, const int *rowptr, const int *col, const float *P, const float *Ef,
                          const float *Wme, const float *bm, float *Zm, float *agg) {
  int i = blockIdx.x, o = threadIdx.x;
  if (i >= N) return;
  float w[GE];
  for (int k = 0; k < GE; k++) w[k] = Wme[o * GE + k];
  float b = bm[o], s = 0.f;
  int e0 = rowptr[i], e1 = rowptr[i + 1];
  for (int e = e0; e < e1; e++) {
    const float *ge = Ef + (size_t)e * GE;
    float z = P[(size_t)col[e] * GW + o] + b;
    for (int k = 0; k < GE; k++) z += w[k] * ge[k];
    if (Zm) Zm[(size_t)e * GW + o] = z;
    s += fmaxf(z, 0.f);
  }
  agg[(size_t)i * GW + o] = s / fmaxf(1.f, (float)(e1 - e0));
}

// H_next = H + relu(U)
__global__ void k_gnn_residual(int n, const float *H, const float *U, float *Hn) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) Hn[i] = H[i] + fmaxf(U[i], 0.f);
}

// edge readout, one warp per row; lane owns hidden units lane and lane + 32
__global__ void k_gnn_readout(int N, const int *rowptr, const int *col, const float *Pr, const float *Qr,
                              const float *Ef, const float *Wrg, const float *br, const float *Wo, const float *bo,
                              const z2g *ratio, const z2g *dinv, float smax, float *Zr, float *Oe, z2g *Mval) {
  int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  int lane = threadIdx.x & 31;
  if (i >= N) return;
  float wg[2][GE], wo[2][GO], bb[2], pi[2];
  for (int t = 0; t < 2; t++) {
    int o = lane + 32 * t;
    for (int k = 0; k < GE; k++) wg[t][k] = Wrg[o * GE + k];
    for (int k = 0; k < GO; k++) wo[t][k] = Wo[k * GW + o];
    bb[t] = br[o];
    pi[t] = Pr[(size_t)i * GW + o];
  }
  for (int e = rowptr[i]; e < rowptr[i + 1]; e++) {
    int j = col[e];
    const float *ge = Ef + (size_t)e * GE;
    float g[GE];
    for (int k = 0; k < GE; k++) g[k] = ge[k];
    float out[GO] = {0, 0, 0, 0};
    for (int t = 0; t < 2; t++) {
      int o = lane + 32 * t;
      float z = pi[t] + Qr[(size_t)j * GW + o] + bb[t];
      for (int k = 0; k < GE; k++) z += wg[t][k] * g[k];
      if (Zr) Zr[(size_t)e * GW + o] = z;
      float y = fmaxf(z, 0.f);
      for (int k = 0; k < GO; k++) out[k] += wo[t][k] * y;
    }
    for (int k = 0; k < GO; k++)
      for (int s = 16; s > 0; s >>= 1) out[k] += __shfl_xor_sync(0xffffffffu, out[k], s);
    if (lane == 0) {
      float o[GO];
      for (int k = 0; k < GO; k++) o[k] = out[k] + bo[k];
      if (Oe)
        for (int k = 0; k < GO; k++) Oe[(size_t)e * GO + k] = o[k];
      z2g c{(i == j ? 1.0 : 0.0) + GNN_CMAX * tanhf(o[0]), (double)(GNN_CMAX * tanhf(o[1]))};
      if (i != j) {
        z2g sr = zmul(z2g{(double)(smax * tanhf(o[2])), (double)(0.5f * smax * tanhf(o[3]))}, ratio[e]);
        c.r -= sr.r;
        c.i -= sr.i;
      }
      Mval[e] = zmul(c, dinv[j]);
    }
  }
}

// W[:, q] = K1 V[:, q], (K1)_ij = A_ij / A_jj = r_e dinv_j / dinv_i off the diagonal
__global__ void k_gnn_k1mv(int N, const int *rowptr, const int *col, const z2g *ratio, const z2g *dinv,
                           const z2g *V, int nv, z2g *W) {
  // eight lanes per row (its entries are contiguous), all nv <= 4 vectors per
  // read of the row; lane partial sums combined by a fixed butterfly
  int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 3, sub = threadIdx.x & 7;
  z2g s[4] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
  if (i < N) {
    int e1 = rowptr[i + 1];
    for (int e = rowptr[i] + sub; e < e1; e += 8) {
      int j = col[e];
      if (j == i) continue;
      z2g rj = zmul(ratio[e], dinv[j]);
#pragma unroll
      for (int q = 0; q < 4; q++)
        if (q < nv) {
          z2g t = zmul(rj, V[(size_t)q * N + j]);
          s[q].r += t.r;
          s[q].i += t.i;
        }
    }
  }
#pragma unroll
  for (int o = 4; o > 0; o >>= 1)
#pragma unroll
    for (int q = 0; q < 4; q++) {
      s[q].r += __shfl_xor_sync(0xffffffffu, s[q].r, o);
      s[q].i += __shfl_xor_sync(0xffffffffu, s[q].i, o);
    }
  if (i < N && sub == 0) {
    z2g ai = zdiv(z2g{1.0, 0.0}, dinv[i]);
    for (int q = 0; q < nv; q++) W[(size_t)q * N + i] = zmul(ai, s[q]);
  }
}

// squared norms of nv columns (one block per column, fixed reduction order)
__global__ void k_gnn_colnorm2(int N, const z2g *V, double *out) {
  const z2g *v = V + (size_t)blockIdx.x * N;
  __shared__ double red[32];
  double s = 0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) s += v[i].r * v[i].r + v[i].i * v[i].i;
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) t += red[k];
    out[blockIdx.x] = t;
  }
}

__global__ void k_gnn_scale_cols(int N, int nv, const double *f, z2g *V) {
  size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= (size_t)N * nv) return;
  double s = f[t / N];
  V[t] = z2g{V[t].r * s, V[t].i * s};
}

// ------------------------------------------------------------------ backward
// output gradients per edge from G = 2 dL/dconj(m):
// t = conj(G) d_j, u = conj(G) r_e d_j ; d(c, s) = (Re t, -Im t, -Re u, Im u)
// (u terms off-diagonal only), then through the bounded tanh maps of o
__global__ void k_gnn_dout(int N, const int *rowptr, const int *col, const z2g *G, double gscale, const z2g *ratio,
                           const z2g *dinv, float smax, const float *Oe, float *dO) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  for (int e = rowptr[i]; e < rowptr[i + 1]; e++) {
    int j = col[e];
    z2g t = zmul(zconj(G[e]), dinv[j]);
    t.r *= gscale;
    t.i *= gscale;
    float *d = dO + (size_t)e * GO;
    d[0] = (float)t.r;
    d[1] = (float)(-t.i);
    if (i != j) {
      z2g u = zmul(t, ratio[e]);
      d[2] = (float)(-u.r);
      d[3] = (float)u.i;
    } else {
      d[2] = d[3] = 0.f;
    }
    for (int k = 0; k < GO; k++) {
      float th = tanhf(Oe[(size_t)e * GO + k]);
      d[k] *= (k < 2 ? GNN_CMAX : (k == 2 ? smax : 0.5f * smax)) * (1.f - th * th);
    }
  }
}

// dZr[e][o] = (sum_k Wo[k][o] dO[e][k]) [Zr > 0]; one block per row, thread per o
__global__ void k_gnn_readout_back(int N, const int *rowptr, const float *Zr, const float *dO, const float *Wo,
                                   float *dZr) {
  int i = blockIdx.x, o = threadIdx.x;
  if (i >= N) return;
  float w[GO];
  for (int k = 0; k < GO; k++) w[k] = Wo[k * GW + o];
  for (int e = rowptr[i]; e < rowptr[i + 1]; e++) {
    float da = 0.f;
    for (int k = 0; k < GO; k++) da += w[k] * dO[(size_t)e * GO + k];
    dZr[(size_t)e * GW + o] = Zr[(size_t)e * GW + o] > 0.f ? da : 0.f;
  }
}

// dWo[k][o] += sum_e dO[e][k] relu(Zr[e][o]); dbo[k] += sum_e dO[e][k] (block o == 0)
__global__ void k_gnn_wo_grad(int E, const float *dO, const float *Zr, float *dWo, float *dbo) {
  int o = blockIdx.x;
  __shared__ float sh[2 * GO];
  if (threadIdx.x < 2 * GO) sh[threadIdx.x] = 0.f;
  __syncthreads();
  float lw[GO] = {0, 0, 0, 0}, lb[GO] = {0, 0, 0, 0};
  for (int e = threadIdx.x; e < E; e += blockDim.x) {
    float y = fmaxf(Zr[(size_t)e * GW + o], 0.f);
    for (int k = 0; k < GO; k++) {
      float d = dO[(size_t)e * GO + k];
      lw[k] += d * y;
      lb[k] += d;
    }
  }
  for (int k = 0; k < GO; k++) {
    atomicAdd(&sh[k], lw[k]);
    atomicAdd(&sh[GO + k], lb[k]);
  }
  __syncthreads();
  if (threadIdx.x < GO) {
    dWo[threadIdx.x * GW + o] += sh[threadIdx.x];
    if (o == 0) dbo[threadIdx.x] += sh[GO + threadIdx.x];
  }
}

// weight gradient of a node map: dW[o][k] += sum_n dY[n][o] X[n][k]; db[o] += sum_n dY[n][o]
__global__ void k_gnn_wgrad(int N, int in, const float *dY, int lddy, const float *X, int ldx, float *dW, float *db) {
  int o = blockIdx.x;
  __shared__ float sh[GW + 1];
  for (int k = threadIdx.x; k <= in; k += blockDim.x) sh[k] = 0.f;
  __syncthreads();
  float loc[GW + 1];
  for (int k = 0; k <= in; k++) loc[k] = 0.f;
  for (int n = threadIdx.x; n < N; n += blockDim.x) {
    float g = dY[(size_t)n * lddy + o];
    if (g == 0.f) continue;
    const float *x = X + (size_t)n * ldx;
    for (int k = 0; k < in; k++) loc[k] += g * x[k];
    loc[in] += g;
  }
  for (int k = 0; k <= in; k++) atomicAdd(&sh[k], loc[k]);
  __syncthreads();
  for (int k = threadIdx.x; k < in; k += blockDim.x) dW[(size_t)o * in + k] += sh[k];
  if (threadIdx.x == 0 && db) db[o] += sh[in];
}

// dX[n][k] (+)= sum_o dY[n][o] W[o][k]
__global__ void k_gnn_dx(int N, int in, int out, const float *dY, int lddy, const float *W, float *dX, int lddx,
                         int accumulate) {
  int n = blockIdx.x, k = threadIdx.x;
  if (n >= N || k >= in) return;
  float s = 0.f;
  for (int o = 0; o < out; o++) s += dY[(size_t)n * lddy + o] * W[(size_t)o * in + k];
  float *p = dX + (size_t)n * lddx + k;
  *p = accumulate ? *p + s : s;
}

// message backward: dZm[e] = dagg_i / deg_i [Zm > 0]
__global__ void k_gnn_msg_back(int N, const int *rowptr, const float *Zm, const float *dagg, float *dZm) {
  int i = blockIdx.x, o = threadIdx.x;
  if (i >= N) return;
  int e0 = rowptr[i], e1 = rowptr[i + 1];
  float da = dagg[(size_t)i * GW + o] / fmaxf(1.f, (float)(e1 - e0));
  for (int e = e0; e < e1; e++) dZm[(size_t)e * GW + o] = Zm[(size_t)e * GW + o] > 0.f ? da : 0.f;
}

// dP[j] = sum over edges e with col(e) = j of dZ[e]  (= sum over row j of dZ[etr])
__global__ void k_gnn_col_gather(int N, const int *rowptr, const int *etr, const float *dZ, float *dP) {
  int j = blockIdx.x, o = threadIdx.x;
  if (j >= N) return;
  float s = 0.f;
  for (int e = rowptr[j]; e < rowptr[j + 1]; e++) s += dZ[(size_t)etr[e] * GW + o];
  dP[(size_t)j * GW + o] = s;
}

// dP[i] = sum over row i of dZ[e]
__global__ void k_gnn_row_sum(int N, const int *rowptr, const float *dZ, float *dP) {
  int i = blockIdx.x, o = threadIdx.x;
  if (i >= N) return;
  float s = 0.f;
  for (int e = rowptr[i]; e < rowptr[i + 1]; e++) s += dZ[(size_t)e * GW + o];
  dP[(size_t)i * GW + o] = s;
}

// dW[o][k] += sum_e dZ[e][o] g_e[k]; db[o] += sum_e dZ[e][o]
__global__ void k_gnn_edge_wgrad(int E, const float *dZ, const float *Ef, float *dW, float *db) {
  int o = blockIdx.x;
  __shared__ float sh[GE + 1];
  if (threadIdx.x <= GE) sh[threadIdx.x] = 0.f;
  __syncthreads();
  float loc[GE + 1];
  for (int k = 0; k <= GE; k++) loc[k] = 0.f;
  for (int e = threadIdx.x; e < E; e += blockDim.x) {
    float g = dZ[(size_t)e * GW + o];
    if (g == 0.f) continue;
    for (int k = 0; k < GE; k++) loc[k] += g * Ef[(size_t)e * GE + k];
    loc[GE] += g;
  }
  for (int k = 0; k <= GE; k++) atomicAdd(&sh[k], loc[k]);
  __syncthreads();
  if (threadIdx.x < GE) dW[o * GE + threadIdx.x] += sh[threadIdx.x];
  if (threadIdx.x == GE) db[o] += sh[GE];
}

__global__ void k_gnn_relu_back(int n, const float *Z, const float *dH, float *dZ) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dZ[i] = Z[i] > 0.f ? dH[i] : 0.f;
}

__global__ void k_gnn_sumsq(int n, const float *g, double *out) {
  double s = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += (double)g[i] * g[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

// Adam with the gradient scaled to global norm <= clip
__global__ void k_gnn_adam(int n, float *p, const float *g, float *m, float *v, const double *sumsq, float lr,
                           float b1, float b2, float c1, float c2, float eps, float clip) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double nrm = sqrt(*sumsq);
  float sc = nrm > clip ? (float)(clip / nrm) : 1.f;
  float gi = g[i] * sc;
  float mi = b1 * m[i] + (1 - b1) * gi, vi = b2 * v[i] + (1 - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// ------------------------------------------------------------------ objective
// G_e = scale sum_q S[i,q] conj(Z[j,q]) + scale2 rb_i conj(b_j)
__global__ void k_gnn_sddmm(int N, const int *rowptr, const int *col, const z2g *S, const z2g *Z, int p,
                            double scale, const z2g *rb, const z2g *b, double scale2, z2g *G) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  for (int e = rowptr[i]; e < rowptr[i + 1]; e++) {
    int j = col[e];
    double gr = 0, gi = 0;
    for (int q = 0; q < p; q++) {
      z2g s = S[(size_t)q * N + i], z = Z[(size_t)q * N + j];
      gr += s.r * z.r + s.i * z.i;
      gi += s.i * z.r - s.r * z.i;
    }
    gr *= scale;
    gi *= scale;
    if (rb) {
      z2g r = rb[i], bb = b[j];
      gr += scale2 * (r.r * bb.r + r.i * bb.i);
      gi += scale2 * (r.i * bb.r - r.r * bb.i);
    }
    G[e] = z2g{gr, gi};
  }
}

// S[c, q] = sum_r conj(A[r, c]) R[r, q]: one warp per column c of A
__global__ void k_gnn_ahr(int N, const z2g *A, size_t lda, const z2g *R, int p, z2g *S) {
  int c = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (c >= N) return;
  double sr[GNN_MAXP], si[GNN_MAXP];
  for (int q = 0; q < GNN_MAXP; q++) sr[q] = si[q] = 0.0;
  const z2g *a = A + (size_t)c * lda;
  for (int r = lane; r < N; r += 32) {
    z2g v = a[r];
#pragma unroll
    for (int q = 0; q < GNN_MAXP; q++)
      if (q < p) {
        z2g x = R[(size_t)q * N + r];
        sr[q] += v.r * x.r + v.i * x.i;
        si[q] += v.r * x.i - v.i * x.r;
      }
  }
  for (int q = 0; q < p; q++) {
    double a0 = sr[q], a1 = si[q];
    for (int o = 16; o > 0; o >>= 1) {
      a0 += __shfl_xor_sync(0xffffffffu, a0, o);
      a1 += __shfl_xor_sync(0xffffffffu, a1, o);
    }
    if (lane == 0) S[(size_t)q * N + c] = z2g{a0, a1};
  }
}

// Y = D^{-1} Z row-wise (d: 1/A_jj), p columns of length N
__global__ void k_gnn_rowscale(int N, int p, const z2g *d, const z2g *Z, z2g *Y) {
  size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= (size_t)N * p) return;
  Y[t] = zmul(d[t % N], Z[t]);
}

// Z[:, q] += W[:, q] and rescale the column to squared norm 2N (one block per column)
__global__ void k_gnn_probe_update(int N, const z2g *W, z2g *Z) {
  int q = blockIdx.x;
  z2g *z = Z + (size_t)q * N;
  const z2g *w = W + (size_t)q * N;
  __shared__ double red[32];
  double s = 0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    z2g v{z[i].r + w[i].r, z[i].i + w[i].i};
    z[i] = v;
    s += v.r * v.r + v.i * v.i;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) t += red[k];
    red[0] = t > 0 ? sqrt(2.0 * N / t) : 1.0;
  }
  __syncthreads();
  double f = red[0];
  for (int i = threadIdx.x; i < N; i += blockDim.x) z[i] = z2g{z[i].r * f, z[i].i * f};
}

__global__ void k_gnn_sub(size_t n, const z2g *A, const z2g *B, z2g *C) {   // C = A - B
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) C[i] = z2g{A[i].r - B[i].r, A[i].i - B[i].i};
}

__global__ void k_gnn_spmm(int N, const int *rowptr, const int *col, const z2g *val, const z2g *X, int p, z2g *Y) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int q = blockIdx.y;
  if (i >= N || q >= p) return;
  double sr = 0, si = 0;
  for (int e = rowptr[i]; e < rowptr[i + 1]; e++) {
    z2g m = val[e], x = X[(size_t)q * N + col[e]];
    sr += m.r * x.r - m.i * x.i;
    si += m.r * x.i + m.i * x.r;
  }
  Y[(size_t)q * N + i] = z2g{sr, si};
}

}  // namespace bg

// =============================================================================
// host side
// =============================================================================
struct bg_gnn {
  float *params = nullptr, *grads = nullptr, *m = nullptr, *v = nullptr;
  double *sumsq = nullptr;
  int step = 0;
};

namespace bg {

// per-call activations (the graph itself is cached in the geometry)
struct GnnBufs {
  int N = 0, E = 0;
  double rho_ref = 0;   // estimate of rho(K1)
  float smax = 0;       // bound of the Neumann coefficient
  const int *rowptr = nullptr, *col = nullptr, *etr = nullptr;
  float *F = nullptr, *Ef = nullptr;
  z2g *ratio = nullptr, *dinv = nullptr;
  float *Z0 = nullptr, *H[GL + 1] = {}, *P = nullptr, *Q = nullptr, *agg[GL] = {}, *U[GL] = {};
  float *Zm[GL] = {}, *Zr = nullptr, *Oe = nullptr;
  // backward
  float *dH = nullptr, *dU = nullptr, *dagg = nullptr, *dZ = nullptr, *dP = nullptr, *dQ = nullptr, *dO = nullptr;
  std::vector<void *> owned;
};

static void bufs_free(GnnBufs &B) {
  for (void *p : B.owned) cudaFree(p);
  B = GnnBufs();
}

template <typename T>
static int balloc(GnnBufs &B, T **p, size_t count) {
  void *q = nullptr;
  cudaError_t e = cudaMalloc(&q, sizeof(T) * std::max<size_t>(count, 1));
  if (e != cudaSuccess) {
    set_error("graph network buffers (%zu bytes): %s", sizeof(T) * count, cudaGetErrorString(e));
    return BG_ERR_NOMEM;
  }
  B.owned.push_back(q);
  *p = (T *)q;
  return BG_OK;
}

// Near-field graph from the geometry's near pairs (same object, >= 1 common
// vertex, a <= b): both directions plus self pairs, sorted columns, reverse map.
static int ensure_graph(bg_geometry *g) {
  if (g->graph.rowptr) return BG_OK;
  int st = bg_geometry_precompute(g);
  if (st) return st;
  int N = g->N, np = g->near.npairs;
  std::vector<int2> pairs(np);
  if (np) BG_CUDA_TRY(cudaMemcpy(pairs.data(), g->near.pairs, sizeof(int2) * np, cudaMemcpyDeviceToHost));
  std::vector<int> deg(N, 1);   // self pair
  for (auto &p : pairs)
    if (p.x != p.y) { deg[p.x]++; deg[p.y]++; }
  std::vector<int> rowptr(N + 1, 0);
  for (int i = 0; i < N; i++) rowptr[i + 1] = rowptr[i] + deg[i];
  int E = rowptr[N];
  std::vector<int> col(E), fill(rowptr.begin(), rowptr.end() - 1);
  for (int i = 0; i < N; i++) col[fill[i]++] = i;
  for (auto &p : pairs)
    if (p.x != p.y) { col[fill[p.x]++] = p.y; col[fill[p.y]++] = p.x; }
  for (int i = 0; i < N; i++) {
    std::sort(col.begin() + rowptr[i], col.begin() + rowptr[i + 1]);
    if (std::adjacent_find(col.begin() + rowptr[i], col.begin() + rowptr[i + 1]) != col.begin() + rowptr[i + 1]) {
      set_error("near graph: duplicate basis-function pair");
      return BG_ERR_STATE;
    }
  }
  std::vector<int> etr(E);
  for (int i = 0; i < N; i++)
    for (int e = rowptr[i]; e < rowptr[i + 1]; e++) {
      int j = col[e];
      auto it = std::lower_bound(col.begin() + rowptr[j], col.begin() + rowptr[j + 1], i);
      if (it == col.begin() + rowptr[j + 1] || *it != i) { set_error("near graph: pattern not symmetric"); return BG_ERR_STATE; }
      etr[e] = (int)(it - col.begin());
    }
  double hsum = 0;
  for (auto &o : g->objs)
    for (int a = 0; a < o.nif; a++) hsum += o.F[a].radius;
  NearGraph G;
  G.E = E;
  G.h = hsum / std::max(1, N);
  BG_CUDA_TRY(cudaMalloc(&G.rowptr, sizeof(int) * (N + 1)));
  BG_CUDA_TRY(cudaMalloc(&G.col, sizeof(int) * E));
  BG_CUDA_TRY(cudaMalloc(&G.etr, sizeof(int) * E));
  BG_CUDA_TRY(cudaMemcpy(G.rowptr, rowptr.data(), sizeof(int) * (N + 1), cudaMemcpyHostToDevice));
  BG_CUDA_TRY(cudaMemcpy(G.col, col.data(), sizeof(int) * E, cudaMemcpyHostToDevice));
  BG_CUDA_TRY(cudaMemcpy(G.etr, etr.data(), sizeof(int) * E, cudaMemcpyHostToDevice));
  g->graph = G;
  return BG_OK;
}

static int bound_coefficient(GnnBufs &B);

static int bufs_alloc(bg_geometry *g, bool train, GnnBufs &B) {
  int st = ensure_graph(g);
  if (st) return st;
  int N = g->N, E = g->graph.E;
  B.N = N;
  B.E = E;
  B.rowptr = g->graph.rowptr;
  B.col = g->graph.col;
  B.etr = g->graph.etr;
  size_t n64 = (size_t)N * GW, e64 = (size_t)E * GW;
  if ((st = balloc(B, &B.F, (size_t)N * GF)) || (st = balloc(B, &B.Ef, (size_t)E * GE)) ||
      (st = balloc(B, &B.ratio, (size_t)E)) || (st = balloc(B, &B.dinv, (size_t)N)) ||
      (st = balloc(B, &B.Z0, n64)) || (st = balloc(B, &B.P, n64)) || (st = balloc(B, &B.Q, n64)))
    return st;
  for (int l = 0; l <= GL; l++)
    if ((st = balloc(B, &B.H[l], n64))) return st;
  for (int l = 0; l < GL; l++)
    if ((st = balloc(B, &B.agg[l], n64)) || (st = balloc(B, &B.U[l], n64))) return st;
  if (train) {
    for (int l = 0; l < GL; l++)
      if ((st = balloc(B, &B.Zm[l], e64))) return st;
    if ((st = balloc(B, &B.Zr, e64)) || (st = balloc(B, &B.dZ, e64)) || (st = balloc(B, &B.dO, (size_t)E * GO)) ||
        (st = balloc(B, &B.Oe, (size_t)E * GO)) ||
        (st = balloc(B, &B.dH, n64)) || (st = balloc(B, &B.dU, n64)) || (st = balloc(B, &B.dagg, n64)) ||
        (st = balloc(B, &B.dP, n64)) || (st = balloc(B, &B.dQ, n64)))
      return st;
  }
  return BG_OK;
}

static int bound_coefficient(GnnBufs &B);

// per-call part: features of (A, omega) and the coefficient bound
static int bufs_compute(bg_geometry *g, bg_matrix *A, double omega, GnnBufs &B) {
  int N = B.N;
  k_gnn_features<<<(N + 127) / 128, 128, 0, stream()>>>(N, B.rowptr, B.col, (const z2g *)A->d, A->ld, g->dev, omega,
                                                        g->graph.h, B.F, B.Ef, B.ratio, B.dinv);
  BG_LAUNCHED();
  return bound_coefficient(B);
}

static int bufs_init(bg_geometry *g, bg_matrix *A, double omega, bool train, GnnBufs &B) {
  int st = bufs_alloc(g, train, B);
  return st ? st : bufs_compute(g, A, omega, B);
}

// The inference buffers (about 15 node-sized and 2 edge-sized arrays) are kept
// with the geometry and reused by every learned preconditioner built for it,
// so a frequency step allocates no graph-network memory.
static int inference_bufs(bg_geometry *g, GnnBufs *&B) {
  int st = ensure_graph(g);
  if (st) return st;
  GnnBufs *c = static_cast<GnnBufs *>(g->gnn_cache);
  if (c && (c->N != g->N || c->E != g->graph.E)) {
    bufs_free(*c);
    delete c;
    c = nullptr;
    g->gnn_cache = nullptr;
  }
  if (!c) {
    c = new GnnBufs();
    if ((st = bufs_alloc(g, false, *c))) {
      bufs_free(*c);
      delete c;
      return st;
    }
    g->gnn_cache = c;
  }
  B = c;
  return BG_OK;
}

void gnn_cache_free(bg_geometry *g) {
  GnnBufs *c = static_cast<GnnBufs *>(g->gnn_cache);
  if (c) {
    bufs_free(*c);
    delete c;
  }
  g->gnn_cache = nullptr;
}

// Power iteration (four seeded vectors in lockstep, GNN_POWER_ITERS steps)
// for the spectral radius of K1; sets the coefficient bound smax.
static int bound_coefficient(GnnBufs &B) {
  const int nv = 4;
  int N = B.N;
  size_t nn = (size_t)N * nv;
  char *w = nullptr;
  BG_CUDA_TRY(cudaMallocAsync((void **)&w, sizeof(z2g) * 2 * nn + sizeof(double) * 2 * nv, stream()));
  z2g *V = (z2g *)w, *W = V + nn;
  double *nrm = (double *)(W + nn), *fac = nrm + nv;
  std::vector<z2g> h(nn);
  uint64_t s = 0x9e3779b97f4a7c15ull;
  for (auto &v : h) {
    s = s * 6364136223846793005ull + 1442695040888963407ull;
    double a = (double)(s >> 11) / 9007199254740992.0 - 0.5;
    s = s * 6364136223846793005ull + 1442695040888963407ull;
    double b = (double)(s >> 11) / 9007199254740992.0 - 0.5;
    v = z2g{a, b};
  }
  int st = BG_OK;
  cudaError_t e = cudaMemcpyAsync(V, h.data(), sizeof(z2g) * nn, cudaMemcpyHostToDevice, stream());
  double rho = 0, hn[nv];
  for (int it = 0; e == cudaSuccess && it <= GNN_POWER_ITERS; it++) {
    // normalise V, then W = K V; the norm of K v for unit v is the estimate
    k_gnn_colnorm2<<<nv, 256, 0, stream()>>>(N, V, nrm);
    if ((e = cudaMemcpyAsync(hn, nrm, sizeof(double) * nv, cudaMemcpyDeviceToHost, stream())) != cudaSuccess) break;
    if ((e = cudaStreamSynchronize(stream())) != cudaSuccess) break;
    g_launches++;
    if (it > 0) {
      rho = 0;
      for (int q = 0; q < nv; q++) rho = std::max(rho, std::sqrt(hn[q]));
      if (it == GNN_POWER_ITERS) break;
    }
    double f[nv];
    for (int q = 0; q < nv; q++) f[q] = hn[q] > 0 ? 1.0 / std::sqrt(hn[q]) : 0.0;
    if ((e = cudaMemcpyAsync(fac, f, sizeof(double) * nv, cudaMemcpyHostToDevice, stream())) != cudaSuccess) break;
    k_gnn_scale_cols<<<(nn + 255) / 256, 256, 0, stream()>>>(N, nv, fac, V);
    k_gnn_k1mv<<<(unsigned)(((size_t)N * 8 + 255) / 256), 256, 0, stream()>>>(N, B.rowptr, B.col, B.ratio, B.dinv, V,
                                                                                nv, W);
    g_launches += 2;
    std::swap(V, W);
  }
  if (e != cudaSuccess) { set_error("near-field spectral estimate: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
  if (!st && !std::isfinite(rho)) { set_error("near-field spectral estimate: non-finite"); st = BG_ERR_NUMERIC; }
  cudaFreeAsync(w, stream());
  B.rho_ref = rho;
  B.smax = (float)(GNN_SREL / std::max(rho, GNN_SREL));
  return st;
}

static int forward(const bg_gnn *net, GnnBufs &B, z2g *Mval) {
  const float *W = net->params;
  int N = B.N, n64 = N * GW, nb = (n64 + 255) / 256;
  k_gnn_linear<<<N, GW, 0, stream()>>>(N, GF, GW, B.F, GF, W + LAY.W0, W + LAY.b0, B.Z0, GW, 0);
  BG_LAUNCHED();
  k_gnn_relu<<<nb, 256, 0, stream()>>>(n64, B.Z0, B.H[0]);
  BG_LAUNCHED();
  for (int l = 0; l < GL; l++) {
    k_gnn_linear<<<N, GW, 0, stream()>>>(N, GW, GW, B.H[l], GW, W + LAY.Wmh[l], nullptr, B.P, GW, 0);
    BG_LAUNCHED();
    k_gnn_msg<<<N, GW, 0, stream()>>>(N, B.rowptr, B.col, B.P, B.Ef, W + LAY.Wme[l], W + LAY.bm[l], B.Zm[l],
                                      B.agg[l]);
    BG_LAUNCHED();
    k_gnn_linear<<<N, GW, 0, stream()>>>(N, GW, GW, B.H[l], GW, W + LAY.Wuh[l], W + LAY.bu[l], B.U[l], GW, 0);
    BG_LAUNCHED();
    k_gnn_linear<<<N, GW, 0, stream()>>>(N, GW, GW, B.agg[l], GW, W + LAY.Wua[l], nullptr, B.U[l], GW, 1);
    BG_LAUNCHED();
    k_gnn_residual<<<nb, 256, 0, stream()>>>(n64, B.H[l], B.U[l], B.H[l + 1]);
    BG_LAUNCHED();
  }
  k_gnn_linear<<<N, GW, 0, stream()>>>(N, GW, GW, B.H[GL], GW, W + LAY.Wri, nullptr, B.P, GW, 0);
  BG_LAUNCHED();
  k_gnn_linear<<<N, GW, 0, stream()>>>(N, GW, GW, B.H[GL], GW, W + LAY.Wrj, nullptr, B.Q, GW, 0);
  BG_LAUNCHED();
  k_gnn_readout<<<(N + 3) / 4, 128, 0, stream()>>>(N, B.rowptr, B.col, B.P, B.Q, B.Ef, W + LAY.Wrg, W + LAY.br,
                                                   W + LAY.Wo, W + LAY.bo, B.ratio, B.dinv, B.smax, B.Zr, B.Oe,
                                                   Mval);
  BG_LAUNCHED();
  return BG_OK;
}

// backward from gscale * G, G = 2 dL/dconj(m); accumulates into net->grads (zeroed by the caller)
static int backward(bg_gnn *net, GnnBufs &B, const z2g *G, double gscale) {
  const float *W = net->params;
  float *dW = net->grads;
  int N = B.N, E = B.E, n64 = N * GW, nb = (n64 + 255) / 256;
  k_gnn_dout<<<(N + 127) / 128, 128, 0, stream()>>>(N, B.rowptr, B.col, G, gscale, B.ratio, B.dinv, B.smax, B.Oe,
                                                    B.dO);
  BG_LAUNCHED();
  k_gnn_wo_grad<<<GW, 256, 0, stream()>>>(E, B.dO, B.Zr, dW + LAY.Wo, dW + LAY.bo);
  BG_LAUNCHED();
  k_gnn_readout_back<<<N, GW, 0, stream()>>>(N, B.rowptr, B.Zr, B.dO, W + LAY.Wo, B.dZ);
  BG_LAUNCHED();
  k_gnn_edge_wgrad<<<GW, 256, 0, stream()>>>(E, B.dZ, B.Ef, dW + LAY.Wrg, dW + LAY.br);
  BG_LAUNCHED();
  k_gnn_row_sum<<<N, GW, 0, stream()>>>(N, B.rowptr, B.dZ, B.dP);
  BG_LAUNCHED();
  k_gnn_col_gather<<<N, GW, 0, stream()>>>(N, B.rowptr, B.etr, B.dZ, B.dQ);
  BG_LAUNCHED();
  k_gnn_wgrad<<<GW, 128, 0, stream()>>>(N, GW, B.dP, GW, B.H[GL], GW, dW + LAY.Wri, nullptr);
  BG_LAUNCHED();
  k_gnn_wgrad<<<GW, 128, 0, stream()>>>(N, GW, B.dQ, GW, B.H[GL], GW, dW + LAY.Wrj, nullptr);
  BG_LAUNCHED();
  k_gnn_dx<<<N, GW, 0, stream()>>>(N, GW, GW, B.dP, GW, W + LAY.Wri, B.dH, GW, 0);
  BG_LAUNCHED();
  k_gnn_dx<<<N, GW, 0, stream()>>>(N, GW, GW, B.dQ, GW, W + LAY.Wrj, B.dH, GW, 1);
  BG_LAUNCHED();
  for (int l = GL - 1; l >= 0; l--) {
    // H_{l+1} = H_l + relu(U_l): dU = dH [U > 0]; dH_l = dH + Wuh^T dU + Wmh^T dP; dagg = Wua^T dU
    k_gnn_relu_back<<<nb, 256, 0, stream()>>>(n64, B.U[l], B.dH, B.dU);
    BG_LAUNCHED();
    k_gnn_wgrad<<<GW, 128, 0, stream()>>>(N, GW, B.dU, GW, B.H[l], GW, dW + LAY.Wuh[l], dW + LAY.bu[l]);
    BG_LAUNCHED();
    k_gnn_wgrad<<<GW, 128, 0, stream()>>>(N, GW, B.dU, GW, B.agg[l], GW, dW + LAY.Wua[l], nullptr);
    BG_LAUNCHED();
    k_gnn_dx<<<N, GW, 0, stream()>>>(N, GW, GW, B.dU, GW, W + LAY.Wuh[l], B.dH, GW, 1);
    BG_LAUNCHED();
    k_gnn_dx<<<N, GW, 0, stream()>>>(N, GW, GW, B.dU, GW, W + LAY.Wua[l], B.dagg, GW, 0);
    BG_LAUNCHED();
    k_gnn_msg_back<<<N, GW, 0, stream()>>>(N, B.rowptr, B.Zm[l], B.dagg, B.dZ);
    BG_LAUNCHED();
    k_gnn_col_gather<<<N, GW, 0, stream()>>>(N, B.rowptr, B.etr, B.dZ, B.dP);
    BG_LAUNCHED();
    k_gnn_edge_wgrad<<<GW, 256, 0, stream()>>>(E, B.dZ, B.Ef, dW + LAY.Wme[l], dW + LAY.bm[l]);
    BG_LAUNCHED();
    k_gnn_wgrad<<<GW, 128, 0, stream()>>>(N, GW, B.dP, GW, B.H[l], GW, dW + LAY.Wmh[l], nullptr);
    BG_LAUNCHED();
    k_gnn_dx<<<N, GW, 0, stream()>>>(N, GW, GW, B.dP, GW, W + LAY.Wmh[l], B.dH, GW, 1);
    BG_LAUNCHED();
  }
  k_gnn_relu_back<<<nb, 256, 0, stream()>>>(n64, B.Z0, B.dH, B.dU);
  BG_LAUNCHED();
  k_gnn_wgrad<<<GW, 128, 0, stream()>>>(N, GF, B.dU, GW, B.F, GF, dW + LAY.W0, dW + LAY.b0);
  BG_LAUNCHED();
  return BG_OK;
}

// objective and G = 2 dL/dconj(M) on the pattern
static int loss_grad(bg_matrix *A, GnnBufs &B, const z2g *Mval, const z2g *Z, int p, const z2g *b, const z2g *x,
                     double lambda, z2g *G, double *loss_out) {
  int N = B.N;
  size_t np = (size_t)N * p;
  z2g *buf = nullptr;
  BG_CUDA_TRY(cudaMallocAsync((void **)&buf, sizeof(z2g) * (4 * np + 2 * (size_t)N), stream()));
  z2g *Y = buf, *W = Y + np, *R = W + np, *S = R + np, *Mb = S + np, *rb = Mb + N;
  int st = BG_OK;
  k_gnn_spmm<<<dim3((N + 127) / 128, p), 128, 0, stream()>>>(N, B.rowptr, B.col, Mval, Z, p, Y);
  BG_LAUNCHED();
  // W = -A Y (the GEMM subtracts into a zeroed buffer); R = A Y - Z; S = A^H R
  BG_CUDA_TRY(cudaMemsetAsync(W, 0, sizeof(z2g) * np, stream()));
  if ((st = zgemm_sub_device(N, p, N, A->d, (int)A->ld, Y, N, W, N))) { cudaFreeAsync(buf, stream()); return st; }
  BG_CUDA_TRY(cudaMemsetAsync(S, 0, sizeof(z2g) * np, stream()));
  k_gnn_sub<<<(np + 255) / 256, 256, 0, stream()>>>(np, S, W, W);
  BG_LAUNCHED();
  k_gnn_sub<<<(np + 255) / 256, 256, 0, stream()>>>(np, W, Z, R);
  BG_LAUNCHED();
  k_gnn_ahr<<<(N + 7) / 8, 256, 0, stream()>>>(N, (const z2g *)A->d, A->ld, R, p, S);
  BG_LAUNCHED();
  double scale = 2.0 / ((double)N * p), scale2 = 0.0, l2 = 0.0;
  if (b && x && lambda > 0) {
    k_gnn_spmm<<<dim3((N + 127) / 128, 1), 128, 0, stream()>>>(N, B.rowptr, B.col, Mval, b, 1, Mb);
    BG_LAUNCHED();
    k_gnn_sub<<<(N + 255) / 256, 256, 0, stream()>>>(N, Mb, x, rb);
    BG_LAUNCHED();
    std::vector<z2g> hx(N), hr(N);
    BG_CUDA_TRY(cudaMemcpyAsync(hx.data(), x, sizeof(z2g) * N, cudaMemcpyDeviceToHost, stream()));
    BG_CUDA_TRY(cudaMemcpyAsync(hr.data(), rb, sizeof(z2g) * N, cudaMemcpyDeviceToHost, stream()));
    BG_CUDA_TRY(cudaStreamSynchronize(stream()));
    double xn = 0, rn = 0;
    for (int i = 0; i < N; i++) {
      xn += hx[i].r * hx[i].r + hx[i].i * hx[i].i;
      rn += hr[i].r * hr[i].r + hr[i].i * hr[i].i;
    }
    scale2 = 2.0 * lambda / std::max(xn, 1e-300);
    l2 = lambda * rn / std::max(xn, 1e-300);
  }
  k_gnn_sddmm<<<(N + 127) / 128, 128, 0, stream()>>>(N, B.rowptr, B.col, S, Z, p, scale, scale2 > 0 ? rb : nullptr,
                                                     b, scale2, G);
  BG_LAUNCHED();
  std::vector<z2g> hR(np);
  BG_CUDA_TRY(cudaMemcpyAsync(hR.data(), R, sizeof(z2g) * np, cudaMemcpyDeviceToHost, stream()));
  BG_CUDA_TRY(cudaStreamSynchronize(stream()));
  double l1 = 0;
  for (auto &r : hR) l1 += r.r * r.r + r.i * r.i;
  *loss_out = l1 / ((double)N * p) + l2;
  cudaFreeAsync(buf, stream());
  return BG_OK;
}

}  // namespace bg

using namespace bg;

extern "C" {

int bg_gnn_create(unsigned long long seed, bg_gnn **out) {
  if (!out) { set_error("bg_gnn_create: null output"); return BG_ERR_ARG; }
  *out = nullptr;
  int st = ensure_device();
  if (st) return st;
  int n = LAY.total;
  std::vector<float> p(n, 0.f);
  // Glorot-uniform weights from a 64-bit LCG; biases and the output map start at zero
  uint64_t s = seed * 6364136223846793005ull + 1442695040888963407ull;
  auto uni = [&]() {
    s = s * 6364136223846793005ull + 1442695040888963407ull;
    return ((s >> 11) * (1.0 / 9007199254740992.0)) * 2 - 1;
  };
  auto fill = [&](int off, int out_, int in_, double gain) {
    double a = gain * std::sqrt(6.0 / (in_ + out_));
    for (int i = 0; i < out_ * in_; i++) p[off + i] = (float)(a * uni());
  };
  fill(LAY.W0, GW, GF, 1.0);
  for (int l = 0; l < GL; l++) {
    fill(LAY.Wmh[l], GW, GW, 1.0);
    fill(LAY.Wme[l], GW, GE, 1.0);
    fill(LAY.Wuh[l], GW, GW, 0.3);
    fill(LAY.Wua[l], GW, GW, 0.3);
  }
  fill(LAY.Wri, GW, GW, 1.0);
  fill(LAY.Wrj, GW, GW, 1.0);
  fill(LAY.Wrg, GW, GE, 1.0);
  size_t nalloc = 4 * (size_t)n + 2;   // params, grads, Adam moments; then one double (8-byte aligned)
  bg_gnn *net = new bg_gnn();
  cudaError_t e = cudaMalloc(&net->params, sizeof(float) * (nalloc + 2));
  if (e != cudaSuccess) { delete net; set_error("bg_gnn_create: %s", cudaGetErrorString(e)); return BG_ERR_NOMEM; }
  net->grads = net->params + n;
  net->m = net->grads + n;
  net->v = net->m + n;
  net->sumsq = (double *)(net->params + ((4 * (size_t)n + 1) & ~(size_t)1));
  e = cudaMemset(net->params, 0, sizeof(float) * (nalloc + 2));
  if (e == cudaSuccess) e = cudaMemcpy(net->params, p.data(), sizeof(float) * n, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(net->params);
    delete net;
    set_error("bg_gnn_create: %s", cudaGetErrorString(e));
    return BG_ERR_CUDA;
  }
  *out = net;
  return BG_OK;
}

void bg_gnn_destroy(bg_gnn *net) {
  if (!net) return;
  if (net->params) cudaFree(net->params);
  delete net;
}

int bg_gnn_num_params(void) { return LAY.total; }

int bg_gnn_get_params(const bg_gnn *net, float *host) {
  if (!net || !host) { set_error("bg_gnn_get_params: bad arguments"); return BG_ERR_ARG; }
  BG_CUDA_TRY(cudaStreamSynchronize(stream()));
  BG_CUDA_TRY(cudaMemcpy(host, net->params, sizeof(float) * LAY.total, cudaMemcpyDeviceToHost));
  return BG_OK;
}

int bg_gnn_set_params(bg_gnn *net, const float *host) {
  if (!net || !host) { set_error("bg_gnn_set_params: bad arguments"); return BG_ERR_ARG; }
  BG_CUDA_TRY(cudaStreamSynchronize(stream()));
  BG_CUDA_TRY(cudaMemcpy(net->params, host, sizeof(float) * LAY.total, cudaMemcpyHostToDevice));
  net->step = 0;
  BG_CUDA_TRY(cudaMemset(net->m, 0, sizeof(float) * 2 * LAY.total));
  return BG_OK;
}

int bg_gnn_get_grads(const bg_gnn *net, float *host) {
  if (!net || !host) { set_error("bg_gnn_get_grads: bad arguments"); return BG_ERR_ARG; }
  BG_CUDA_TRY(cudaStreamSynchronize(stream()));
  BG_CUDA_TRY(cudaMemcpy(host, net->grads, sizeof(float) * LAY.total, cudaMemcpyDeviceToHost));
  return BG_OK;
}

int bg_precond_create_learned(bg_geometry *g, bg_matrix *A, double omega, const bg_gnn *net, bg_precond **out) {
  if (!g || !A || !net || !out || A->precision != BG_C128 || A->N != g->N) {
    set_error("bg_precond_create_learned: bad arguments");
    return BG_ERR_ARG;
  }
  *out = nullptr;
  if (A->factored) { set_error("bg_precond_create_learned: matrix holds LU factors"); return BG_ERR_STATE; }
  GnnBufs *Bp = nullptr;
  prof_start(PROF_GNN);
  int st = inference_bufs(g, Bp);
  if (st) {
    prof_stop(PROF_GNN, 0.0);
    return st;
  }
  GnnBufs &B = *Bp;
  st = bufs_compute(g, A, omega, B);
  bg_precond *P = nullptr;
  if (!st) {
    P = new bg_precond();
    P->N = B.N;
    P->nnz = B.E;

    cudaError_t e = cudaMallocAsync((void **)&P->rowptr, sizeof(int) * (B.N + 1), stream());
    if (e == cudaSuccess) e = cudaMallocAsync((void **)&P->col, sizeof(int) * B.E, stream());
    if (e == cudaSuccess) e = cudaMallocAsync((void **)&P->val, sizeof(z2g) * B.E, stream());
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(P->rowptr, B.rowptr, sizeof(int) * (B.N + 1), cudaMemcpyDeviceToDevice, stream());
    if (e == cudaSuccess) e = cudaMemcpyAsync(P->col, B.col, sizeof(int) * B.E, cudaMemcpyDeviceToDevice, stream());
    if (e != cudaSuccess) { set_error("learned preconditioner: %s", cudaGetErrorString(e)); st = BG_ERR_NOMEM; }
  }
  if (!st) st = forward(net, B, (z2g *)P->val);
  if (!st) {
    P->rho = B.rho_ref;
    P->theta = B.smax;
  }
  prof_stop(PROF_GNN, 0.0);
  if (st) {
    bg_precond_destroy(P);
    return st;
  }
  *out = P;
  return BG_OK;
}

// One training step on one matrix: forward, objective, backward of log L, Adam (lr > 0).
int bg_gnn_train_step(bg_gnn *net, bg_geometry *g, bg_matrix *A, double omega, const double *Z_host, int p,
                      int probe_power, const double *b_host, const double *x_host, double lambda, double lr,
                      double *loss_out) {
  if (!net || !g || !A || !Z_host || p <= 0 || p > GNN_MAXP || A->precision != BG_C128 || A->N != g->N || lr < 0 ||
      probe_power < 0 || probe_power > 64) {
    set_error("bg_gnn_train_step: bad arguments (at most %d probes)", GNN_MAXP);
    return BG_ERR_ARG;
  }
  if (A->factored) { set_error("bg_gnn_train_step: matrix holds LU factors"); return BG_ERR_STATE; }
  GnnBufs B;
  int st = bufs_init(g, A, omega, true, B);
  int N = g->N;
  z2g *dbuf = nullptr;
  if (!st) {
    size_t bytes = sizeof(z2g) * (3 * (size_t)N * p + 2 * (size_t)N + 2 * (size_t)B.E);
    cudaError_t e = cudaMallocAsync((void **)&dbuf, bytes, stream());
    if (e != cudaSuccess) { set_error("train step: %s", cudaGetErrorString(e)); st = BG_ERR_NOMEM; }
  }
  bool rhs = b_host && x_host && lambda > 0;
  z2g *Z = dbuf, *b = Z + (size_t)N * p, *x = b + N, *Mval = x + N, *Gg = Mval + B.E, *Y = Gg + B.E,
      *W = Y + (size_t)N * p;
  if (!st) {
    cudaError_t e = cudaMemcpyAsync(Z, Z_host, sizeof(z2g) * (size_t)N * p, cudaMemcpyHostToDevice, stream());
    if (e == cudaSuccess && rhs) e = cudaMemcpyAsync(b, b_host, sizeof(z2g) * N, cudaMemcpyHostToDevice, stream());
    if (e == cudaSuccess && rhs) e = cudaMemcpyAsync(x, x_host, sizeof(z2g) * N, cudaMemcpyHostToDevice, stream());
    if (e != cudaSuccess) { set_error("train step: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
  }
  // probes through the Jacobi error map: Z <- Z - A D^{-1} Z, rescaled
  for (int k = 0; !st && k < probe_power; k++) {
    size_t np = (size_t)N * p;
    k_gnn_rowscale<<<(np + 255) / 256, 256, 0, stream()>>>(N, p, B.dinv, Z, Y);
    g_launches++;
    cudaError_t e = cudaMemsetAsync(W, 0, sizeof(z2g) * np, stream());
    if (e != cudaSuccess) { set_error("train step: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; break; }
    if ((st = zgemm_sub_device(N, p, N, A->d, (int)A->ld, Y, N, W, N))) break;   // W = -A D^{-1} Z
    k_gnn_probe_update<<<p, 512, 0, stream()>>>(N, W, Z);
    g_launches++;
  }
  if (!st) st = forward(net, B, Mval);
  double loss = 0;
  if (!st) st = loss_grad(A, B, Mval, Z, p, rhs ? b : nullptr, rhs ? x : nullptr, lambda, Gg, &loss);
  if (!st) {
    cudaError_t e = cudaMemsetAsync(net->grads, 0, sizeof(float) * LAY.total, stream());
    if (e != cudaSuccess) { set_error("train step: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
  }
  if (!st && !(loss > 0 && std::isfinite(loss))) { set_error("train step: objective %g", loss); st = BG_ERR_NUMERIC; }
  if (!st) st = backward(net, B, Gg, 1.0 / loss);
  if (!st && lr > 0) {
    net->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    float c1 = 1.f - std::pow(b1, (float)net->step), c2 = 1.f - std::pow(b2, (float)net->step);
    cudaError_t e = cudaMemsetAsync(net->sumsq, 0, sizeof(double), stream());
    if (e != cudaSuccess) { set_error("train step: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
    if (!st) {
      k_gnn_sumsq<<<64, 256, 0, stream()>>>(LAY.total, net->grads, net->sumsq);
      g_launches++;
      k_gnn_adam<<<(LAY.total + 255) / 256, 256, 0, stream()>>>(LAY.total, net->params, net->grads, net->m, net->v,
                                                                net->sumsq, (float)lr, b1, b2, c1, c2, 1e-8f, 1.0f);
      g_launches++;
    }
  }
  if (dbuf) cudaFreeAsync(dbuf, stream());
  cudaError_t e2 = cudaStreamSynchronize(stream());
  if (!st && e2 != cudaSuccess) { set_error("train step: %s", cudaGetErrorString(e2)); st = BG_ERR_CUDA; }
  bufs_free(B);
  if (loss_out) *loss_out = loss;
  return st;
}

int bg_precond_bound(const bg_precond *P, double *rho, double *smax) {
  if (!P) { set_error("bg_precond_bound: null"); return BG_ERR_ARG; }
  if (rho) *rho = P->rho;
  if (smax) *smax = P->theta;
  return BG_OK;
}

int bg_precond_download(const bg_precond *P, int *rowptr, int *col, double *val) {
  if (!P) { set_error("bg_precond_download: null"); return BG_ERR_ARG; }
  BG_CUDA_TRY(cudaStreamSynchronize(stream()));
  if (rowptr) BG_CUDA_TRY(cudaMemcpy(rowptr, P->rowptr, sizeof(int) * (P->N + 1), cudaMemcpyDeviceToHost));
  if (col) BG_CUDA_TRY(cudaMemcpy(col, P->col, sizeof(int) * P->nnz, cudaMemcpyDeviceToHost));
  if (val) BG_CUDA_TRY(cudaMemcpy(val, P->val, sizeof(z2g) * P->nnz, cudaMemcpyDeviceToHost));
  return BG_OK;
}

}  // extern "C"
