// Static integrals of tetrahedron pairs sharing 2, 3 or 4 vertices (the
// singular near-field pairs), computed once per geometry as 24 moments per
// ordered pair:
//   per kernel K in {1/(4 pi r), 1/(4 pi), r/(8 pi)}:
//     int K,  int K (x - o),  int K (y - o),  int K (x - o).(y - o)
// in the unit-simplex measure, o = the first common vertex.
//
// The reference integrates these pairs with its generalised Taylor-Duffy code
// and an adaptive cubature at relative tolerance 1e-6 (TTaylorDuffy.cc:284-343,
// tolerance set at SWGGeometry.cc:46-47; called from GMatrixElements.cc:174-263,
// 343-353).  Here the rule is a relative-coordinate polar rule: barycentrics
// lambda (row tetrahedron A) and mu (column tetrahedron B), common vertices
// first; d = (lambda_k - mu_k | lambda_A-own | -mu_B-own) makes x - y linear
// and homogeneous in d; the admissible d form the polytope {sum d = 0,
// |d|_1 <= 2} whose faces away from the origin are Delta_{p-1} x Delta_{q-1},
// one per sign pattern S of the common components.  With d = rho zeta the
// remaining common barycentrics span a (c-1)-simplex of size 1 - rho and
//   dlambda dmu = rho^{m-1} (1 - rho)^{c-1} drho dzeta dt,  m = 7 - c,
// so the t- and rho-integrals are closed-form Beta integrals and only the
// 6 - c angular dimensions of each face cube [0,1]^{6-c} need a rule.
//
// Two stages:
//  * k_sing_fixed, one CTA per pair: collapsed Gauss-Legendre product rules
//    of orders n and n + 2 over every face cube.  Where all 24 moments of the
//    two orders agree to flag_tol of their scale (|M0|, |M0| h, |M0| h^2 for
//    the zeroth, first and second moments of each kernel, h = diameter of A)
//    the order n + 2 values are final; otherwise the pair is queued.
//  * k_sing_refine, persistent, one CTA per queued pair at a time: each face
//    cube is refined level by level.  Every open box is halved along each of
//    its dimensions in turn (a 6^{6-c}-point rule per half); the split that
//    changes the box value most is taken; the box closes when that change is
//    within tol of the scale (its two halves are kept) or stays open as two
//    boxes for the next level.  At most SG_MAXBOX boxes are open per level
//    and SG_MAXLEVEL levels are run; a box that cannot be opened for lack of
//    room, or is still open after the last level, keeps its halves and sets
//    bit 0 / bit 1 of the pair's status (never silently: the bits are OR-ed
//    into the geometry's status word, bg_geometry_singular_stats).
// With the fixed rule only (bg_geometry_set_singular_refine off) the order n
// values are kept for every pair, as before refinement existed.
//
// Every sum has a fixed order (thread-strided points, fixed shuffle trees,
// boxes closed in level and box order), so results are deterministic.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "internal.h"

namespace bg {

#define SG_THREADS 256
#define SG_NG 6            // Gauss points per dimension of a refinement box
#define SG_MAXBOX 2048     // boxes open per level, at most (per pair)
#define SG_MAXLEVEL 40
#define SG_TASKS 256       // half-box evaluations per chunk (their sums live in shared memory)
#define SG_CHUNK_BOXES 64  // boxes per chunk, at most (SG_TASKS / (2 x 2 dimensions))
#define SG_REC 33          // doubles per box record: lo[4], hi[4], val[24], S

// Gauss-Legendre rules on [0,1]: row n holds the n-point rule (n <= 16)
__constant__ double c_sgx[17][16], c_sgw[17][16];
static bool s_sg_tables = false;

static int sg_tables() {
  if (s_sg_tables) return BG_OK;
  static double x[17][16], w[17][16];
  for (int n = 1; n <= 16; n++) gauss_legendre01(n, x[n], w[n]);
  BG_CUDA_TRY(cudaMemcpyToSymbol(c_sgx, x, sizeof x));
  BG_CUDA_TRY(cudaMemcpyToSymbol(c_sgw, w, sizeof w));
  s_sg_tables = true;
  return BG_OK;
}

// per-pair data: vertices relative to the first common vertex, the closed-form
// moments of the common simplex (ub, W) and the Beta factors G
struct SgPair {
  double VA[4][3], VB[4][3];
  double ub[3], W;
  double G[3][3];
  int c;
};

__device__ __forceinline__ double sg_fact(int n) {
  double r = 1.0;
  for (int i = 2; i <= n; i++) r *= i;
  return r;
}

__device__ void sg_setup(const DevGeom &g, int4 oa, int4 ob, int c, SgPair &X) {
  const int via[4] = {oa.x, oa.y, oa.z, oa.w}, vib[4] = {ob.x, ob.y, ob.z, ob.w};
  double o[3] = {g.V4[4 * (size_t)via[0]], g.V4[4 * (size_t)via[0] + 1], g.V4[4 * (size_t)via[0] + 2]};
  for (int i = 0; i < 4; i++)
    for (int k = 0; k < 3; k++) {
      X.VA[i][k] = g.V4[4 * (size_t)via[i] + k] - o[k];
      X.VB[i][k] = g.V4[4 * (size_t)vib[i] + k] - o[k];
    }
  c = c < 2 ? 2 : c > 4 ? 4 : c;   // two tetrahedra share at most 4 vertices
  X.c = c;
  int nn = c - 1, m = 7 - c;
  double s2 = 0, sv[3] = {0, 0, 0};
  for (int i = 0; i < c; i++)
    for (int k = 0; k < 3; k++) { sv[k] += X.VA[i][k]; s2 += X.VA[i][k] * X.VA[i][k]; }
  for (int k = 0; k < 3; k++) X.ub[k] = sv[k] / (nn + 1);
  X.W = (s2 + sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2]) / ((nn + 1.0) * (nn + 2.0));
  for (int p = 0; p < 3; p++)
    for (int j = 0; j < 3; j++) {
      int a = m - 2 + p;   // m - 1 + (p - 1)
      X.G[p][j] = sg_fact(a + j) / sg_fact(a + j + nn + 1);
    }
}

__device__ __forceinline__ double sel4(const double *a, int i) {
  return i == 0 ? a[0] : i == 1 ? a[1] : i == 2 ? a[2] : a[3];
}

// collapsed map of u[0..k-1] (k <= 3) onto the k+1 barycentrics of Delta_k;
// returns the Jacobian (1-u0)^{k-1} (1-u1)^{k-2} ...
__device__ __forceinline__ double sg_collapse(int k, const double *u, double *b) {
  double rest = 1.0, J = 1.0;
#pragma unroll
  for (int i = 0; i < 3; i++)
    if (i < k) {
      b[i] = rest * u[i];
      rest *= 1.0 - u[i];
      if (i < k - 1) J *= rest;
    }
#pragma unroll
  for (int i = 0; i < 4; i++)
    if (i == k) b[i] = rest;
  return J;
}

// One angular point of face S with barycentrics al (A side) and be (B side)
// and weight w.  The 24 moments are linear in eight raw sums per kernel
// power R^p (p = -1, 0, 1): sum w R^p, sum w R^p A1, sum w R^p B1,
// sum w R^p A1.B1 (A1, B1: the points of A and B relative to the first
// common vertex, which is the origin, so VA[0] = 0), so only those are
// accumulated per point; sg_raw_to_moments applies the Beta factors and the
// common-simplex moments once per box.
template <int C>
__device__ __forceinline__ void sg_point(const SgPair &X_, int S, const double *al, const double *be, double w,
                                         double raw[24]) {
  // read the vertices per point (not hoisted into registers for the whole loop)
  const volatile SgPair &X = X_;
  double A1[3] = {0, 0, 0}, B1[3] = {0, 0, 0};
  int ja = 0, jb = 0;
#pragma unroll
  for (int k = 0; k < C; k++) {
    if ((S >> k) & 1) {
      double z = sel4(al, ja++);
      if (k > 0) {
#pragma unroll
        for (int x = 0; x < 3; x++) A1[x] += z * X.VA[k][x];
      }
    } else {
      double z = sel4(be, jb++);
      if (k > 0) {
#pragma unroll
        for (int x = 0; x < 3; x++) B1[x] += z * X.VA[k][x];
      }
    }
  }
#pragma unroll
  for (int k = C; k < 4; k++) {
    double za = sel4(al, ja++), zb = sel4(be, jb++);
#pragma unroll
    for (int x = 0; x < 3; x++) { A1[x] += za * X.VA[k][x]; B1[x] += zb * X.VB[k][x]; }
  }
  double L0 = A1[0] - B1[0], L1 = A1[1] - B1[1], L2 = A1[2] - B1[2];
  double R = sqrt(L0 * L0 + L1 * L1 + L2 * L2);
  double AB = A1[0] * B1[0] + A1[1] * B1[1] + A1[2] * B1[2];
  double wp[3] = {w / R, w, w * R};
#pragma unroll
  for (int pk = 0; pk < 3; pk++) {
    double t = wp[pk];
    raw[8 * pk] += t;
#pragma unroll
    for (int x = 0; x < 3; x++) {
      raw[8 * pk + 1 + x] += t * A1[x];
      raw[8 * pk + 4 + x] += t * B1[x];
    }
    raw[8 * pk + 7] += t * AB;
  }
}

// moment i of the pair from the raw sums (Beta factors G, common-simplex
// moments ub and W)
__device__ __forceinline__ double sg_raw_to_moment(const SgPair &X, const double *raw, int i) {
  int pk = i / 8, j = i % 8;
  double G0 = X.G[pk][0], G1 = X.G[pk][1], G2 = X.G[pk][2];
  const double *r = raw + 8 * pk;
  if (j == 0) return G0 * r[0];
  if (j < 4) return G1 * r[j] + X.ub[j - 1] * (G0 - G1) * r[0];
  if (j < 7) return G1 * r[j] + X.ub[j - 4] * (G0 - G1) * r[0];
  double uAB = X.ub[0] * (r[1] + r[4]) + X.ub[1] * (r[2] + r[5]) + X.ub[2] * (r[3] + r[6]);
  return G2 * r[7] + (G1 - G2) * uAB + X.W * (G0 - 2.0 * G1 + G2) * r[0];
}

// all 24 moments from raw sums held in registers (constant indices only)
__device__ __forceinline__ void sg_moments_from_raw(const SgPair &X, const double raw[24], double out[24]) {
#pragma unroll
  for (int pk = 0; pk < 3; pk++) {
    double G0 = X.G[pk][0], G1 = X.G[pk][1], G2 = X.G[pk][2];
    const double *r = raw + 8 * pk;
    double *m = out + 8 * pk;
    m[0] = G0 * r[0];
#pragma unroll
    for (int x = 0; x < 3; x++) {
      m[1 + x] = G1 * r[1 + x] + X.ub[x] * (G0 - G1) * r[0];
      m[4 + x] = G1 * r[4 + x] + X.ub[x] * (G0 - G1) * r[0];
    }
    double uAB = X.ub[0] * (r[1] + r[4]) + X.ub[1] * (r[2] + r[5]) + X.ub[2] * (r[3] + r[6]);
    m[7] = G2 * r[7] + (G1 - G2) * uAB + X.W * (G0 - 2.0 * G1 + G2) * r[0];
  }
}


// point t (digits of base ng, first dimension least significant) of the
// ng^k product rule (k = 6 - C) on box [lo, hi] of face S; the first ka
// collapsed coordinates map onto A's simplex, the next kb onto B's
template <int C>
__device__ __forceinline__ void sg_box_point(const SgPair &X, int S, int ka, int ng, const double *lo,
                                             const double *hi, int t, double raw[24]) {
  constexpr int K = 6 - C;
  const int kb = K - ka;
  double u[K], w = 1.0;
#pragma unroll
  for (int d = 0; d < K; d++) {
    int i = t % ng;
    t /= ng;
    u[d] = lo[d] + (hi[d] - lo[d]) * c_sgx[ng][i];
    w *= (hi[d] - lo[d]) * c_sgw[ng][i];
  }
  double uA[3], uB[3];
#pragma unroll
  for (int e = 0; e < 3; e++) {
    uA[e] = e < K ? u[e < K ? e : 0] : 0.0;
    double v = 0.0;
#pragma unroll
    for (int d = 0; d < K; d++)
      if (d - ka == e) v = u[d];
    uB[e] = v;
  }
  double al[4], be[4];
  double ja = sg_collapse(ka, uA, al);
  double jb = sg_collapse(kb, uB, be);
  w *= ja * jb;
  sg_point<C>(X, S, al, be, w, raw);
}

__device__ __forceinline__ int sg_face_S(int c, int f) { return c == 4 ? f + 1 : f; }
__device__ __forceinline__ int sg_nfaces(int c) { return c == 4 ? 14 : (1 << c); }

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// sums part[24] over the block into out[24] (shared) in a fixed order
__device__ void sg_block_sum(double part[24], double (*red)[24], double *out) {
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < 24; i++) {
    double v = warp_sum_d(part[i]);
    if (lane == 0) red[wid][i] = v;
  }
  __syncthreads();
  if (threadIdx.x < 24) {
    double s = 0.0;
    for (int w = 0; w < SG_THREADS / 32; w++) s += red[w][threadIdx.x];
    out[threadIdx.x] = s;
  }
  __syncthreads();
}

__constant__ double c_sg_gpre[3] = {0.25 / M_PI, 0.25 / M_PI, 0.125 / M_PI};

// whole-face product rule of order n, points strided over the block (raw sums)
template <int C>
__device__ void sg_fixed_pass(const SgPair &X, int n, double raw[24]) {
  constexpr int nown = 4 - C, K = 6 - C, nf = C == 4 ? 14 : (1 << C);
  int per = 1;
#pragma unroll
  for (int i = 0; i < K; i++) per *= n;
#pragma unroll
  for (int i = 0; i < 24; i++) raw[i] = 0.0;
  const double lo[K] = {}, hi[K] = {};
  double one[K];
#pragma unroll
  for (int d = 0; d < K; d++) one[d] = 1.0;
  (void)hi;
#pragma unroll 1
  for (int f = threadIdx.x; f < nf * per; f += SG_THREADS) {
    int face = f / per, t = f - face * per;
    int S = sg_face_S(C, face), ns = __popc(S);
    sg_box_point<C>(X, S, ns + nown - 1, n, lo, one, t, raw);
  }
}

// h^2 = squared diameter of tetrahedron A; scales of the 24 moments from the
// order n + 2 values f1 (which include the kernel prefactors)
__device__ void sg_scales(const SgPair &X, const double *f1, double *scale) {
  double h2 = 0.0;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      double s2 = 0.0;
      for (int x = 0; x < 3; x++) s2 += (X.VA[i][x] - X.VA[j][x]) * (X.VA[i][x] - X.VA[j][x]);
      h2 = fmax(h2, s2);
    }
  double h = sqrt(h2);
  for (int pk = 0; pk < 3; pk++) {
    double m0 = fabs(f1[8 * pk]) / c_sg_gpre[pk];
    scale[8 * pk] = m0;
    for (int x = 1; x < 7; x++) scale[8 * pk + x] = m0 * h;
    scale[8 * pk + 7] = m0 * h2;
  }
}

struct SgLists {
  int *list;        // flagged pair indices, by class (c = 2, 3, 4) at start[c-2]
  int *cnt;         // 3 counters
  int start[3];
  unsigned char *flag;   // per singular pair: bit 0 flagged, bits 1-2 refinement status
  int *work;        // work counter of the refinement kernel
  unsigned int *status;
  unsigned long long *evals;
};

template <int C>
__device__ void sg_fixed_pair(const SgPair &X, int pidx, int first, double *mom, int n, int refine,
                              double flag_tol, const SgLists &L, double (*red)[24], double *f0, double *f1) {
  double part[24];
  sg_fixed_pass<C>(X, n, part);
  sg_block_sum(part, red, f1);
  if (threadIdx.x < 24) f0[threadIdx.x] = sg_raw_to_moment(X, f1, threadIdx.x) * c_sg_gpre[threadIdx.x / 8];
  __syncthreads();
  if (!refine) {
    if (threadIdx.x < 24) mom[24 * (size_t)pidx + threadIdx.x] = f0[threadIdx.x];
    return;
  }
  sg_fixed_pass<C>(X, n + 2, part);
  sg_block_sum(part, red, f1);
  double m1 = threadIdx.x < 24 ? sg_raw_to_moment(X, f1, threadIdx.x) * c_sg_gpre[threadIdx.x / 8] : 0.0;
  __syncthreads();
  if (threadIdx.x < 24) f1[threadIdx.x] = m1;
  __syncthreads();
  if (threadIdx.x == 0) {
    double scale[24];
    sg_scales(X, f1, scale);
    double flag = 0.0;
    for (int i = 0; i < 24; i++) flag = fmax(flag, fabs(f1[i] - f0[i]) / c_sg_gpre[i / 8] / scale[i]);
    for (int i = 0; i < 24; i++) mom[24 * (size_t)pidx + i] = f1[i];
    bool flagged = !(flag <= flag_tol);
    L.flag[pidx - first] = flagged ? 1 : 0;
    if (flagged) {
      int pos = atomicAdd(&L.cnt[C - 2], 1);
      L.list[L.start[C - 2] + pos] = pidx;
    }
  }
}

__global__ void __launch_bounds__(SG_THREADS, 2) k_sing_fixed(DevGeom g, const int4 *tp, const int4 *ordA,
                                                              const int4 *ordB, int first, double *mom, int n,
                                                              int refine, double flag_tol, SgLists L) {
  __shared__ SgPair X;
  __shared__ double red[SG_THREADS / 32][24];
  __shared__ double f0[24], f1[24];
  const int pidx = first + blockIdx.x;
  if (threadIdx.x == 0) sg_setup(g, ordA[pidx], ordB[pidx], tp[pidx].z, X);
  __syncthreads();
  switch (X.c) {
    case 2: sg_fixed_pair<2>(X, pidx, first, mom, n, refine, flag_tol, L, red, f0, f1); break;
    case 3: sg_fixed_pair<3>(X, pidx, first, mom, n, refine, flag_tol, L, red, f0, f1); break;
    default: sg_fixed_pair<4>(X, pidx, first, mom, n, refine, flag_tol, L, red, f0, f1); break;
  }
}

// shared state of the refinement kernel
struct SgShared {
  SgPair X;
  double scale[24], acc[24];
  double blo[SG_CHUNK_BOXES][4], bhi[SG_CHUNK_BOXES][4];
  int bS[SG_CHUNK_BOXES], bd[SG_CHUNK_BOXES], bopen[SG_CHUNK_BOXES], bpos[SG_CHUNK_BOXES];
  double tb[SG_THREADS / 4][8];   // per lane group: the bounds (lo, hi) of its current task
  int pidx, nn, status;
  unsigned long long evals;
};

// Evaluates ntasks boxes of the chunk into sres (24 moments each, unit
// measure, no kernel prefactor).  split: task t is box t / 2K halved along
// dimension (t % 2K) / 2, half t % 2; otherwise task t is box t whole.
// G lanes share a task (a fixed shuffle tree sums their points).
template <int C>
__device__ void sg_eval_tasks(SgShared &sh, double *sres, int ntasks, bool split) {
  constexpr int K = 6 - C, nown = 4 - C;
  constexpr int G = C == 2 ? 32 : C == 3 ? 8 : 4;
  constexpr int P = SG_NG * SG_NG * (K > 2 ? SG_NG : 1) * (K > 3 ? SG_NG : 1);
  const int gl = threadIdx.x % G, grp = threadIdx.x / G;
  constexpr int ngrp = SG_THREADS / G;
  for (int base = 0; base < ntasks; base += ngrp) {
    int t = base + grp;
    double part[24];
#pragma unroll
    for (int i = 0; i < 24; i++) part[i] = 0.0;
    int j = split ? t / (2 * K) : t;
    __syncwarp();   // the group's previous task has finished reading its bounds
    if (t < ntasks && gl == 0) {
      int sd = split ? (t % (2 * K)) / 2 : -1, h = t & 1;
#pragma unroll
      for (int d = 0; d < 4; d++) {
        double lo = sh.blo[j][d], hi = sh.bhi[j][d];
        if (d == sd) {
          double mid = 0.5 * (lo + hi);
          if (h == 0) hi = mid; else lo = mid;
        }
        sh.tb[grp][d] = lo;
        sh.tb[grp][4 + d] = hi;
      }
    }
    __syncwarp();
    if (t < ntasks) {
      int S = sh.bS[j], ns = __popc(S);
      // bounds read per point from shared memory (keeps registers for the point)
      const volatile double *tb = sh.tb[grp];
#pragma unroll 1
      for (int p = gl; p < P; p += G) {
        double lo[K], hi[K];
#pragma unroll
        for (int d = 0; d < K; d++) { lo[d] = tb[d]; hi[d] = tb[4 + d]; }
        sg_box_point<C>(sh.X, S, ns + nown - 1, SG_NG, lo, hi, p, part);
      }
    }
#pragma unroll
    for (int i = 0; i < 24; i++) {
      double v = part[i];
#pragma unroll
      for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      part[i] = v;
    }
    if (t < ntasks && gl == 0) {
#pragma unroll
      for (int i = 0; i < 24; i++) sres[24 * t + i] = part[i];
    }
  }
  // raw sums -> moments, one thread per task
  __syncthreads();
  for (int t = threadIdx.x; t < ntasks; t += SG_THREADS) {
    double r[24], m[24];
#pragma unroll
    for (int i = 0; i < 24; i++) r[i] = sres[24 * t + i];
    sg_moments_from_raw(sh.X, r, m);
#pragma unroll
    for (int i = 0; i < 24; i++) sres[24 * t + i] = m[i];
  }
}

template <int C>
__device__ void sg_refine_pair(SgShared &sh, double *sres, double *cur, double *nxt, double tol) {
  constexpr int K = 6 - C, nf = C == 4 ? 14 : (1 << C);
  constexpr int P = SG_NG * SG_NG * (K > 2 ? SG_NG : 1) * (K > 3 ? SG_NG : 1);
  constexpr int CB = SG_TASKS / (2 * K);
  // level 0 boxes: the whole face cubes
  if (threadIdx.x < nf) {
    sh.bS[threadIdx.x] = sg_face_S(C, threadIdx.x);
    for (int d = 0; d < 4; d++) { sh.blo[threadIdx.x][d] = 0.0; sh.bhi[threadIdx.x][d] = 1.0; }
  }
  __syncthreads();
  sg_eval_tasks<C>(sh, sres, nf, false);
  __syncthreads();
  for (int idx = threadIdx.x; idx < nf * SG_REC; idx += SG_THREADS) {
    int j = idx / SG_REC, f = idx % SG_REC;
    double v = f < 4 ? 0.0 : f < 8 ? 1.0 : f < 32 ? sres[24 * j + f - 8] : (double)sh.bS[j];
    cur[(size_t)j * SG_REC + f] = v;
  }
  if (threadIdx.x == 0) sh.evals += (unsigned long long)nf * P;
  __syncthreads();
  int ncur = nf;
  for (int level = 0; level < SG_MAXLEVEL && ncur > 0; level++) {
    if (threadIdx.x == 0) sh.nn = 0;
    for (int cb = 0; cb < ncur; cb += CB) {
      const int nb = min(CB, ncur - cb);
      for (int idx = threadIdx.x; idx < nb * 9; idx += SG_THREADS) {
        int j = idx / 9, f = idx % 9;
        const double *r = cur + (size_t)(cb + j) * SG_REC;
        if (f < 4) sh.blo[j][f] = r[f];
        else if (f < 8) sh.bhi[j][f - 4] = r[f];
        else sh.bS[j] = (int)r[32];
      }
      __syncthreads();
      sg_eval_tasks<C>(sh, sres, nb * 2 * K, true);
      __syncthreads();
      // the split that changes each box most, and whether it stays open
      if (threadIdx.x < nb) {
        int j = threadIdx.x;
        const double *val = cur + (size_t)(cb + j) * SG_REC + 8;
        double best = -1.0;
        int bestd = 0;
        for (int d = 0; d < K; d++) {
          const double *v0 = sres + 24 * (j * 2 * K + 2 * d), *v1 = v0 + 24;
          double e = 0.0;
          for (int i = 0; i < 24; i++) e = fmax(e, fabs(v0[i] + v1[i] - val[i]) / sh.scale[i]);
          if (e > best) { best = e; bestd = d; }
        }
        sh.bd[j] = bestd;
        sh.bopen[j] = best > tol;
      }
      __syncthreads();
      // positions of the opened boxes in the next level, in box order
      if (threadIdx.x == 0) {
        int nn = sh.nn;
        for (int j = 0; j < nb; j++) {
          if (!sh.bopen[j]) continue;
          if (nn + 2 > SG_MAXBOX) { sh.bopen[j] = 0; sh.status |= 1; continue; }
          if (level == SG_MAXLEVEL - 1) { sh.bopen[j] = 0; sh.status |= 2; continue; }
          sh.bpos[j] = nn;
          nn += 2;
        }
        sh.nn = nn;
        sh.evals += (unsigned long long)nb * 2 * K * P;
      }
      __syncthreads();
      for (int idx = threadIdx.x; idx < nb * 2 * SG_REC; idx += SG_THREADS) {
        int j = idx / (2 * SG_REC), r = idx % (2 * SG_REC), h = r / SG_REC, f = r % SG_REC;
        if (!sh.bopen[j]) continue;
        int d = sh.bd[j];
        double v;
        if (f < 8) {
          int dd = f & 3;
          double lo = sh.blo[j][dd], hi = sh.bhi[j][dd];
          if (dd == d) {
            double mid = 0.5 * (lo + hi);
            if (h == 0) hi = mid; else lo = mid;
          }
          v = f < 4 ? lo : hi;
        } else if (f < 32) {
          v = sres[24 * (j * 2 * K + 2 * d + h) + f - 8];
        } else {
          v = (double)sh.bS[j];
        }
        nxt[(size_t)(sh.bpos[j] + h) * SG_REC + f] = v;
      }
      if (threadIdx.x < 24) {
        double a = sh.acc[threadIdx.x];
        for (int j = 0; j < nb; j++) {
          if (sh.bopen[j]) continue;
          const double *v0 = sres + 24 * (j * 2 * K + 2 * sh.bd[j]);
          a += v0[threadIdx.x] + v0[24 + threadIdx.x];
        }
        sh.acc[threadIdx.x] = a;
      }
      __syncthreads();
    }
    double *t = cur;
    cur = nxt;
    nxt = t;
    ncur = sh.nn;
    __syncthreads();
  }
}

// Refinement of the flagged pairs; pool: 2 x SG_MAXBOX box records per CTA.
__global__ void __launch_bounds__(SG_THREADS, 1) k_sing_refine(DevGeom g, const int4 *tp, const int4 *ordA,
                                                               const int4 *ordB, int first, double *mom, double tol,
                                                               double *pool, SgLists L) {
  extern __shared__ double sres[];   // SG_TASKS x 24 half-box moments
  __shared__ SgShared sh;
  double *cur = pool + (size_t)blockIdx.x * 2 * SG_MAXBOX * SG_REC;
  double *nxt = cur + (size_t)SG_MAXBOX * SG_REC;
  const int total = L.cnt[0] + L.cnt[1] + L.cnt[2];
  for (;;) {
    if (threadIdx.x == 0) {
      int w = atomicAdd(L.work, 1);
      int pidx = -1;
      if (w < L.cnt[0]) pidx = L.list[L.start[0] + w];
      else if (w < L.cnt[0] + L.cnt[1]) pidx = L.list[L.start[1] + w - L.cnt[0]];
      else if (w < total) pidx = L.list[L.start[2] + w - L.cnt[0] - L.cnt[1]];
      sh.pidx = pidx;
      if (pidx >= 0) {
        sg_setup(g, ordA[pidx], ordB[pidx], tp[pidx].z, sh.X);
        double f1[24];
        for (int i = 0; i < 24; i++) f1[i] = mom[24 * (size_t)pidx + i];
        sg_scales(sh.X, f1, sh.scale);
      }
      sh.status = 0;
      sh.evals = 0;
    }
    if (threadIdx.x < 24) sh.acc[threadIdx.x] = 0.0;
    __syncthreads();
    const int pidx = sh.pidx;
    if (pidx < 0) return;
    switch (sh.X.c) {
      case 2: sg_refine_pair<2>(sh, sres, cur, nxt, tol); break;
      case 3: sg_refine_pair<3>(sh, sres, cur, nxt, tol); break;
      default: sg_refine_pair<4>(sh, sres, cur, nxt, tol); break;
    }
    if (threadIdx.x < 24) mom[24 * (size_t)pidx + threadIdx.x] = sh.acc[threadIdx.x] * c_sg_gpre[threadIdx.x / 8];
    if (threadIdx.x == 0) {
      L.flag[pidx - first] |= (unsigned char)(sh.status << 1);
      if (sh.status) atomicOr(L.status, (unsigned int)sh.status);
      atomicAdd(L.evals, sh.evals);
    }
    __syncthreads();
  }
}

// Singular pairs of the near table: [ntp_reg, ntp), sorted by class (2, 3, 4
// common vertices).  Fills tpMom and the geometry's singular statistics.
int singular_precompute(bg_geometry *g) {
  NearData &nd = g->near;
  const int nsing = nd.ntp - nd.ntp_reg;
  for (int i = 0; i < 6; i++) g->sing_stats[i] = 0;
  if (nsing <= 0) return BG_OK;
  int st = sg_tables();
  if (st) return st;
  const int n = g->singular_order;
  const bool refine = g->sing_refine;
  // points of the fixed passes (host arithmetic, per class)
  long long fixed_pts = 0;
  for (int cls = 0; cls < 3; cls++) {
    int c = cls + 2, nf = c == 4 ? 14 : (1 << c);
    long long p0 = 1, p1 = 1;
    for (int i = 0; i < 6 - c; i++) { p0 *= n; p1 *= n + 2; }
    fixed_pts += (long long)nd.nsing_c[cls] * nf * (p0 + (refine ? p1 : 0));
  }
  g->sing_stats[0] = nsing;
  g->sing_stats[2] = fixed_pts;
  // small device block: counters (3), work counter, status, evals, then the
  // list and the per-pair flags
  size_t hdr = 64, bytes = hdr + sizeof(int) * (size_t)nsing + (size_t)nsing;
  char *blk = nullptr;
  BG_CUDA_TRY(cudaMallocAsync((void **)&blk, bytes, stream()));
  SgLists L;
  L.cnt = (int *)blk;
  L.work = (int *)(blk + 16);
  L.status = (unsigned int *)(blk + 20);
  L.evals = (unsigned long long *)(blk + 24);
  L.list = (int *)(blk + hdr);
  L.flag = (unsigned char *)(blk + hdr + sizeof(int) * (size_t)nsing);
  L.start[0] = 0;
  L.start[1] = nd.nsing_c[0];
  L.start[2] = nd.nsing_c[0] + nd.nsing_c[1];
  int rc = BG_OK;
  double *pool = nullptr;
  do {
    if (cudaMemsetAsync(blk, 0, bytes, stream()) != cudaSuccess) { rc = BG_ERR_CUDA; break; }
    k_sing_fixed<<<nsing, SG_THREADS, 0, stream()>>>(g->dev, nd.tp, nd.tpOrdA, nd.tpOrdB, nd.ntp_reg, nd.tpMom, n,
                                                     refine ? 1 : 0, g->sing_flag_tol, L);
    if (cudaGetLastError() != cudaSuccess) { rc = BG_ERR_CUDA; break; }
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (refine) {
      const size_t smem = sizeof(double) * SG_TASKS * 24;
      static bool attr = false;
      if (!attr) {
        if (cudaFuncSetAttribute(k_sing_refine, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess) { rc = BG_ERR_CUDA; break; }
        attr = true;
      }
      int dev = 0, nsm = 0, per = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_sing_refine, SG_THREADS, smem);
      int grid = std::max(1, nsm * std::max(1, per));
      grid = std::min(grid, nsing);
      size_t pbytes = sizeof(double) * (size_t)grid * 2 * SG_MAXBOX * SG_REC;
      if (cudaMallocAsync((void **)&pool, pbytes, stream()) != cudaSuccess) { rc = BG_ERR_NOMEM; break; }
      k_sing_refine<<<grid, SG_THREADS, smem, stream()>>>(g->dev, nd.tp, nd.tpOrdA, nd.tpOrdB, nd.ntp_reg, nd.tpMom,
                                                          g->sing_tol, pool, L);
      if (cudaGetLastError() != cudaSuccess) { rc = BG_ERR_CUDA; break; }
      g_launches.fetch_add(1, std::memory_order_relaxed);
    }
    struct { int cnt[4]; int work; unsigned int status; unsigned long long evals; } h;
    if (cudaMemcpyAsync(&h, blk, sizeof h, cudaMemcpyDeviceToHost, stream()) != cudaSuccess) { rc = BG_ERR_CUDA; break; }
    if (!nd.tpFlag && cudaMallocAsync((void **)&nd.tpFlag, (size_t)nsing, stream()) != cudaSuccess) {
      rc = BG_ERR_NOMEM;
      break;
    }
    if (cudaMemcpyAsync(nd.tpFlag, L.flag, (size_t)nsing, cudaMemcpyDeviceToDevice, stream()) != cudaSuccess) {
      rc = BG_ERR_CUDA;
      break;
    }
    if (cudaStreamSynchronize(stream()) != cudaSuccess) { rc = BG_ERR_CUDA; break; }
    g->sing_stats[1] = (long long)h.cnt[0] + h.cnt[1] + h.cnt[2];
    g->sing_stats[3] = (long long)h.evals;
    g->sing_stats[4] = h.status;
    g->sing_stats[5] = refine ? 1 : 0;
  } while (0);
  if (rc == BG_ERR_CUDA) set_error("singular near-field precompute: %s", cudaGetErrorString(cudaGetLastError()));
  else if (rc == BG_ERR_NOMEM) set_error("singular near-field precompute: cannot allocate the refinement box pool");
  if (pool) cudaFreeAsync(pool, stream());
  cudaFreeAsync(blk, stream());
  if (rc == BG_OK) BG_CUDA_TRY(cudaStreamSynchronize(stream()));
  return rc;
}

}  // namespace bg
