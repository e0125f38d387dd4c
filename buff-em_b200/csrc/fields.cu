// Fields of the solved currents at evaluation points: SWGGeometry::GetFields
// (GetFields.cc:287-382) with Get1BFFields (GetFields.cc:265-281) and the
// volume integrand GetFields_VIntegrand (GetFields.cc:176-201).
//
// The reference sums, per point X and basis function a, J_a times the fields
// of b_a integrated over both tetrahedra with the 4-point rule when
// |X - centroid_a| / radius_a > 10, else the 16-point rule.  Both rules are
// fully symmetric, so their points depend only on the tetrahedron, and the
// sum over the (up to four) basis functions living on one tetrahedron T is a
// single linear current per rule:
//
//   sum_a J_a b_a(y) * 6 vol_T = sum_k g_k (y - V_k),   g_k = 2 s_k A_k J_k
//
// (k runs over T's faces that carry a basis function, V_k is the vertex
// opposite face k, s_k = +1 on the basis function's P side, -1 on its M side,
// A_k the face area).  The kernel therefore walks tetrahedra, not basis
// functions: each (point, tetrahedron) pair costs 4 quadrature points when all
// of T's faces are far from X, and 4 + 16 (split by face) otherwise --
// a quarter of the per-basis-function work, with the same quadrature points
// and the same rule choice per basis function as the reference.
//
// Field kernels (e^{-i w t}, vacuum, g = e^{ikr}/(4 pi r), R = X - y, Rh = R/r):
//   E = i w Z0 g [(1 + i/kr - 1/kr^2) J + (-1 - 3i/kr + 3/kr^2) (Rh.J) Rh]
//   H = g (ik - 1/r) Rh x J
// which are the G and C dyadics of the reference's CalcGC with its prefactors.
// The incident plane wave adds E0 e^{ik nhat.X} and nhat x E / Z0.
//
// HBM layout (per tetrahedron, built once per geometry):
//   fieldTet  16 doubles: V0..V3 (12), centroid (3), R_all (1), where
//             |X - centroid| > R_all implies every face of T is far from X
//   fieldFace 16 doubles: per local face k, (centroid, radius), radius 0 if the
//             face carries no basis function
//   coef       8 doubles per call: g_k (4 complex) from J
// Work split: a block owns 128 x tpt tetrahedra (tpt = 1 with the
// tetrahedron's data held in registers across the points while the partials
// stay small; else tpt grows to ~8 blocks per SM) and 32 points; each
// warp reduces its lanes per point into shared memory and the block writes one
// partial per (tetrahedron block, point), summed in a fixed order by the
// finishing kernel (deterministic).
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "internal.h"

namespace bg {
namespace {

constexpr int FTHREADS = 128;
constexpr int FPCH = 32;           // points per block
constexpr double ZVAC_F = 376.73031346177;

// 16-point rule (TetCR.cc): orbit patterns as in the assembly kernels
__constant__ double c_fr16[64];
static bool s_fr16_ok = false;

int init_rule16() {
  if (s_fr16_ok) return BG_OK;
  const double v[5] = {0.771642902067237, 0.076119032644254315, 0.07183164526766925, 0.11970052779780202,
                       0.40423391346726440};
  const char *pat[2] = {"ABB BAB BBA BBB", "CDE CED CEE DCE DEC DEE ECD ECE EDC EDE EEC EED"};
  const double w[2] = {8.3956323500204695e-3, 0.011090344772215399};
  double h[64];
  int np = 0;
  for (int o = 0; o < 2; o++)
    for (const char *p = pat[o]; *p;) {
      if (*p == ' ') { p++; continue; }
      h[4 * np] = v[p[0] - 'A']; h[4 * np + 1] = v[p[1] - 'A']; h[4 * np + 2] = v[p[2] - 'A'];
      h[4 * np + 3] = w[o];
      np++;
      p += 3;
    }
  BG_CUDA_TRY(cudaMemcpyToSymbol(c_fr16, h, sizeof h));
  s_fr16_ok = true;
  return BG_OK;
}

struct z { double r, i; };
__device__ __forceinline__ z zmul(z a, z b) { return z{a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r}; }

struct FieldK {
  z k;       // wavenumber (= omega in the reference's units)
  z invik;   // 1 / (i k)
  z ik;      // i k
};

// one quadrature point: current alpha y - beta at y with weight w
template <bool REALK>
__device__ __forceinline__ void field_point(const FieldK &K, const double *x, const double *y, double w, z al,
                                            const z *be, double *acc) {
  z J[3];
#pragma unroll
  for (int c = 0; c < 3; c++) J[c] = z{al.r * y[c] - be[c].r, al.i * y[c] - be[c].i};
  double R[3] = {x[0] - y[0], x[1] - y[1], x[2] - y[2]};
  double r2 = R[0] * R[0] + R[1] * R[1] + R[2] * R[2];
  if (r2 < 1e-24) return;
  double ir = rsqrt(r2), r = r2 * ir;
  double s, c;
  sincos(K.k.r * r, &s, &c);
  double m = w * ir;
  if (!REALK) m *= exp(-K.k.i * r);
  z g{m * c, m * s};                       // w e^{ikr} / r
  z u{K.invik.r * ir, K.invik.i * ir};     // 1/(ikr)
  z u2 = zmul(u, u);
  z t1{1.0 - u.r + u2.r, -u.i + u2.i};
  z t2{-1.0 + 3.0 * (u.r - u2.r), 3.0 * (u.i - u2.i)};
  double Rh[3] = {R[0] * ir, R[1] * ir, R[2] * ir};
  z RJ{Rh[0] * J[0].r + Rh[1] * J[1].r + Rh[2] * J[2].r, Rh[0] * J[0].i + Rh[1] * J[1].i + Rh[2] * J[2].i};
  z c1 = zmul(g, t1), c2 = zmul(zmul(g, t2), RJ), ch = zmul(g, z{K.ik.r - ir, K.ik.i});
#pragma unroll
  for (int q = 0; q < 3; q++) {
    z e = zmul(c1, J[q]);
    acc[2 * q] += e.r + c2.r * Rh[q];
    acc[2 * q + 1] += e.i + c2.i * Rh[q];
  }
  z X0{Rh[1] * J[2].r - Rh[2] * J[1].r, Rh[1] * J[2].i - Rh[2] * J[1].i};
  z X1{Rh[2] * J[0].r - Rh[0] * J[2].r, Rh[2] * J[0].i - Rh[0] * J[2].i};
  z X2{Rh[0] * J[1].r - Rh[1] * J[0].r, Rh[0] * J[1].i - Rh[1] * J[0].i};
  z h0 = zmul(ch, X0), h1 = zmul(ch, X1), h2 = zmul(ch, X2);
  acc[6] += h0.r; acc[7] += h0.i;
  acc[8] += h1.r; acc[9] += h1.i;
  acc[10] += h2.r; acc[11] += h2.i;
}

template <bool REALK>
__device__ __forceinline__ void rule4(const FieldK &K, const double *x, const double (*V)[3], z al, const z *be,
                                      double *acc) {
  // barycentric (B, A, A, A) and permutations, weight 1/24 (TetCR.cc 4-point rule)
  const double A = 0.13819660112501051, B = 0.58541019662496850;
  double S[3];
#pragma unroll
  for (int c = 0; c < 3; c++) S[c] = A * (V[0][c] + V[1][c] + V[2][c] + V[3][c]);
#pragma unroll
  for (int i = 0; i < 4; i++) {
    double y[3];
#pragma unroll
    for (int c = 0; c < 3; c++) y[c] = S[c] + (B - A) * V[i][c];
    field_point<REALK>(K, x, y, 1.0 / 24.0, al, be, acc);
  }
}

template <bool REALK>
__device__ __forceinline__ void rule16(const FieldK &K, const double *x, const double (*V)[3], z al, const z *be,
                                       double *acc) {
#pragma unroll 1
  for (int i = 0; i < 16; i++) {
    const double *u = c_fr16 + 4 * i;
    double y[3];
#pragma unroll
    for (int c = 0; c < 3; c++)
      y[c] = V[0][c] + u[0] * (V[1][c] - V[0][c]) + u[1] * (V[2][c] - V[0][c]) + u[2] * (V[3][c] - V[0][c]);
    field_point<REALK>(K, x, y, u[3], al, be, acc);
  }
}

// g_k per tetrahedron from the basis-function coefficients
__global__ void k_fields_coef(DevGeom g, const z *J, z *coef) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.NT) return;
  int4 fi = g.tetFI[t];
  int f[4] = {fi.x, fi.y, fi.z, fi.w};
#pragma unroll
  for (int k = 0; k < 4; k++) {
    z v{0.0, 0.0};
    int a = f[k];
    if (a >= 0) {
      double s = (g.bfTet[a].x == t ? 2.0 : -2.0) * g.bfArea[a];
      z Ja = J[a];
      v = z{s * Ja.r, s * Ja.i};
    }
    coef[4 * t + k] = v;
  }
}

// one tetrahedron's data for the field sums: vertices, the all-faces-far
// sphere, and the linear current alpha y - beta of all its basis functions
struct TetData {
  double V[4][3], ctr[3], Rall;
  z al, be[3];
};

__device__ __forceinline__ void load_tet(const double *__restrict__ tetT, const z *__restrict__ coef, int t,
                                         TetData &T) {
  const double2 *T2 = reinterpret_cast<const double2 *>(tetT + 16 * (size_t)t);
  double2 a0 = T2[0], a1 = T2[1], a2 = T2[2], a3 = T2[3], a4 = T2[4], a5 = T2[5], a6 = T2[6], a7 = T2[7];
  T.V[0][0] = a0.x; T.V[0][1] = a0.y; T.V[0][2] = a1.x; T.V[1][0] = a1.y; T.V[1][1] = a2.x; T.V[1][2] = a2.y;
  T.V[2][0] = a3.x; T.V[2][1] = a3.y; T.V[2][2] = a4.x; T.V[3][0] = a4.y; T.V[3][1] = a5.x; T.V[3][2] = a5.y;
  T.ctr[0] = a6.x; T.ctr[1] = a6.y; T.ctr[2] = a7.x; T.Rall = a7.y;
  T.al = z{0.0, 0.0};
#pragma unroll
  for (int c = 0; c < 3; c++) T.be[c] = z{0.0, 0.0};
#pragma unroll
  for (int k = 0; k < 4; k++) {
    z gk = coef[4 * (size_t)t + k];
    T.al.r += gk.r; T.al.i += gk.i;
#pragma unroll
    for (int c = 0; c < 3; c++) { T.be[c].r += gk.r * T.V[k][c]; T.be[c].i += gk.i * T.V[k][c]; }
  }
}

// fields at x of tetrahedron t (data T): the 4-point rule for all of it when
// every face is far, else split by face with the reference's rule choice
template <bool REALK>
__device__ __forceinline__ void tet_point(const FieldK &K, const double *x, const TetData &T,
                                          const double *__restrict__ tetF, const z *__restrict__ coef, int t,
                                          double *acc) {
  double d2 = (x[0] - T.ctr[0]) * (x[0] - T.ctr[0]) + (x[1] - T.ctr[1]) * (x[1] - T.ctr[1]) +
              (x[2] - T.ctr[2]) * (x[2] - T.ctr[2]);
  if (d2 > T.Rall * T.Rall) {
    rule4<REALK>(K, x, T.V, T.al, T.be, acc);
    return;
  }
  // per face: the reference's rule choice |X - centroid| / radius > 10
  z a4{0.0, 0.0}, b4[3] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
  z a16{0.0, 0.0}, b16[3] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
  bool any4 = false, any16 = false;
  const double4 *F4 = reinterpret_cast<const double4 *>(tetF + 16 * (size_t)t);
#pragma unroll
  for (int k = 0; k < 4; k++) {
    double4 f = F4[k];
    z gk = coef[4 * (size_t)t + k];
    double dx = x[0] - f.x, dy = x[1] - f.y, dz = x[2] - f.z;
    bool live = f.w != 0.0;
    bool far = live && sqrt(dx * dx + dy * dy + dz * dz) / f.w > 10.0;
    bool near = live && !far;
    double m4 = far ? 1.0 : 0.0, m16 = near ? 1.0 : 0.0;
    a4.r += m4 * gk.r; a4.i += m4 * gk.i;
    a16.r += m16 * gk.r; a16.i += m16 * gk.i;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      b4[c].r += m4 * gk.r * T.V[k][c]; b4[c].i += m4 * gk.i * T.V[k][c];
      b16[c].r += m16 * gk.r * T.V[k][c]; b16[c].i += m16 * gk.i * T.V[k][c];
    }
    any4 |= far;
    any16 |= near;
  }
  if (any4) rule4<REALK>(K, x, T.V, a4, b4, acc);
  if (any16) rule16<REALK>(K, x, T.V, a16, b16, acc);
}

// warp sum of the 12 accumulators of point p into the warp's shared slot
__device__ __forceinline__ void warp_flush(double *acc, double (*slot)[12], int p, int lane) {
#pragma unroll
  for (int q = 0; q < 12; q++) {
    double v = acc[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    acc[q] = v;
  }
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < 12; q++) slot[p][q] = acc[q];
  }
}

template <bool REALK, bool ONE>
__global__ void __launch_bounds__(FTHREADS, 3)
k_fields(const double *__restrict__ tetT, const double *__restrict__ tetF, const z *__restrict__ coef, int NT,
         int tpt, const double *__restrict__ X, int P, FieldK K, double *__restrict__ part) {
  __shared__ double sx[FPCH][3];
  __shared__ double sacc[FTHREADS / 32][FPCH][12];
  int p0 = blockIdx.x * FPCH, np = min(FPCH, P - p0);
  for (int i = threadIdx.x; i < 3 * np; i += FTHREADS) sx[i / 3][i % 3] = X[3 * p0 + i];
  __syncthreads();
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int tbase = blockIdx.y * FTHREADS * tpt + threadIdx.x;
  if (ONE) {
    // one tetrahedron per thread: its data stays in registers for all points
    bool live = tbase < NT;
    TetData T;
    if (live) load_tet(tetT, coef, tbase, T);
    for (int p = 0; p < np; p++) {
      double x[3] = {sx[p][0], sx[p][1], sx[p][2]};
      double acc[12];
#pragma unroll
      for (int q = 0; q < 12; q++) acc[q] = 0.0;
      if (live) tet_point<REALK>(K, x, T, tetF, coef, tbase, acc);
      warp_flush(acc, sacc[warp], p, lane);
    }
  } else {
    for (int p = 0; p < np; p++) {
      double x[3] = {sx[p][0], sx[p][1], sx[p][2]};
      double acc[12];
#pragma unroll
      for (int q = 0; q < 12; q++) acc[q] = 0.0;
      for (int j = 0; j < tpt; j++) {
        int t = tbase + j * FTHREADS;
        if (t >= NT) break;
        TetData T;
        load_tet(tetT, coef, t, T);
        tet_point<REALK>(K, x, T, tetF, coef, t, acc);
      }
      warp_flush(acc, sacc[warp], p, lane);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 12 * np; i += FTHREADS) {
    int p = i / 12, q = i % 12;
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < FTHREADS / 32; w++) s += sacc[w][p][q];
    part[((size_t)blockIdx.y * P + p0 + p) * 12 + q] = s;
  }
}

struct FieldInc { z E0[3]; double nh[3]; int on; };

__global__ void k_fields_finish(const double *__restrict__ part, int nblk, int P, const double *__restrict__ X,
                                FieldK K, z epre, FieldInc inc, z *out) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  double s[12];
  for (int q = 0; q < 12; q++) s[q] = 0.0;
  for (int b = 0; b < nblk; b++)
    for (int q = 0; q < 12; q++) s[q] += part[((size_t)b * P + p) * 12 + q];
  z F[6];
  const double inv4pi = 0.25 / M_PI;
  for (int c = 0; c < 3; c++) {
    F[c] = zmul(epre, z{s[2 * c], s[2 * c + 1]});
    F[3 + c] = z{inv4pi * s[6 + 2 * c], inv4pi * s[7 + 2 * c]};
  }
  if (inc.on) {
    double ph = inc.nh[0] * X[3 * p] + inc.nh[1] * X[3 * p + 1] + inc.nh[2] * X[3 * p + 2];
    double sn, cs;
    sincos(K.k.r * ph, &sn, &cs);
    double m = K.k.i == 0.0 ? 1.0 : exp(-K.k.i * ph);
    z e{m * cs, m * sn}, E[3];
    for (int c = 0; c < 3; c++) E[c] = zmul(inc.E0[c], e);
    const double *n = inc.nh;
    z H[3] = {{(n[1] * E[2].r - n[2] * E[1].r) / ZVAC_F, (n[1] * E[2].i - n[2] * E[1].i) / ZVAC_F},
              {(n[2] * E[0].r - n[0] * E[2].r) / ZVAC_F, (n[2] * E[0].i - n[0] * E[2].i) / ZVAC_F},
              {(n[0] * E[1].r - n[1] * E[0].r) / ZVAC_F, (n[0] * E[1].i - n[1] * E[0].i) / ZVAC_F}};
    for (int c = 0; c < 3; c++) {
      F[c].r += E[c].r; F[c].i += E[c].i;
      F[3 + c].r += H[c].r; F[3 + c].i += H[c].i;
    }
  }
  for (int c = 0; c < 6; c++) out[6 * (size_t)p + c] = F[c];
}

}  // namespace

// per-tetrahedron field tables, built on first use
static int field_tables(bg_geometry *g) {
  if (g->d_fieldTet && g->d_fieldFace) return BG_OK;
  std::vector<double> T, F;
  T.reserve(16 * (size_t)g->NT);
  F.reserve(16 * (size_t)g->NT);
  for (const Object &o : g->objs) {
    for (int t = 0; t < o.nt; t++) {
      double ctr[3] = {0, 0, 0};
      for (int k = 0; k < 4; k++)
        for (int c = 0; c < 3; c++) {
          double v = o.V[3 * o.VI[4 * t + k] + c];
          T.push_back(v);
          ctr[c] += 0.25 * v;
        }
      double Rall = 0.0;
      for (int k = 0; k < 4; k++) {
        int f = o.FI[4 * t + k];
        if (f >= 0 && f < o.nif) {
          const Face &Fc = o.F[f];
          double d = std::sqrt((Fc.cen[0] - ctr[0]) * (Fc.cen[0] - ctr[0]) + (Fc.cen[1] - ctr[1]) * (Fc.cen[1] - ctr[1]) +
                               (Fc.cen[2] - ctr[2]) * (Fc.cen[2] - ctr[2]));
          Rall = std::fmax(Rall, 10.0 * Fc.radius + d);
          F.insert(F.end(), {Fc.cen[0], Fc.cen[1], Fc.cen[2], Fc.radius});
        } else {
          F.insert(F.end(), {0.0, 0.0, 0.0, 0.0});
        }
      }
      // margin so that rounding never calls a face far that the per-face test would not
      Rall = Rall * (1.0 + 1e-12) + 1e-300;
      T.insert(T.end(), {ctr[0], ctr[1], ctr[2], Rall});
    }
  }
  double *dT = nullptr, *dF = nullptr;
  cudaError_t e = cudaMalloc(&dT, sizeof(double) * T.size());
  if (e == cudaSuccess) e = cudaMalloc(&dF, sizeof(double) * F.size());
  if (e == cudaSuccess) e = cudaMemcpy(dT, T.data(), sizeof(double) * T.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dF, F.data(), sizeof(double) * F.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    // both tables or neither: a failed build leaves the geometry as it was
    cudaFree(dT);
    cudaFree(dF);
    set_error("GetFields tables: %s", cudaGetErrorString(e));
    return BG_ERR_CUDA;
  }
  g->d_fieldTet = dT;
  g->d_fieldFace = dF;
  return BG_OK;
}

int get_fields(bg_geometry *g, double wr, double wi, const void *dJ, const double *E0, const double *nhat,
               int npts, const double *dX, void *dOut) {
  int st = upload_geometry(g);
  if (st || (st = init_rule16()) || (st = field_tables(g))) return st;
  if (npts == 0) return BG_OK;
  FieldK K;
  K.k = z{wr, wi};
  K.ik = z{-wi, wr};
  double d = wr * wr + wi * wi;
  K.invik = z{-wi / d, -wr / d};      // 1/(ik) = -i/k
  // i w Z0 / (4 pi)
  const double f = ZVAC_F * 0.25 / M_PI;
  z epre{-wi * f, wr * f};
  FieldInc inc{};
  if (E0 && nhat) {
    inc.on = 1;
    for (int c = 0; c < 3; c++) { inc.E0[c] = z{E0[2 * c], E0[2 * c + 1]}; inc.nh[c] = nhat[c]; }
  }
  int NT = g->NT;
  int ny = (npts + FPCH - 1) / FPCH, tpt = 1;
  int nbx = dJ ? (NT + FTHREADS - 1) / FTHREADS : 0;
  // one tetrahedron per thread (data in registers) while the partial sums
  // (96 bytes per tetrahedron block and point) stay under 256 MiB; beyond
  // that, longer tetrahedron blocks until the grid is about 8 blocks per SM,
  // which amortises the per-point warp reductions over many tetrahedra
  bool one = 96.0 * nbx * npts <= 268435456.0 && nbx <= 65535;
  while (!one && (nbx > 65535 || (nbx > 1 && (long)nbx * ny > 8L * 148))) {
    tpt *= 2;
    nbx = (NT + FTHREADS * tpt - 1) / (FTHREADS * tpt);
  }
  double *part = nullptr;
  z *coef = nullptr;
  if (nbx) {
    BG_CUDA_TRY(cudaMallocAsync(&part, sizeof(double) * 12 * (size_t)nbx * npts, stream()));
    cudaError_t e = cudaMallocAsync(&coef, sizeof(z) * 4 * (size_t)NT, stream());
    if (e != cudaSuccess) {
      cudaFreeAsync(part, stream());
      set_error("GetFields scratch: %s", cudaGetErrorString(e));
      return BG_ERR_CUDA;
    }
    k_fields_coef<<<(NT + 255) / 256, 256, 0, stream()>>>(g->dev, (const z *)dJ, coef);
    BG_LAUNCHED();
    dim3 grid(ny, nbx);
    auto kern = wi == 0.0 ? (one ? k_fields<true, true> : k_fields<true, false>)
                          : (one ? k_fields<false, true> : k_fields<false, false>);
    kern<<<grid, FTHREADS, 0, stream()>>>(g->d_fieldTet, g->d_fieldFace, coef, NT, tpt, dX, npts, K, part);
    BG_LAUNCHED();
  }
  k_fields_finish<<<(npts + 127) / 128, 128, 0, stream()>>>(part, nbx, npts, dX, K, epre, inc, (z *)dOut);
  BG_LAUNCHED();
  if (part) cudaFreeAsync(part, stream());
  if (coef) cudaFreeAsync(coef, stream());
  return BG_OK;
}

}  // namespace bg
