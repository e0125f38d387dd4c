// sm_100a kernels of the VIE assembly path: far-field G entries, the
// frequency-independent near-field integrals (regular 16x16 rule and the
// singular relative-coordinate rule, both as tetrahedron-pair moments), the
// per-frequency near entries, V^-1 Gram blocks, plane-wave RHS and the
// absorbed/scattered power (EMT and overlap).
//
// Reference semantics (HomerReid/buff-em, src/libs/libbuff):
//   GMatrixElements.cc:59-167,270-424   kernels and dispatcher
//   Cubature.cc:161-527, TetCR.cc:35-95 fixed tetrahedron rules
//   VIEMatrix.cc:51-72,122-316,321-460  Gram blocks and assembly
//   RHSVector.cc:62-124                 plane-wave RHS
//   EMTPFT.cc:151-493, OPFT.cc:62-119   power
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <vector>

#include "internal.h"

namespace bg {

// ----------------------------------------------------------------- tables
// Fixed tetrahedron rules (TetCR.cc:35-95): points (u1,u2,u3) in the unit
// simplex, weights summing to 1/6.  All orbits are complete, so the point set
// does not depend on which vertex is taken as origin.
__constant__ double c_tcr16[64];
__constant__ double c_tcr33[132];
static double h_tcr16[64], h_tcr33[132];
static int s_tables_ok = 0;

static void fill_rule(double *dst, const char *pat, const double *vals, double w, int *np) {
  for (const char *p = pat; *p;) {
    if (*p == ' ') { p++; continue; }
    double *q = dst + 4 * (*np);
    q[0] = vals[p[0] - 'A']; q[1] = vals[p[1] - 'A']; q[2] = vals[p[2] - 'A']; q[3] = w;
    (*np)++;
    p += 3;
  }
}

static int init_tables() {
  if (s_tables_ok) return BG_OK;
  int np;
  const double v16[5] = {0.771642902067237, 0.076119032644254315, 0.07183164526766925, 0.11970052779780202,
                         0.40423391346726440};
  np = 0;
  fill_rule(h_tcr16, "ABB BAB BBA BBB", v16, 8.3956323500204695e-3, &np);
  fill_rule(h_tcr16, "CDE CED CEE DCE DEC DEE ECD ECE EDC EDE EEC EED", v16, 0.011090344772215399, &np);
  const double v33[11] = {0.25, 0.31407428362944793, 0.05777714911165610, 0.06254680497480394,
                          0.81235958507558810, 0.04120213879937276, 0.30021473119185615, 0.61738099120939840,
                          0.05292032110257111, 0.25198057383388334, 0.44311853122966216};
  np = 0;
  fill_rule(h_tcr33, "AAA", v33, 0.017783308938202055, &np);
  fill_rule(h_tcr33, "BBB CBB BCB BBC", v33, -0.019099406118263309, &np);
  fill_rule(h_tcr33, "DDD EDD DED DDE", v33, 3.8252276536630236e-3, &np);
  fill_rule(h_tcr33, "FFG FFH FGF FGH FHF FHG GFF GFH GHF HFF HFG HGF", v33, 0.0035475499144103266, &np);
  fill_rule(h_tcr33, "IJJ IJK IKJ JIJ JIK JJI JJK JKI JKJ KIJ KJI KJJ", v33, 0.013950789384495153, &np);
  BG_CUDA_TRY(cudaMemcpyToSymbol(c_tcr16, h_tcr16, sizeof h_tcr16));
  BG_CUDA_TRY(cudaMemcpyToSymbol(c_tcr33, h_tcr33, sizeof h_tcr33));
  s_tables_ok = 1;
  return BG_OK;
}

void gauss_legendre01(int n, double *x, double *w) {
  for (int i = 0; i < n; i++) {
    double z = std::cos(M_PI * (i + 0.75) / (n + 0.5)), pp = 0.0;
    for (int it = 0; it < 100; it++) {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 1; j <= n; j++) {
        double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      double z1 = z;
      z = z1 - p1 / pp;
      if (std::fabs(z - z1) < 1e-16) break;
    }
    x[i] = 0.5 * (1.0 - z);
    w[i] = 1.0 / ((1.0 - z * z) * pp * pp);
  }
}

// ----------------------------------------------------------------- complex
struct cd { double r, i; };
__device__ __forceinline__ cd cmk(double r, double i) { return cd{r, i}; }
__device__ __forceinline__ cd cadd(cd a, cd b) { return cd{a.r + b.r, a.i + b.i}; }
__device__ __forceinline__ cd csub(cd a, cd b) { return cd{a.r - b.r, a.i - b.i}; }
__device__ __forceinline__ cd cmul(cd a, cd b) { return cd{a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r}; }
__device__ __forceinline__ cd cscale(cd a, double s) { return cd{a.r * s, a.i * s}; }
__device__ __forceinline__ cd cdiv(cd a, cd b) {
  double d = b.r * b.r + b.i * b.i;
  return cd{(a.r * b.r + a.i * b.i) / d, (a.i * b.r - a.r * b.i) / d};
}
__device__ __forceinline__ double cnorm2(cd a) { return a.r * a.r + a.i * a.i; }
// exp(i k r) for complex k
__device__ __forceinline__ cd expikr(cd k, double r) {
  double s, c;
  sincos(k.r * r, &s, &c);
  double m = (k.i == 0.0) ? 1.0 : exp(-k.i * r);
  return cd{m * c, m * s};
}

// exp(i x) for |x| <= 1: Taylor series of cos and sin at y = x/2 in Horner
// form (one fused multiply-add per term), then cos x = c^2 - s^2,
// sin x = 2 c s.  Terms to y^14 / y^15: the first omitted terms, y^16/16!
// and y^17/17!, are below 1e-18 for |y| <= 1/2.  expi_small_short serves
// |x| <= 1/4 (|y| <= 1/8) with terms to y^10 / y^11 (first omitted terms
// below 2e-20).
#define EXPI_C(n, f) (((n) & 1 ? -1.0 : 1.0) / (f))
__device__ __forceinline__ cd expi_halfangle(double c, double sn) { return cd{c * c - sn * sn, 2.0 * c * sn}; }
__device__ __forceinline__ cd expi_small(double x) {
  double y = 0.5 * x, y2 = y * y;
  double c = EXPI_C(7, 87178291200.0);           // 1/14!
  c = fma(c, y2, EXPI_C(6, 479001600.0));        // 1/12!
  c = fma(c, y2, EXPI_C(5, 3628800.0));
  c = fma(c, y2, EXPI_C(4, 40320.0));
  c = fma(c, y2, EXPI_C(3, 720.0));
  c = fma(c, y2, EXPI_C(2, 24.0));
  c = fma(c, y2, EXPI_C(1, 2.0));
  c = fma(c, y2, 1.0);
  double sn = EXPI_C(7, 1307674368000.0);        // 1/15!
  sn = fma(sn, y2, EXPI_C(6, 6227020800.0));     // 1/13!
  sn = fma(sn, y2, EXPI_C(5, 39916800.0));
  sn = fma(sn, y2, EXPI_C(4, 362880.0));
  sn = fma(sn, y2, EXPI_C(3, 5040.0));
  sn = fma(sn, y2, EXPI_C(2, 120.0));
  sn = fma(sn, y2, EXPI_C(1, 6.0));
  sn = fma(sn, y2, 1.0) * y;
  return expi_halfangle(c, sn);
}
__device__ __forceinline__ cd expi_small_short(double x) {
  double y = 0.5 * x, y2 = y * y;
  double c = EXPI_C(5, 3628800.0);               // 1/10!
  c = fma(c, y2, EXPI_C(4, 40320.0));
  c = fma(c, y2, EXPI_C(3, 720.0));
  c = fma(c, y2, EXPI_C(2, 24.0));
  c = fma(c, y2, EXPI_C(1, 2.0));
  c = fma(c, y2, 1.0);
  double sn = EXPI_C(5, 39916800.0);             // 1/11!
  sn = fma(sn, y2, EXPI_C(4, 362880.0));
  sn = fma(sn, y2, EXPI_C(3, 5040.0));
  sn = fma(sn, y2, EXPI_C(2, 120.0));
  sn = fma(sn, y2, EXPI_C(1, 6.0));
  sn = fma(sn, y2, 1.0) * y;
  return expi_halfangle(c, sn);
}

// e^x - 1 - x - x^2/2: GetExpRelTable(x,3,3), GMatrixElements.cc:59-93 -- the
// series from n=4 is stopped once |term|^2 < 1e-16 |sum|^2 (or n = 100).
__device__ __forceinline__ cd exprel3(cd x) {
  cd term = cmul(cscale(x, 0.5), x);   // x^2/2
  term = cmul(term, cscale(x, 1.0 / 3.0));
  cd first = term, sum = cmk(0, 0);
  for (int n = 4; n < 100; n++) {
    term = cmul(term, cscale(x, 1.0 / n));
    sum = cadd(sum, term);
    if (cnorm2(term) < 1.0e-16 * cnorm2(sum)) break;
  }
  return cadd(first, sum);
}

// complex functions of the SVTENSOR programs, from their definitions in
// terms of the real exp, log, sincos, sinh, cosh, sqrt, hypot and atan2
__device__ cd cx_exp(cd z) {
  double s, c, e = exp(z.r);
  sincos(z.i, &s, &c);
  return cd{e * c, e * s};
}
__device__ cd cx_log(cd z) { return cd{log(hypot(z.r, z.i)), atan2(z.i, z.r)}; }
__device__ cd cx_sqrt(cd z) {   // principal branch
  double r = hypot(z.r, z.i);
  if (r == 0.0) return cd{0.0, 0.0};
  if (z.r >= 0.0) {
    double t = sqrt(0.5 * (r + z.r));
    return cd{t, z.i / (2.0 * t)};
  }
  double t = sqrt(0.5 * (r - z.r));
  return cd{fabs(z.i) / (2.0 * t), copysign(t, z.i)};
}
__device__ cd cx_sin(cd z) {
  double s, c;
  sincos(z.r, &s, &c);
  return cd{s * cosh(z.i), c * sinh(z.i)};
}
__device__ cd cx_cos(cd z) {
  double s, c;
  sincos(z.r, &s, &c);
  return cd{c * cosh(z.i), -s * sinh(z.i)};
}
__device__ cd cx_sinh(cd z) {
  double s, c;
  sincos(z.i, &s, &c);
  return cd{sinh(z.r) * c, cosh(z.r) * s};
}
__device__ cd cx_cosh(cd z) {
  double s, c;
  sincos(z.i, &s, &c);
  return cd{cosh(z.r) * c, sinh(z.r) * s};
}
// asin z = -i log(iz + sqrt(1 - z^2)), acos z = pi/2 - asin z,
// atan z = (i/2) [log(1 - iz) - log(1 + iz)]
__device__ cd cx_asin(cd z) {
  cd w = cx_log(cadd(cd{-z.i, z.r}, cx_sqrt(csub(cd{1.0, 0.0}, cmul(z, z)))));
  return cd{w.i, -w.r};
}
__device__ cd cx_atan(cd z) {
  cd a = cx_log(cd{1.0 + z.i, -z.r}), b = cx_log(cd{1.0 - z.i, z.r});
  cd d = csub(a, b);
  return cd{-0.5 * d.i, 0.5 * d.r};
}
__device__ cd cx_pow(cd x, cd y) {
  // integer powers by repeated squaring, as the host evaluator (matprop.cpp)
  if (y.i == 0.0 && y.r == floor(y.r) && fabs(y.r) <= 64.0) {
    long n = (long)y.r;
    bool inv = n < 0;
    unsigned long m = inv ? (unsigned long)(-n) : (unsigned long)n;
    cd r{1.0, 0.0};
    while (m) {
      if (m & 1) r = cmul(r, x);
      x = cmul(x, x);
      m >>= 1;
    }
    return inv ? cdiv(cd{1.0, 0.0}, r) : r;
  }
  return cx_exp(cmul(y, cx_log(x)));
}

// one component program of a compiled SVTENSOR (DevExpr) at point x
__device__ cd expr_eval(const DevExpr &e, int comp, const double *x) {
  cd st[BG_EXPR_STACK];
  int sp = 0;
  const int b = e.start[comp], n = e.len[comp];
  for (int k = 0; k < n; k++) {
    const int w = e.op[b + k], code = w >> 16, arg = w & 0xffff;
    switch (code) {
      case 0: st[sp++] = cd{e.con[2 * arg], e.con[2 * arg + 1]}; break;
      case 1: {
        double v;
        if (arg < 3) v = x[arg];
        else if (arg == 3) v = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
        else if (arg == 4) v = atan2(sqrt(x[0] * x[0] + x[1] * x[1]), x[2]);
        else v = atan2(x[1], x[0]);
        st[sp++] = cd{v, 0.0};
        break;
      }
      case 2: st[sp - 1] = csub(cd{0.0, 0.0}, st[sp - 1]); break;
      case 8: {
        cd a = st[sp - 1], r;
        switch (arg) {
          case 0: r = cx_exp(a); break;
          case 1: r = cx_log(a); break;
          case 2: r = cx_sqrt(a); break;
          case 3: r = cx_sin(a); break;
          case 4: r = cx_cos(a); break;
          case 5: r = cdiv(cx_sin(a), cx_cos(a)); break;
          case 6: r = cx_sinh(a); break;
          case 7: r = cx_cosh(a); break;
          case 8: r = cdiv(cx_sinh(a), cx_cosh(a)); break;
          case 9: r = cx_asin(a); break;
          case 10: r = csub(cd{0.5 * M_PI, 0.0}, cx_asin(a)); break;
          case 11: r = cx_atan(a); break;
          case 12: r = cd{hypot(a.r, a.i), 0.0}; break;
          default: r = cd{a.r < 0.0 ? 0.0 : 1.0, 0.0}; break;
        }
        st[sp - 1] = r;
        break;
      }
      default: {
        cd bb = st[--sp], aa = st[sp - 1];
        st[sp - 1] = code == 3 ? cadd(aa, bb) : code == 4 ? csub(aa, bb) : code == 5 ? cmul(aa, bb)
                   : code == 6 ? cdiv(aa, bb) : cx_pow(aa, bb);
        break;
      }
    }
  }
  return st[0];
}

// permittivity functor (SVTensor::Evaluate semantics, SVTensor.cc:306-373);
// ex: the object's compiled program when m.kind == BG_MAT_EXPR
__device__ void mat_eval(const bg_material &m, const DevExpr *ex, const double *x, cd E[3][3]) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) E[i][j] = cmk(0, 0);
  if (m.kind == BG_MAT_EXPR) {
    // components not given keep the identity, off-diagonal pairs are
    // averaged, yy and zz follow xx when only xx is given (SVTensor.cc:344-372)
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++)
        E[i][j] = ex->len[3 * i + j] ? expr_eval(*ex, 3 * i + j, x) : cmk(i == j ? 1.0 : 0.0, 0.0);
    for (int mu = 0; mu < 3; mu++) {
      int nu = (mu + 1) % 3;
      cd a = cscale(cadd(E[mu][nu], E[nu][mu]), 0.5);
      E[mu][nu] = E[nu][mu] = a;
    }
    if (ex->len[0]) {
      if (!ex->len[4]) E[1][1] = E[0][0];
      if (!ex->len[8]) E[2][2] = E[0][0];
    }
    return;
  }
  if (m.kind == BG_MAT_CONST_TENSOR) {
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) E[i][j] = cmk(m.eps[2 * (3 * i + j)], m.eps[2 * (3 * i + j) + 1]);
    for (int mu = 0; mu < 3; mu++) {
      int nu = (mu + 1) % 3;
      cd a = cscale(cadd(E[mu][nu], E[nu][mu]), 0.5);
      E[mu][nu] = E[nu][mu] = a;
    }
    return;
  }
  cd e;
  if (m.kind == BG_MAT_CONST_ISO) e = cmk(m.eps[0], m.eps[1]);
  else if (m.kind == BG_MAT_JANUS_Z) e = (x[2] > m.center[2]) ? cmk(m.eps[0], m.eps[1]) : cmk(m.eps2[0], m.eps2[1]);
  else {
    double d0 = x[0] - m.center[0], d1 = x[1] - m.center[1], d2 = x[2] - m.center[2];
    double r2 = (d0 * d0 + d1 * d1 + d2 * d2) / (m.width * m.width);
    double g = exp(-r2);
    e = cmk(m.eps[0] + m.amp[0] * g, m.eps[1] + m.amp[1] * g);
  }
  E[0][0] = E[1][1] = E[2][2] = e;
}

// Invert3x3Matrix, VIEMatrix.cc:51-72
__device__ void inv3(cd M[3][3], cd W[3][3]) {
  cd M11 = M[0][0], M12 = M[0][1], M13 = M[0][2];
  cd M21 = M[1][0], M22 = M[1][1], M23 = M[1][2];
  cd M31 = M[2][0], M32 = M[2][1], M33 = M[2][2];
  cd Det = csub(csub(csub(cadd(cadd(cmul(cmul(M12, M23), M31), cmul(cmul(M13, M21), M32)), cmul(cmul(M11, M22), M33)),
                          cmul(cmul(M13, M22), M31)),
                     cmul(cmul(M11, M23), M32)),
                cmul(cmul(M12, M21), M33));
  W[0][0] = cdiv(csub(cmul(M22, M33), cmul(M23, M32)), Det);
  W[0][1] = cdiv(csub(cmul(M13, M32), cmul(M12, M33)), Det);
  W[0][2] = cdiv(csub(cmul(M12, M23), cmul(M13, M22)), Det);
  W[1][0] = cdiv(csub(cmul(M23, M31), cmul(M21, M33)), Det);
  W[1][1] = cdiv(csub(cmul(M11, M33), cmul(M13, M31)), Det);
  W[1][2] = cdiv(csub(cmul(M13, M21), cmul(M11, M23)), Det);
  W[2][0] = cdiv(csub(cmul(M21, M32), cmul(M22, M31)), Det);
  W[2][1] = cdiv(csub(cmul(M12, M31), cmul(M11, M32)), Det);
  W[2][2] = cdiv(csub(cmul(M11, M22), cmul(M12, M21)), Det);
}

__device__ __forceinline__ void load3(const double *V4, int v, double *x) {
  x[0] = V4[4 * v]; x[1] = V4[4 * v + 1]; x[2] = V4[4 * v + 2];
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// =========================================================================
// far field (GetGME_BFBFInt, GMatrixElements.cc:270-288; BFBFInt,
// Cubature.cc:476-527): for a basis-function pair (a, b) with no common
// vertex, 4 tetrahedron pairs x 4x4 points of the Helmholtz kernel.  With
// w = 6V w_i (w_i = 1/24) and b = +-A/(3V)(x - Q) the volume cancels:
//   w_a b_a . w_b b_b = s_a s_b A_a A_b (x-Q_a).(y-Q_b)/144,
//   w_a Div b_a w_b Div b_b = s_a s_b A_a A_b / 16,
// so with x~ = x - o_A, y~ = y - o_B (o = tetrahedron centroid) and
// q = Q - o each tetrahedron pair contributes through 8 complex moments of
// phi = exp(ikr)/(4 pi r):
//   M0 = sum phi, M1 = sum x~ phi, M1' = sum y~ phi, M2 = sum x~.y~ phi,
//   entry += s s' A A' [M2/144 - M0/(16k^2) - q'.M1/144 - q.M1'/144 + q.q' M0/144].
// The moments depend on the two tetrahedra only, and a tile of 32
// consecutive basis functions touches about 29 distinct tetrahedra (face
// numbering follows the mesh), so a CTA computes each distinct tetrahedron
// pair of its 32 x 32 tile once (about 850 instead of 4096 pairs of 16
// kernel evaluations).  The thread that computes a pair's 8 moments forms,
// while they are in registers, the terms of every basis-function pair of
// the tile that uses it (side sa of row ra on tetrahedron iA, side sb of
// column rb on tetrahedron jB: term slot (ra, rb, 2 sa + sb), written by
// exactly one thread); after one barrier each basis-function pair adds its
// four slots in a fixed order.
// Phase: for real k, exp(ikr) = exp(ik rc) exp(ik (r - rc)) with rc the
// centroid distance and |r - rc| <= rA + rB (triangle inequality, rA the
// largest distance of a rule point from its centroid); when |k| (rA + rB)
// <= 1 the second factor is a short Taylor series (expi_small), so one
// sincos serves the 16 point pairs.
// =========================================================================
#define FT 16        // PFT tiles (k_pft_far): 16 x 16 basis functions
#define FTF BG_FAR_TILE
#define FTT BG_FAR_TILE_TETS
#define FTHR 256     // threads of the far kernel

struct FarSmem {
  cd slot[FTF][FTF][4];         // term (sa, sb) of the basis-function pair (row ra, column rb) of the tile
  double pA[FTT][4][3], pB[FTT][4][3];
  double oA[FTT][3], oB[FTT][3];
  double rA[FTT], rB[FTT];      // largest distance of a rule point from its centroid
  double uA[FTF][2][4], uB[FTF][2][4];   // s A (1, Q - o) per side
  int lA[FTF][2], lB[FTF][2];            // tile-local tetrahedron of each side, -1 past N
  int vA[FTF][5], vB[FTF][5];
  unsigned char sA[FTT][4], sB[FTT][4];  // sides on each tetrahedron: row << 1 | side
  int nsA[FTT], nsB[FTT];
};

// Frequency-parameterised launches: when fq (device, {Re w, Im w}) is
// given, the kernels below read omega from it instead of their by-value
// arguments, so that one captured CUDA graph serves every frequency.
__device__ __forceinline__ cd dev_invk2(double wr, double wi) {
  double d = (wr * wr - wi * wi) * (wr * wr - wi * wi) + 4 * wr * wr * wi * wi;
  return cd{(wr * wr - wi * wi) / d, -2 * wr * wi / d};
}

__device__ void far_stage_tets(const DevGeom &g, int tile, double (*P)[4][3], int tid) {
  int nt = g.tileNT[tile];
  for (int e = tid; e < nt * 12; e += FTHR) {
    int t = e / 12, r = e % 12;
    int tet = g.tileTet[(size_t)tile * FTT + t];
    P[t][r / 3][r % 3] = g.tetP4[16 * (size_t)tet + 4 * (r / 3) + (r % 3)];
  }
}

__device__ void far_stage_bfs(const DevGeom &g, int tile, double (*P)[4][3], double (*u)[2][4], int (*l)[2],
                              int (*v)[5], int tid) {
  if (tid < 2 * FTF) {
    int r = tid >> 1, s = tid & 1;
    int bf = tile * FTF + r;
    l[r][s] = -1;
    if (bf < g.N) {
      int2 loc = g.bfTileLoc[bf];
      int lt = s == 0 ? loc.x : loc.y;
      int2 qq = g.bfQ[bf];
      double Q[3];
      load3(g.V4, s == 0 ? qq.x : qq.y, Q);
      double coef = (s == 0 ? 1.0 : -1.0) * g.bfArea[bf];
      u[r][s][0] = coef;
      for (int c = 0; c < 3; c++) {
        double o = 0.25 * (P[lt][0][c] + P[lt][1][c] + P[lt][2][c] + P[lt][3][c]);
        u[r][s][1 + c] = coef * (Q[c] - o);
      }
      l[r][s] = lt;
      if (s == 0) {
        int4 vv = g.bfV[bf];
        v[r][0] = qq.x; v[r][1] = vv.x; v[r][2] = vv.y; v[r][3] = vv.z; v[r][4] = qq.y;
      }
    }
  }
}

// centroid, point radius and the sides resting on tetrahedron t of a tile
__device__ void far_stage_tet_info(int t, const double (*P)[4][3], double (*o)[3], double *rad, const int (*l)[2],
                                   unsigned char (*sides)[4], int *ns) {
  for (int c = 0; c < 3; c++) o[t][c] = 0.25 * (P[t][0][c] + P[t][1][c] + P[t][2][c] + P[t][3][c]);
  double r2 = 0.0;
  for (int i = 0; i < 4; i++) {
    double a2 = 0.0;
    for (int c = 0; c < 3; c++) {
      double d = P[t][i][c] - o[t][c];
      a2 += d * d;
    }
    r2 = fmax(r2, a2);
  }
  rad[t] = sqrt(r2);
  int n = 0;
  for (int r = 0; r < FTF; r++)
    for (int s = 0; s < 2; s++)
      if (l[r][s] == t && n < 4) sides[t][n++] = (unsigned char)(r << 1 | s);
  ns[t] = n;
}

// one CTA per 32 x 32 tile of basis-function pairs (upper triangle of tiles).
// MODE, the phase of exp(ikr) per point pair, fixed per launch so that one
// code path is compiled into each instantiation: 2 = ec * (short series)
// (|k| (rA + rB) <= 1/4 for every pair of the mesh), 1 = ec * (series)
// (<= 1), 0 = sincos per point pair (complex k or coarse pairs), 3 = chosen
// per tetrahedron pair (launches that read omega from device memory, whose
// frequency the host does not know when it launches them).
template <int MODE>
__global__ void __launch_bounds__(FTHR, 2) k_far(DevGeom g, cd k, cd invk2, cd *M, size_t ld, const double *fq,
                                                  float2 *F, size_t ldf) {
  if (fq) {
    k = cd{fq[0], fq[1]};
    invk2 = dev_invk2(fq[0], fq[1]);
  }
  int bx = blockIdx.x, by = blockIdx.y;
  if (bx > by) return;
  extern __shared__ __align__(16) unsigned char far_smem_raw[];
  FarSmem &S = *reinterpret_cast<FarSmem *>(far_smem_raw);
  const int tid = threadIdx.x;
  const int nA = g.tileNT[bx], nB = g.tileNT[by];
  far_stage_tets(g, bx, S.pA, tid);
  far_stage_tets(g, by, S.pB, tid);
  __syncthreads();
  far_stage_bfs(g, bx, S.pA, S.uA, S.lA, S.vA, tid);
  far_stage_bfs(g, by, S.pB, S.uB, S.lB, S.vB, tid);
  __syncthreads();
  if (tid < FTT) {
    if (tid < nA) far_stage_tet_info(tid, S.pA, S.oA, S.rA, S.lA, S.sA, S.nsA);
  } else if (tid < 2 * FTT) {
    if (tid - FTT < nB) far_stage_tet_info(tid - FTT, S.pB, S.oB, S.rB, S.lB, S.sB, S.nsB);
  }
  __syncthreads();
  const double inv4pi = 0.25 / M_PI;
  for (int p = tid; p < nA * nB; p += FTHR) {
    const int iA = p / nB, tB = p - iA * nB;
    cd m[8];
#pragma unroll
    for (int q = 0; q < 8; q++) m[q] = cmk(0, 0);
    // phase about the centroid distance rc (see above); mode 2: |k|(rA+rB)
    // <= 1/4 (every pair of a fine mesh at moderate frequency), mode 1:
    // <= 1, mode 0: a sincos per point pair.  1/(4 pi) rides on ec.
    const double e0 = S.oA[iA][0] - S.oB[tB][0], e1 = S.oA[iA][1] - S.oB[tB][1], e2 = S.oA[iA][2] - S.oB[tB][2];
    const double rc = sqrt(e0 * e0 + e1 * e1 + e2 * e2);
    const double span = fabs(k.r) * (S.rA[iA] + S.rB[tB]);
    const int mode = MODE != 3 ? MODE : (k.i != 0.0 ? 0 : (span <= 0.25 ? 2 : (span <= 1.0 ? 1 : 0)));
    const cd ec = mode ? cscale(expikr(k, rc), inv4pi) : cmk(inv4pi, 0.0);
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const double xt0 = S.pA[iA][i][0] - S.oA[iA][0], xt1 = S.pA[iA][i][1] - S.oA[iA][1],
                   xt2 = S.pA[iA][i][2] - S.oA[iA][2];
      cd phiI = cmk(0, 0);
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const double y0 = S.pB[tB][j][0], y1 = S.pB[tB][j][1], y2 = S.pB[tB][j][2];
        double R0 = S.pA[iA][i][0] - y0, R1 = S.pA[iA][i][1] - y1, R2 = S.pA[iA][i][2] - y2;
        double r2 = R0 * R0 + R1 * R1 + R2 * R2;
        if (r2 < 1.0e-24) continue;           // r < 1e-12
        double ir = rsqrt(r2), r = r2 * ir;   // one reciprocal square root instead of sqrt and a division
        cd ph = mode == 2 ? cmul(ec, expi_small_short(k.r * (r - rc)))
                          : (mode == 1 ? cmul(ec, expi_small(k.r * (r - rc))) : cscale(expikr(k, r), inv4pi));
        cd phi = cscale(ph, ir);
        const double yt0 = y0 - S.oB[tB][0], yt1 = y1 - S.oB[tB][1], yt2 = y2 - S.oB[tB][2];
        phiI = cadd(phiI, phi);
        m[4] = cadd(m[4], cscale(phi, yt0));
        m[5] = cadd(m[5], cscale(phi, yt1));
        m[6] = cadd(m[6], cscale(phi, yt2));
        m[7] = cadd(m[7], cscale(phi, xt0 * yt0 + xt1 * yt1 + xt2 * yt2));
      }
      m[0] = cadd(m[0], phiI);
      m[1] = cadd(m[1], cscale(phiI, xt0));
      m[2] = cadd(m[2], cscale(phiI, xt1));
      m[3] = cadd(m[3], cscale(phiI, xt2));
    }
    // terms of the basis-function pairs on (iA, tB):
    //   s s' A A' [M2/144 - M0/(16 k^2) - q'.M1/144 - q.M1'/144 + q.q' M0/144]
    const cd kM0 = cmul(invk2, m[0]);
    const int na = S.nsA[iA], nb = S.nsB[tB];
    for (int ia = 0; ia < na; ia++) {
      const int ca = S.sA[iA][ia], ra = ca >> 1, sa = ca & 1;
      const double *u = S.uA[ra][sa];
      const double u0 = u[0], u1 = u[1], u2 = u[2], u3 = u[3];
      // the row side's part: u0 M2 - u0 (.M1 with v) ... arranged per column below
      for (int ib = 0; ib < nb; ib++) {
        const int cb = S.sB[tB][ib], rb = cb >> 1, sb = cb & 1;
        const double *v = S.uB[rb][sb];
        double uv = u1 * v[1] + u2 * v[2] + u3 * v[3];
        cd t = cscale(m[7], u0 * v[0]);
        t = csub(t, cscale(cadd(cadd(cscale(m[1], v[1]), cscale(m[2], v[2])), cscale(m[3], v[3])), u0));
        t = csub(t, cscale(cadd(cadd(cscale(m[4], u1), cscale(m[5], u2)), cscale(m[6], u3)), v[0]));
        t = cadd(t, cscale(m[0], uv));
        t = csub(cscale(t, 1.0 / 144.0), cscale(kM0, u0 * v[0] / 16.0));
        S.slot[ra][rb][2 * sa + sb] = t;
      }
    }
  }
  __syncthreads();
  // this thread's 2 x 2 basis-function pairs: rows tx, tx + 16; columns ty, ty + 16
  const int tx = tid & 15, ty = tid >> 4;
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 2; j++) {
      int ra = tx + 16 * i, rb = ty + 16 * j;
      int a = bx * FTF + ra, b = by * FTF + rb;
      if (!(a < g.N && b < g.N && a <= b)) continue;
      // CompareBFs (SWGVolume.cc:295-344): pairs with a common vertex are near
      int ncv = 0;
      for (int p = 0; p < 5; p++)
        for (int q = 0; q < 5; q++) ncv += (S.vA[ra][p] == S.vB[rb][q]);
      if (ncv) continue;
      const cd *sl = S.slot[ra][rb];
      cd v = cadd(cadd(cadd(sl[0], sl[1]), sl[2]), sl[3]);
      M[(size_t)a + (size_t)b * ld] = v;
      if (a != b) M[(size_t)b + (size_t)a * ld] = v;
      if (F) {   // the complex64 copy, as k_c128_to_c64 would convert it
        const float2 f = make_float2((float)v.r, (float)v.i);
        F[(size_t)a + (size_t)b * ldf] = f;
        if (a != b) F[(size_t)b + (size_t)a * ldf] = f;
      }
    }
}

int assemble_far(bg_geometry *g, double wr, double wi, void *M, size_t ld, const double *fq, void *F, size_t ldf) {
  int st = init_tables();
  if (st) return st;
  cd k{wr, wi};
  // 1/k^2
  double d = (wr * wr - wi * wi) * (wr * wr - wi * wi) + 4 * wr * wr * wi * wi;
  cd invk2{(wr * wr - wi * wi) / d, -2 * wr * wi / d};
  int nb = (g->N + FTF - 1) / FTF;
  dim3 grid(nb, nb);
  static bool attr = false;
  if (!attr) {
    const int sm = (int)sizeof(FarSmem);
    BG_CUDA_TRY(cudaFuncSetAttribute(k_far<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    BG_CUDA_TRY(cudaFuncSetAttribute(k_far<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    BG_CUDA_TRY(cudaFuncSetAttribute(k_far<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    BG_CUDA_TRY(cudaFuncSetAttribute(k_far<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    attr = true;
  }
  // the largest phase span |k| (rA + rB) of any tetrahedron pair of the mesh
  const double span = std::fabs(wr) * 2.0 * g->rule_rmax;
  const int mode = fq ? 3 : (wi != 0.0 ? 0 : (span <= 0.25 ? 2 : (span <= 1.0 ? 1 : 0)));
  const size_t sm = sizeof(FarSmem);
  switch (mode) {
    case 0: k_far<0><<<grid, FTHR, sm, stream()>>>(g->dev, k, invk2, (cd *)M, ld, fq, (float2 *)F, ldf); break;
    case 1: k_far<1><<<grid, FTHR, sm, stream()>>>(g->dev, k, invk2, (cd *)M, ld, fq, (float2 *)F, ldf); break;
    case 2: k_far<2><<<grid, FTHR, sm, stream()>>>(g->dev, k, invk2, (cd *)M, ld, fq, (float2 *)F, ldf); break;
    default: k_far<3><<<grid, FTHR, sm, stream()>>>(g->dev, k, invk2, (cd *)M, ld, fq, (float2 *)F, ldf); break;
  }
  BG_LAUNCHED();
  return BG_OK;
}

// =========================================================================
// near field, frequency independent: tetrahedron-pair moments
//   M0 = sum K,  M1 = sum K (x-o_A),  M1' = sum K (y-o_B),  M2 = sum K (x-o_A).(y-o_B)
// for K in {1/(4 pi r), 1/(4 pi), r/(8 pi)} (GMEIntegrand KERNEL_STATIC,
// GMatrixElements.cc:153-165), in the unit-simplex measure (rule weights sum
// to 1/6 per tetrahedron).  Layout: 24 doubles per pair, [kernel][M0, M1(3),
// M1'(3), M2].  The per-basis-function-pair numbers of
// GetGME_TetTetInt(KERNEL_STATIC) follow from
//   int (x-Q).(y-Q') K = M2 - q.M1' - q'.M1 + q.q' M0,  q = Q-o_A, q' = Q'-o_B.
// =========================================================================

// regular pairs (<= 1 common vertex): 16x16 rule (GMatrixElements.cc:329-341),
// one warp per tetrahedron pair, origins o_A, o_B = first vertex of each tet.
__global__ void k_tp_regular(DevGeom g, const int4 *tp, int ntp, double *mom) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= ntp) return;
  int4 p = tp[warp];
  int4 A = g.tetVI[p.x], B = g.tetVI[p.y];
  double oA[3], oB[3], LA[3][3], LB[3][3];
  load3(g.V4, A.x, oA); load3(g.V4, B.x, oB);
  int va[3] = {A.y, A.z, A.w}, vb[3] = {B.y, B.z, B.w};
  for (int i = 0; i < 3; i++) {
    double t[3];
    load3(g.V4, va[i], t);
    for (int c = 0; c < 3; c++) LA[i][c] = t[c] - oA[c];
    load3(g.V4, vb[i], t);
    for (int c = 0; c < 3; c++) LB[i][c] = t[c] - oB[c];
  }
  double d0 = oA[0] - oB[0], d1 = oA[1] - oB[1], d2 = oA[2] - oB[2];
  double acc[24];
#pragma unroll
  for (int i = 0; i < 24; i++) acc[i] = 0.0;
  const double inv4pi = 0.25 / M_PI, inv8pi = 0.125 / M_PI;
  for (int idx = lane; idx < 256; idx += 32) {
    int i = idx >> 4, j = idx & 15;
    double xa[3], yb[3];
    for (int c = 0; c < 3; c++) {
      xa[c] = c_tcr16[4 * i] * LA[0][c] + c_tcr16[4 * i + 1] * LA[1][c] + c_tcr16[4 * i + 2] * LA[2][c];
      yb[c] = c_tcr16[4 * j] * LB[0][c] + c_tcr16[4 * j + 1] * LB[1][c] + c_tcr16[4 * j + 2] * LB[2][c];
    }
    double w = c_tcr16[4 * i + 3] * c_tcr16[4 * j + 3];
    double R0 = d0 + xa[0] - yb[0], R1 = d1 + xa[1] - yb[1], R2 = d2 + xa[2] - yb[2];
    double r = sqrt(R0 * R0 + R1 * R1 + R2 * R2);
    if (r < 1.0e-12) continue;
    double K[3] = {inv4pi / r, inv4pi, r * inv8pi};
    double xy = xa[0] * yb[0] + xa[1] * yb[1] + xa[2] * yb[2];
#pragma unroll
    for (int pk = 0; pk < 3; pk++) {
      double wk = w * K[pk];
      acc[8 * pk] += wk;
      acc[8 * pk + 1] += wk * xa[0]; acc[8 * pk + 2] += wk * xa[1]; acc[8 * pk + 3] += wk * xa[2];
      acc[8 * pk + 4] += wk * yb[0]; acc[8 * pk + 5] += wk * yb[1]; acc[8 * pk + 6] += wk * yb[2];
      acc[8 * pk + 7] += wk * xy;
    }
  }
#pragma unroll
  for (int i = 0; i < 24; i++) acc[i] = warp_sum(acc[i]);
  if (lane == 0)
    for (int i = 0; i < 24; i++) mom[24 * (size_t)warp + i] = acc[i];
}

// singular pairs (2..4 common vertices): singular.cu (singular_precompute)

// combine the 4 tetrahedron pairs of each near basis-function pair into the
// 6 numbers of GetGME_TetTetInt(KERNEL_STATIC) (GMatrixElements.cc:295-365):
// per kernel {4 A A' int (x-Q).(y-Q') K, 36 A A' int K} with sign +1 for PP/MM,
// -1 for PM/MP.
__device__ __forceinline__ void tp_origin(const DevGeom &g, const int4 *tp, const int4 *ordA, int id, bool first,
                                          double *o) {
  int4 p = tp[id];
  if (p.z >= 2) load3(g.V4, ordA[id].x, o);
  else load3(g.V4, first ? g.tetVI[p.x].x : g.tetVI[p.y].x, o);
}

__global__ void k_fibbi_combine(DevGeom g, NearData nd) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nd.npairs) return;
  int2 ab = nd.pairs[k];
  int a = ab.x, b = ab.y;
  int4 t4 = nd.pairTP[k];
  int tid[4] = {t4.x, t4.y, t4.z, t4.w};
  int2 qa = g.bfQ[a], qb = g.bfQ[b];
  double AA = g.bfArea[a] * g.bfArea[b];
  double out[6] = {0, 0, 0, 0, 0, 0};
  for (int sa = 0; sa < 2; sa++)
    for (int sb = 0; sb < 2; sb++) {
      int code = tid[2 * sa + sb];
      bool sw = (code >> 30) & 1;
      int id = code & ~(1 << 30);
      const double *M = nd.tpMom + 24 * (size_t)id;
      double ox[3], oy[3], Q[3], QP[3];
      tp_origin(g, nd.tp, nd.tpOrdA, id, !sw, ox);
      tp_origin(g, nd.tp, nd.tpOrdA, id, sw, oy);
      load3(g.V4, sa == 0 ? qa.x : qa.y, Q);
      load3(g.V4, sb == 0 ? qb.x : qb.y, QP);
      double q[3] = {Q[0] - ox[0], Q[1] - ox[1], Q[2] - ox[2]};
      double qp[3] = {QP[0] - oy[0], QP[1] - oy[1], QP[2] - oy[2]};
      double s = (sa == sb) ? 1.0 : -1.0;
      for (int pk = 0; pk < 3; pk++) {
        const double *m = M + 8 * pk;
        const double *m1 = sw ? m + 4 : m + 1;   // moment of the x (row) tetrahedron
        const double *m1p = sw ? m + 1 : m + 4;  // moment of the y (column) tetrahedron
        double J = m[7] - (q[0] * m1p[0] + q[1] * m1p[1] + q[2] * m1p[2]) -
                   (qp[0] * m1[0] + qp[1] * m1[1] + qp[2] * m1[2]) +
                   (q[0] * qp[0] + q[1] * qp[1] + q[2] * qp[2]) * m[0];
        out[2 * pk] += s * 4.0 * AA * J;
        out[2 * pk + 1] += s * 36.0 * AA * m[0];
      }
    }
  for (int i = 0; i < 6; i++) nd.fibbi[6 * (size_t)k + i] = out[i];
}

int precompute_near(bg_geometry *g) {
  int st = init_tables();
  if (st) return st;
  NearData &nd = g->near;
  if (nd.ntp_reg > 0) {
    int threads = 256, blocks = (nd.ntp_reg * 32 + threads - 1) / threads;
    k_tp_regular<<<blocks, threads, 0, stream()>>>(g->dev, nd.tp, nd.ntp_reg, nd.tpMom);
    BG_LAUNCHED();
  }
  if ((st = singular_precompute(g))) return st;
  if (nd.npairs > 0) {
    k_fibbi_combine<<<(nd.npairs + 127) / 128, 128, 0, stream()>>>(g->dev, nd);
    BG_LAUNCHED();
  }
  BG_CUDA_TRY(cudaStreamSynchronize(stream()));
  return BG_OK;
}

// =========================================================================
// near field per frequency: desingularised 64-point BF-pair integral plus the
// cached static numbers (GetGMatrixElement, GMatrixElements.cc:400-420):
//   G = BFBFInt[(e^{ikr}-1-ikr-(ikr)^2/2)/4 pi r] + (F0-F1/k^2) + ik(F2-F3/k^2)
//       + (ik)^2 (F4-F5/k^2)
// =========================================================================
__global__ void k_near(DevGeom g, NearData nd, cd k, cd invk2, cd *M, size_t ld, const double *fq, float2 *Fc,
                       size_t ldf) {
  if (fq) {
    k = cd{fq[0], fq[1]};
    invk2 = dev_invk2(fq[0], fq[1]);
  }
  int kk = blockIdx.x * blockDim.x + threadIdx.x;
  if (kk >= nd.npairs) return;
  int2 ab = nd.pairs[kk];
  int a = ab.x, b = ab.y;
  int2 ta = g.bfTet[a], tb = g.bfTet[b], qa = g.bfQ[a], qb = g.bfQ[b];
  double Aa = g.bfArea[a], Ab = g.bfArea[b];
  const double inv4pi = 0.25 / M_PI;
  cd ik = cmk(-k.i, k.r);
  cd acc = cmk(0, 0);
  for (int sa = 0; sa < 2; sa++) {
    int t1 = sa == 0 ? ta.x : ta.y;
    double Q[3];
    load3(g.V4, sa == 0 ? qa.x : qa.y, Q);
    for (int sb = 0; sb < 2; sb++) {
      int t2 = sb == 0 ? tb.x : tb.y;
      double QP[3];
      load3(g.V4, sb == 0 ? qb.x : qb.y, QP);
      double cc = (sa == 0 ? 1.0 : -1.0) * (sb == 0 ? 1.0 : -1.0) * Aa * Ab;
      cd part = cmk(0, 0);
      for (int i = 0; i < 4; i++) {
        const double *x = g.tetP4 + 16 * (size_t)t1 + 4 * i;
        for (int j = 0; j < 4; j++) {
          const double *y = g.tetP4 + 16 * (size_t)t2 + 4 * j;
          double R0 = x[0] - y[0], R1 = x[1] - y[1], R2 = x[2] - y[2];
          double r = sqrt(R0 * R0 + R1 * R1 + R2 * R2);
          if (r < 1.0e-12) continue;
          double dot = (x[0] - Q[0]) * (y[0] - QP[0]) + (x[1] - Q[1]) * (y[1] - QP[1]) + (x[2] - Q[2]) * (y[2] - QP[2]);
          cd phi = cscale(exprel3(cscale(ik, r)), inv4pi / r);
          cd pe = cmk(dot * (1.0 / 144.0) - invk2.r * (1.0 / 16.0), -invk2.i * (1.0 / 16.0));
          part = cadd(part, cmul(pe, phi));
        }
      }
      acc = cadd(acc, cscale(part, cc));
    }
  }
  const double *F = nd.fibbi + 6 * (size_t)kk;
  cd t0 = cadd(cmk(F[0], 0), cscale(invk2, -F[1]));
  cd t1 = cmul(ik, cadd(cmk(F[2], 0), cscale(invk2, -F[3])));
  cd t2 = cmul(cmul(ik, ik), cadd(cmk(F[4], 0), cscale(invk2, -F[5])));
  acc = cadd(acc, cadd(t0, cadd(t1, t2)));
  M[(size_t)a + (size_t)b * ld] = acc;
  if (a != b) M[(size_t)b + (size_t)a * ld] = acc;
  if (Fc) {   // the complex64 copy
    const float2 f = make_float2((float)acc.r, (float)acc.i);
    Fc[(size_t)a + (size_t)b * ldf] = f;
    if (a != b) Fc[(size_t)b + (size_t)a * ldf] = f;
  }
}

int assemble_near(bg_geometry *g, double wr, double wi, void *M, size_t ld, const double *fq, void *F, size_t ldf) {
  NearData &nd = g->near;
  if (nd.npairs == 0) return BG_OK;
  double d = (wr * wr - wi * wi) * (wr * wr - wi * wi) + 4 * wr * wr * wi * wi;
  cd invk2{(wr * wr - wi * wi) / d, -2 * wr * wi / d};
  k_near<<<(nd.npairs + 127) / 128, 128, 0, stream()>>>(g->dev, nd, cd{wr, wi}, invk2, (cd *)M, ld, fq,
                                                       (float2 *)F, ldf);
  BG_LAUNCHED();
  return BG_OK;
}

// =========================================================================
// V^-1 Gram block of one row (GetOverlaps, VIEMatrix.cc:200-316):
//   -(1/w^2) int_T F_a . (eps(x)-1)^-1 . F_b, 33-point rule with w = 6V w_i,
// w = real(omega), over the faces of both tetrahedra of basis function a.
// Added to M(a,b) and M(b,a) for b >= a (the reference adds the full row and
// its symmetric fill then overwrites the lower triangle with the upper).
// =========================================================================
__global__ void k_gram(DevGeom g, double w, cd *M, size_t ld, const double *fq, float2 *F, size_t ldf) {
  if (fq) w = fq[0];
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= g.N) return;
  int2 tt = g.bfTet[a], qq = g.bfQ[a];
  double Aa = g.bfArea[a];
  int nnz = 1;
  int idx[8];
  cd val[8];
  idx[0] = a;
  val[0] = cmk(0, 0);
  const double pre = -1.0 / (w * w);
  for (int side = 0; side < 2; side++) {
    int t = side == 0 ? tt.x : tt.y;
    int obj = g.tetObj[t];
    const bg_material &mat = g.mats[obj];
    const DevExpr *mex = g.expr ? g.expr + obj : nullptr;
    double vol = g.tetVol[t];
    double QA[3];
    load3(g.V4, side == 0 ? qq.x : qq.y, QA);
    double pa = (side == 0 ? 1.0 : -1.0) * Aa / (3.0 * vol);
    int4 vi = g.tetVI[t];
    double V0[3], L[3][3];
    load3(g.V4, vi.x, V0);
    int vv[3] = {vi.y, vi.z, vi.w};
    for (int i = 0; i < 3; i++) {
      double tmp[3];
      load3(g.V4, vv[i], tmp);
      for (int c = 0; c < 3; c++) L[i][c] = tmp[c] - V0[c];
    }
    int4 fi = g.tetFI[t];
    int fl[4] = {fi.x, fi.y, fi.z, fi.w};
    for (int ifb = 0; ifb < 4; ifb++) {
      int b = fl[ifb];
      if (b < 0) continue;
      int2 tb = g.bfTet[b], qb = g.bfQ[b];
      double QB[3], pb;
      if (tb.x == t) { load3(g.V4, qb.x, QB); pb = g.bfArea[b] / (3.0 * vol); }
      else { load3(g.V4, qb.y, QB); pb = -g.bfArea[b] / (3.0 * vol); }
      cd accv = cmk(0, 0);
      for (int i = 0; i < 33; i++) {
        const double *u = c_tcr33 + 4 * i;
        double wt = 6.0 * vol * u[3], x[3];
        for (int c = 0; c < 3; c++) x[c] = V0[c] + u[0] * L[0][c] + u[1] * L[1][c] + u[2] * L[2][c];
        cd E[3][3], Ei[3][3];
        mat_eval(mat, mex, x, E);
        E[0][0].r -= 1.0; E[1][1].r -= 1.0; E[2][2].r -= 1.0;
        inv3(E, Ei);
        double FA[3], FB[3];
        for (int c = 0; c < 3; c++) { FA[c] = pa * (x[c] - QA[c]); FB[c] = pb * (x[c] - QB[c]); }
        cd v = cmk(0, 0);
        for (int mu = 0; mu < 3; mu++)
          for (int nu = 0; nu < 3; nu++) v = cadd(v, cscale(Ei[mu][nu], FA[mu] * FB[nu]));
        accv = cadd(accv, cscale(v, pre * wt));
      }
      if (b == a) val[0] = cadd(val[0], accv);
      else { idx[nnz] = b; val[nnz] = accv; nnz++; }
    }
  }
  for (int i = 0; i < nnz; i++) {
    int b = idx[i];
    if (b < a) continue;
    cd *p = M + (size_t)a + (size_t)b * ld;
    const cd v = cadd(*p, val[i]);
    *p = v;
    if (b != a) {
      cd *q = M + (size_t)b + (size_t)a * ld;
      *q = cadd(*q, val[i]);
    }
    if (F) {   // the final value of these entries: the complex64 copy
      F[(size_t)a + (size_t)b * ldf] = make_float2((float)v.r, (float)v.i);
      if (b != a) {
        const cd *q = M + (size_t)b + (size_t)a * ld;
        F[(size_t)b + (size_t)a * ldf] = make_float2((float)q->r, (float)q->i);
      }
    }
  }
}

int assemble_gram(bg_geometry *g, double wr, double wi, void *M, size_t ld, const double *fq, void *F, size_t ldf) {
  if (g->dispersive && fq) { set_error("frequency-dependent materials need a host frequency"); return BG_ERR_ARG; }
  int st = refresh_materials(g, wr, wi);
  if (st) return st;
  k_gram<<<(g->N + 127) / 128, 128, 0, stream()>>>(g->dev, wr, (cd *)M, ld, fq, (float2 *)F, ldf);
  BG_LAUNCHED();
  return BG_OK;
}

// =========================================================================
// plane-wave RHS (RHSVector.cc:85-124): v_a = -1/(i w Z0) BFInt[b . E],
// E = E0 exp(i k nhat.x), 33-point rule on both tetrahedra of a.
// =========================================================================
struct PWave { cd E0[3]; double nh[3]; cd k; };

__device__ __forceinline__ cd bf_dot_field(const DevGeom &g, int a, const PWave &pw) {
  int2 tt = g.bfTet[a], loc = g.bfLoc[a];
  double Aa = g.bfArea[a];
  cd tot = cmk(0, 0);
  for (int side = 0; side < 2; side++) {
    int t = side == 0 ? tt.x : tt.y, iq = side == 0 ? loc.x : loc.y;
    int4 vi = g.tetVI[t];
    int v[4] = {vi.x, vi.y, vi.z, vi.w};
    double Q[3], L[3][3];
    load3(g.V4, v[iq], Q);
    for (int i = 0; i < 3; i++) {
      double tmp[3];
      load3(g.V4, v[(iq + 1 + i) % 4], tmp);
      for (int c = 0; c < 3; c++) L[i][c] = tmp[c] - Q[c];
    }
    double vol = g.tetVol[t];
    double pf = (side == 0 ? 1.0 : -1.0) * Aa / (3.0 * vol);
    cd acc = cmk(0, 0);
    for (int i = 0; i < 33; i++) {
      const double *u = c_tcr33 + 4 * i;
      double wt = 6.0 * vol * u[3], x[3], b[3];
      for (int c = 0; c < 3; c++) {
        b[c] = u[0] * L[0][c] + u[1] * L[1][c] + u[2] * L[2][c];
        x[c] = Q[c] + b[c];
        b[c] *= pf;
      }
      double ph = pw.nh[0] * x[0] + pw.nh[1] * x[1] + pw.nh[2] * x[2];
      cd e = expikr(pw.k, ph);
      cd be = cadd(cadd(cscale(pw.E0[0], b[0]), cscale(pw.E0[1], b[1])), cscale(pw.E0[2], b[2]));
      acc = cadd(acc, cscale(cmul(be, e), wt));
    }
    tot = cadd(tot, acc);
  }
  return tot;
}

__global__ void k_rhs(DevGeom g, PWave pw, cd pre, cd *out, const double *fq) {
  if (fq) {
    // -1/(i w Z0) = i/(w Z0)
    double wr = fq[0], wi = fq[1], d = (wr * wr + wi * wi) * 376.73031346177;
    pw.k = cd{wr, wi};
    pre = cd{wi / d, wr / d};
  }
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= g.N) return;
  out[a] = cmul(pre, bf_dot_field(g, a, pw));
}

static PWave make_pw(double wr, double wi, const double *E0, const double *nhat) {
  PWave pw;
  for (int i = 0; i < 3; i++) { pw.E0[i] = cd{E0[2 * i], E0[2 * i + 1]}; pw.nh[i] = nhat[i]; }
  pw.k = cd{wr, wi};
  return pw;
}

int rhs_planewave(bg_geometry *g, double wr, double wi, const double *E0, const double *nhat, void *out,
                  const double *fq) {
  int st = init_tables();
  if (st) return st;
  PWave pw = make_pw(wr, wi, E0, nhat);
  // -1/(i w Z0) = i/(w Z0)
  const double Z0 = 376.73031346177;
  double d = (wr * wr + wi * wi) * Z0;
  cd pre{wi / d, wr / d};
  k_rhs<<<(g->N + 127) / 128, 128, 0, stream()>>>(g->dev, pw, pre, (cd *)out, fq);
  BG_LAUNCHED();
  return BG_OK;
}

// =========================================================================
// EMT power (EMTPFT.cc:324-493): PScat = sum_{a<=b} Re(Z0 J_a^* J_b) Im Q_ab
// (same object; Im Q = w BFBFInt[PEFIE sin(kr)/(4 pi r)], series for kr<2e-2)
// and -1/2 Re(Z0 J_a^* J_b i Q_ab) across objects (full e^{ikr}/(4 pi r));
// rule 4/16/33 points by common vertices and kR>5 (EMTPFT.cc:305-313).
// Extinction 1/2 Re(J_a^* BFInt[b.E_inc]) (EMTPFT.cc:151-211).
// Partial sums per block and object pair are reduced on the host in a fixed
// order.
// =========================================================================
struct PftArgs {
  DevGeom g;
  const cd *J;
  double w;      // real(omega)
  double absw;   // |omega|
  int nobj;
  const cd *DR = nullptr;   // dressed Rytov matrix (column-major, ldr) in place of J
  size_t ldr = 0;
};

__device__ __forceinline__ void rule_point(int npts, int i, double *u) {
  if (npts == 16) { u[0] = c_tcr16[4 * i]; u[1] = c_tcr16[4 * i + 1]; u[2] = c_tcr16[4 * i + 2]; u[3] = c_tcr16[4 * i + 3]; }
  else { u[0] = c_tcr33[4 * i]; u[1] = c_tcr33[4 * i + 1]; u[2] = c_tcr33[4 * i + 2]; u[3] = c_tcr33[4 * i + 3]; }
}

// Full EMT PFT (EMTPFT.cc:85-127 extinction, 216-291 scattered, 396-491 sum).
// Ten quantities per pair, NPQ order: PScat, force (3), torque from b_A x b_B
// (3), torque from (x_A - c_A) x R (3); c_A = torque centre (object origin).
#define NPQ 10
#define TEN_THIRDS (10.0 / 3.0)

// BFBFInt of the scattered integrand (EMTPFT.cc:216-291); lanes [lane, nl)
// split the point pairs; q: this lane's partial integrals
__device__ void scat_q(const PftArgs &P, int a, int b, int npts, bool same, int lane, int nl, cd q[NPQ]) {
  const DevGeom &g = P.g;
  int2 ta = g.bfTet[a], tb = g.bfTet[b], la = g.bfLoc[a], lb = g.bfLoc[b];
  double k = P.w, k2 = k * k;
  for (int n = 0; n < NPQ; n++) q[n] = cmk(0, 0);
  const double inv4pi = 0.25 / M_PI;
  int oa = g.bfV[a].w;
  const double *tc = g.objOrigin + 3 * oa;
  for (int sa = 0; sa < 2; sa++)
    for (int sb = 0; sb < 2; sb++) {
      int t1 = sa == 0 ? ta.x : ta.y, t2 = sb == 0 ? tb.x : tb.y;
      int i1 = sa == 0 ? la.x : la.y, i2 = sb == 0 ? lb.x : lb.y;
      int4 v1 = g.tetVI[t1], v2 = g.tetVI[t2];
      int va[4] = {v1.x, v1.y, v1.z, v1.w}, vb[4] = {v2.x, v2.y, v2.z, v2.w};
      double Q1[3], Q2[3], L1[3][3], L2[3][3];
      load3(g.V4, va[i1], Q1);
      load3(g.V4, vb[i2], Q2);
      for (int i = 0; i < 3; i++) {
        double tmp[3];
        load3(g.V4, va[(i1 + 1 + i) % 4], tmp);
        for (int c = 0; c < 3; c++) L1[i][c] = tmp[c] - Q1[c];
        load3(g.V4, vb[(i2 + 1 + i) % 4], tmp);
        for (int c = 0; c < 3; c++) L2[i][c] = tmp[c] - Q2[c];
      }
      double V1 = g.tetVol[t1], V2 = g.tetVol[t2];
      double p1 = (sa == 0 ? 1.0 : -1.0) * g.bfArea[a] / (3.0 * V1);
      double p2 = (sb == 0 ? 1.0 : -1.0) * g.bfArea[b] / (3.0 * V2);
      int np2 = npts * npts;
      for (int idx = lane; idx < np2; idx += nl) {
        int i = idx / npts, j = idx % npts;
        double u[4], v[4];
        if (npts == 4) {
          const double qa = 0.13819660112501051, qb = 0.58541019662496850;
          u[0] = (i == 1) ? qb : qa; u[1] = (i == 2) ? qb : qa; u[2] = (i == 3) ? qb : qa; u[3] = 1.0 / 24.0;
          v[0] = (j == 1) ? qb : qa; v[1] = (j == 2) ? qb : qa; v[2] = (j == 3) ? qb : qa; v[3] = 1.0 / 24.0;
        } else {
          rule_point(npts, i, u);
          rule_point(npts, j, v);
        }
        double xa[3], xb[3], ba[3], bb[3];
        for (int c = 0; c < 3; c++) {
          ba[c] = u[0] * L1[0][c] + u[1] * L1[1][c] + u[2] * L1[2][c];
          xa[c] = Q1[c] + ba[c];
          ba[c] *= p1;
          bb[c] = v[0] * L2[0][c] + v[1] * L2[1][c] + v[2] * L2[2][c];
          xb[c] = Q2[c] + bb[c];
          bb[c] *= p2;
        }
        double wt = 6.0 * V1 * u[3] * 6.0 * V2 * v[3];
        double R[3] = {xa[0] - xb[0], xa[1] - xb[1], xa[2] - xb[2]};
        double r2 = R[0] * R[0] + R[1] * R[1] + R[2] * R[2], r = sqrt(r2), kr = k * r;
        double pefie = ba[0] * bb[0] + ba[1] * bb[1] + ba[2] * bb[2] - (3.0 * p1) * (3.0 * p2) / k2;
        cd phi, psi;
        if (same) {
          double imphi, impsi;
          if (fabs(kr) < 2.0e-2) {
            imphi = (1.0 - kr * kr / 6.0) * k * inv4pi;
            impsi = -(1.0 - kr * kr / 10.0) * k2 * k / (12.0 * M_PI);
          } else {
            double s, c;
            sincos(kr, &s, &c);
            imphi = s * inv4pi / r;
            impsi = (kr * c - s) * inv4pi / (r * r2);
          }
          phi = cmk(0, imphi);
          psi = cmk(0, impsi);
        } else {
          double s, c;
          sincos(kr, &s, &c);
          phi = cmk(c * inv4pi / r, s * inv4pi / r);
          psi = cscale(cmul(phi, cmk(-1.0, kr)), 1.0 / r2);     // phi (ikr - 1) / r^2
        }
        double XT[3] = {xa[0] - tc[0], xa[1] - tc[1], xa[2] - tc[2]};
        q[0] = cadd(q[0], cscale(phi, P.w * pefie * wt));
        cd pp = cscale(psi, TEN_THIRDS * pefie * wt), pf = cscale(phi, TEN_THIRDS * wt);
        for (int m = 0; m < 3; m++) {
          int m1 = (m + 1) % 3, m2 = (m + 2) % 3;
          q[1 + m] = cadd(q[1 + m], cscale(pp, R[m]));
          q[4 + m] = cadd(q[4 + m], cscale(pf, ba[m1] * bb[m2] - ba[m2] * bb[m1]));
          q[7 + m] = cadd(q[7 + m], cscale(pp, XT[m1] * R[m2] - XT[m2] * R[m1]));
        }
      }
    }
}

// contributions of pair (a, b) to the per-object-pair sums (EMTPFT.cc:416-436)
__device__ __forceinline__ void scat_terms(const PftArgs &P, int a, int b, const cd q[NPQ], bool same, double d[NPQ]) {
  const double Z0 = 376.73031346177;
  // u0JJ = Z0 GetJJ(a, b) (GetPFT.cc:108-115): Z0 DR(b, a) for a dressed
  // Rytov matrix, else Z0 conj(Ja) Jb
  cd u;
  if (P.DR) {
    cd v = P.DR[(size_t)b + (size_t)a * P.ldr];
    u = cmk(Z0 * v.r, Z0 * v.i);
  } else {
    cd Ja = P.J[a], Jb = P.J[b];
    u = cmk(Z0 * (Ja.r * Jb.r + Ja.i * Jb.i), Z0 * (Ja.r * Jb.i - Ja.i * Jb.r));
  }
  if (same) {
    d[0] = u.r * q[0].i;
    for (int n = 1; n < NPQ; n++) d[n] = a != b ? u.i * q[n].i : 0.0;
  } else {
    // -0.5 Re(u i q) = 0.5 Im(u q);  -0.5 Im(u i q) = -0.5 Re(u q)
    cd uq = cmul(u, q[0]);
    d[0] = 0.5 * uq.i;
    for (int n = 1; n < NPQ; n++) d[n] = -0.5 * cmul(u, q[n]).r;
  }
}

#define PMAXOBJ 4
// far pairs (no common vertex): one thread per pair; partial sums per block
// and object pair: part[block][noa*NO + nob][NPQ]
__global__ void __launch_bounds__(FT * FT) k_pft_far(PftArgs P, double *part) {
  int bx = blockIdx.x, by = blockIdx.y;
  int a = bx * FT + threadIdx.x, b = by * FT + threadIdx.y;
  const DevGeom &g = P.g;
  double d[NPQ];
  for (int n = 0; n < NPQ; n++) d[n] = 0.0;
  int pairid = 0;
  if (bx <= by && a < g.N && b < g.N && a <= b) {
    int4 va = g.bfV[a], vb = g.bfV[b];
    int2 qa = g.bfQ[a], qb = g.bfQ[b];
    int A5[5] = {qa.x, va.x, va.y, va.z, qa.y}, B5[5] = {qb.x, vb.x, vb.y, vb.z, qb.y};
    int ncv = 0;
    for (int i = 0; i < 5; i++)
      for (int j = 0; j < 5; j++) ncv += A5[i] == B5[j];
    if (ncv == 0) {
      double kR = P.absw * fmax(g.bfRadius[a], g.bfRadius[b]);
      int npts = kR > 5.0 ? 16 : 4;
      bool same = va.w == vb.w;
      cd q[NPQ];
      scat_q(P, a, b, npts, same, 0, 1, q);
      scat_terms(P, a, b, q, same, d);
      pairid = va.w * P.nobj + vb.w;
    }
  }
  __shared__ double red[FT * FT / 32][PMAXOBJ * PMAXOBJ][NPQ];
  int tid = threadIdx.y * FT + threadIdx.x, lane = tid & 31, wid = tid >> 5;
  for (int pid = 0; pid < P.nobj * P.nobj; pid++)
    for (int n = 0; n < NPQ; n++) {
      double v = warp_sum(pid == pairid ? d[n] : 0.0);
      if (lane == 0) red[wid][pid][n] = v;
    }
  __syncthreads();
  int nv = P.nobj * P.nobj * NPQ;
  for (int e = tid; e < nv; e += FT * FT) {
    int pid = e / NPQ, n = e % NPQ;
    double s = 0;
    for (int w = 0; w < FT * FT / 32; w++) s += red[w][pid][n];
    part[((size_t)by * gridDim.x + bx) * nv + e] = s;
  }
}

// near pairs (same object, common vertex): one warp per pair, lanes split the
// point pairs; partial sums per block and object: part[block][no][NPQ]
__global__ void k_pft_near(PftArgs P, NearData nd, double *part) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  double d[NPQ];
  for (int n = 0; n < NPQ; n++) d[n] = 0.0;
  if (warp < nd.npairs) {
    int2 ab = nd.pairs[warp];
    const DevGeom &g = P.g;
    double kR = P.absw * fmax(g.bfRadius[ab.x], g.bfRadius[ab.y]);
    int npts = kR > 5.0 ? 33 : 16;
    cd q[NPQ];
    scat_q(P, ab.x, ab.y, npts, true, lane, 32, q);
    for (int n = 0; n < NPQ; n++) {
      q[n].r = warp_sum(q[n].r);
      q[n].i = warp_sum(q[n].i);
    }
    if (lane == 0) scat_terms(P, ab.x, ab.y, q, true, d);
  }
  __shared__ double red[8][NPQ];
  __shared__ int objs[8];
  int wid = threadIdx.x >> 5;
  if (lane == 0) {
    for (int n = 0; n < NPQ; n++) red[wid][n] = d[n];
    objs[wid] = (warp < nd.npairs) ? P.g.bfV[nd.pairs[warp].x].w : 0;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < P.nobj * NPQ; e += blockDim.x) {
    int o = e / NPQ, n = e % NPQ;
    double s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++)
      if (objs[w] == o) s += red[w][n];
    part[(size_t)blockIdx.x * P.nobj * NPQ + e] = s;
  }
}

// extinction (EMTPFT.cc:85-127, 151-211) for a plane wave (grad E = ik nhat E):
// per basis function q0 = int b.E, qx = int (x - c) b.E, t1 = int b x E;
// e[0] = Re(J* q0), e[1+i] = Im(J* ik nhat_i q0), e[4+i] = Im(J* t1_i),
// e[7+i] = Im(J* ik (qx x nhat)_i); partial sums per block and object
__global__ void k_pft_ext(PftArgs P, PWave pw, double *part) {
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  double e[NPQ];
  for (int n = 0; n < NPQ; n++) e[n] = 0.0;
  int obj = 0;
  if (a < P.g.N) {
    const DevGeom &g = P.g;
    obj = g.bfV[a].w;
    const double *tc = g.objOrigin + 3 * obj;
    int2 tt = g.bfTet[a], loc = g.bfLoc[a];
    double Aa = g.bfArea[a];
    cd q0 = cmk(0, 0), qx[3] = {cmk(0, 0), cmk(0, 0), cmk(0, 0)}, t1[3] = {cmk(0, 0), cmk(0, 0), cmk(0, 0)};
    for (int side = 0; side < 2; side++) {
      int t = side == 0 ? tt.x : tt.y, iq = side == 0 ? loc.x : loc.y;
      int4 vi = g.tetVI[t];
      int v[4] = {vi.x, vi.y, vi.z, vi.w};
      double Q[3], L[3][3];
      load3(g.V4, v[iq], Q);
      for (int i = 0; i < 3; i++) {
        double tmp[3];
        load3(g.V4, v[(iq + 1 + i) % 4], tmp);
        for (int c = 0; c < 3; c++) L[i][c] = tmp[c] - Q[c];
      }
      double vol = g.tetVol[t];
      double pf = (side == 0 ? 1.0 : -1.0) * Aa / (3.0 * vol);
      for (int i = 0; i < 33; i++) {
        const double *u = c_tcr33 + 4 * i;
        double wt = 6.0 * vol * u[3], x[3], bv[3];
        for (int c = 0; c < 3; c++) {
          bv[c] = u[0] * L[0][c] + u[1] * L[1][c] + u[2] * L[2][c];
          x[c] = Q[c] + bv[c];
          bv[c] *= pf;
        }
        cd ph = expikr(pw.k, pw.nh[0] * x[0] + pw.nh[1] * x[1] + pw.nh[2] * x[2]);
        cd E[3];
        for (int c = 0; c < 3; c++) E[c] = cscale(cmul(pw.E0[c], ph), wt);
        cd be = cadd(cadd(cscale(E[0], bv[0]), cscale(E[1], bv[1])), cscale(E[2], bv[2]));
        q0 = cadd(q0, be);
        for (int c = 0; c < 3; c++) qx[c] = cadd(qx[c], cscale(be, x[c] - tc[c]));
        t1[0] = cadd(t1[0], csub(cscale(E[2], bv[1]), cscale(E[1], bv[2])));
        t1[1] = cadd(t1[1], csub(cscale(E[0], bv[2]), cscale(E[2], bv[0])));
        t1[2] = cadd(t1[2], csub(cscale(E[1], bv[0]), cscale(E[0], bv[1])));
      }
    }
    cd Jc = cmk(P.J[a].r, -P.J[a].i);
    cd ik = cmk(-pw.k.i, pw.k.r);
    e[0] = cmul(Jc, q0).r;
    for (int i = 0; i < 3; i++) {
      int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
      e[1 + i] = cmul(Jc, cscale(cmul(ik, q0), pw.nh[i])).i;
      e[4 + i] = cmul(Jc, t1[i]).i;
      cd qxn = csub(cscale(qx[i1], pw.nh[i2]), cscale(qx[i2], pw.nh[i1]));
      e[7 + i] = cmul(Jc, cmul(ik, qxn)).i;
    }
  }
  __shared__ double red[4][PMAXOBJ][NPQ];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int o = 0; o < P.nobj; o++)
    for (int n = 0; n < NPQ; n++) {
      double v = warp_sum(o == obj ? e[n] : 0.0);
      if (lane == 0) red[wid][o][n] = v;
    }
  __syncthreads();
  for (int x = threadIdx.x; x < P.nobj * NPQ; x += blockDim.x) {
    int o = x / NPQ, n = x % NPQ;
    double s = 0;
    for (int w = 0; w < 4; w++) s += red[w][o][n];
    part[(size_t)blockIdx.x * P.nobj * NPQ + x] = s;
  }
}

// OPFT absorbed power (OPFT.cc:62-119, OverlapIntegrand_PFT PAbs term,
// OverlapIntegrals.cc:79-170,242-298): sum Re(conj(Ja) Jb ME_ab),
// ME_ab = 1/2 int b_a . (i Z0/w)(eps-1)^-1 . b_b on the shared tetrahedron.
__global__ void k_opft(PftArgs P, cd omega, double *part, const double *fq) {
  if (fq) {
    omega = cd{fq[0], fq[1]};
    P.w = fq[0];
    P.absw = sqrt(fq[0] * fq[0] + fq[1] * fq[1]);
  }
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  const DevGeom &g = P.g;
  double contrib = 0.0;
  int obj = 0;
  if (a < g.N) {
    obj = g.bfV[a].w;
    const bg_material &mat = g.mats[obj];
    const DevExpr *mex = g.expr ? g.expr + obj : nullptr;
    int2 tt = g.bfTet[a], loc = g.bfLoc[a];
    cd Ja = P.J[a];
    const double Z0 = 376.73031346177;
    cd pre = cdiv(cmk(0, Z0), omega);
    for (int side = 0; side < 2; side++) {
      int t = side == 0 ? tt.x : tt.y, iq = side == 0 ? loc.x : loc.y;
      double vol = g.tetVol[t];
      double pa = (side == 0 ? 1.0 : -1.0) * g.bfArea[a] / (3.0 * vol);
      int4 vi = g.tetVI[t];
      int v[4] = {vi.x, vi.y, vi.z, vi.w};
      double QA[3], L[3][3];
      load3(g.V4, v[iq], QA);
      for (int i = 0; i < 3; i++) {
        double tmp[3];
        load3(g.V4, v[(iq + 1 + i) % 4], tmp);
        for (int c = 0; c < 3; c++) L[i][c] = tmp[c] - QA[c];
      }
      int4 fi = g.tetFI[t];
      int fl[4] = {fi.x, fi.y, fi.z, fi.w};
      for (int ifb = 0; ifb < 4; ifb++) {
        int b = fl[ifb];
        if (b < 0) continue;
        int2 tb = g.bfTet[b], qb = g.bfQ[b];
        double QB[3], pb;
        if (tb.x == t) { load3(g.V4, qb.x, QB); pb = g.bfArea[b] / (3.0 * vol); }
        else { load3(g.V4, qb.y, QB); pb = -g.bfArea[b] / (3.0 * vol); }
        cd me = cmk(0, 0);
        for (int i = 0; i < 33; i++) {
          const double *u = c_tcr33 + 4 * i;
          double wt = 6.0 * vol * u[3], x[3], bA[3], bB[3];
          for (int c = 0; c < 3; c++) {
            bA[c] = u[0] * L[0][c] + u[1] * L[1][c] + u[2] * L[2][c];
            x[c] = bA[c] + QA[c];
            bB[c] = pb * (x[c] - QB[c]);
            bA[c] *= pa;
          }
          cd E[3][3], Ei[3][3];
          mat_eval(mat, mex, x, E);
          E[0][0].r -= 1.0; E[1][1].r -= 1.0; E[2][2].r -= 1.0;
          inv3(E, Ei);
          cd vsum = cmk(0, 0);
          for (int mu = 0; mu < 3; mu++) {
            cd e = cmk(0, 0);
            for (int nu = 0; nu < 3; nu++) e = cadd(e, cscale(cmul(pre, Ei[mu][nu]), bB[nu]));
            vsum = cadd(vsum, cscale(e, 0.5 * bA[mu]));
          }
          me = cadd(me, cscale(vsum, wt));
        }
        cd Jb = P.J[b];
        cd jj = cmk(Ja.r * Jb.r + Ja.i * Jb.i, Ja.r * Jb.i - Ja.i * Jb.r);
        contrib += cmul(jj, me).r;
      }
    }
  }
  __shared__ double red[4][PMAXOBJ];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int o = 0; o < P.nobj; o++) {
    double v = warp_sum(o == obj ? contrib : 0.0);
    if (lane == 0) red[wid][o] = v;
  }
  __syncthreads();
  if (threadIdx.x < P.nobj) {
    double s = 0;
    for (int w = 0; w < 4; w++) s += red[w][threadIdx.x];
    part[(size_t)blockIdx.x * P.nobj + threadIdx.x] = s;
  }
}

static int ensure_scratch(bg_geometry *g, size_t bytes) {
  if (g->scratch_bytes >= bytes) return BG_OK;
  if (g->d_scratch) cudaFree(g->d_scratch);
  g->d_scratch = nullptr;
  g->scratch_bytes = 0;
  BG_CUDA_TRY(cudaMalloc(&g->d_scratch, bytes));
  g->scratch_bytes = bytes;
  return BG_OK;
}

int pft(bg_geometry *g, double wr, double wi, const void *dJ, const double *E0, const double *nhat, int method,
        double *out) {
  int st = init_tables();
  if (st) return st;
  int NO = (int)g->objs.size();
  if (NO > PMAXOBJ) { set_error("PFT supports at most %d objects", PMAXOBJ); return BG_ERR_ARG; }
  PftArgs P{g->dev, (const cd *)dJ, wr, std::sqrt(wr * wr + wi * wi), NO};
  int nrow = (g->N + 127) / 128;
  if (method == BG_PFT_OVERLAP) {
    if ((st = ensure_scratch(g, sizeof(double) * nrow * NO))) return st;
    if ((st = refresh_materials(g, wr, wi))) return st;
    k_opft<<<nrow, 128, 0, stream()>>>(P, cd{wr, wi}, g->d_scratch, nullptr);
    BG_LAUNCHED();
    std::vector<double> h((size_t)nrow * NO);
    BG_CUDA_TRY(cudaMemcpyAsync(h.data(), g->d_scratch, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, stream()));
    BG_CUDA_TRY(cudaStreamSynchronize(stream()));
    for (int o = 0; o < NO; o++) {
      double s = 0;
      for (int b = 0; b < nrow; b++) s += h[(size_t)b * NO + o];
      out[2 * o] = s;
      out[2 * o + 1] = 0.0;
    }
    return BG_OK;
  }
  double full[8 * PMAXOBJ];
  if ((st = pft_emt_full(g, wr, wi, dJ, E0, nhat, full))) return st;
  for (int o = 0; o < NO; o++) {
    out[2 * o] = full[8 * o];
    out[2 * o + 1] = full[8 * o + 1];
  }
  return BG_OK;
}

// GetPFTMatrix with EMT (GetPFT.cc:133-189, EMTPFT.cc:324-493): out[8*no + c],
// c = PAbs, PScat, Fx, Fy, Fz, Tx, Ty, Tz (force and torque in the
// reference's units, TENTHIRDS = 10/3), plane-wave incident field
static int pft_emt_impl(bg_geometry *g, double wr, double wi, const void *dJ, const void *dDR, size_t ldr,
                        const double *E0, const double *nhat, double *out) {
  int st = init_tables();
  if (st) return st;
  int NO = (int)g->objs.size();
  if (NO > PMAXOBJ) { set_error("PFT supports at most %d objects", PMAXOBJ); return BG_ERR_ARG; }
  PftArgs P{g->dev, (const cd *)dJ, wr, std::sqrt(wr * wr + wi * wi), NO, (const cd *)dDR, ldr};
  int nrow = (g->N + 127) / 128;
  if ((st = build_near_lists(g))) return st;
  int nb = (g->N + FT - 1) / FT;
  size_t nfar = (size_t)nb * nb * NO * NO * NPQ;
  int nnear_blocks = (g->near.npairs * 32 + 255) / 256;
  size_t nnear = (size_t)std::max(nnear_blocks, 1) * NO * NPQ;
  size_t next = (size_t)nrow * NO * NPQ;
  if ((st = ensure_scratch(g, sizeof(double) * (nfar + nnear + next)))) return st;
  double *pfar = g->d_scratch, *pnear = pfar + nfar, *pext = pnear + nnear;
  k_pft_far<<<dim3(nb, nb), dim3(FT, FT), 0, stream()>>>(P, pfar);
  BG_LAUNCHED();
  if (g->near.npairs > 0) {
    k_pft_near<<<nnear_blocks, 256, 0, stream()>>>(P, g->near, pnear);
    BG_LAUNCHED();
  }
  if (E0) {
    PWave pw = make_pw(wr, wi, E0, nhat);
    k_pft_ext<<<nrow, 128, 0, stream()>>>(P, pw, pext);
    BG_LAUNCHED();
  } else {
    BG_CUDA_TRY(cudaMemsetAsync(pext, 0, sizeof(double) * next, stream()));
  }
  std::vector<double> h(nfar + nnear + next);
  BG_CUDA_TRY(cudaMemcpyAsync(h.data(), g->d_scratch, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, stream()));
  BG_CUDA_TRY(cudaStreamSynchronize(stream()));
  // scat[noa][nob][n]: pair sums; ext[no][n]
  std::vector<double> scat((size_t)NO * NO * NPQ, 0.0), ext((size_t)NO * NPQ, 0.0);
  for (size_t blk = 0; blk < (size_t)nb * nb; blk++)
    for (size_t e = 0; e < (size_t)NO * NO * NPQ; e++) scat[e] += h[blk * NO * NO * NPQ + e];
  if (g->near.npairs > 0)
    for (int blk = 0; blk < nnear_blocks; blk++)
      for (int o = 0; o < NO; o++)
        for (int n = 0; n < NPQ; n++) scat[((size_t)o * NO + o) * NPQ + n] += h[nfar + ((size_t)blk * NO + o) * NPQ + n];
  for (int blk = 0; blk < nrow; blk++)
    for (size_t e = 0; e < (size_t)NO * NPQ; e++) ext[e] += h[nfar + nnear + (size_t)blk * NO * NPQ + e];
  double ftf = 0.5 * TEN_THIRDS / wr;
  for (int o = 0; o < NO; o++) {
    double s[NPQ] = {0};
    for (int ob = 0; ob < NO; ob++)
      for (int n = 0; n < NPQ; n++) s[n] += scat[((size_t)o * NO + ob) * NPQ + n];
    const double *e = ext.data() + (size_t)o * NPQ;
    double *r = out + 8 * o;
    r[0] = 0.5 * e[0] - s[0];
    r[1] = s[0];
    for (int i = 0; i < 3; i++) {
      r[2 + i] = ftf * e[1 + i] - s[1 + i];
      r[5 + i] = ftf * (e[4 + i] + e[7 + i]) - s[4 + i] - s[7 + i];
    }
  }
  return BG_OK;
}

int pft_emt_full(bg_geometry *g, double wr, double wi, const void *dJ, const double *E0, const double *nhat,
                 double *out) {
  return pft_emt_impl(g, wr, wi, dJ, nullptr, 0, E0, nhat, out);
}

// GetPFTMatrix(0, Omega, {EMT, DRMatrix}) as buff-neq calls it (GetFlux.cc:391-399):
// the pair sums with JJ = DR(b, a) and no incident field
int pft_emt_dr(bg_geometry *g, double wr, double wi, const void *dDR, size_t ldr, double *out) {
  return pft_emt_impl(g, wr, wi, nullptr, dDR, ldr, nullptr, nullptr, out);
}

// =========================================================================
// Overlap blocks for buff-neq (GetOverlaps, VIEMatrix.cc:122-316, and
// GetOverlapElements, SWGVolume.cc:405-481), row a: up to 7 columns b with
//   S_ab  = int b_a . b_b (closed form),
//   V_ab  = -w^2 int b_a . (eps - 1) b_b,
//   R_ab  = 4 w / (pi Z0) int b_a . Im(eps - 1) b_b   (uniform temperature),
// w = real(omega), the V and R integrals by the 33-point rule on each
// tetrahedron of a.  Slot 0 is the diagonal; cnt[a] is the number of slots.
// =========================================================================
__global__ void k_neq_overlaps(DevGeom g, double w, int *idx, double *S, cd *V, double *R, int *cnt) {
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= g.N) return;
  int2 tt = g.bfTet[a], qq = g.bfQ[a];
  int4 fv = g.bfV[a];
  double Aa = g.bfArea[a];
  double cen[3], P1[3], P2[3], P3[3];
  load3(g.V4, fv.x, P1); load3(g.V4, fv.y, P2); load3(g.V4, fv.z, P3);
  for (int c = 0; c < 3; c++) cen[c] = (P1[c] + P2[c] + P3[c]) / 3.0;
  int nnz = 1;
  int ix[8];
  double sv[8], rv[8];
  cd vv[8];
  ix[0] = a; sv[0] = 0.0; rv[0] = 0.0; vv[0] = cmk(0, 0);
  const double rpre = 4.0 * w / (M_PI * 376.73031346177), vpre = -w * w;
  for (int side = 0; side < 2; side++) {
    int t = side == 0 ? tt.x : tt.y;
    double sa = side == 0 ? 1.0 : -1.0;
    const bg_material &mat = g.mats[g.tetObj[t]];
    const DevExpr *mex = g.expr ? g.expr + g.tetObj[t] : nullptr;
    double vol = g.tetVol[t];
    double QA[3];
    load3(g.V4, side == 0 ? qq.x : qq.y, QA);
    // closed-form Gram terms of this tetrahedron
    double L2s = 0.0, XmQ[3], XmQ2 = 0.0;
    for (int c = 0; c < 3; c++) {
      double d1 = P1[c] - QA[c], d2 = P2[c] - QA[c], d3 = P3[c] - QA[c];
      L2s += d1 * d1 + d2 * d2 + d3 * d3;
      XmQ[c] = cen[c] - QA[c];
      XmQ2 += XmQ[c] * XmQ[c];
    }
    sv[0] += Aa * Aa * (XmQ2 / 20.0 + L2s / 180.0) / vol;
    double pa = sa * Aa / (3.0 * vol);
    int4 vi = g.tetVI[t];
    double V0[3], L[3][3];
    load3(g.V4, vi.x, V0);
    int vq[3] = {vi.y, vi.z, vi.w};
    for (int i = 0; i < 3; i++) {
      double tmp[3];
      load3(g.V4, vq[i], tmp);
      for (int c = 0; c < 3; c++) L[i][c] = tmp[c] - V0[c];
    }
    int4 fi = g.tetFI[t];
    int fl[4] = {fi.x, fi.y, fi.z, fi.w};
    for (int ifb = 0; ifb < 4; ifb++) {
      int b = fl[ifb];
      if (b < 0) continue;
      int2 tb = g.bfTet[b], qb = g.bfQ[b];
      double QB[3], pb, sb;
      if (tb.x == t) { load3(g.V4, qb.x, QB); sb = 1.0; }
      else { load3(g.V4, qb.y, QB); sb = -1.0; }
      pb = sb * g.bfArea[b] / (3.0 * vol);
      cd accv = cmk(0, 0);
      double accr = 0.0;
      for (int i = 0; i < 33; i++) {
        const double *u = c_tcr33 + 4 * i;
        double wt = 6.0 * vol * u[3], x[3];
        for (int c = 0; c < 3; c++) x[c] = V0[c] + u[0] * L[0][c] + u[1] * L[1][c] + u[2] * L[2][c];
        cd E[3][3];
        mat_eval(mat, mex, x, E);
        E[0][0].r -= 1.0; E[1][1].r -= 1.0; E[2][2].r -= 1.0;
        double FA[3], FB[3];
        for (int c = 0; c < 3; c++) { FA[c] = pa * (x[c] - QA[c]); FB[c] = pb * (x[c] - QB[c]); }
        cd v = cmk(0, 0);
        double r = 0.0;
        for (int mu = 0; mu < 3; mu++)
          for (int nu = 0; nu < 3; nu++) {
            v = cadd(v, cscale(E[mu][nu], FA[mu] * FB[nu]));
            r += FA[mu] * E[mu][nu].i * FB[nu];
          }
        accv = cadd(accv, cscale(v, vpre * wt));
        accr += rpre * r * wt;
      }
      if (b == a) {
        vv[0] = cadd(vv[0], accv);
        rv[0] += accr;
      } else {
        double pf = 2.0 * sa * sb * Aa * g.bfArea[b] / (3.0 * vol);
        double xd = XmQ[0] * (QA[0] - QB[0]) + XmQ[1] * (QA[1] - QB[1]) + XmQ[2] * (QA[2] - QB[2]);
        ix[nnz] = b;
        sv[nnz] = pf * (3.0 * XmQ2 / 40.0 + L2s / 120.0 + xd / 8.0);
        vv[nnz] = accv;
        rv[nnz] = accr;
        nnz++;
      }
    }
  }
  for (int i = 0; i < 8; i++) {
    size_t o = 8 * (size_t)a + i;
    idx[o] = i < nnz ? ix[i] : -1;
    S[o] = i < nnz ? sv[i] : 0.0;
    V[o] = i < nnz ? vv[i] : cmk(0, 0);
    R[o] = i < nnz ? rv[i] : 0.0;
  }
  cnt[a] = nnz;
}

int neq_overlaps(bg_geometry *g, double w, int *idx, double *S, void *V, double *R, int *cnt) {
  int st = init_tables();
  if (st) return st;
  if ((st = refresh_materials(g, w, 0.0))) return st;
  k_neq_overlaps<<<(g->N + 127) / 128, 128, 0, stream()>>>(g->dev, w, idx, S, (cd *)V, R, cnt);
  BG_LAUNCHED();
  return BG_OK;
}

// Absorbed power per object by the overlap method with every number kept on
// the device (for captured graphs): partial sums into part (ceil(N/128) x NO
// doubles), then out[o] = sum over blocks, o < NO.
__global__ void k_opft_reduce(int nrow, int nobj, const double *part, double *out) {
  int o = blockIdx.x;
  double s = 0;
  for (int b = threadIdx.x; b < nrow; b += blockDim.x) s += part[(size_t)b * nobj + o];
  s = warp_sum(s);
  __shared__ double red[8];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
    out[o] = t;
  }
}

int opft_enqueue(bg_geometry *g, double wr, double wi, const void *dJ, const double *fq, double *part,
                 double *out_dev) {
  if (g->dispersive && fq) { set_error("frequency-dependent materials need a host frequency"); return BG_ERR_ARG; }
  int NO = (int)g->objs.size();
  if (NO > PMAXOBJ) { set_error("PFT supports at most %d objects", PMAXOBJ); return BG_ERR_ARG; }
  PftArgs P{g->dev, (const cd *)dJ, wr, std::sqrt(wr * wr + wi * wi), NO};
  int nrow = (g->N + 127) / 128;
  k_opft<<<nrow, 128, 0, stream()>>>(P, cd{wr, wi}, part, fq);
  BG_LAUNCHED();
  k_opft_reduce<<<NO, 256, 0, stream()>>>(nrow, NO, part, out_dev);
  BG_LAUNCHED();
  return BG_OK;
}

}  // namespace bg
