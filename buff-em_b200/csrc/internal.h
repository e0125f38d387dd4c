// Internal declarations shared by the host geometry code, the C-ABI layer and
// the CUDA kernels of the B200 BUFF-EM hot path.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "../../include/buffem_b200.h"

namespace bg {

#define BG_FAR_TILE 32                      // basis functions per far-field tile
#define BG_FAR_TILE_TETS (2 * BG_FAR_TILE)  // distinct tetrahedra per tile, at most

// ---------------------------------------------------------------- errors
void set_error(const char *fmt, ...);
extern std::atomic<long long> g_launches;

#define BG_CUDA_TRY(expr)                                                          \
  do {                                                                             \
    cudaError_t _e = (expr);                                                       \
    if (_e != cudaSuccess) {                                                       \
      ::bg::set_error("%s:%d: %s: %s", __FILE__, __LINE__, #expr,                  \
                      cudaGetErrorString(_e));                                     \
      return BG_ERR_CUDA;                                                          \
    }                                                                              \
  } while (0)

#define BG_LAUNCHED()                                                              \
  do {                                                                             \
    ::bg::g_launches.fetch_add(1, std::memory_order_relaxed);                      \
    cudaError_t _e = cudaGetLastError();                                           \
    if (_e != cudaSuccess) {                                                       \
      ::bg::set_error("%s:%d: kernel launch: %s", __FILE__, __LINE__,              \
                      cudaGetErrorString(_e));                                     \
      return BG_ERR_CUDA;                                                          \
    }                                                                              \
  } while (0)

cudaStream_t stream();
void set_thread_stream(cudaStream_t s);   // nullptr: back to the library stream
int ensure_device();

// kernel-class profiling (CUDA events around launches when enabled)
enum {
  PROF_GEMM = 0, PROF_PANEL = 1, PROF_LASWP = 2, PROF_TRSM = 3, PROF_ASM_FAR = 4, PROF_ASM_NEAR = 5,
  PROF_MATVEC = 6, PROF_GNN = 7, PROF_ORTHO = 8, PROF_PRECOND = 9, PROF_TRSV = 10, PROF_RESID = 11,
  PROF_NCLASS = 12
};
bool prof_on();
void prof_start(int cls);
void prof_stop(int cls, double flops);

// ---------------------------------------------------------------- host mesh
struct Face {
  int iV1, iV2, iV3, iQP, iQM, iPTet, iMTet, PIndex, MIndex, Index;
  double cen[3], area, radius;
};

// A MATERIAL ... ENDMATERIAL section: constants and Eps(w) (matprop.cpp).
struct MatPropFn;

struct SVTensorFn;

struct Object {
  std::string meshfile, label;
  std::shared_ptr<const MatPropFn> matprop;   // frequency-dependent eps, or null
  std::shared_ptr<const SVTensorFn> svt;      // frequency-dependent tensor (SVTENSOR file), or null
  int nv = 0, nt = 0, nif = 0, ntf = 0;
  std::vector<double> V;       // 3*nv (after displacement)
  std::vector<int> VI, FI;     // 4*nt each
  std::vector<double> vol;     // signed volume per tet
  std::vector<Face> F;         // interior faces first
  bg_material mat{};
  double origin[3] = {0, 0, 0};
};

// Reads a gmsh mesh (ReadGMSHFile.cc:66-261) and builds the face list
// (InitFaceList.cc:69-279).  xf, when not null, is the object's one-time
// transformation XP = M X + D as 12 doubles (M row-major, then D), applied to
// the vertices before the merge and to the origin.  Returns BG_OK or an error
// status.
int load_object(Object &o, const char *meshfile, const double *xf);

// One OBJECT ... ENDOBJECT section of a .buffgeo file.
struct GeoObject {
  std::string label, mesh;
  bg_material mat{};
  std::shared_ptr<const MatPropFn> matprop;   // MATERIAL naming a MATERIAL section
  std::shared_ptr<const SVTensorFn> svt;      // SVTENSOR file
  double xf[12];
};

// MATERIAL <name> ... ENDMATERIAL body lines (with their line numbers) into
// out; errors name path:line.
int matprop_parse_section(const std::string &name, const std::vector<std::string> &lines,
                          const std::vector<int> &lineno, const char *path, std::shared_ptr<const MatPropFn> &out);
// eps(Omega), Omega in units of 3e14 rad/s, into eps[2] (re, im)
void matprop_eps(const MatPropFn &m, double omega_re, double omega_im, double eps[2]);

// MATERIAL sections seen so far in a geometry's files, in order
typedef std::vector<std::pair<std::string, std::shared_ptr<const MatPropFn>>> MatDB;

// An SVTENSOR file (matprop.cpp).  Parsing adds its MATERIAL sections to db.
int svtensor_parse_file(const std::string &path, MatDB &db, std::shared_ptr<const SVTensorFn> &out);
bool svtensor_position_dependent(const SVTensorFn &t);
// the device program of a position-dependent tensor at Omega (w, Eps1-3 and
// the constants folded in); BG_ERR_ARG with a message if it is too long
struct DevExpr;
int svtensor_compile(const SVTensorFn &t, double omega_re, double omega_im, DevExpr *out);
// the tensor at Omega and point x into Q (3x3 complex, row-major re/im)
void svtensor_eval(const SVTensorFn &t, double omega_re, double omega_im, const double *x, double Q[18]);

// Parses a .buffgeo file (SWGGeometry.cc:52-158, 214-383) or a special
// MESH__<mesh>__MAT__<material> name (SWGGeometry.cc:167-209).
int parse_buffgeo(const char *path, std::vector<GeoObject> &objs);

// One transformation of a .trans file: a tag and, per named object, a
// transformation (12 doubles, M row-major then D).
struct TransEntry {
  struct Op {
    std::string label;
    double xf[12];
  };
  std::string tag;
  std::vector<Op> ops;
};
int parse_trans_file(const char *path, std::vector<TransEntry> &out);
// composes e's transformations after the named objects' own
int apply_trans(const TransEntry &e, std::vector<GeoObject> &objs);

// ---------------------------------------------------------------- device SoA
// All indices are global over the objects of a geometry (vertex and tet
// indices carry per-object offsets), so basis functions of different objects
// never share a vertex index, matching CompareBFs' OA != OB rule.
// An SVTENSOR permittivity that depends on position, compiled per frequency
// into postfix programs (one per tensor component, row-major) for the device
// (matprop.cpp: svtensor_compile; kernels.cu: mat_eval).  op = code << 16 |
// argument: 0 push constant con[arg], 1 push position variable arg (x, y, z,
// r, Theta, Phi), 2 negate, 3 add, 4 subtract, 5 multiply, 6 divide, 7 power,
// 8 function arg (exp log sqrt sin cos tan sinh cosh tanh asin acos atan abs
// step).
#define BG_MAT_EXPR 16           // internal material kind: eps from DevGeom::expr[object]
#define BG_EXPR_MAXOPS 512
#define BG_EXPR_MAXCON 128
#define BG_EXPR_STACK 24
struct DevExpr {
  int start[9], len[9];          // component (row-major) program; len 0: not given
  int op[BG_EXPR_MAXOPS];
  double con[2 * BG_EXPR_MAXCON];
};

struct DevGeom {
  int N = 0, NT = 0, NV = 0;
  double *V4 = nullptr;      // 4 doubles per vertex (x, y, z, 0)
  int4 *tetVI = nullptr;     // global vertex indices
  double *tetVol = nullptr;  // signed volume
  double *tetP4 = nullptr;   // 4-point rule points: 16 doubles per tet (x,y,z,0)*4
  int *tetObj = nullptr;
  // per basis function (global index a), side s in {0: P, 1: M}
  int2 *bfTet = nullptr;     // (PTet, MTet) global tet indices
  int2 *bfQ = nullptr;       // (QP, QM) global vertex indices
  int2 *bfLoc = nullptr;     // (PIndex, MIndex): local index of Q in each tet
  int4 *tetFI = nullptr;     // global basis-function index of the face opposite vertex k, -1 if exterior
  int4 *bfV = nullptr;       // (V1, V2, V3, obj)
  double *bfArea = nullptr;
  double *bfRadius = nullptr;
  bg_material *mats = nullptr;  // per object
  DevExpr *expr = nullptr;      // per object (allocated when some object is BG_MAT_EXPR)
  double *objOrigin = nullptr;  // 3 per object
  // far-field tiles of BG_FAR_TILE consecutive basis functions: the distinct
  // tetrahedra of each tile (<= 2 per basis function) and, per basis
  // function, the positions of its P and M tetrahedra in its tile's list
  int *tileTet = nullptr;       // BG_FAR_TILE_TETS per tile, -1 padded
  int *tileNT = nullptr;        // number of distinct tetrahedra per tile
  int2 *bfTileLoc = nullptr;
};

struct NearData {
  // near basis-function pairs (same object, >=1 common vertex), a <= b
  int npairs = 0;
  int2 *pairs = nullptr;       // (a, b)
  int4 *pairTP = nullptr;      // indices of the 4 tet pairs (PP, PM, MP, MM); sign bit 30 => swapped
  double *fibbi = nullptr;     // 6 per pair
  // distinct tetrahedron pairs feeding the near pairs
  int ntp = 0, ntp_reg = 0;    // first ntp_reg are regular (<=1 common vertex)
  int4 *tp = nullptr;          // (tA, tB, c, 0); singular pairs: vertex order in tpOrd
  int4 *tpOrdA = nullptr, *tpOrdB = nullptr;  // common-first vertex orders (global vertex ids)
  double *tpMom = nullptr;     // 24 moments per tet pair
  int nsing_c[3] = {0, 0, 0};  // singular pairs with 2, 3, 4 common vertices (in that order after ntp_reg)
  unsigned char *tpFlag = nullptr;  // per singular pair: bit 0 refined, bits 1-2 refinement status
};

// near-field graph of the basis functions for the learned preconditioner:
// CSR of pairs with a common vertex (both directions, self pairs included,
// columns sorted), reverse-edge map, mean face radius; built once per geometry
struct NearGraph {
  int E = 0;
  int *rowptr = nullptr, *col = nullptr, *etr = nullptr;
  double h = 0;
};

}  // namespace bg

struct bg_geometry {
  std::vector<bg::Object> objs;
  std::vector<int> bfOffset, vOffset, tOffset;
  int N = 0, NV = 0, NT = 0;
  bg::DevGeom dev;
  bg::NearData near;
  int singular_order = 10;
  // refined singular rule (singular.cu): on by default; flag and box tolerances
  bool sing_refine = true;
  double sing_flag_tol = 1e-8, sing_tol = 1e-9;
  // singular pairs, refined pairs, fixed-rule points, refinement points,
  // refinement status bits (1: box pool full, 2: level limit), refinement on
  long long sing_stats[6] = {0, 0, 0, 0, 0, 0};
  bool uploaded = false, precomputed = false;
  bool dispersive = false;      // some object's eps comes from a MATERIAL section
  double rule_rmax = 0.0;       // largest distance of a 4-point rule point from its tetrahedron's centroid
  bg::NearGraph graph;
  double *d_scratch = nullptr;  // general scratch (PFT partial sums etc.)
  double *d_fieldTet = nullptr, *d_fieldFace = nullptr;  // GetFields tables, 16 doubles per tet each
  void *gnn_cache = nullptr;    // graph-network inference buffers, reused across learned preconditioners
  size_t scratch_bytes = 0;
};

struct bg_precond {
  int N = 0, nnz = 0;
  int *rowptr = nullptr, *col = nullptr;   // CSR on the device
  void *val = nullptr;                     // complex128 values
  double rho = 0, theta = 0;               // learned: estimate of rho(K1) and the coefficient bound smax
  bool jacobi = false;                     // the diagonal preconditioner
};

struct bg_matrix {
  bg_geometry *g = nullptr;
  int N = 0, precision = BG_C128;
  size_t ld = 0;
  void *d = nullptr;
  int *d_ipiv = nullptr;       // 1-based pivots (LAPACK)
  bool factored = false;
  int info = 0;
  void *d_work = nullptr;      // LU workspace
  size_t work_bytes = 0;
  int *d_perm = nullptr;       // row permutation of the factors + solve flags/tickets
  int solve_epoch = 0;
  bool symmetric = false;      // contents known to satisfy M = M^T (assembled, or converted from such)
};

namespace bg {
// kernels entry points (implemented in .cu files); all return BG status
int upload_geometry(bg_geometry *g);
int build_near_lists(bg_geometry *g);
int precompute_near(bg_geometry *g);
int singular_precompute(bg_geometry *g);
// fq (optional, device {Re w, Im w}): omega read on the device instead of wr, wi
// F (optional): a complex64 matrix (leading dimension ldf) that receives the
// complex64 value of every entry the kernel leaves in M
int assemble_far(bg_geometry *g, double wr, double wi, void *M, size_t ld, const double *fq = nullptr,
                 void *F = nullptr, size_t ldf = 0);
int assemble_near(bg_geometry *g, double wr, double wi, void *M, size_t ld, const double *fq = nullptr,
                  void *F = nullptr, size_t ldf = 0);
int assemble_gram(bg_geometry *g, double wr, double wi, void *M, size_t ld, const double *fq = nullptr,
                  void *F = nullptr, size_t ldf = 0);
// Frequency-dependent materials: eps(Omega) of every object with a MATERIAL
// section into its host bg_material and, once uploaded, into the device copy
// (a no-op for geometries without such materials).
int refresh_materials(bg_geometry *g, double wr, double wi);
int rhs_planewave(bg_geometry *g, double wr, double wi, const double *E0, const double *nhat, void *out,
                  const double *fq = nullptr);
int opft_enqueue(bg_geometry *g, double wr, double wi, const void *dJ, const double *fq, double *part,
                 double *out_dev);
int pft(bg_geometry *g, double wr, double wi, const void *dJ, const double *E0, const double *nhat, int method,
        double *out);
// fields at npts points (device X: 3 per point; out: 6 complex per point);
// dJ may be null (incident field only), E0/nhat null (no incident field)
int get_fields(bg_geometry *g, double wr, double wi, const void *dJ, const double *E0, const double *nhat,
               int npts, const double *dX, void *dOut);
// frees the graph-network inference buffers kept with a geometry
void gnn_cache_free(bg_geometry *g);
// EMT PFT with a dressed Rytov matrix (device, column-major ldr) and no incident field
int pft_emt_dr(bg_geometry *g, double wr, double wi, const void *dDR, size_t ldr, double *out);
// buff-neq overlap rows: 8 slots per basis function (idx -1 past cnt[a])
int neq_overlaps(bg_geometry *g, double w, int *idx, double *S, void *V, double *R, int *cnt);
// B <- A^{-1} B for many right-hand sides (GEMM-based triangular solves; complex128)
int lu_solve_many(bg_matrix *m, void *dB, size_t ldb, int nrhs);
int pft_emt_full(bg_geometry *g, double wr, double wi, const void *dJ, const double *E0, const double *nhat,
                 double *out);
int lu_factor(bg_matrix *m);
int lu_solve(bg_matrix *m, void *dB, int ldb, int nrhs);
int lu_solve_status(bg_matrix *m);
int lu_solve_noalloc(bg_matrix *m, void *dB, int ldb, int nrhs);
// the allocation-free solve's size limits (BG_ERR_ARG with a message beyond them)
int lu_noalloc_check(const bg_matrix *m, int nrhs);
// capture-safe factor/solve (batched sweeps; complex128)
int lu_capture_prepare(bg_matrix *m);
int lu_factor_enqueue(bg_matrix *m);
int *lu_capture_info_ptr(bg_matrix *m);
int *lu_capture_solve_err_ptr(bg_matrix *m);
int lu_solve_enqueue(bg_matrix *m, void *dB, int ldb, int nrhs, void *dT);
void lu_set_panel_rows(int rows);
int lu_get_panel_rows();
void lu_set_gemm_tile(int tile);   // complex128 GEMM CTA tile: 0 64x64, 1 128x64, 2 64x128
int lu_get_gemm_tile();
int gmres_solve(bg_matrix *A, const bg_precond *P, void *dB, int ldb, int nrhs, double tol, int restart, int maxit,
                double *stats, const bg_precond *Palt = nullptr, int *cycle = nullptr);
// what the last mixed-precision solve of this thread did beyond its stats
struct GmInfo {
  int steps = 0, sweeps = 0;
  double relres = 0;
  int switched = 0;        // the given preconditioner stagnated: the rest ran with Jacobi
  int gave_up = 0;         // stopped early: the observed rate could not reach the target
  int longest_cycle = 0;   // longest restart cycle used
};
GmInfo gmres_last_info();
int gmres_solve_mixed(bg_matrix *A, bg_matrix *F, const bg_precond *P, void *dB, int ldb, int nrhs, double tol,
                      int restart, int maxit, double inner_tol, double *stats);
int precond_jacobi(bg_matrix *A, bg_precond **out);
int zgemm_sub_device(int M, int N, int K, const void *A, int lda, const void *B, int ldb, void *C, int ldc);
int cgemm_sub_device(int M, int N, int K, const void *A, int lda, const void *B, int ldb, void *C, int ldc);
int matrix_convert(const bg_matrix *src, bg_matrix *dst);
int solve_refined(bg_matrix *A, bg_matrix *F, void *dB, int ldb, int nrhs, double tol, int maxit, double *stats);
void gauss_legendre01(int n, double *x, double *w);
}  // namespace bg
