/*
 * buffem_b200.h -- C-ABI of the B200-native BUFF-EM dense VIE hot path.
 *
 * Plain C types only (opaque handles, pointers, sizes); no torch or C++
 * types cross this boundary.  Every entry point returns an int status:
 *   0 (BG_OK)  success
 *   > 0        LAPACK-style info from the LU (1-based index of an exactly zero pivot)
 *   < 0        error; bg_last_error() returns a thread-local message.
 * No exception crosses the ABI.  There is no CPU fallback: every compute
 * entry point runs hand-written sm_100a CUDA kernels and fails with
 * BG_ERR_CUDA when no usable GPU is present.
 *
 * Units and conventions follow libbuff: omega in units of 3e14 rad/s,
 * lengths in microns, k = omega in vacuum, complex numbers as interleaved
 * (re, im) doubles, matrices column-major N x N complex128 (LAPACK layout;
 * the VIE matrix is complex-symmetric, M = M^T).
 *
 * Each declaration cites the libbuff / libhmat interface it replaces
 * (paths relative to the HomerReid/buff-em source tree).
 */
#ifndef BUFFEM_B200_H
#define BUFFEM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define BG_OK 0
#define BG_ERR_ARG (-1)       /* invalid argument / wrong-size object */
#define BG_ERR_IO (-2)        /* unreadable or malformed mesh / geometry file */
#define BG_ERR_TOPOLOGY (-3)  /* mesh face shared by more than two tetrahedra */
#define BG_ERR_CUDA (-4)      /* CUDA runtime error or no usable GPU */
#define BG_ERR_NOMEM (-5)     /* device or host allocation failed */
#define BG_ERR_STATE (-6)     /* call out of order (e.g. solve before factor) */
#define BG_ERR_NUMERIC (-7)   /* non-finite value detected */

/* matrix storage precisions */
#define BG_C128 0             /* complex128 (the plain FP64 path) */
#define BG_C64 1              /* complex64 (precision form)          */

/* permittivity functors (replace SVTensor / MatProp expressions,
   SVTensor.cc:41-114,306-373; off-diagonals are symmetrised on evaluation) */
#define BG_MAT_CONST_ISO 0     /* eps[0]+i eps[1]                               */
#define BG_MAT_CONST_TENSOR 1  /* eps[0..17]: 3x3 complex, row-major            */
#define BG_MAT_JANUS_Z 2       /* eps (z > center[2]) / eps2 (z <= center[2])   */
#define BG_MAT_GAUSSIAN 3      /* eps + amp*exp(-|x-center|^2/width^2)          */

typedef struct bg_material {
  int kind;
  double eps[18];
  double eps2[2];
  double center[3];
  double amp[2];
  double width;
} bg_material;

/* PFT methods (GetPFT.cc:133-189) */
#define BG_PFT_EMT 0          /* energy/momentum transfer (BUFF default, GetPFT.cc:205) */
#define BG_PFT_OVERLAP 1      /* overlap method (OPFT.cc:62-119) */

typedef struct bg_geometry bg_geometry;
typedef struct bg_matrix bg_matrix;
typedef struct bg_precond bg_precond;

/* Thread-local description of the last error (replaces ErrExit's message). */
const char *bg_last_error(void);

/* ---------------------------------------------------------------------------
 * geometry -- replaces buff::SWGGeometry (libbuff.h:200-272)
 * ------------------------------------------------------------------------- */

/* SWGGeometry::SWGGeometry(const char *GeoFileName), SWGGeometry.cc:214-383.
   Parses MESHPATH lines, MATERIAL <name> ... ENDMATERIAL sections (complex
   constants and Eps(w), w in rad/s; used at every frequency the geometry is
   assembled at, except in bg_batch_sweep) and OBJECT <label> ... ENDOBJECT
   sections holding MESHFILE, MATERIAL (CONST_EPS_<value>, VACUUM or the name
   of a MATERIAL section above) or SVTENSOR <file> (a permittivity tensor of
   frequency and position, evaluated on the device), and any number of
   DISPLACED dx dy dz / ROTATED theta ABOUT ax ay az lines, composed in order
   and applied to the mesh before its vertex merge (SWGGeometry.cc:52-158);
   the special name MESH__<mesh>__MAT__<material> stands for a one-object
   file (SWGGeometry.cc:167-209).  Meshes are gmsh .msh/.vmsh read with the
   semantics of ReadGMSHFile.cc:66-261 and numbered by InitFaceList.cc:69-279.
   Errors carry "<file>:<line>: <message>" as the reference's ErrExit does. */
int bg_geometry_create(const char *buffgeo_path, bg_geometry **out);

/* Transformation lists (.trans files of buff-neq's --TransFile, read by
   ReadTransFile into GTComplex lists, CreateBNEQData.cc:58-66): lines
   TRANS <tag> OBJECT <label> DISP dx dy dz [ROT theta ABOUT ax ay az]
   [OBJECT ...], or TRANS <tag> followed by OBJECT lines and ENDTRANS.
   bg_trans_file_count returns the number of transformations;
   bg_trans_file_tag copies tag k into buf (as bg_geometry_object_label) and
   returns its length. */
int bg_trans_file_count(const char *trans_path);
int bg_trans_file_tag(const char *trans_path, int k, char *buf, int cap);

/* The geometry of a .buffgeo file with transformation k of a .trans file
   applied (SWGGeometry::Transform, SWGGeometry.cc:426-439: each named
   object's transformation follows its one-time DISPLACED / ROTATED ones).
   One handle per transformation replaces the reference's transform /
   untransform of a single geometry; an unknown object label is an error. */
int bg_geometry_create_transformed(const char *buffgeo_path, const char *trans_path, int k, bg_geometry **out);

/* Same as bg_geometry_create from explicit per-object mesh files, displacements
   (3*nobj doubles or NULL) and permittivity functors (SWGGeometry.cc:52-158). */
int bg_geometry_create_objects(int nobj, const char *const *meshfiles, const double *displacements,
                               const bg_material *materials, bg_geometry **out);

/* SWGGeometry::~SWGGeometry, SWGGeometry.cc:388-397 */
void bg_geometry_destroy(bg_geometry *g);

/* SWGGeometry::TotalBFs / NumObjects / BFIndexOffset (libbuff.h:262-263) */
int bg_geometry_num_bfs(const bg_geometry *g);
int bg_geometry_num_objects(const bg_geometry *g);
int bg_geometry_bf_offset(const bg_geometry *g, int obj);

/* Permittivity of object obj at Omega (units of 3e14 rad/s) into eps[2]
   (re, im): a MATERIAL ... ENDMATERIAL section's Eps(w) at w = Omega x 3e14
   rad/s (SVTensor::Evaluate -> MatProp::GetEps, SVTensor.cc:306-316), the
   xx component of an SVTENSOR object's tensor (the scalar SVTensor::Evaluate,
   SVTensor.cc:375-380), or the constant of a CONST_EPS / VACUUM / constant
   isotropic object.  Returns 1 for a frequency-dependent material, 0 for a
   constant one, or BG_ERR_ARG (constant tensors and the eps(x) functors of
   bg_geometry_create_objects: bg_geometry_material_tensor). */
int bg_geometry_material_eps(const bg_geometry *g, int obj, double omega_re, double omega_im, double *eps);

/* The permittivity tensor of object obj at Omega and point x[3] into
   Q[18] (3x3 complex, row-major, re/im), as the device evaluates it
   (SVTensor::Evaluate, SVTensor.cc:306-373): SVTENSOR files, MATERIAL
   sections, and the bg_material functors (constant tensors with their
   off-diagonal pairs averaged). */
int bg_geometry_material_tensor(const bg_geometry *g, int obj, double omega_re, double omega_im, const double *x,
                                double *Q);

/* SWGGeometry::GetObjectByLabel (SWGGeometry.cc:405-419): index of the first
   object whose label matches, ignoring case, or BG_ERR_ARG if none does.
   Labels are the OBJECT names of a .buffgeo file, or the mesh file names
   given to bg_geometry_create_objects. */
int bg_geometry_object_index(const bg_geometry *g, const char *label);

/* SWGVolume::Label of object obj into buf (cap bytes, NUL-terminated,
   truncated to fit; buf may be NULL when cap is 0).  Returns the label's
   length or a negative status. */
int bg_geometry_object_label(const bg_geometry *g, int obj, char *buf, int cap);

/* SWGVolume::Vertices / NumVertices / Origin (libbuff.h:73-195) of object
   obj: 3 doubles per vertex into xyz (mesh nodes in file order after the
   one-time transformation; merged duplicates stay in place) and the object's
   origin, the transformed (0,0,0) about which torques are taken, into
   origin[3].  Either pointer may be NULL.  Returns the vertex count or a
   negative status. */
int bg_geometry_vertices(const bg_geometry *g, int obj, double *xyz, double *origin);

/* Face table of object obj, 9 ints per interior face:
   iV1 iV2 iV3 iQP iQM iPTet iMTet PIndex MIndex (SWGFace, libbuff.h:97-115). */
int bg_geometry_faces(const bg_geometry *g, int obj, int *out);

/* Frequency-independent near-field integrals (the FIBBI cache of
   FIBBICache.cc:211-245 / ComputeFIBBIData, GMatrixElements.cc:370-375),
   computed on the device and kept resident.  Called implicitly by the first
   bg_assemble; exposed for timing.  The SWGGeometry statics
   TaylorDuffyTolerance / MaxTaylorDuffyEvals (libbuff.h:254-255) are replaced by
   bg_geometry_set_singular_order: Gauss points per angular dimension of the
   singular rule (default 10; must be set before the first precompute). */
int bg_geometry_precompute(bg_geometry *g);
int bg_geometry_set_singular_order(bg_geometry *g, int n);

/* Replaces the statics SWGGeometry::TaylorDuffyTolerance / MaxTaylorDuffyEvals
   (libbuff.h:254-255, set at SWGGeometry.cc:46-47) that bound the reference's
   adaptive Taylor-Duffy integrals (TTaylorDuffy.cc:284-343) of tetrahedron
   pairs sharing 2-4 vertices.  on = 1 (the default, flag_tol 1e-8, tol 1e-9):
   every such pair is integrated with the singular rule at orders n and n+2
   (n = the singular order, at most 14 here); where any of its 24 moments
   differ by more than flag_tol of their scale, the face cubes are refined
   level by level (6 Gauss points per dimension per box, boxes closed when a
   split changes them by at most tol of the scale; at most 2048 open boxes per
   level and 40 levels per pair).  on = 0: the fixed rule of order n alone.
   Must be set before the first precompute (BG_ERR_STATE otherwise). */
int bg_geometry_set_singular_refine(bg_geometry *g, int on, double flag_tol, double tol);

/* Statistics of the singular pairs (runs the precompute if needed), 6 values:
   [0] tetrahedron pairs sharing 2-4 vertices, [1] pairs refined,
   [2] angular points of the fixed rules, [3] angular points of the
   refinement, [4] status bits OR-ed over the pairs (1: a pair's box pool was
   full, 2: a pair still had open boxes after the last level; its halves are
   kept either way), [5] 1 if the refined rule is on. */
int bg_geometry_singular_stats(bg_geometry *g, long long *out);

/* The frequency-independent moments of the singular tetrahedron pairs as the
   device keeps them (the tetrahedron-pair form of ComputeFIBBIData's
   Taylor-Duffy branch, GMatrixElements.cc:343-353): *count pairs; per pair
   pairs[4i..] = row tetrahedron, column tetrahedron, common vertices,
   flags (bit 0 refined, bits 1-2 status); verts[8i..] = the two
   tetrahedra's global vertex indices, common vertices first in the row
   tetrahedron's order (CompareTets, SWGVolume.cc:357-400); mom[24i..] = per
   kernel 1/(4 pi r), 1/(4 pi), r/(8 pi): int K, int K (x-o) (3),
   int K (y-o) (3), int K (x-o).(y-o), unit-simplex measure, o = the first
   common vertex.  Any output pointer may be NULL. */
int bg_geometry_singular_moments(bg_geometry *g, int *count, int *pairs, int *verts, double *mom);

/* Copies the 6 frequency-independent near-field numbers of every near
   basis-function pair: pairs[2*k] = a, pairs[2*k+1] = b (a <= b, global
   indices), data[6*k..6*k+5] (GMatrixElements.cc:404-420 ordering).
   *count receives the number of pairs; pass pairs=data=NULL to query it. */
int bg_geometry_near_data(bg_geometry *g, int *count, int *pairs, double *data);

/* ---------------------------------------------------------------------------
 * VIE matrix -- replaces AllocateVIEMatrix / AssembleVIEMatrix and HMatrix
 * ------------------------------------------------------------------------- */

/* SWGGeometry::AllocateVIEMatrix(bool), VIEMatrix.cc:465-471.  The matrix is
   device-resident (N x N column-major, precision BG_C128 or BG_C64). */
int bg_matrix_create(bg_geometry *g, int precision, bg_matrix **out);
void bg_matrix_destroy(bg_matrix *m);

/* SWGGeometry::AssembleVIEMatrix(cdouble Omega, HMatrix *M), VIEMatrix.cc:431-460:
   G blocks (AssembleGBlock, :365-426) + V^-1 Gram blocks (AssembleOverlapBlocks,
   :321-360) + symmetric fill.  A matrix of the wrong size is an error
   (BG_ERR_ARG) instead of the reference's silent reallocation. */
int bg_assemble(bg_geometry *g, double omega_re, double omega_im, bg_matrix *m);
/* bg_assemble into m (BG_C128) that also writes f (BG_C64, same N) = m
   converted to complex64 (as bg_matrix_convert would) in the same kernels:
   the copy the mixed-precision solvers run on, without a separate pass over
   the complex128 matrix.  No reference counterpart (the reference assembles
   one precision). */
int bg_assemble_with_copy(bg_geometry *g, double omega_re, double omega_im, bg_matrix *m, bg_matrix *f);

/* HMatrix::GetEntries / ExportToMATLAB equivalent: copy the whole matrix
   (or its LU factors after bg_lu_factor) to host memory, column-major,
   2*N*N doubles (BG_C128) or 2*N*N floats (BG_C64). */
int bg_matrix_download(const bg_matrix *m, void *host);
/* HMatrix::GetEntries for whole rows: rows[k] of the matrix (or of its
   factors) into host row-major nrows x N (complex128 or complex64 as the
   matrix), without copying the rest of the matrix. */
int bg_matrix_get_rows(const bg_matrix *m, int nrows, const int *rows, void *host);
/* Upload a host matrix (same layout) into m, e.g. for factoring user data. */
int bg_matrix_upload(bg_matrix *m, const void *host);
/* Device pointer and leading dimension of the storage (no copy). */
int bg_matrix_device_ptr(bg_matrix *m, void **dptr, int *ld);

/* HMatrix::LUFactorize() -> LAPACK zgetrf (call site buff-scatter.cc:285).
   Right-looking blocked LU with partial pivoting on the device.  Returns
   > 0 (LAPACK info) for an exactly singular pivot. */
int bg_lu_factor(bg_matrix *m);
/* 1-based pivot indices (LAPACK ipiv), N ints, to host. */
int bg_lu_pivots(const bg_matrix *m, int *ipiv_host);

/* HMatrix::LUSolve(HVector *) -> zgetrs (call site buff-scatter.cc:314).
   B is a host column-major N x nrhs complex128 array, overwritten by X (for a
   BG_C64 matrix the solve runs in complex64 and B is rounded on the way). */
int bg_lu_solve(bg_matrix *m, double *B_host, int nrhs);
/* Same with B already on the device (leading dimension ldb, complex128). */
int bg_lu_solve_device(bg_matrix *m, void *B_dev, int ldb, int nrhs);

/* No counterpart in the reference.  bg_lu_solve_device for callers that
   cannot allocate GPU memory at solve time (an application whose framework
   has already reserved the device memory for its own pool, or a time-critical
   loop that cannot accept an allocation's possible failure or implicit
   synchronisation): the solve's gather buffer is a fixed 4 MiB device array
   in the library instead of an allocation.  Limits: nrhs <= 4 and
   N * nrhs * (16 bytes for complex128, 8 for complex64) <= 4 MiB, otherwise
   BG_ERR_ARG.  The array is shared by all calls and keeps the last call's
   contents; calls whose GPU work overlaps would race on it.  The first call
   on a device looks up the array's device address. */
int bg_lu_solve_device_noalloc(bg_matrix *m, void *B_dev, int ldb, int nrhs);

/* C <- C - A*B for device column-major complex128 matrices (A: M x K, B: K x N,
   C: M x N), the FP64 tensor-core GEMM of the LU trailing update.  Also the
   building block of buff-neq's dressed-Rytov chain (GetFlux.cc:155-272, four
   GEMMs per source object).  Runs on the library stream. */
int bg_zgemm_sub_device(int M, int N, int K, const void *A, int lda, const void *B, int ldb, void *C, int ldc);

/* C <- C - A*B for device column-major complex64 matrices: the tcgen05
   (kind::tf32) tensor-core GEMM of the precision form's LU trailing update
   (no reference counterpart).  TF32 products, FP32 accumulation.  B is read
   through a tensor map: it must start on a 16-byte boundary and ldb must be
   even (BG_ERR_ARG otherwise).  Synchronises the library stream; a pipeline
   timeout inside the kernel is reported as BG_ERR_CUDA. */
int bg_cgemm_sub_device(int M, int N, int K, const void *A, int lda, const void *B, int ldb, void *C, int ldc);

/* ---------------------------------------------------------------------------
 * precision form: complex64 tensor-core LU + FP64 iterative refinement
 * (no reference counterpart; the reference factors in complex128 only)
 * ------------------------------------------------------------------------- */

/* Copy a complex128 matrix into a complex64 one of the same size (device). */
int bg_matrix_convert(const bg_matrix *src, bg_matrix *dst);

/* Solve A X = B with the complex64 LU factors F of A (bg_lu_factor on a
   BG_C64 matrix runs the trailing updates on the tcgen05 tensor cores in
   TF32) and FP64 iterative refinement against the complex128 matrix A:
   x += F^{-1} (b - A x) until max_j |b_j - A x_j| / |b_j| <= tol or maxit
   sweeps.  B: host N x nrhs complex128 (nrhs <= 4), overwritten by X.
   stats (3 doubles, may be NULL): sweeps, final and first relative residual.
   Returns BG_ERR_NUMERIC if the residual becomes non-finite. */
int bg_lu_solve_refined(bg_matrix *A, bg_matrix *F, double *B_host, int nrhs, double tol, int maxit, double *stats);
int bg_lu_solve_refined_device(bg_matrix *A, bg_matrix *F, void *B_dev, int ldb, int nrhs, double tol, int maxit,
                               double *stats);

/* ---------------------------------------------------------------------------
 * learned form: GMRES with a sparse near-field preconditioner
 * (no reference counterpart; the reference solves by LU only)
 * ------------------------------------------------------------------------- */

/* Diagonal (Jacobi) preconditioner of an assembled complex128 matrix. */
int bg_precond_create_jacobi(bg_matrix *A, bg_precond **out);
void bg_precond_destroy(bg_precond *P);
/* Number of stored entries (complex128) of a preconditioner. */
int bg_precond_nnz(const bg_precond *P);

/* Restarted GMRES(restart) in FP64 on the device with right preconditioner P
   (NULL: none) for A X = B; up to 4 right-hand sides advance in lockstep so
   each step reads A once.  Stops when max_j |b_j - A x_j| / |b_j| <= tol or
   after maxit matrix-vector steps.  A cycle that gains fewer than 0.025
   digits of the true residual per step doubles the next cycle's length (up
   to 4 x restart, at most 200; a GMRES(restart) converging faster than that
   is unchanged), and, once at that length, the solve returns early,
   unconverged, when the last cycle's rate could not reach tol within the
   remaining steps even if it doubled.  stats (3 doubles, may be NULL):
   steps, final and initial relative residual.  B: host N x nrhs complex128. */
int bg_gmres_solve(bg_matrix *A, const bg_precond *P, double *B_host, int nrhs, double tol, int restart, int maxit,
                   double *stats);
int bg_gmres_solve_device(bg_matrix *A, const bg_precond *P, void *B_dev, int ldb, int nrhs, double tol, int restart,
                          int maxit, double *stats);

/* Mixed-precision GMRES: Krylov solves against the complex64 copy F of A
   (bg_matrix_convert; 8 N^2 bytes per step) to relative residual inner_tol,
   FP64 iterative refinement with the complex128 A between them, until
   max_j |b_j - A x_j| / |b_j| <= tol or maxit Krylov steps in total.
   stats (3 doubles, may be NULL): Krylov steps, final relative residual,
   refinement sweeps.  P as for bg_gmres_solve (built from A); when a cycle
   of the longest length with a given P still gains less than a factor 10,
   the solve continues with the diagonal (Jacobi) preconditioner of A
   (bg_gmres_last_info reports it). */
int bg_gmres_solve_mixed(bg_matrix *A, bg_matrix *F, const bg_precond *P, double *B_host, int nrhs, double tol,
                         int restart, int maxit, double inner_tol, double *stats);
int bg_gmres_solve_mixed_device(bg_matrix *A, bg_matrix *F, const bg_precond *P, void *B_dev, int ldb, int nrhs,
                                double tol, int restart, int maxit, double inner_tol, double *stats);

/* The learned form's solve: bg_gmres_solve_mixed, and when it misses tol
   within maxit Krylov steps (or its residual turns non-finite), LU
   factorisation of F (tcgen05 complex64) and the FP64-refined LU solve of the
   original right-hand sides (F then holds factors).  stats (4 doubles, may be
   NULL): Krylov steps, final relative residual, refinement sweeps, 1 if the
   LU fallback ran. */
int bg_gmres_solve_lu_fallback(bg_matrix *A, bg_matrix *F, const bg_precond *P, double *B_host, int nrhs,
                               double tol, int restart, int maxit, double inner_tol, double *stats);
/* What the calling thread's last mixed-precision solve did (6 doubles):
   Krylov steps, final relative residual, refinement sweeps, 1 if the given
   preconditioner was replaced by Jacobi, 1 if the Krylov solve stopped early
   on its convergence rate, the longest restart cycle used. */
int bg_gmres_last_info(double *out);
int bg_gmres_solve_lu_fallback_device(bg_matrix *A, bg_matrix *F, const bg_precond *P, void *B_dev, int ldb,
                                      int nrhs, double tol, int restart, int maxit, double inner_tol,
                                      double *stats);

/* Graph network (3 message-passing layers of width 64 over the near-field
   pattern of the basis functions) that predicts the entries of a sparse
   approximate inverse on that pattern,
     m_ij = [delta_ij + c_ij - [i != j] s_ij A_ij / A_ii] / A_jj,
   |Re c|, |Im c| < 0.1, |Re s| < smax, |Im s| < smax / 2, where
   smax = 0.7 / max(0.7, rho(K1)) and rho(K1) is a power-iteration estimate of
   the spectral radius of the scaled near-field part K1_ij = A_ij / A_jj
   (i != j on the pattern).  Parameters live on the device; the untrained
   network (seeded Glorot weights, zero readout) reproduces Jacobi. */
typedef struct bg_gnn bg_gnn;
int bg_gnn_create(unsigned long long seed, bg_gnn **out);
void bg_gnn_destroy(bg_gnn *net);
int bg_gnn_num_params(void);
int bg_gnn_get_params(const bg_gnn *net, float *host);
int bg_gnn_set_params(bg_gnn *net, const float *host);
int bg_gnn_get_grads(const bg_gnn *net, float *host);
/* One Adam step (lr > 0; lr == 0 computes loss and gradients only) on
   log L, L = |A M Z - Z|_F^2 / (N p) + lambda |M b - x|^2 / |x|^2, for the
   assembled complex128 matrix A of geometry g at frequency omega.  Z: host
   N x p complex128 probes (p <= 16), first mapped probe_power times
   (0..64) through z <- z - A D^{-1} z (D = diag A) and rescaled to
   |z|^2 = 2N; b, x: host right-hand side and its solution, or NULL.
   loss: L before the update; the stored gradients (bg_gnn_get_grads) are
   those of log L. */
int bg_gnn_train_step(bg_gnn *net, bg_geometry *g, bg_matrix *A, double omega, const double *Z_host, int p,
                      int probe_power, const double *b_host, const double *x_host, double lambda, double lr,
                      double *loss);
/* Preconditioner predicted by the network for the assembled matrix A. */
int bg_precond_create_learned(bg_geometry *g, bg_matrix *A, double omega, const bg_gnn *net, bg_precond **out);
/* Learned preconditioners: the estimate of rho(K1) and the coefficient bound
   smax used (Jacobi: 0 and 0). */
int bg_precond_bound(const bg_precond *P, double *rho, double *smax);
/* Copies a preconditioner's CSR (rowptr N+1 ints, col nnz ints, val 2*nnz
   doubles) to the host; any pointer may be NULL. */
int bg_precond_download(const bg_precond *P, int *rowptr, int *col, double *val);

/* ---------------------------------------------------------------------------
 * batching form: frequency sweeps over several geometries
 * (no reference counterpart; the reference assembles and factors one
 * frequency at a time: SWGGeometry::AssembleVIEMatrix, VIEMatrix.cc:431-460,
 * then HMatrix::LUFactorize / LUSolve)
 * ------------------------------------------------------------------------- */

#define BG_BATCH_MAXOBJ 4          /* objects per geometry in a sweep */
#define BG_BATCH_NO_GRAPHS 1       /* flags: launch every job directly, no CUDA graphs */

/* For every geometry geoms[i] and every omega[j] (complex, 2 doubles each):
   assemble the complex128 VIE matrix, LU-factor it, solve the plane wave
   (E0: 3 complex, nhat: 3 real) and write the absorbed power of each object
   (overlap method, as bg_pft with BG_PFT_OVERLAP) to
   pabs[(i * nomega + j) * BG_BATCH_MAXOBJ + object] (unused entries 0).
   Each geometry's launch sequence is recorded once per concurrent slot into
   a CUDA graph whose kernels read omega from device memory, and replayed per
   frequency; up to max_streams slots run concurrently.  An online autotuner
   picks, per size class (N rounded up to 1024), the LU panel slice height
   (16/32/64 rows per CTA), the CTA tile of the complex128 tensor-core GEMM
   (0: 64 x 64, 1: 128 x 64, 2: 64 x 128) and the slot count (1, 2, 4, ...
   <= max_streams) by timing the sweep's own first jobs, and keeps the
   choice for later geometries of that class.  stats (may be NULL;
   4 + 4*ngeom doubles): wall seconds, jobs, graphs requested, 1 if a capture
   fell back to direct launches; then per geometry the chosen panel rows,
   slots, seconds per job measured while tuning (0 if the class was already
   tuned) and GEMM tile.
   Returns BG_ERR_NUMERIC if a matrix was singular. */
int bg_batch_sweep(bg_geometry *const *geoms, int ngeom, const double *omega, int nomega, const double *E0,
                   const double *nhat, int max_streams, int flags, double *pabs, double *stats);

/* ---------------------------------------------------------------------------
 * right-hand side and post-processing
 * ------------------------------------------------------------------------- */

/* SWGGeometry::AssembleRHSVector(Omega, PlaneWave(E0, nHat), RHS),
   RHSVector.cc:85-124: v_a = -1/(i w Z0) * int b_a . E0 exp(i k nhat.x).
   E0: 3 complex (6 doubles); nhat: 3 doubles; out: N complex (host). */
int bg_rhs_planewave(bg_geometry *g, double omega_re, double omega_im, const double *E0,
                     const double *nhat, double *out_host);
/* Same, writing to a device buffer of N complex128. */
int bg_rhs_planewave_device(bg_geometry *g, double omega_re, double omega_im, const double *E0,
                            const double *nhat, void *out_dev);

/* SWGGeometry::GetPFTMatrix(J, Omega, Options), GetPFT.cc:133-189, absorbed and
   scattered power columns (PFT_PABS, PFT_PSCAT) per object: out[2*obj+0] =
   PAbs, out[2*obj+1] = PScat.  method = BG_PFT_EMT (EMTPFT.cc:324-493, with the
   plane wave E0/nhat as incident field) or BG_PFT_OVERLAP (OPFT.cc:62-119;
   PScat is not defined there and is returned as 0).  J: N complex (host). */
int bg_pft(bg_geometry *g, double omega_re, double omega_im, const double *J_host, const double *E0,
           const double *nhat, int method, double *out);

/* SWGGeometry::GetPFTMatrix(J, Omega, Options) with the EMT method, all
   columns (GetPFT.cc:133-189, EMTPFT.cc:85-127,216-291,324-493): out[8*obj +
   c], c = PAbs, PScat, Fx, Fy, Fz, Tx, Ty, Tz, for the plane wave E0/nhat as
   incident field.  Forces and torques use the reference's units (its 10/3
   factor); torques are about each object's displacement (its origin).
   J: N complex (host). */
int bg_pft_full(bg_geometry *g, double omega_re, double omega_im, const double *J_host, const double *E0,
                const double *nhat, double *out);

/* SWGGeometry::GetFields(IF, J, Omega, XMatrix, FMatrix), GetFields.cc:287-382:
   total fields at npts points X (host, 3 doubles per point): the plane wave
   E0/nhat (pass E0 = NULL for none; IF = 0 in the reference) plus the fields
   of the currents J (N complex on the host, or NULL for none; J = 0 in the
   reference), each basis function integrated with the 4-point rule when
   |X - centroid| / radius > 10 and the 16-point rule otherwise
   (Get1BFFields, GetFields.cc:265-281).  out: npts x 6 complex, point-major
   (Ex, Ey, Ez, Hx, Hy, Hz per point), the rows of the reference's FMatrix.
   A point closer than 1e-12 to a quadrature point skips that point. */
int bg_get_fields(bg_geometry *g, double omega_re, double omega_im, const double *J_host, const double *E0,
                  const double *nhat, int npts, const double *X_host, double *out_host);
/* Same on device buffers (J_dev may be NULL); synchronizes the library stream. */
int bg_get_fields_device(bg_geometry *g, double omega_re, double omega_im, const void *J_dev, const double *E0,
                         const double *nhat, int npts, const double *X_dev, void *out_dev);

/* ---------------------------------------------------------------------------
 * buff-neq flux chain (GetFlux, GetFlux.cc:291-436; ComputeDressedRytovMatrix,
 * GetFlux.cc:155-272) for one geometry as it stands (one transform) and a
 * uniform temperature per object.  A handle keeps the frequency-independent
 * inverse Gram matrix S^-1 (CreateBNEQData.cc:122-141) and three N x N
 * complex128 work matrices on the device (4 N^2 x 16 bytes in total).
 * ------------------------------------------------------------------------- */
typedef struct bg_neq bg_neq;
int bg_neq_create(bg_geometry *g, bg_neq **out);
void bg_neq_destroy(bg_neq *h);
/* Flux spectral densities at omega (real part nonzero): flux[(s*NO + d)*8 + q],
   s = source object, d = destination object, q = PAbs, PRad (PScat), Fx, Fy,
   Fz, Tx, Ty, Tz -- GetPFTMatrix(0, Omega, {EMT, DR_s}) per source object, the
   numbers buff-neq writes to .SIFlux.EMTPFT.  W = (1 + S^-1 V S^-1 G)^-1 is
   factored once per frequency and shared by the source objects. */
int bg_neq_flux(bg_neq *h, double omega_re, double omega_im, double *flux);
/* The dressed Rytov matrix DR_s = W S^-1 R_s S^-1 W^H of source object src,
   N x N complex column-major, copied to the host. */
int bg_neq_dressed_rytov(bg_neq *h, double omega_re, double omega_im, int src, void *out_host);
/* GetPFTMatrix(0, Omega, {EMT, DRMatrix}) (EMTPFT.cc:324-493 with GetJJ =
   DR(b, a), GetPFT.cc:108-115) for a device matrix DR (column-major, ld >= N):
   out[8*obj + q] as bg_pft_full without the incident-field terms. */
int bg_pft_dr_device(bg_geometry *g, double omega_re, double omega_im, const void *DR_dev, int ld, double *out);

/* The reference's FIBBI cache file (FIBBICache::Store / PreLoad,
   FIBBICache.cc:272-463): "FIBBI_GCACHE\0", then records of 27 float keys
   (GetFIBBICacheKey, FIBBICache.cc:133-160) and the 6 static near-field
   integrals of a basis-function pair of one object.  Store writes the near
   table of object obj (computing it first if needed); load replaces the
   entries of obj's near table whose keys appear in the file (for instance a
   cache written by the reference's own tools) and reports how many did.
   Keys are compared bit for bit, as the reference's map does, so a displaced
   copy of an object matches only the records whose float key differences
   the displacement leaves unchanged. */
int bg_fibbi_store(bg_geometry *g, int obj, const char *path, int *written);
int bg_fibbi_load(bg_geometry *g, int obj, const char *path, int *matched);

/* ---------------------------------------------------------------------------
 * instrumentation
 * ------------------------------------------------------------------------- */

/* Number of CUDA kernels this library has launched since load (all streams). */
long long bg_kernel_launch_count(void);
/* Synchronise the library's stream (timing helpers). */
int bg_synchronize(void);
/* cudaStream_t of the library (as void*), so callers can time on it. */
void *bg_stream(void);

/* Kernel-class timing with CUDA events on the library stream (off by default).
   bg_profile_begin() clears and enables it; bg_profile_read() synchronises and
   returns, per kernel class, the number of timed regions, summed
   milliseconds and an algorithmic work count (counts/ms/flops arrays of
   length n <= 12): 0 LU trailing GEMM (flops), 1 LU panel (flops), 2 row
   interchanges, 3 triangular-solve leaves (flops), 4 far-field assembly
   (point-pair kernel evaluations, 64 per basis-function pair), 5 near-field
   and Gram assembly, 6 GMRES dense matrix-vector products (matrix bytes
   read), 7 learned-preconditioner inference, 8 GMRES Gram-Schmidt steps
   (including their host reads), 9 preconditioner applications, 10 the two
   triangular sweeps of an LU solve (factor bytes read), 11 the complex128
   residual products of iterative refinement (matrix bytes read). */
int bg_profile_begin(void);
int bg_profile_read(int n, long long *counts, double *ms, double *flops);
int bg_profile_end(void);

#ifdef __cplusplus
}
#endif

#endif /* BUFFEM_B200_H */
