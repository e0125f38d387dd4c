// Test infrastructure: C entry points over the reference's own libbuff code
// (compiled in place from the reference's sources with the project-written
// SCUFF-EM stand-ins of shim.cc), used only to generate the golden fixtures
// under tests/golden/ in a container that holds the reference.  Nothing in
// the library or its benchmark loads this.
//
// Call sequence as the reference's drivers (buff-scatter.cc:236-347,
// unit-test-LFField.cc:50-71): SWGGeometry(buffgeo), AssembleVIEMatrix,
// AssembleRHSVector(PlaneWave), GetPFTMatrix, GetFields.
//
// Frequency-independent near-field data (the FIBBI cache) is either
// preloaded by the reference's own FIBBICache constructor from
// ${BUFF_CACHE_PATH}/<mesh>.cache (FIBBICache.cc:108-160) or computed by the
// reference itself, Taylor-Duffy included (TTaylorDuffy.cc, compiled with
// the project's adaptive cubature and kernel functions, shim.cc), at the
// tolerance set by rp_set_taylor_duffy.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "libbuff.h"

using namespace buff;

namespace buff {
void GetFIBBICacheKey(SWGVolume *OA, int nfA, SWGVolume *OB, int nfB, float *K);
void ComputeFIBBIData(SWGVolume *OA, int nfA, SWGVolume *OB, int nfB, double GFI[FIBBIDATALEN]);

// PFT methods of the reference that the pin does not compile (MomentPFT.cc,
// DSIPFT.cc need more of SCUFF-EM); selecting them ends the process.
HMatrix *GetMomentPFTMatrix(SWGGeometry *, cdouble, IncField *, HVector *, HMatrix *, HMatrix *, bool) {
  ErrExit("the moment PFT method is not part of the pinned path");
  return 0;
}
void GetDSIPFT(SWGGeometry *, cdouble, IncField *, HVector *, double *, GTransformation *, GTransformation *,
               PFTOptions *) {
  ErrExit("the DSI PFT method is not part of the pinned path");
}
void GetDSIPFTTrace(SWGGeometry *, cdouble, HMatrix *, double *, GTransformation *, GTransformation *,
                    PFTOptions *) {
  ErrExit("the DSI PFT method is not part of the pinned path");
}
}  // namespace buff

extern "C" {

void *rp_geometry(const char *buffgeo) {
  SWGGeometry *G = new SWGGeometry(buffgeo);
  G->LogLevel = BUFF_NO_LOGGING;
  return G;
}

// SWGGeometry::TaylorDuffyTolerance and MaxTaylorDuffyEvals (defaults 1e-6
// and 1e4, SWGGeometry.cc:46-47).
void rp_set_taylor_duffy(double reltol, int maxevals) {
  SWGGeometry::TaylorDuffyTolerance = reltol;
  SWGGeometry::MaxTaylorDuffyEvals = maxevals;
}

// The near-field record of the basis-function pair (a, b) of object no,
// computed by the reference (ComputeFIBBIData, GMatrixElements.cc:362-368):
// the 16x16 rule for tetrahedron pairs sharing <= 1 vertex, Taylor-Duffy for
// the others.  n pairs, 6 doubles each; OpenMP over the pairs.
void rp_fibbi(void *g, int no, int n, const int *pairs, double *out) {
  SWGVolume *O = ((SWGGeometry *)g)->Objects[no];
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < n; i++) ComputeFIBBIData(O, pairs[2 * i], O, pairs[2 * i + 1], out + 6 * i);
}

void rp_geometry_free(void *g) { delete (SWGGeometry *)g; }

int rp_total_bfs(void *g) { return ((SWGGeometry *)g)->TotalBFs; }
int rp_num_objects(void *g) { return ((SWGGeometry *)g)->NumObjects; }
int rp_object_bfs(void *g, int no) { return ((SWGGeometry *)g)->Objects[no]->NumInteriorFaces; }

// Face table of object no: per interior face iV1 iV2 iV3 iQP iQM iPTet iMTet
// PIndex MIndex (9 ints), in the reference's basis-function order.
void rp_faces(void *g, int no, int *out) {
  SWGVolume *O = ((SWGGeometry *)g)->Objects[no];
  for (int nf = 0; nf < O->NumInteriorFaces; nf++) {
    SWGFace *F = O->Faces[nf];
    int v[9] = {F->iV1, F->iV2, F->iV3, F->iQP, F->iQM, F->iPTet, F->iMTet, F->PIndex, F->MIndex};
    memcpy(out + 9 * nf, v, sizeof v);
  }
}

// The whole VIE matrix, column-major complex128 (N x N).
void rp_assemble(void *g, double re_w, double im_w, double *out) {
  SWGGeometry *G = (SWGGeometry *)g;
  HMatrix *M = G->AssembleVIEMatrix(cdouble(re_w, im_w), 0);
  memcpy(out, (void *)M->ZM, sizeof(cdouble) * (size_t)G->TotalBFs * G->TotalBFs);
  delete M;
}

// Entries of the Green's-function block only (no V^-1 term) for the listed
// (row, column) pairs of one object, with its near-field cache: the reference's
// GetGMatrixElement for selected entries of a large mesh.
void rp_gme(void *g, int no, double re_w, double im_w, int n, const int *rows, const int *cols, double *out) {
  SWGGeometry *G = (SWGGeometry *)g;
  SWGVolume *O = G->Objects[no];
  if (G->ObjectGCaches[no] == 0) G->ObjectGCaches[no] = new FIBBICache(O->MeshFileName);
  FIBBICache *C = G->ObjectGCaches[no];
  cdouble *z = (cdouble *)out;
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < n; i++) z[i] = GetGMatrixElement(O, rows[i], O, cols[i], cdouble(re_w, im_w), C);
}

// Basis-function pairs (a <= b) of object no whose near-field record needs
// the Taylor-Duffy integrator: CompareBFs > 0 and some tetrahedron pair of
// the two supports shares two or more vertices (GetGME_TetTetInt,
// GMatrixElements.cc:310-356).  Writes up to max pairs; returns the count.
int rp_singular_pairs(void *g, int no, int *out, int max) {
  SWGVolume *O = ((SWGGeometry *)g)->Objects[no];
  int n = 0;
  for (int a = 0; a < O->NumInteriorFaces; a++)
    for (int b = a; b < O->NumInteriorFaces; b++) {
      if (CompareBFs(O, a, O, b) == 0) continue;
      SWGFace *FA = O->Faces[a], *FB = O->Faces[b];
      int ta[2] = {FA->iPTet, FA->iMTet}, tb[2] = {FB->iPTet, FB->iMTet}, worst = 0;
      for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
          int c = CompareTets(O, ta[i], O, tb[j]);
          if (c > worst) worst = c;
        }
      if (worst < 2) continue;
      if (n < max) {
        out[2 * n] = a;
        out[2 * n + 1] = b;
      }
      n++;
    }
  return n;
}

// The reference's near-field cache key of the pair (a, b) of object no
// (GetFIBBICacheKey, FIBBICache.cc:171-201): 27 floats.
void rp_cache_key(void *g, int no, int a, int b, float *out) {
  SWGVolume *O = ((SWGGeometry *)g)->Objects[no];
  GetFIBBICacheKey(O, a, O, b, out);
}

// Vertex coordinates of object no as the reference holds them (after its
// mesh reader's node merge and any DISPLACED/ROTATED transformation).
int rp_vertices(void *g, int no, double *out) {
  SWGVolume *O = ((SWGGeometry *)g)->Objects[no];
  if (out) memcpy(out, O->Vertices, sizeof(double) * 3 * (size_t)O->NumVertices);
  return O->NumVertices;
}

// Near-field cache records held for object no (after a preload or assembly).
int rp_cache_size(void *g, int no) {
  SWGGeometry *G = (SWGGeometry *)g;
  return G->ObjectGCaches[no] ? G->ObjectGCaches[no]->Size() : -1;
}

// V^-1 overlap entries of object no, added into a zeroed N x N matrix
// (AssembleOverlapBlocks in its matrix mode, VIEMatrix.cc:321-360).
void rp_overlap_block(void *g, int no, double re_w, double im_w, double *out) {
  SWGGeometry *G = (SWGGeometry *)g;
  int N = G->Objects[no]->NumInteriorFaces;
  HMatrix M(N, N, LHM_COMPLEX);
  M.Zero();
  G->AssembleOverlapBlocks(no, cdouble(re_w, im_w), 0, 0.0, 0.0, 0, 0, 0, &M, 0);
  memcpy(out, (void *)M.ZM, sizeof(cdouble) * (size_t)N * N);
}

// Right-hand side for a plane wave (E0 as 3 complex = 6 doubles).
void rp_rhs(void *g, double re_w, double im_w, const double *E0, const double *nhat, double *out) {
  SWGGeometry *G = (SWGGeometry *)g;
  const cdouble *e = (const cdouble *)E0;
  PlaneWave PW(e, nhat);
  HVector *V = G->AssembleRHSVector(cdouble(re_w, im_w), &PW, G->AllocateRHSVector());
  memcpy(out, (void *)V->ZV, sizeof(cdouble) * (size_t)G->TotalBFs);
  delete V;
}

// PFT matrix (NumObjects x 8, row-major out) for current J; method 0 =
// overlap, 1 = energy/momentum transfer (needs the plane wave).
void rp_pft(void *g, const double *J, double re_w, double im_w, const double *E0, const double *nhat, int method,
            double *out) {
  SWGGeometry *G = (SWGGeometry *)g;
  int N = G->TotalBFs;
  HVector JV(N, LHM_COMPLEX);
  memcpy((void *)JV.ZV, J, sizeof(cdouble) * (size_t)N);
  PlaneWave PW((const cdouble *)E0, nhat);
  PFTOptions *Opt = BUFF_InitPFTOptions(0);
  Opt->PFTMethod = (method == 0) ? SCUFF_PFT_OVERLAP : SCUFF_PFT_EMT;
  Opt->IF = &PW;
  PW.SetFrequency(cdouble(re_w, im_w), true);
  HMatrix *P = G->GetPFTMatrix(&JV, cdouble(re_w, im_w), Opt, 0);
  for (int no = 0; no < G->NumObjects; no++)
    for (int q = 0; q < NUMPFT; q++) out[no * NUMPFT + q] = P->GetEntryD(no, q);
  delete P;
  free(Opt);
}

// Scattered fields (incident field left out) at np points: out is np x 6
// complex, row-major (Ex Ey Ez Hx Hy Hz per point).
void rp_fields(void *g, const double *J, double re_w, double im_w, int np, const double *X, double *out) {
  SWGGeometry *G = (SWGGeometry *)g;
  int N = G->TotalBFs;
  HVector JV(N, LHM_COMPLEX);
  memcpy((void *)JV.ZV, J, sizeof(cdouble) * (size_t)N);
  HMatrix XM(np, 3, LHM_REAL);
  for (int p = 0; p < np; p++)
    for (int i = 0; i < 3; i++) XM.SetEntry(p, i, X[3 * p + i]);
  HMatrix *F = G->GetFields(0, &JV, cdouble(re_w, im_w), &XM, 0);
  cdouble *z = (cdouble *)out;
  for (int p = 0; p < np; p++)
    for (int i = 0; i < 6; i++) z[6 * p + i] = F->GetEntry(p, i);
  delete F;
}

}  // extern "C"
