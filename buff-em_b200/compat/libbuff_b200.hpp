// libbuff_b200.hpp -- header-only C++ layer that recreates the libbuff /
// libhmat names used on the VIE hot path on top of the C-ABI of
// include/buffem_b200.h, so a buff-scatter-style driver switches by changing
// its include and namespace:
//
//   buff::SWGGeometry *G = new buff::SWGGeometry(GeoFile);   // SWGGeometry.cc:214
//   HMatrix *M = G->AllocateVIEMatrix();                      // VIEMatrix.cc:465
//   HVector *J = G->AllocateRHSVector();                      // RHSVector.cc:49
//   G->AssembleVIEMatrix(Omega, M);                           // VIEMatrix.cc:431
//   M->LUFactorize();                                         // buff-scatter.cc:285
//   G->AssembleRHSVector(Omega, IF, J);                       // RHSVector.cc:85
//   M->LUSolve(J);                                            // buff-scatter.cc:314
//   HMatrix *PFT = G->GetPFTMatrix(J, Omega, IF);             // GetPFT.cc:133
//   G->GetFields(IF, J, Omega, X, EH);                        // GetFields.cc:387
//   BNEQ(G).GetFlux(Omega)                                    // buff-neq GetFlux.cc:291
//
// Differences from the reference: errors throw buff_b200::Error (carrying the
// C-ABI status and message) instead of calling ErrExit; the matrix lives on the
// device and GetEntry copies it to the host lazily; the incident field is a
// plane wave (libIncField's PlaneWave, E0 exp(i k nhat.x)).
#pragma once

#include <complex>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/buffem_b200.h"

namespace buff_b200 {

typedef std::complex<double> cdouble;

struct Error : std::runtime_error {
  int status;
  Error(int st, const char *msg) : std::runtime_error(std::string(msg)), status(st) {}
};

inline int check(int st) {
  if (st < 0) throw Error(st, bg_last_error());
  return st;
}

class HVector {
 public:
  int N;
  std::vector<cdouble> v;
  explicit HVector(int n) : N(n), v((size_t)n) {}
  cdouble GetEntry(int i) const { return v[(size_t)i]; }
  void SetEntry(int i, cdouble x) { v[(size_t)i] = x; }
  double *data() { return reinterpret_cast<double *>(v.data()); }
};

class HMatrix {
 public:
  int NR, NC;
  bg_matrix *m = nullptr;
  HMatrix(bg_geometry *g, int nr, int precision = BG_C128) : NR(nr), NC(nr) {
    check(bg_matrix_create(g, precision, &m));
  }
  ~HMatrix() { bg_matrix_destroy(m); }
  HMatrix(const HMatrix &) = delete;
  HMatrix &operator=(const HMatrix &) = delete;

  // HMatrix::LUFactorize -> zgetrf semantics; returns LAPACK info
  int LUFactorize() {
    int info = check(bg_lu_factor(m));
    host_.clear();
    if (info > 0) throw Error(info, "LUFactorize: singular matrix");
    return info;
  }
  // HMatrix::LUSolve(HVector*) -> zgetrs
  HVector *LUSolve(HVector *X) {
    check(bg_lu_solve(m, X->data(), 1));
    return X;
  }
  // multi-RHS form: column-major N x nrhs
  void LUSolve(cdouble *B, int nrhs) { check(bg_lu_solve(m, reinterpret_cast<double *>(B), nrhs)); }

  cdouble GetEntry(int r, int c) {
    if (host_.empty()) {
      host_.resize((size_t)NR * NC);
      check(bg_matrix_download(m, host_.data()));
    }
    return host_[(size_t)r + (size_t)c * NR];
  }
  void invalidate() { host_.clear(); }

 private:
  std::vector<cdouble> host_;
};

// SCUFF-EM PlaneWave(E0, nHat)
struct PlaneWave {
  cdouble E0[3];
  double nHat[3];
  PlaneWave(const cdouble pE0[3], const double pnHat[3]) {
    for (int i = 0; i < 3; i++) { E0[i] = pE0[i]; nHat[i] = pnHat[i]; }
  }
};

// The host-side fields of SWGVolume (libbuff.h:127-195) that the path's
// callers read: vertices after the one-time DISPLACED / ROTATED
// transformation, the origin about which torques are taken, counts, index.
struct SWGVolume {
  std::string Label;
  int Index = 0, NumVertices = 0, NumInteriorFaces = 0;
  std::vector<double> Vertices;   // 3 * NumVertices
  double Origin[3] = {0, 0, 0};
};

class SWGGeometry {
 public:
  int NumObjects = 0, TotalBFs = 0;
  std::vector<int> BFIndexOffset;
  std::vector<std::unique_ptr<SWGVolume>> Objects;   // Objects[no]->Vertices as in libbuff
  bg_geometry *g = nullptr;

  explicit SWGGeometry(const char *GeoFileName) {
    check(bg_geometry_create(GeoFileName, &g));
    init();
  }
  // the geometry with transformation k of a .trans file applied
  // (SWGGeometry::Transform, SWGGeometry.cc:426-439; one object per
  // transformation instead of Transform / UnTransform on one)
  SWGGeometry(const char *GeoFileName, const char *TransFile, int k) {
    check(bg_geometry_create_transformed(GeoFileName, TransFile, k, &g));
    init();
  }
  SWGGeometry(int nobj, const char *const *meshes, const double *disp, const bg_material *mats) {
    check(bg_geometry_create_objects(nobj, meshes, disp, mats, &g));
    init();
  }
  ~SWGGeometry() { bg_geometry_destroy(g); }
  SWGGeometry(const SWGGeometry &) = delete;
  SWGGeometry &operator=(const SWGGeometry &) = delete;

  // eps of object no at Omega (SVT->Evaluate for a homogeneous isotropic
  // object, SVTensor.cc:306-316; MATERIAL sections are evaluated at
  // w = Omega x 3e14 rad/s)
  cdouble GetEps(int no, cdouble Omega) const {
    double e[2];
    check(bg_geometry_material_eps(g, no, Omega.real(), Omega.imag(), e));
    return cdouble(e[0], e[1]);
  }

  // the permittivity tensor of object no at Omega and point X
  // (SVTensor::Evaluate, SVTensor.cc:306-373), for every kind of material
  void GetEpsTensor(int no, cdouble Omega, const double X[3], cdouble Q[3][3]) const {
    double q[18];
    check(bg_geometry_material_tensor(g, no, Omega.real(), Omega.imag(), X, q));
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) Q[a][b] = cdouble(q[2 * (3 * a + b)], q[2 * (3 * a + b) + 1]);
  }

  // SWGGeometry::GetObjectByLabel (SWGGeometry.cc:405-419)
  SWGVolume *GetObjectByLabel(const char *Label, int *pno = nullptr) {
    if (pno) *pno = -1;
    if (!Label) return nullptr;
    int no = bg_geometry_object_index(g, Label);
    if (no < 0) return nullptr;
    if (pno) *pno = no;
    return Objects[no].get();
  }

  HMatrix *AllocateVIEMatrix(bool PureImagFreq = false) {
    (void)PureImagFreq;
    return new HMatrix(g, TotalBFs);
  }
  HMatrix *AssembleVIEMatrix(cdouble Omega, HMatrix *M) {
    if (!M) M = AllocateVIEMatrix();
    check(bg_assemble(g, Omega.real(), Omega.imag(), M->m));
    M->invalidate();
    return M;
  }
  HVector *AllocateRHSVector() { return new HVector(TotalBFs); }
  HVector *AssembleRHSVector(cdouble Omega, const PlaneWave *IF, HVector *RHS) {
    if (!RHS) RHS = AllocateRHSVector();
    check(bg_rhs_planewave(g, Omega.real(), Omega.imag(), reinterpret_cast<const double *>(IF->E0), IF->nHat,
                           RHS->data()));
    return RHS;
  }
  // rows = objects; columns PAbs, PScat (PFT_PABS, PFT_PSCAT)
  std::vector<double> GetPFTMatrix(HVector *J, cdouble Omega, const PlaneWave *IF, int method = BG_PFT_EMT) {
    std::vector<double> out(2 * (size_t)NumObjects);
    check(bg_pft(g, Omega.real(), Omega.imag(), J->data(), IF ? reinterpret_cast<const double *>(IF->E0) : nullptr,
                 IF ? IF->nHat : nullptr, method, out.data()));
    return out;
  }
  // all eight EMT columns per object: PAbs, PScat, Fx, Fy, Fz, Tx, Ty, Tz (GetPFT.cc:133-189)
  std::vector<double> GetPFTMatrixFull(HVector *J, cdouble Omega, const PlaneWave *IF) {
    std::vector<double> out(8 * (size_t)NumObjects);
    check(bg_pft_full(g, Omega.real(), Omega.imag(), J->data(), reinterpret_cast<const double *>(IF->E0), IF->nHat,
                      out.data()));
    return out;
  }
  // SWGGeometry::GetFields(IF, J, Omega, XMatrix, FMatrix) (GetFields.cc:287-382):
  // X holds npts x 3 coordinates row by row; the result holds npts x 6 values
  // (Ex, Ey, Ez, Hx, Hy, Hz) row by row.  IF and J may be null, as in the reference.
  std::vector<cdouble> GetFields(const PlaneWave *IF, HVector *J, cdouble Omega, const std::vector<double> &X) {
    int npts = (int)(X.size() / 3);
    std::vector<cdouble> F(6 * (size_t)npts);
    check(bg_get_fields(g, Omega.real(), Omega.imag(), J ? J->data() : nullptr,
                        IF ? reinterpret_cast<const double *>(IF->E0) : nullptr, IF ? IF->nHat : nullptr, npts,
                        X.data(), reinterpret_cast<double *>(F.data())));
    return F;
  }
  // the one-point form (GetFields.cc:387-395)
  void GetFields(const PlaneWave *IF, HVector *J, cdouble Omega, const double X[3], cdouble EH[6]) {
    std::vector<cdouble> F = GetFields(IF, J, Omega, std::vector<double>(X, X + 3));
    for (int i = 0; i < 6; i++) EH[i] = F[i];
  }
  // FIBBICache::Store / PreLoad (FIBBICache.cc:272-463) for one object; return
  // the number of records written / matched
  int StoreFIBBICache(int obj, const char *path) {
    int n = 0;
    check(bg_fibbi_store(g, obj, path, &n));
    return n;
  }
  int PreloadFIBBICache(int obj, const char *path) {
    int n = 0;
    check(bg_fibbi_load(g, obj, path, &n));
    return n;
  }

 private:
  void init() {
    NumObjects = bg_geometry_num_objects(g);
    TotalBFs = bg_geometry_num_bfs(g);
    for (int i = 0; i <= NumObjects; i++) BFIndexOffset.push_back(bg_geometry_bf_offset(g, i));
    for (int i = 0; i < NumObjects; i++) {
      std::unique_ptr<SWGVolume> O(new SWGVolume);
      O->Index = i;
      O->NumVertices = check(bg_geometry_vertices(g, i, nullptr, nullptr));
      O->NumInteriorFaces = BFIndexOffset[i + 1] - BFIndexOffset[i];
      O->Vertices.resize(3 * (size_t)O->NumVertices);
      check(bg_geometry_vertices(g, i, O->Vertices.data(), O->Origin));
      std::vector<char> label(check(bg_geometry_object_label(g, i, nullptr, 0)) + 1);
      check(bg_geometry_object_label(g, i, label.data(), (int)label.size()));
      O->Label = label.data();
      Objects.push_back(std::move(O));
    }
  }
};

// buff-neq's flux chain for one geometry (GetFlux, GetFlux.cc:291-436):
// GetFlux(Omega)[(s * NO + d) * 8 + q], source s, destination d,
// q = PAbs, PRad, Fx, Fy, Fz, Tx, Ty, Tz (EMT, uniform temperature per object)
class BNEQ {
 public:
  explicit BNEQ(SWGGeometry &G) : NO(G.NumObjects) { check(bg_neq_create(G.g, &h)); }
  ~BNEQ() { bg_neq_destroy(h); }
  BNEQ(const BNEQ &) = delete;
  BNEQ &operator=(const BNEQ &) = delete;
  std::vector<double> GetFlux(cdouble Omega) {
    std::vector<double> out((size_t)NO * NO * 8);
    check(bg_neq_flux(h, Omega.real(), Omega.imag(), out.data()));
    return out;
  }

 private:
  int NO;
  bg_neq *h = nullptr;
};

}  // namespace buff_b200
