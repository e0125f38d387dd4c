// Test infrastructure: a project-written stand-in for the dense-matrix and
// vector classes of SCUFF-EM's libhmat, reduced to the members the
// reference's libbuff sources use (entry access, zeroing, the element type
// flag, wrapping caller memory).  Storage is column-major, double for
// LHM_REAL and complex128 for LHM_COMPLEX, so that a complex matrix can be
// handed to LAPACK by the caller.  Factorisation is not provided: the pin
// drivers export the matrix and factor it with LAPACK zgetrf on the Python
// side.
#ifndef REFPIN_LIBHMAT_H
#define REFPIN_LIBHMAT_H

#include "libhrutil.h"

#define LHM_REAL 0
#define LHM_COMPLEX 1
#define LHM_NORMAL 0

class HMatrix {
 public:
  // Data != null wraps caller memory of the given type (not freed)
  HMatrix(int NR, int NC, int RealComplex = LHM_REAL, int StorageType = LHM_NORMAL, void *Data = 0);
  ~HMatrix();
  void Zero();
  void SetEntry(int r, int c, cdouble v);
  void SetEntry(int r, int c, double v) { SetEntry(r, c, cdouble(v, 0.0)); }
  void AddEntry(int r, int c, cdouble v);
  void AddEntry(int r, int c, double v) { AddEntry(r, c, cdouble(v, 0.0)); }
  cdouble GetEntry(int r, int c) const;
  double GetEntryD(int r, int c) const { return real(GetEntry(r, c)); }
  // SetEntriesD(row, ":", values): a whole row from NC doubles
  void SetEntriesD(int r, const char *cols, const double *v);

  int NR, NC, RealComplex;
  double *DM;
  cdouble *ZM;
  bool Owns;
};

class HVector {
 public:
  HVector(int N, int RealComplex = LHM_REAL);
  ~HVector();
  void Zero();
  void SetEntry(int i, cdouble v);
  void SetEntry(int i, double v) { SetEntry(i, cdouble(v, 0.0)); }
  cdouble GetEntry(int i) const { return RealComplex == LHM_REAL ? cdouble(DV[i], 0.0) : ZV[i]; }
  double GetEntryD(int i) const { return real(GetEntry(i)); }

  int N, RealComplex;
  double *DV;
  cdouble *ZV;
};

// Sparse matrices appear in the reference's signatures only for the
// buff-neq overlap blocks; the hot path passes null pointers.  Any use
// ends the process.
class SMatrix {
 public:
  void SetEntry(int r, int c, cdouble v);
  void SetEntry(int r, int c, double v);
};

#endif
