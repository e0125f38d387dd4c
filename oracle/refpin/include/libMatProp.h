// Test infrastructure: a project-written stand-in for SCUFF-EM's MatProp
// (isotropic material properties), reduced to what the reference's SVTensor
// uses: construction from a name, GetEps(Omega), Name, ErrMsg and the
// frequency unit.  Names understood: VACUUM, CONST_EPS_<complex number>
// (e.g. CONST_EPS_4+0.2i) and materials defined by MATERIAL ... ENDMATERIAL
// sections (constants "NAME = value" and "Eps(w) = expression of w" in
// rad/s), registered by AddMaterialToMatPropDataBase.
#ifndef REFPIN_LIBMATPROP_H
#define REFPIN_LIBMATPROP_H

#include "libhrutil.h"

class MatProp {
 public:
  MatProp(const char *Name);
  ~MatProp();
  cdouble GetEps(cdouble Omega);
  char *Name;
  char *ErrMsg;
  static double FreqUnit;   // rad/s per unit of the solver's Omega (3e14)

  cdouble Constant;         // CONST_EPS_ / VACUUM value
  void *EpsExpr;            // parsed Eps(w) of a MATERIAL section, or null
};

char *AddMaterialToMatPropDataBase(FILE *f, char *FileName, char *MatName, int *LineNum);

#endif
