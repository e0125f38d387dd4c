// Test infrastructure: a project-written stand-in for SCUFF-EM's incident
// fields, reduced to the plane wave in vacuum that the reference's RHS and
// EMT power routines evaluate: E = E0 exp(i k nHat.x), H = nHat x E / Z0,
// k = Omega (Omega in units of c / 1 um), with the x-derivatives.
#ifndef REFPIN_LIBINCFIELD_H
#define REFPIN_LIBINCFIELD_H

#include "libhrutil.h"

class IncField {
 public:
  IncField() : Next(0), Omega(0.0) {}
  virtual ~IncField() {}
  virtual void GetFields(const double X[3], cdouble EH[6]) = 0;
  virtual void GetFieldGradients(const double X[3], cdouble dEH[3][6]) = 0;
  void SetFrequency(cdouble W, bool Traverse = true);
  IncField *Next;
  cdouble Omega;
};

class PlaneWave : public IncField {
 public:
  PlaneWave(const cdouble E0[3], const double nHat[3]);
  void GetFields(const double X[3], cdouble EH[6]);
  void GetFieldGradients(const double X[3], cdouble dEH[3][6]);
  cdouble E0[3];
  double nHat[3];
};

#endif
