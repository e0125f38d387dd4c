// Test infrastructure: the options structure and column indices of the
// power/force/torque (PFT) routines, as the reference's GetPFT.cc, EMTPFT.cc
// and OPFT.cc use them (the header itself belongs to SCUFF-EM, which is not
// vendored).  Column order: absorbed power, scattered power, force x/y/z,
// torque x/y/z.
#ifndef REFPIN_PFTOPTIONS_H
#define REFPIN_PFTOPTIONS_H

#include "libhmat.h"
#include "libIncField.h"

#define SCUFF_PFT_OVERLAP 0
#define SCUFF_PFT_EMT 1
#define SCUFF_PFT_MOMENTS 2
#define SCUFF_PFT_DSI 3

#define PFT_PABS 0
#define PFT_PSCAT 1
#define PFT_XFORCE 2
#define PFT_YFORCE 3
#define PFT_ZFORCE 4
#define PFT_XTORQUE 5
#define PFT_YTORQUE 6
#define PFT_ZTORQUE 7

namespace scuff {

typedef struct PFTOptions {
  int PFTMethod;
  HMatrix *DRMatrix;
  HVector *RHSVector;
  IncField *IF;
  char *DSIMesh;
  double DSIRadius;
  int DSIPoints;
} PFTOptions;

// overlap-method defaults; the pin drivers set the method they test
void InitPFTOptions(PFTOptions *Options);

}  // namespace scuff

#endif
