// Test infrastructure: the triangle-rule lookup the reference's face
// integrals name; unused on the volume hot path, so shim.cc returns null.
#ifndef REFPIN_LIBTRIINT_H
#define REFPIN_LIBTRIINT_H
double *GetTCR(int Order, int *NumPts);
#endif
