// Test infrastructure: declarations of the adaptive-cubature entry points
// the reference's Cubature.cc names (the cubature library is third-party and
// not vendored).  The hot path of the pin never calls them -- fixed-rule
// cubature only -- so shim.cc defines them to end the process.
#ifndef REFPIN_LIBSGJC_H
#define REFPIN_LIBSGJC_H

#include <cstddef>

typedef int (*integrand)(unsigned ndim, const double *x, void *fdata, unsigned fdim, double *fval);
typedef enum { ERROR_INDIVIDUAL = 0, ERROR_PAIRED, ERROR_L2, ERROR_L1, ERROR_LINF } error_norm;

int hcubature(unsigned fdim, integrand f, void *fdata, unsigned dim, const double *xmin, const double *xmax,
              size_t maxEval, double reqAbsError, double reqRelError, error_norm norm, double *val, double *err);
int CCCubature(int Order, unsigned fdim, integrand f, void *fdata, unsigned dim, const double *xmin,
               const double *xmax, size_t maxEval, double reqAbsError, double reqRelError, error_norm norm,
               double *val, double *err);

#endif
