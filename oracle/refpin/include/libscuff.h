// Test infrastructure: the reference's libbuff sources include SCUFF-EM's
// libscuff header for its namespace, the geometric-transformation classes and
// a few helpers; this stand-in provides the namespace and pulls in the
// reference's own GTransformation.h (whose member functions are defined, by
// the project, in shim.cc).
#ifndef REFPIN_LIBSCUFF_H
#define REFPIN_LIBSCUFF_H

#include "libhrutil.h"
#include "libhmat.h"
#include "GTransformation.h"

namespace scuff {}

#endif
