// Test infrastructure: a project-written stand-in for the utility surface of
// SCUFF-EM's libhrutil that the reference's libbuff sources include.  Only the
// names, argument meanings and return values the reference's hot-path files
// use are provided; every body is in shim.cc.  SCUFF-EM is not vendored with
// the reference, so nothing here is its code.
#ifndef REFPIN_LIBHRUTIL_H
#define REFPIN_LIBHRUTIL_H

#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <strings.h>

typedef std::complex<double> cdouble;
typedef std::complex<float> cfloat;
using std::abs;
using std::conj;
using std::exp;
using std::imag;
using std::norm;
using std::real;
using std::sqrt;

#ifndef ZVAC
#define ZVAC 376.73031346177
#endif
// the reference's unit constant: Omega in units of 3e14 rad/s with lengths
// in um makes force prefactors carry 10/3
#ifndef TENTHIRDS
#define TENTHIRDS (10.0 / 3.0)
#endif
#ifndef ONEMEG
#define ONEMEG 1048576
#endif

// messages: ErrExit prints and exits the process (the reference's error path)
void ErrExit(const char *format, ...);
void Warn(const char *format, ...);
void Log(const char *format, ...);
void LogPercent(int n, int N, int Tenths = 10);

// allocation that exits on failure; mallocEC returns zeroed memory
void *mallocEC(size_t size);
void *reallocEC(void *p, size_t size);
char *strdupEC(const char *s);
char *vstrdup(const char *format, ...);
char *vstrappend(char *s, const char *format, ...);
void vsnprintfEC(char *buf, size_t n, const char *format, va_list ap);

void fprintVecCR(FILE *f, cdouble *v, int n);

// a complex number as text, for log messages (static buffer)
const char *z2s(cdouble z);

// strings and files
int Tokenize(char *s, char **Tokens, int MaxTokens);
int StrCaseCmp(const char *a, const char *b);
FILE *fopenPath(const char *Path, const char *FileName, const char *Mode, char **WhichDir = 0);
FILE *vfopen(const char *format, const char *mode, ...);
char *GetFileBase(const char *FileName);
char *GetFileExtension(const char *FileName);

// timing and resources
double Secs();
int GetNumThreads();
unsigned long GetMemoryUsage(unsigned long *MemoryUsage = 0);

// 3-vectors: the result goes to the last argument, which is returned
double *VecSub(const double *a, const double *b, double *c);
double *VecAdd(const double *a, const double *b, double *c);
double *VecCross(const double *a, const double *b, double *c);
double *VecScale(double *a, double s);
double *VecPlusEquals(double *a, double s, const double *b);
// length-N forms: a[0..N) += s b[0..N)
double *VecPlusEquals(double *a, double s, const double *b, int N);
cdouble *VecPlusEquals(cdouble *a, double s, const cdouble *b, int N);
double *VecCopy(const double *a, double *b);
double VecDot(const double *a, const double *b);
double VecNorm(const double *a);
double VecNorm2(const double *a);
double VecNormalize(double *a);
double VecDistance(const double *a, const double *b);

#endif
