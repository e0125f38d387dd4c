// Test infrastructure: bodies of the project-written stand-ins declared in
// include/ for the SCUFF-EM surface (libhrutil, libhmat, libMatProp,
// libIncField, cmatheval, the scuff GTransformation members) that the
// reference's libbuff sources need to compile and link.  SCUFF-EM is not
// vendored with the reference; every body here is the project's own, written
// from what the reference's call sites require of it.
//
// Entry points that the pinned hot path must never reach (the moment and
// displaced-surface PFT methods, sparse matrices, Helmholtz Taylor-Duffy
// kernels) end the process with a message, so that a fixture can never
// silently contain a stand-in's value.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <sys/time.h>
#include <vector>
#include <omp.h>

#include "libhrutil.h"
#include "libhmat.h"
#include "libMatProp.h"
#include "libIncField.h"
#include "libSGJC.h"
#include "libTriInt.h"
#include "cmatheval.h"
#include "PFTOptions.h"
#include "GTransformation.h"

/* ------------------------------------------------------------ messages */
static int g_verbose = -1;
static bool verbose() {
  if (g_verbose < 0) g_verbose = getenv("REFPIN_VERBOSE") ? 1 : 0;
  return g_verbose == 1;
}

void ErrExit(const char *format, ...) {
  va_list ap;
  va_start(ap, format);
  fprintf(stderr, "reference error: ");
  vfprintf(stderr, format, ap);
  fprintf(stderr, "\n");
  va_end(ap);
  exit(1);
}

void Warn(const char *format, ...) {
  va_list ap;
  va_start(ap, format);
  fprintf(stderr, "reference warning: ");
  vfprintf(stderr, format, ap);
  fprintf(stderr, "\n");
  va_end(ap);
}

void Log(const char *format, ...) {
  if (!verbose()) return;
  va_list ap;
  va_start(ap, format);
  vfprintf(stderr, format, ap);
  fprintf(stderr, "\n");
  va_end(ap);
}

void LogPercent(int, int, int) {}

/* ------------------------------------------------------------ memory */
void *mallocEC(size_t size) {
  void *p = calloc(1, size ? size : 1);
  if (!p) ErrExit("out of memory (%zu bytes)", size);
  return p;
}

void *reallocEC(void *p, size_t size) {
  void *q = realloc(p, size ? size : 1);
  if (!q) ErrExit("out of memory (%zu bytes)", size);
  return q;
}

char *strdupEC(const char *s) {
  char *p = strdup(s ? s : "");
  if (!p) ErrExit("out of memory");
  return p;
}

static char *vformat(const char *format, va_list ap) {
  va_list aq;
  va_copy(aq, ap);
  int n = vsnprintf(0, 0, format, aq);
  va_end(aq);
  char *s = (char *)mallocEC((size_t)n + 1);
  vsnprintf(s, (size_t)n + 1, format, ap);
  return s;
}

char *vstrdup(const char *format, ...) {
  va_list ap;
  va_start(ap, format);
  char *s = vformat(format, ap);
  va_end(ap);
  return s;
}

char *vstrappend(char *s, const char *format, ...) {
  va_list ap;
  va_start(ap, format);
  char *t = vformat(format, ap);
  va_end(ap);
  size_t a = s ? strlen(s) : 0, b = strlen(t);
  char *r = (char *)reallocEC(s, a + b + 1);
  memcpy(r + a, t, b + 1);
  free(t);
  return r;
}

void vsnprintfEC(char *buf, size_t n, const char *format, va_list ap) {
  int k = vsnprintf(buf, n, format, ap);
  if (k < 0 || (size_t)k >= n) ErrExit("string too long: %s", format);
}

const char *z2s(cdouble z) {
  static thread_local char buf[64];
  snprintf(buf, sizeof buf, "(%g,%g)", real(z), imag(z));
  return buf;
}

/* ------------------------------------------------------------ strings, files */
// Splits s in place at blanks; a token starting with '#' ends the line.
int Tokenize(char *s, char **Tokens, int MaxTokens) {
  int n = 0;
  char *p = s;
  while (*p && n < MaxTokens) {
    while (*p && isspace((unsigned char)*p)) p++;
    if (!*p || *p == '#') break;
    Tokens[n++] = p;
    while (*p && !isspace((unsigned char)*p)) p++;
    if (*p) *p++ = 0;
  }
  return n;
}

int StrCaseCmp(const char *a, const char *b) { return strcasecmp(a, b); }

// Opens FileName as given, else in each directory of the colon-separated Path.
FILE *fopenPath(const char *Path, const char *FileName, const char *Mode, char **WhichDir) {
  FILE *f = fopen(FileName, Mode);
  if (f) {
    if (WhichDir) *WhichDir = strdupEC(".");
    return f;
  }
  if (!Path) return 0;
  std::string all(Path);
  size_t start = 0;
  while (start <= all.size()) {
    size_t end = all.find(':', start);
    if (end == std::string::npos) end = all.size();
    std::string dir = all.substr(start, end - start);
    if (!dir.empty()) {
      std::string full = dir + "/" + FileName;
      f = fopen(full.c_str(), Mode);
      if (f) {
        if (WhichDir) *WhichDir = strdupEC(dir.c_str());
        return f;
      }
    }
    start = end + 1;
  }
  return 0;
}

FILE *vfopen(const char *format, const char *mode, ...) {
  va_list ap;
  va_start(ap, mode);
  char *name = vformat(format, ap);
  va_end(ap);
  FILE *f = fopen(name, mode);
  free(name);
  return f;
}

// File name without directories and without its last extension (static buffer).
char *GetFileBase(const char *FileName) {
  static thread_local char buf[1024];
  const char *s = strrchr(FileName, '/');
  s = s ? s + 1 : FileName;
  snprintf(buf, sizeof buf, "%s", s);
  char *dot = strrchr(buf, '.');
  if (dot && dot != buf) *dot = 0;
  return buf;
}

char *GetFileExtension(const char *FileName) {
  const char *s = strrchr(FileName, '/');
  s = s ? s + 1 : FileName;
  const char *dot = strrchr(s, '.');
  return (char *)(dot ? dot + 1 : 0);
}

double Secs() {
  struct timeval tv;
  gettimeofday(&tv, 0);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

int GetNumThreads() { return omp_get_max_threads(); }

unsigned long GetMemoryUsage(unsigned long *MemoryUsage) {
  if (MemoryUsage) MemoryUsage[0] = 0;
  return 0;
}

/* ------------------------------------------------------------ 3-vectors */
double *VecSub(const double *a, const double *b, double *c) {
  for (int i = 0; i < 3; i++) c[i] = a[i] - b[i];
  return c;
}
double *VecAdd(const double *a, const double *b, double *c) {
  for (int i = 0; i < 3; i++) c[i] = a[i] + b[i];
  return c;
}
double *VecCross(const double *a, const double *b, double *c) {
  double x = a[1] * b[2] - a[2] * b[1], y = a[2] * b[0] - a[0] * b[2], z = a[0] * b[1] - a[1] * b[0];
  c[0] = x;
  c[1] = y;
  c[2] = z;
  return c;
}
double *VecScale(double *a, double s) {
  for (int i = 0; i < 3; i++) a[i] *= s;
  return a;
}
double *VecPlusEquals(double *a, double s, const double *b) { return VecPlusEquals(a, s, b, 3); }
double *VecPlusEquals(double *a, double s, const double *b, int N) {
  for (int i = 0; i < N; i++) a[i] += s * b[i];
  return a;
}
cdouble *VecPlusEquals(cdouble *a, double s, const cdouble *b, int N) {
  for (int i = 0; i < N; i++) a[i] += s * b[i];
  return a;
}
double *VecCopy(const double *a, double *b) {
  for (int i = 0; i < 3; i++) b[i] = a[i];
  return b;
}
double VecDot(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
double VecNorm2(const double *a) { return VecDot(a, a); }
double VecNorm(const double *a) { return sqrt(VecNorm2(a)); }
double VecNormalize(double *a) {
  double n = VecNorm(a);
  if (n > 0) VecScale(a, 1.0 / n);
  return n;
}
double VecDistance(const double *a, const double *b) {
  double d[3];
  return VecNorm(VecSub(a, b, d));
}

/* ------------------------------------------------------------ dense matrices */
HMatrix::HMatrix(int nr, int nc, int rc, int, void *Data) : NR(nr), NC(nc), RealComplex(rc), DM(0), ZM(0) {
  Owns = (Data == 0);
  size_t n = (size_t)nr * nc;
  if (rc == LHM_REAL)
    DM = Data ? (double *)Data : (double *)mallocEC(n * sizeof(double));
  else
    ZM = Data ? (cdouble *)Data : (cdouble *)mallocEC(n * sizeof(cdouble));
}
HMatrix::~HMatrix() {
  if (Owns) {
    free(DM);
    free(ZM);
  }
}
void HMatrix::Zero() {
  size_t n = (size_t)NR * NC;
  if (DM) memset(DM, 0, n * sizeof(double));
  if (ZM) memset((void *)ZM, 0, n * sizeof(cdouble));
}
void HMatrix::SetEntry(int r, int c, cdouble v) {
  size_t i = r + (size_t)NR * c;
  if (DM)
    DM[i] = real(v);
  else
    ZM[i] = v;
}
void HMatrix::AddEntry(int r, int c, cdouble v) {
  size_t i = r + (size_t)NR * c;
  if (DM)
    DM[i] += real(v);
  else
    ZM[i] += v;
}
cdouble HMatrix::GetEntry(int r, int c) const {
  size_t i = r + (size_t)NR * c;
  return DM ? cdouble(DM[i], 0.0) : ZM[i];
}
void HMatrix::SetEntriesD(int r, const char *cols, const double *v) {
  if (strcmp(cols, ":")) ErrExit("SetEntriesD: only ':' column ranges are supported");
  for (int c = 0; c < NC; c++) SetEntry(r, c, v[c]);
}

HVector::HVector(int n, int rc) : N(n), RealComplex(rc), DV(0), ZV(0) {
  if (rc == LHM_REAL)
    DV = (double *)mallocEC((size_t)n * sizeof(double));
  else
    ZV = (cdouble *)mallocEC((size_t)n * sizeof(cdouble));
}
HVector::~HVector() {
  free(DV);
  free(ZV);
}
void HVector::Zero() {
  if (DV) memset(DV, 0, (size_t)N * sizeof(double));
  if (ZV) memset((void *)ZV, 0, (size_t)N * sizeof(cdouble));
}
void HVector::SetEntry(int i, cdouble v) {
  if (DV)
    DV[i] = real(v);
  else
    ZV[i] = v;
}

void SMatrix::SetEntry(int, int, cdouble) { ErrExit("sparse matrices are not part of the pinned path"); }
void SMatrix::SetEntry(int, int, double) { ErrExit("sparse matrices are not part of the pinned path"); }

/* ------------------------------------------------------------ expressions */
// Recursive-descent parser into a small tree; variables are looked up by
// name at evaluation (bound by index through cevaluator_set_var_index, or
// fixed through cevaluator_set_var).
namespace {

struct Node {
  char op;            // 'n' number, 'v' variable, 'f' function, '~' negate, or + - * / ^
  cdouble val;
  std::string name;   // variable or function name
  int a = -1, b = -1;
};

struct Expr {
  std::vector<Node> nodes;
  int root = -1;
  std::vector<std::pair<std::string, int>> index;      // name -> position in the values array
  std::vector<std::pair<std::string, cdouble>> fixed;  // name -> constant value
};

struct Parser {
  const char *s;
  size_t p = 0;
  Expr &e;
  std::string err;
  Parser(const char *str, Expr &ex) : s(str), e(ex) {}
  void ws() {
    while (s[p] && isspace((unsigned char)s[p])) p++;
  }
  int add(Node n) {
    e.nodes.push_back(n);
    return (int)e.nodes.size() - 1;
  }
  int primary() {
    ws();
    char c = s[p];
    if (c == '(') {
      p++;
      int r = sum();
      ws();
      if (s[p] != ')') {
        err = "missing )";
        return -1;
      }
      p++;
      return r;
    }
    if (isdigit((unsigned char)c) || c == '.') {
      char *end;
      double v = strtod(s + p, &end);
      p = end - s;
      Node n;
      n.op = 'n';
      n.val = v;
      // an imaginary literal: a number followed directly by i
      if (s[p] == 'i' && !isalnum((unsigned char)s[p + 1]) && s[p + 1] != '_') {
        p++;
        n.val = cdouble(0.0, v);
      }
      return add(n);
    }
    if (isalpha((unsigned char)c) || c == '_') {
      size_t q = p;
      while (isalnum((unsigned char)s[p]) || s[p] == '_') p++;
      std::string name(s + q, p - q);
      ws();
      if (s[p] == '(') {
        p++;
        int arg = sum();
        ws();
        if (s[p] != ')') {
          err = "missing ) after function argument";
          return -1;
        }
        p++;
        Node n;
        n.op = 'f';
        n.name = name;
        n.a = arg;
        return add(n);
      }
      Node n;
      if (name == "i" || name == "I") {
        n.op = 'n';
        n.val = cdouble(0.0, 1.0);
      } else if (name == "pi") {
        n.op = 'n';
        n.val = M_PI;
      } else {
        n.op = 'v';
        n.name = name;
      }
      return add(n);
    }
    err = std::string("unexpected character in expression: ") + (c ? c : '?');
    return -1;
  }
  int unary() {
    ws();
    if (s[p] == '-') {
      p++;
      Node n;
      n.op = '~';
      n.a = unary();
      return add(n);
    }
    if (s[p] == '+') {
      p++;
      return unary();
    }
    return power();
  }
  int power() {
    int a = primary();
    ws();
    if (s[p] == '^') {
      p++;
      Node n;
      n.op = '^';
      n.a = a;
      n.b = unary();   // right-associative
      return add(n);
    }
    return a;
  }
  int product() {
    int a = unary();
    for (;;) {
      ws();
      char c = s[p];
      if (c != '*' && c != '/') return a;
      p++;
      Node n;
      n.op = c;
      n.a = a;
      n.b = unary();
      a = add(n);
    }
  }
  int sum() {
    int a = product();
    for (;;) {
      ws();
      char c = s[p];
      if (c != '+' && c != '-') return a;
      p++;
      Node n;
      n.op = c;
      n.a = a;
      n.b = product();
      a = add(n);
    }
  }
};

cdouble lookup(const Expr &e, const std::string &name, int count, char **names, cdouble *values) {
  for (auto &f : e.fixed)
    if (f.first == name) return f.second;
  for (auto &ix : e.index)
    if (ix.first == name && ix.second < count) return values[ix.second];
  for (int k = 0; k < count; k++)
    if (names && names[k] && name == names[k]) return values[k];
  ErrExit("expression uses undefined name %s", name.c_str());
  return 0.0;
}

cdouble eval(const Expr &e, int i, int count, char **names, cdouble *values) {
  const Node &n = e.nodes[i];
  switch (n.op) {
    case 'n': return n.val;
    case 'v': return lookup(e, n.name, count, names, values);
    case '~': return -eval(e, n.a, count, names, values);
    case '+': return eval(e, n.a, count, names, values) + eval(e, n.b, count, names, values);
    case '-': return eval(e, n.a, count, names, values) - eval(e, n.b, count, names, values);
    case '*': return eval(e, n.a, count, names, values) * eval(e, n.b, count, names, values);
    case '/': return eval(e, n.a, count, names, values) / eval(e, n.b, count, names, values);
    case '^': {
      cdouble a = eval(e, n.a, count, names, values), b = eval(e, n.b, count, names, values);
      if (imag(b) == 0.0 && real(b) == std::floor(real(b)) && std::fabs(real(b)) <= 64) {
        int k = (int)real(b);
        cdouble r = 1.0, x = (k < 0) ? 1.0 / a : a;
        for (int j = 0; j < std::abs(k); j++) r *= x;
        return r;
      }
      return std::pow(a, b);
    }
    case 'f': {
      cdouble x = eval(e, n.a, count, names, values);
      const std::string &f = n.name;
      if (f == "exp") return std::exp(x);
      if (f == "log") return std::log(x);
      if (f == "sqrt") return std::sqrt(x);
      if (f == "sin") return std::sin(x);
      if (f == "cos") return std::cos(x);
      if (f == "tan") return std::tan(x);
      if (f == "sinh") return std::sinh(x);
      if (f == "cosh") return std::cosh(x);
      if (f == "tanh") return std::tanh(x);
      if (f == "abs") return std::abs(x);
      if (f == "step") return real(x) < 0 ? 0.0 : 1.0;
      ErrExit("unknown function %s", f.c_str());
    }
  }
  ErrExit("bad expression node");
  return 0.0;
}

}  // namespace

void *cevaluator_create(char *string) {
  Expr *e = new Expr;
  Parser ps(string, *e);
  e->root = ps.sum();
  ps.ws();
  if (e->root < 0 || !ps.err.empty() || string[ps.p]) {
    delete e;
    return 0;
  }
  return e;
}

void cevaluator_destroy(void *ev) { delete (Expr *)ev; }

void cevaluator_set_var_index(void *ev, const char *name, int index) {
  ((Expr *)ev)->index.push_back({name, index});
}

void cevaluator_set_var(void *ev, const char *name, cdouble value) {
  ((Expr *)ev)->fixed.push_back({name, value});
}

cdouble cevaluator_evaluate(void *ev, int count, char **names, cdouble *values) {
  const Expr *e = (const Expr *)ev;
  return eval(*e, e->root, count, names, values);
}

/* ------------------------------------------------------------ materials */
double MatProp::FreqUnit = 3.0e14;

namespace {
struct MaterialDef {
  std::string name;
  std::vector<std::pair<std::string, cdouble>> constants;
  std::string eps;   // expression of w (rad/s)
};
std::vector<MaterialDef> g_materials;
}  // namespace

static bool parse_complex(const char *s, cdouble *v) {
  void *e = cevaluator_create((char *)s);
  if (!e) return false;
  *v = cevaluator_evaluate(e, 0, 0, 0);
  cevaluator_destroy(e);
  return true;
}

MatProp::MatProp(const char *name) : Name(strdupEC(name)), ErrMsg(0), Constant(1.0), EpsExpr(0) {
  if (!strcasecmp(name, "VACUUM")) return;
  if (!strncasecmp(name, "CONST_EPS_", 10)) {
    if (!parse_complex(name + 10, &Constant)) ErrMsg = vstrdup("invalid constant permittivity %s", name);
    return;
  }
  for (auto &m : g_materials)
    if (!strcasecmp(m.name.c_str(), name)) {
      Expr *e = (Expr *)cevaluator_create((char *)m.eps.c_str());
      if (!e) {
        ErrMsg = vstrdup("invalid Eps(w) for material %s", name);
        return;
      }
      for (auto &c : m.constants) e->fixed.push_back(c);
      e->index.push_back({"w", 0});
      EpsExpr = e;
      return;
    }
  ErrMsg = vstrdup("unknown material %s", name);
}

MatProp::~MatProp() {
  free(Name);
  if (EpsExpr) cevaluator_destroy(EpsExpr);
}

cdouble MatProp::GetEps(cdouble Omega) {
  if (!EpsExpr) return Constant;
  cdouble w = Omega * FreqUnit;
  return cevaluator_evaluate(EpsExpr, 1, 0, &w);
}

// MATERIAL name ... ENDMATERIAL: "NAME = value" constants (each may use the
// ones before it) and "Eps(w) = expression".
char *AddMaterialToMatPropDataBase(FILE *f, char *FileName, char *MatName, int *LineNum) {
  MaterialDef m;
  m.name = MatName;
  char line[4096];
  while (fgets(line, sizeof line, f)) {
    if (LineNum) (*LineNum)++;
    char *s = line;
    while (isspace((unsigned char)*s)) s++;
    char *semi = strchr(s, ';');
    if (semi) *semi = 0;
    char *nl = strpbrk(s, "\r\n#");
    if (nl) *nl = 0;
    if (!*s) continue;
    if (!strncasecmp(s, "ENDMATERIAL", 11)) {
      if (m.eps.empty()) return vstrdup("%s: material %s has no Eps(w)", FileName, MatName);
      g_materials.push_back(m);
      return 0;
    }
    char *eq = strchr(s, '=');
    if (!eq) return vstrdup("%s:%d: syntax error", FileName, LineNum ? *LineNum : 0);
    *eq = 0;
    std::string lhs(s), rhs(eq + 1);
    while (!lhs.empty() && isspace((unsigned char)lhs.back())) lhs.pop_back();
    if (!strncasecmp(lhs.c_str(), "Eps(w)", 6)) {
      m.eps = rhs;
    } else if (!strncasecmp(lhs.c_str(), "Mu(w)", 5)) {
      // non-magnetic volume problem: ignored
    } else {
      Expr *e = (Expr *)cevaluator_create((char *)rhs.c_str());
      if (!e) return vstrdup("%s: bad constant %s", FileName, lhs.c_str());
      for (auto &c : m.constants) e->fixed.push_back(c);
      m.constants.push_back({lhs, cevaluator_evaluate(e, 0, 0, 0)});
      cevaluator_destroy(e);
    }
  }
  return vstrdup("%s: MATERIAL %s without ENDMATERIAL", FileName, MatName);
}

/* ------------------------------------------------------------ incident field */
void IncField::SetFrequency(cdouble W, bool Traverse) {
  Omega = W;
  if (Traverse)
    for (IncField *n = Next; n; n = n->Next) n->Omega = W;
}

PlaneWave::PlaneWave(const cdouble e0[3], const double nh[3]) {
  for (int i = 0; i < 3; i++) {
    E0[i] = e0[i];
    nHat[i] = nh[i];
  }
}

void PlaneWave::GetFields(const double X[3], cdouble EH[6]) {
  cdouble k = Omega;   // vacuum exterior: k = Omega in units of 1/um
  cdouble ph = std::exp(cdouble(0.0, 1.0) * k * (nHat[0] * X[0] + nHat[1] * X[1] + nHat[2] * X[2]));
  cdouble E[3] = {E0[0] * ph, E0[1] * ph, E0[2] * ph};
  for (int i = 0; i < 3; i++) EH[i] = E[i];
  EH[3] = (nHat[1] * E[2] - nHat[2] * E[1]) / ZVAC;
  EH[4] = (nHat[2] * E[0] - nHat[0] * E[2]) / ZVAC;
  EH[5] = (nHat[0] * E[1] - nHat[1] * E[0]) / ZVAC;
}

void PlaneWave::GetFieldGradients(const double X[3], cdouble dEH[3][6]) {
  cdouble EH[6];
  GetFields(X, EH);
  cdouble ik = cdouble(0.0, 1.0) * Omega;
  for (int mu = 0; mu < 3; mu++)
    for (int n = 0; n < 6; n++) dEH[mu][n] = ik * nHat[mu] * EH[n];
}

/* ------------------------------------------------------------ adaptive cubature */
// h-adaptive cubature over a box, the published algorithm of A. C. Genz and
// A. A. Malik, "An adaptive algorithm for numerical integration over an
// N-dimensional rectangular region", J. Comput. Appl. Math. 6 (1980) 295-302:
// a degree-7 fully symmetric rule with an embedded degree-5 rule; the box with
// the largest error estimate |I7 - I5| is halved along the coordinate with the
// largest fourth divided difference until every component's summed error is
// within max(reqAbsError, reqRelError |I|) (ERROR_INDIVIDUAL) or maxEval
// evaluations are spent (maxEval 0: no limit).  The cubature library the
// reference links (SGJ's) is not vendored; this is the project's own code.
namespace {
struct Box {
  std::vector<double> c, h;       // centre, half-widths
  std::vector<double> I, E;       // integral and error per component
  int split;                      // coordinate to halve next
  double key;                     // largest error component
};

int gm_eval(integrand f, void *fdata, unsigned n, unsigned fdim, Box &b, size_t &evals) {
  const double l2 = sqrt(9.0 / 70.0), l4 = sqrt(9.0 / 10.0), l5 = sqrt(9.0 / 19.0);
  const double nn = n;
  const double w1 = (12824.0 - 9120.0 * nn + 400.0 * nn * nn) / 19683.0, w2 = 980.0 / 6561.0,
               w3 = (1820.0 - 400.0 * nn) / 19683.0, w4 = 200.0 / 19683.0, w5 = 6859.0 / 19683.0 / ldexp(1.0, n);
  const double v1 = (729.0 - 950.0 * nn + 50.0 * nn * nn) / 729.0, v2 = 245.0 / 486.0,
               v3 = (265.0 - 100.0 * nn) / 1458.0, v4 = 25.0 / 729.0;
  std::vector<double> x(n), f0(fdim), fp(fdim), fm(fdim), s2(fdim, 0), s3(fdim, 0), s4(fdim, 0), s5(fdim, 0);
  double vol = 1.0;
  for (unsigned i = 0; i < n; i++) vol *= 2.0 * b.h[i];
  auto at = [&](std::vector<double> &fv) {
    if (f(n, x.data(), fdata, fdim, fv.data())) return 1;
    evals++;
    return 0;
  };
  x = b.c;
  if (at(f0)) return 1;
  double best = -1;
  b.split = 0;
  for (unsigned i = 0; i < n; i++) {
    std::vector<double> a2(fdim), a3(fdim);
    for (int sgn = 0; sgn < 2; sgn++) {
      x = b.c;
      x[i] += (sgn ? -1 : 1) * l2 * b.h[i];
      if (at(sgn ? fm : fp)) return 1;
    }
    for (unsigned k = 0; k < fdim; k++) {
      a2[k] = fp[k] + fm[k];
      s2[k] += a2[k];
    }
    for (int sgn = 0; sgn < 2; sgn++) {
      x = b.c;
      x[i] += (sgn ? -1 : 1) * l4 * b.h[i];
      if (at(sgn ? fm : fp)) return 1;
    }
    for (unsigned k = 0; k < fdim; k++) {
      a3[k] = fp[k] + fm[k];
      s3[k] += a3[k];
    }
    // fourth difference along i, summed over the components
    double diff = 0;
    for (unsigned k = 0; k < fdim; k++)
      diff += std::fabs(a2[k] - 2 * f0[k] - (l2 * l2 / (l4 * l4)) * (a3[k] - 2 * f0[k]));
    if (diff > best * (1 + 1e-12)) {
      best = diff;
      b.split = i;
    }
  }
  for (unsigned i = 0; i < n; i++)
    for (unsigned j = i + 1; j < n; j++)
      for (int si = 0; si < 2; si++)
        for (int sj = 0; sj < 2; sj++) {
          x = b.c;
          x[i] += (si ? -1 : 1) * l4 * b.h[i];
          x[j] += (sj ? -1 : 1) * l4 * b.h[j];
          if (at(fp)) return 1;
          for (unsigned k = 0; k < fdim; k++) s4[k] += fp[k];
        }
  for (unsigned m = 0; m < (1u << n); m++) {
    for (unsigned i = 0; i < n; i++) x[i] = b.c[i] + (((m >> i) & 1) ? -1 : 1) * l5 * b.h[i];
    if (at(fp)) return 1;
    for (unsigned k = 0; k < fdim; k++) s5[k] += fp[k];
  }
  b.I.assign(fdim, 0);
  b.E.assign(fdim, 0);
  b.key = 0;
  for (unsigned k = 0; k < fdim; k++) {
    double i7 = vol * (w1 * f0[k] + w2 * s2[k] + w3 * s3[k] + w4 * s4[k] + w5 * s5[k]);
    double i5 = vol * (v1 * f0[k] + v2 * s2[k] + v3 * s3[k] + v4 * s4[k]);
    b.I[k] = i7;
    b.E[k] = std::fabs(i7 - i5);
    if (b.E[k] > b.key) b.key = b.E[k];
  }
  return 0;
}
}  // namespace

int hcubature(unsigned fdim, integrand f, void *fdata, unsigned dim, const double *xmin, const double *xmax,
              size_t maxEval, double reqAbsError, double reqRelError, error_norm, double *val, double *err) {
  std::vector<Box> heap(1);
  heap[0].c.resize(dim);
  heap[0].h.resize(dim);
  for (unsigned i = 0; i < dim; i++) {
    heap[0].c[i] = 0.5 * (xmin[i] + xmax[i]);
    heap[0].h[i] = 0.5 * (xmax[i] - xmin[i]);
  }
  size_t evals = 0;
  if (gm_eval(f, fdata, dim, fdim, heap[0], evals)) return 1;
  auto cmp = [](const Box &a, const Box &b) { return a.key < b.key; };
  std::vector<double> I(heap[0].I), E(heap[0].E);
  for (;;) {
    bool done = true;
    for (unsigned k = 0; k < fdim; k++)
      if (E[k] > reqAbsError && E[k] > reqRelError * std::fabs(I[k])) done = false;
    if (done || (maxEval && evals >= maxEval)) break;
    std::pop_heap(heap.begin(), heap.end(), cmp);
    Box b = heap.back();
    heap.pop_back();
    Box c1 = b, c2 = b;
    int s = b.split;
    c1.h[s] = c2.h[s] = 0.5 * b.h[s];
    c1.c[s] = b.c[s] - c1.h[s];
    c2.c[s] = b.c[s] + c2.h[s];
    if (gm_eval(f, fdata, dim, fdim, c1, evals) || gm_eval(f, fdata, dim, fdim, c2, evals)) return 1;
    for (unsigned k = 0; k < fdim; k++) {
      I[k] += c1.I[k] + c2.I[k] - b.I[k];
      E[k] += c1.E[k] + c2.E[k] - b.E[k];
    }
    heap.push_back(c1);
    std::push_heap(heap.begin(), heap.end(), cmp);
    heap.push_back(c2);
    std::push_heap(heap.begin(), heap.end(), cmp);
    // summed estimates drift by rounding over many splits: re-sum now and then
    if (heap.size() % 256 == 0) {
      std::fill(I.begin(), I.end(), 0.0);
      std::fill(E.begin(), E.end(), 0.0);
      for (auto &h : heap)
        for (unsigned k = 0; k < fdim; k++) {
          I[k] += h.I[k];
          E[k] += h.E[k];
        }
    }
  }
  for (unsigned k = 0; k < fdim; k++) {
    val[k] = 0;
    if (err) err[k] = 0;
  }
  for (auto &h : heap)
    for (unsigned k = 0; k < fdim; k++) {
      val[k] += h.I[k];
      if (err) err[k] += h.E[k];
    }
  return 0;
}

// The reference calls this for integrals of dimension <= 2 (and for fixed
// orders); here it is the same adaptive rule.
int CCCubature(int, unsigned fdim, integrand f, void *fdata, unsigned dim, const double *xmin, const double *xmax,
               size_t maxEval, double reqAbsError, double reqRelError, error_norm norm, double *val, double *err) {
  return hcubature(fdim, f, fdata, dim, xmin, xmax, maxEval, reqAbsError, reqRelError, norm, val, err);
}

double *GetTCR(int, int *NumPts) {
  if (NumPts) *NumPts = 0;
  return 0;
}

void fprintVecCR(FILE *f, cdouble *v, int n) {
  for (int i = 0; i < n; i++) fprintf(f, "%+.8e %+.8e ", real(v[i]), imag(v[i]));
  fprintf(f, "\n");
}

namespace scuff {
// The kernel functions of the generalised Taylor-Duffy method (M. T. H. Reid,
// J. K. White, S. G. Johnson, IEEE Trans. Antennas Propag. 63(1), 2015):
// K_n(X) = int_0^1 w^n K(w X) dw for n = nMin..nMax (stored at index n).
// For the power kernels K(r) = r^p (TTD_RP, p = real(KParam)) this is
// X^p / (n + p + 1).  The Helmholtz kernels are not part of the pinned path
// (the near field is assembled from static integrals).
void GetScriptK(int WhichK, cdouble KParam, double X, int nMin, int nMax, cdouble *KVector) {
  if (WhichK != 0) ErrExit("only the power kernels of Taylor-Duffy are part of the pinned path");
  double p = real(KParam);
  for (int n = nMin; n <= nMax; n++) KVector[n] = std::pow(X, p) / (n + p + 1.0);
}

// Homogeneous dyadic Green's functions of the field routine (restated from
// their definitions, SCUFF-EM's own CalcGC is not vendored), R = R1 - R2:
//   G_mn = [delta_mn + d_m d_n / k^2] phi,   C_mn = (1 / ik) eps_mnr d_r phi,
//   phi = exp(ikr) / (4 pi r),  k = Omega sqrt(EpsR MuR).
// The derivative arrays are not used on the pinned path.
void CalcGC(double R1[3], double R2[3], cdouble Omega, cdouble EpsR, cdouble MuR, cdouble GMuNu[3][3],
            cdouble CMuNu[3][3], cdouble GMuNuRho[3][3][3], cdouble CMuNuRho[3][3][3]) {
  if (GMuNuRho || CMuNuRho) ErrExit("CalcGC derivatives are not part of the pinned path");
  double R[3] = {R1[0] - R2[0], R1[1] - R2[1], R1[2] - R2[2]};
  double r = VecNorm(R);
  cdouble k = Omega * std::sqrt(EpsR * MuR), ik = cdouble(0.0, 1.0) * k;
  cdouble phi = std::exp(ik * r) / (4.0 * M_PI * r);
  cdouble d1 = phi * (ik - 1.0 / r);                                       // dphi/dr
  cdouble d2 = phi * ((ik - 1.0 / r) * (ik - 1.0 / r) + 1.0 / (r * r));    // d2phi/dr2
  for (int m = 0; m < 3; m++)
    for (int n = 0; n < 3; n++) {
      double rr = R[m] * R[n] / (r * r);
      cdouble dmn = rr * d2 + ((m == n ? 1.0 : 0.0) - rr) * d1 / r;      // d_m d_n phi
      GMuNu[m][n] = (m == n ? phi : 0.0) + dmn / (k * k);
    }
  cdouble c = d1 / (ik * r);   // (1/ik) dphi/dr / r, times R_r below
  for (int m = 0; m < 3; m++) {
    CMuNu[m][m] = 0.0;
    int n = (m + 1) % 3, q = (m + 2) % 3;   // eps_{m n q} = +1
    CMuNu[m][n] = c * R[q];
    CMuNu[n][m] = -c * R[q];
  }
}

void InitPFTOptions(PFTOptions *o) {
  memset(o, 0, sizeof *o);
  o->PFTMethod = SCUFF_PFT_OVERLAP;
  o->DSIRadius = 5.0;
  o->DSIPoints = 110;
}

/* ------------------------------------------------------------ transformations */
// XP = M X + DX
GTransformation::GTransformation() { Reset(); }
GTransformation::GTransformation(const double dx[3]) {
  Reset();
  Displace(dx);
}
GTransformation::GTransformation(const double ZHat[3], double ThetaDegrees) {
  Reset();
  Rotate(ZHat, ThetaDegrees);
}
GTransformation::GTransformation(const char *s, char **ErrMsg) {
  Reset();
  Parse(s, ErrMsg);
}
GTransformation::GTransformation(char **Tokens, int NumTokens, char **ErrMsg, int *TokensConsumed) {
  Reset();
  Parse(Tokens, NumTokens, ErrMsg, TokensConsumed);
}
GTransformation::GTransformation(const GTransformation &G) { *this = G; }
GTransformation::GTransformation(const GTransformation *G) { *this = *G; }
void GTransformation::operator=(const GTransformation &G) {
  memcpy(DX, G.DX, sizeof DX);
  memcpy(M, G.M, sizeof M);
}
void GTransformation::Reset() {
  for (int i = 0; i < 3; i++) {
    DX[i] = 0;
    for (int j = 0; j < 3; j++) M[i][j] = (i == j) ? 1.0 : 0.0;
  }
}
void GTransformation::Displace(const double dx[3]) {
  for (int i = 0; i < 3; i++) DX[i] += dx[i];
}
// rotation by ThetaDegrees about the axis ZHat (right-hand rule), applied after this one
void GTransformation::Rotate(const double ZHat[3], double ThetaDegrees) {
  double a[3] = {ZHat[0], ZHat[1], ZHat[2]};
  VecNormalize(a);
  double t = ThetaDegrees * M_PI / 180.0, c = cos(t), s = sin(t), R[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) R[i][j] = (1 - c) * a[i] * a[j] + ((i == j) ? c : 0.0);
  R[0][1] -= s * a[2];
  R[0][2] += s * a[1];
  R[1][0] += s * a[2];
  R[1][2] -= s * a[0];
  R[2][0] -= s * a[1];
  R[2][1] += s * a[0];
  GTransformation G;
  memcpy(G.M, R, sizeof R);
  Transform(&G);
}
// this <- G * this
void GTransformation::Transform(const GTransformation *G) {
  double NM[3][3], ND[3];
  for (int i = 0; i < 3; i++) {
    ND[i] = G->DX[i];
    for (int j = 0; j < 3; j++) {
      NM[i][j] = 0;
      for (int k = 0; k < 3; k++) NM[i][j] += G->M[i][k] * M[k][j];
      ND[i] += G->M[i][j] * DX[j];
    }
  }
  memcpy(M, NM, sizeof M);
  memcpy(DX, ND, sizeof DX);
}
void GTransformation::Invert() { *this = Inverse(); }
GTransformation GTransformation::Inverse() const {
  GTransformation G;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) G.M[i][j] = M[j][i];   // rotations only
  for (int i = 0; i < 3; i++) {
    G.DX[i] = 0;
    for (int j = 0; j < 3; j++) G.DX[i] -= G.M[i][j] * DX[j];
  }
  return G;
}
bool GTransformation::Parse(const char *s, char **ErrMsg) {
  char *copy = strdupEC(s), *Tokens[50];
  int n = Tokenize(copy, Tokens, 50), used = 0;
  bool ok = Parse(Tokens, n, ErrMsg, &used);
  free(copy);
  return ok;
}
// DISPLACED dx dy dz | ROTATED theta ABOUT ax ay az, repeated
bool GTransformation::Parse(char **Tokens, int NumTokens, char **ErrMsg, int *TokensConsumed) {
  if (ErrMsg) *ErrMsg = 0;
  int p = 0;
  while (p < NumTokens) {
    if (!strcasecmp(Tokens[p], "DISPLACED") && p + 3 < NumTokens) {
      double d[3] = {atof(Tokens[p + 1]), atof(Tokens[p + 2]), atof(Tokens[p + 3])};
      GTransformation G(d);
      Transform(&G);
      p += 4;
    } else if (!strcasecmp(Tokens[p], "ROTATED") && p + 5 < NumTokens && !strcasecmp(Tokens[p + 2], "ABOUT")) {
      double ax[3] = {atof(Tokens[p + 3]), atof(Tokens[p + 4]), atof(Tokens[p + 5])};
      Rotate(ax, atof(Tokens[p + 1]));
      p += 6;
    } else
      break;
  }
  if (TokensConsumed) *TokensConsumed = p;
  if (p == 0 && ErrMsg) *ErrMsg = strdupEC("invalid transformation");
  return p > 0;
}
GTransformation GTransformation::operator+(const GTransformation &G) const {
  GTransformation R(this);
  R.Transform(&G);
  return R;
}
GTransformation GTransformation::operator-(const GTransformation &G) const {
  GTransformation R(this), Gi = G.Inverse();
  R.Transform(&Gi);
  return R;
}
void GTransformation::Apply(const double *X, double *XP, int NX) const {
  for (int n = 0; n < NX; n++) {
    double x[3] = {X[3 * n], X[3 * n + 1], X[3 * n + 2]};
    for (int i = 0; i < 3; i++) XP[3 * n + i] = DX[i] + M[i][0] * x[0] + M[i][1] * x[1] + M[i][2] * x[2];
  }
}
void GTransformation::UnApply(const double *X, double *XP, int NX) const {
  GTransformation G = Inverse();
  G.Apply(X, XP, NX);
}
void GTransformation::ApplyRotation(const double X[3], double XP[3]) const {
  double x[3] = {X[0], X[1], X[2]};
  for (int i = 0; i < 3; i++) XP[i] = M[i][0] * x[0] + M[i][1] * x[1] + M[i][2] * x[2];
}
void GTransformation::UnApplyRotation(const double X[3], double XP[3]) const {
  double x[3] = {X[0], X[1], X[2]};
  for (int i = 0; i < 3; i++) XP[i] = M[0][i] * x[0] + M[1][i] * x[1] + M[2][i] * x[2];
}
}  // namespace scuff
