// Frequency-dependent isotropic materials of .buffgeo files:
//
//   MATERIAL Gold
//     wp = 1.37e16;
//     gamma = 5.32e13;
//     Eps(w) = 1 - wp^2 / (w * (w + i*gamma));
//   ENDMATERIAL
//
// The reference hands these sections to SCUFF-EM's MatProp database
// (AddMaterialToMatPropDataBase, SWGGeometry.cc:318-330; SVTensor.cc:306-316),
// which evaluates them with the complex expression library cmatheval; neither
// is vendored.  This file restates what those sections mean: constants are
// complex expressions evaluated once, in order, each able to use the ones
// before it; Eps(w) is an expression of the angular frequency w in rad/s,
// i.e. Omega times 3e14 (Omega in units of c / 1 um, the solver's unit).
// Mu(w) is accepted and ignored (the VIE path is non-magnetic).
//
// SVTENSOR files (SVTensor.cc:41-300) give the permittivity tensor as
// expressions "Eps = ...", "Q = ..." (isotropic) or "Qxy = ...", "EpsXY = ...",
// "Eps12 = ..." per component, of w (rad/s, Omega x 3e14: SVTensor.cc:332),
// x, y, z, r, Theta, Phi and MP_<name> (the eps of a MATERIAL section or a
// CONST_EPS_ name at that frequency), with "NAME = number" constants and
// MATERIAL sections of their own.  Components not given keep the identity;
// off-diagonal pairs are averaged; Qyy and Qzz default to Qxx when only Qxx
// is given (SVTensor.cc:344-372).  Expressions
// use + - * / ^ (right-associative), unary signs, parentheses, numbers with
// exponents, the constants i, pi and e, and the functions exp, log, sqrt,
// sin, cos, tan, sinh, cosh, tanh, asin, acos, atan, abs and step (0 for a
// negative real part, else 1).
#include <algorithm>
#include <cctype>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"

namespace bg {

typedef std::complex<double> cplx;

struct ExprNode {
  enum Kind { NUM, VAR, NEG, ADD, SUB, MUL, DIV, POW, FUN } kind;
  cplx value{0.0, 0.0};  // NUM
  int var = 0;           // VAR: 0 = w, k > 0 = constant k-1
  int fun = 0;           // FUN
  int a = -1, b = -1;    // children
};

static const char *kFuncs[] = {"exp", "log", "sqrt", "sin", "cos", "tan", "sinh", "cosh", "tanh",
                               "asin", "acos", "atan", "abs", "step"};
static const int kNumFuncs = (int)(sizeof kFuncs / sizeof kFuncs[0]);

struct MatPropFn {
  std::string name;
  std::vector<std::string> const_names;
  std::vector<cplx> const_values;
  std::vector<ExprNode> nodes;
  int eps_root = -1;
};

struct SVTensorFn {
  std::string file;
  std::vector<std::string> const_names;
  std::vector<cplx> const_values;
  std::vector<ExprNode> nodes;
  int root[3][3];
  std::vector<std::shared_ptr<const MatPropFn>> mps;   // Eps1, Eps2, Eps3
  bool position = false;                               // uses x, y, z, r, Theta or Phi
};

namespace {

struct Parser {
  const std::string &s;
  size_t p = 0;
  std::vector<ExprNode> &nodes;
  const std::vector<std::string> &names;  // constants visible to this expression
  bool allow_w;
  const std::vector<std::string> *extra = nullptr;  // further variables (VAR -1, -2, ...)
  std::string err;

  Parser(const std::string &src, std::vector<ExprNode> &n, const std::vector<std::string> &nm, bool w)
      : s(src), nodes(n), names(nm), allow_w(w) {}

  void skip() { while (p < s.size() && std::isspace((unsigned char)s[p])) p++; }
  int add(ExprNode n) { nodes.push_back(n); return (int)nodes.size() - 1; }
  int fail(const std::string &m) { if (err.empty()) err = m; return -1; }

  // expr := term (('+'|'-') term)*
  int expr() {
    int l = term();
    while (l >= 0) {
      skip();
      if (p < s.size() && (s[p] == '+' || s[p] == '-')) {
        char op = s[p++];
        int r = term();
        if (r < 0) return -1;
        ExprNode n{op == '+' ? ExprNode::ADD : ExprNode::SUB};
        n.a = l; n.b = r;
        l = add(n);
      } else break;
    }
    return l;
  }
  // term := unary (('*'|'/') unary)*
  int term() {
    int l = unary();
    while (l >= 0) {
      skip();
      if (p < s.size() && (s[p] == '*' || s[p] == '/')) {
        char op = s[p++];
        int r = unary();
        if (r < 0) return -1;
        ExprNode n{op == '*' ? ExprNode::MUL : ExprNode::DIV};
        n.a = l; n.b = r;
        l = add(n);
      } else break;
    }
    return l;
  }
  // unary := ('+'|'-') unary | power
  int unary() {
    skip();
    if (p < s.size() && (s[p] == '+' || s[p] == '-')) {
      char op = s[p++];
      int a = unary();
      if (a < 0 || op == '+') return a;
      ExprNode n{ExprNode::NEG};
      n.a = a;
      return add(n);
    }
    return power();
  }
  // power := primary ('^' unary)?      (right-associative; -x^2 = -(x^2))
  int power() {
    int l = primary();
    if (l < 0) return -1;
    skip();
    if (p < s.size() && s[p] == '^') {
      p++;
      int r = unary();
      if (r < 0) return -1;
      ExprNode n{ExprNode::POW};
      n.a = l; n.b = r;
      return add(n);
    }
    return l;
  }
  int primary() {
    skip();
    if (p >= s.size()) return fail("unexpected end of expression");
    char c = s[p];
    if (c == '(') {
      p++;
      int e = expr();
      skip();
      if (e < 0) return -1;
      if (p >= s.size() || s[p] != ')') return fail("missing )");
      p++;
      return e;
    }
    if (std::isdigit((unsigned char)c) || c == '.') {
      const char *b = s.c_str() + p;
      char *end;
      double v = std::strtod(b, &end);
      if (end == b) return fail("bad number");
      p += (size_t)(end - b);
      ExprNode n{ExprNode::NUM};
      n.value = cplx(v, 0.0);
      return add(n);
    }
    if (std::isalpha((unsigned char)c) || c == '_') {
      size_t q = p;
      while (q < s.size() && (std::isalnum((unsigned char)s[q]) || s[q] == '_')) q++;
      std::string id = s.substr(p, q - p);
      p = q;
      skip();
      if (p < s.size() && s[p] == '(') {
        for (int f = 0; f < kNumFuncs; f++)
          if (id == kFuncs[f]) {
            p++;
            int a = expr();
            skip();
            if (a < 0) return -1;
            if (p >= s.size() || s[p] != ')') return fail("missing ) after " + id);
            p++;
            ExprNode n{ExprNode::FUN};
            n.fun = f; n.a = a;
            return add(n);
          }
        return fail("unknown function " + id);
      }
      // constants defined in the section shadow the built-in names
      for (size_t k = names.size(); k-- > 0;)
        if (names[k] == id) {
          ExprNode n{ExprNode::VAR};
          n.var = (int)k + 1;
          return add(n);
        }
      if (extra)
        for (size_t k = 0; k < extra->size(); k++)
          if ((*extra)[k] == id) {
            ExprNode n{ExprNode::VAR};
            n.var = -(int)k - 1;
            return add(n);
          }
      if (id == "w") {
        if (!allow_w) return fail("w may only appear in Eps(w) or Mu(w)");
        ExprNode n{ExprNode::VAR};
        n.var = 0;
        return add(n);
      }
      ExprNode n{ExprNode::NUM};
      if (id == "i") n.value = cplx(0.0, 1.0);
      else if (id == "pi") n.value = cplx(M_PI, 0.0);
      else if (id == "e") n.value = cplx(M_E, 0.0);
      else return fail("unknown name " + id);
      return add(n);
    }
    return fail(std::string("unexpected character '") + c + "'");
  }
};

cplx ipow(cplx x, long n) {
  bool inv = n < 0;
  unsigned long m = inv ? (unsigned long)(-n) : (unsigned long)n;
  cplx r(1.0, 0.0);
  while (m) {
    if (m & 1) r *= x;
    x *= x;
    m >>= 1;
  }
  return inv ? cplx(1.0, 0.0) / r : r;
}

cplx eval(const std::vector<ExprNode> &nodes, int id, cplx w, const std::vector<cplx> &consts,
          const cplx *extra = nullptr) {
  const ExprNode &n = nodes[id];
  switch (n.kind) {
    case ExprNode::NUM: return n.value;
    case ExprNode::VAR: return n.var == 0 ? w : n.var > 0 ? consts[n.var - 1] : extra[-n.var - 1];
    case ExprNode::NEG: return cplx(0.0, 0.0) - eval(nodes, n.a, w, consts, extra);   // -(4) is (-4, +0): sqrt(-4) = 2i
    case ExprNode::ADD: return eval(nodes, n.a, w, consts, extra) + eval(nodes, n.b, w, consts, extra);
    case ExprNode::SUB: return eval(nodes, n.a, w, consts, extra) - eval(nodes, n.b, w, consts, extra);
    case ExprNode::MUL: return eval(nodes, n.a, w, consts, extra) * eval(nodes, n.b, w, consts, extra);
    case ExprNode::DIV: return eval(nodes, n.a, w, consts, extra) / eval(nodes, n.b, w, consts, extra);
    case ExprNode::POW: {
      cplx x = eval(nodes, n.a, w, consts, extra), y = eval(nodes, n.b, w, consts, extra);
      // integer powers by repeated multiplication (wp^2 is then exact)
      if (y.imag() == 0.0 && y.real() == std::floor(y.real()) && std::fabs(y.real()) <= 64.0)
        return ipow(x, (long)y.real());
      return std::pow(x, y);
    }
    case ExprNode::FUN: {
      cplx x = eval(nodes, n.a, w, consts, extra);
      switch (n.fun) {
        case 0: return std::exp(x);
        case 1: return std::log(x);
        case 2: return std::sqrt(x);
        case 3: return std::sin(x);
        case 4: return std::cos(x);
        case 5: return std::tan(x);
        case 6: return std::sinh(x);
        case 7: return std::cosh(x);
        case 8: return std::tanh(x);
        case 9: return std::asin(x);
        case 10: return std::acos(x);
        case 11: return std::atan(x);
        case 12: return cplx(std::abs(x), 0.0);
        default: return cplx(x.real() < 0.0 ? 0.0 : 1.0, 0.0);   // Heaviside step of the real part
      }
    }
  }
  return cplx(0.0, 0.0);
}

std::string trim(const std::string &s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) a++;
  while (b > a && std::isspace((unsigned char)s[b - 1])) b--;
  return s.substr(a, b - a);
}

std::string upper(std::string s) {
  for (auto &c : s) c = (char)std::toupper((unsigned char)c);
  return s;
}

}  // namespace

// One statement "name = expr" or "Eps(w) = expr" of a MATERIAL section; the
// Eps(w) expression is only recorded here (in eps_src) and parsed once the
// whole section, with every constant, has been read.
static bool matprop_statement(MatPropFn &m, const std::string &stmt, std::string &eps_src, std::string &err) {
  size_t eq = stmt.find('=');
  if (eq == std::string::npos) { err = "expected NAME = EXPRESSION"; return false; }
  std::string lhs = trim(stmt.substr(0, eq)), rhs = stmt.substr(eq + 1);
  std::string L = upper(lhs);
  std::string nospace;
  for (char c : L) if (!std::isspace((unsigned char)c)) nospace += c;
  bool is_eps = nospace == "EPS(W)" || nospace == "EPS", is_mu = nospace == "MU(W)" || nospace == "MU";
  if (!is_eps && !is_mu) {
    if (lhs.empty() || !(std::isalpha((unsigned char)lhs[0]) || lhs[0] == '_')) { err = "bad name " + lhs; return false; }
    for (char c : lhs)
      if (!std::isalnum((unsigned char)c) && c != '_') { err = "bad name " + lhs; return false; }
  }
  if (is_eps) { eps_src = rhs; return true; }
  std::vector<ExprNode> nodes;
  Parser P(rhs, nodes, m.const_names, is_mu);
  int root = P.expr();
  P.skip();
  if (root >= 0 && P.p != rhs.size()) P.fail("junk after expression");
  if (!P.err.empty()) { err = P.err + " in " + trim(rhs); return false; }
  if (!is_mu) {
    m.const_names.push_back(lhs);
    m.const_values.push_back(eval(nodes, root, cplx(0.0, 0.0), m.const_values));
  }
  return true;
}

int matprop_parse_section(const std::string &name, const std::vector<std::string> &lines,
                          const std::vector<int> &lineno, const char *path, std::shared_ptr<const MatPropFn> &out) {
  auto m = std::make_shared<MatPropFn>();
  m->name = name;
  std::string eps_src;
  int eps_line = 0;
  for (size_t l = 0; l < lines.size(); l++) {
    std::string line = lines[l];
    size_t hash = line.find('#');
    if (hash != std::string::npos) line = line.substr(0, hash);
    size_t a = 0;
    while (a <= line.size()) {
      size_t b = line.find(';', a);
      if (b == std::string::npos) b = line.size();
      std::string stmt = trim(line.substr(a, b - a));
      std::string err, src;
      if (!stmt.empty() && !matprop_statement(*m, stmt, src, err)) {
        set_error("%s:%d: MATERIAL %s: %s", path, lineno[l], name.c_str(), err.c_str());
        return BG_ERR_IO;
      }
      if (!src.empty()) { eps_src = src; eps_line = lineno[l]; }
      a = b + 1;
    }
  }
  if (eps_src.empty()) {
    set_error("%s:%d: MATERIAL %s defines no Eps(w)", path, lineno.empty() ? 0 : lineno.back(), name.c_str());
    return BG_ERR_IO;
  }
  Parser P(eps_src, m->nodes, m->const_names, true);
  m->eps_root = P.expr();
  P.skip();
  if (m->eps_root >= 0 && P.p != eps_src.size()) P.fail("junk after expression");
  if (!P.err.empty()) {
    set_error("%s:%d: MATERIAL %s: %s in %s", path, eps_line, name.c_str(), P.err.c_str(), trim(eps_src).c_str());
    return BG_ERR_IO;
  }
  out = m;
  return BG_OK;
}

// eps at the solver frequency Omega (units of 3e14 rad/s), as
// SVTensor::Evaluate -> MatProp::GetEps does for a homogeneous isotropic
// material (SVTensor.cc:312-317, w = Omega * MatProp::FreqUnit).
void matprop_eps(const MatPropFn &m, double omega_re, double omega_im, double eps[2]) {
  const double kFreqUnit = 3.0e14;
  cplx v = eval(m.nodes, m.eps_root, cplx(omega_re * kFreqUnit, omega_im * kFreqUnit), m.const_values);
  eps[0] = v.real();
  eps[1] = v.imag();
}


// ---------------------------------------------------------------- SVTENSOR
static const std::vector<std::string> kSvtVars = {"x", "y", "z", "r", "Theta", "Phi", "Eps1", "Eps2", "Eps3"};

// the smallest k in 1..3 such that the expression reads Eps<k> although only
// nmat MP_ materials exist (k > nmat), or 0
static int uses_material_beyond(const std::vector<ExprNode> &nodes, int id, int nmat) {
  if (id < 0) return 0;
  const ExprNode &n = nodes[id];
  if (n.kind == ExprNode::VAR && n.var < 0) {
    int k = -n.var - 1 - 6 + 1;   // Eps1..Eps3 are extra variables 6..8
    return (k >= 1 && k <= 3 && k > nmat) ? k : 0;
  }
  int a = uses_material_beyond(nodes, n.a, nmat), b = uses_material_beyond(nodes, n.b, nmat);
  if (a && b) return std::min(a, b);
  return a ? a : b;
}

static bool uses_position(const std::vector<ExprNode> &nodes, int id) {
  const ExprNode &n = nodes[id];
  if (n.kind == ExprNode::VAR) return n.var < 0 && -n.var - 1 < 6;
  bool r = false;
  if (n.a >= 0) r = r || uses_position(nodes, n.a);
  if (n.b >= 0) r = r || uses_position(nodes, n.b);
  return r;
}

// MP_<name> -> Eps<k>, resolving <name> against the MATERIAL sections seen so
// far (latest first, ignoring case) or a CONST_EPS_ / VACUUM name
static bool replace_mps(std::string &expr, SVTensorFn &t, const MatDB &db, std::string &err) {
  size_t p;
  while ((p = expr.find("MP_")) != std::string::npos) {
    size_t q = p + 3;
    while (q < expr.size() && (std::isalnum((unsigned char)expr[q]) || expr[q] == '_' || expr[q] == '.' ||
                               ((expr[q] == '+' || expr[q] == '-') && upper(expr.substr(p + 3, q - p - 3)).rfind("CONST_EPS_", 0) == 0)))
      q++;
    std::string name = expr.substr(p + 3, q - p - 3);
    std::shared_ptr<const MatPropFn> fn;
    for (size_t k = db.size(); k-- > 0 && !fn;)
      if (upper(db[k].first) == upper(name)) fn = db[k].second;
    if (!fn) {
      std::string U = upper(name), body;
      if (U == "VACUUM") body = "1";
      else if (U.rfind("CONST_EPS_", 0) == 0) {
        // <re>, <re>+<im>i, <re>-<im>i or <im>i, as in a CONST_EPS_ MATERIAL
        const char *c0 = name.c_str() + 10;
        char *e1, *e2;
        double a = std::strtod(c0, &e1), b = 0.0;
        bool ok = e1 != c0;
        if (ok && (*e1 == 'i' || *e1 == 'j' || *e1 == 'I') && e1[1] == 0) { b = a; a = 0.0; }
        else if (ok && *e1 != 0) {
          b = std::strtod(e1, &e2);
          ok = e2 != e1 && (*e2 == 'i' || *e2 == 'j' || *e2 == 'I') && e2[1] == 0;
        }
        if (ok) {
          char tmp[96];
          std::snprintf(tmp, sizeof tmp, "(%.17g) + (%.17g)*i", a, b);
          body = tmp;
        }
      }
      if (body.empty()) { err = "unknown material MP_" + name; return false; }
      std::shared_ptr<const MatPropFn> c;
      std::vector<std::string> lines{"Eps(w) = " + body};
      std::vector<int> ln{0};
      if (matprop_parse_section(name, lines, ln, "MP_", c)) { err = "bad material MP_" + name; return false; }
      fn = c;
    }
    size_t k = 0;
    while (k < t.mps.size() && t.mps[k] != fn) k++;
    if (k == t.mps.size()) {
      if (t.mps.size() == 3) { err = "too many MP_ statements (at most 3 materials)"; return false; }
      t.mps.push_back(fn);
    }
    expr.replace(p, q - p, "Eps" + std::to_string(k + 1));
  }
  return true;
}

int svtensor_parse_file(const std::string &path, MatDB &db, std::shared_ptr<const SVTensorFn> &out) {
  FILE *f = std::fopen(path.c_str(), "r");
  if (!f) { set_error("could not find file %s", path.c_str()); return BG_ERR_IO; }
  auto t = std::make_shared<SVTensorFn>();
  t->file = path;
  for (auto &r : t->root) for (int &x : r) x = -1;
  std::vector<std::string> all;
  {
    std::string line;
    char buf[1024];
    while (std::fgets(buf, sizeof buf, f)) {
      line += buf;
      if (!line.empty() && line.back() == '\n') { line.pop_back(); all.push_back(line); line.clear(); }
    }
    if (!line.empty()) all.push_back(line);
  }
  std::fclose(f);
  auto fail = [&](size_t l, const std::string &m) {
    set_error("%s:%d: %s", path.c_str(), (int)l + 1, m.c_str());
    return BG_ERR_IO;
  };
  // The whole file is read before any component expression is parsed
  // (SVTensor.cc:88-113 sets every constant on every expression after
  // parsing), so a constant or MATERIAL section may come after its use.
  struct Component {
    size_t line;
    int M, N;
    std::string rhs;
  };
  std::vector<Component> comps;
  for (size_t l = 0; l < all.size(); l++) {
    std::string p = trim(all[l]);
    if (p.empty() || p[0] == '#') continue;
    size_t semi = p.find(';');
    if (semi != std::string::npos) p = trim(p.substr(0, semi));
    if (p.compare(0, 8, "MATERIAL") == 0 && (p.size() == 8 || std::isspace((unsigned char)p[8]))) {
      std::string name = trim(p.substr(8));
      if (name.empty()) return fail(l, "no name given for MATERIAL");
      if (name.find_first_of(" \t") != std::string::npos) return fail(l, "syntax error");
      std::vector<std::string> body;
      std::vector<int> ln;
      size_t e = l + 1;
      while (e < all.size() && upper(trim(all[e])).compare(0, 11, "ENDMATERIAL") != 0) {
        body.push_back(all[e]);
        ln.push_back((int)e + 1);
        e++;
      }
      if (e == all.size()) return fail(l, "MATERIAL without ENDMATERIAL");
      std::shared_ptr<const MatPropFn> fn;
      int st = matprop_parse_section(name, body, ln, path.c_str(), fn);
      if (st) return st;
      db.emplace_back(name, fn);
      l = e;
      continue;
    }
    size_t eq = p.find('=');
    if (eq == std::string::npos) return fail(l, "syntax error");
    std::string lhs = trim(p.substr(0, eq)), rhs = p.substr(eq + 1), L = upper(lhs);
    int M = -1, N = -1;
    std::string comp;
    if (L == "Q" || L == "EPS") M = N = 0;
    else if (L.size() == 3 && L[0] == 'Q') comp = L.substr(1);
    else if (L.size() == 5 && L.compare(0, 3, "EPS") == 0) comp = L.substr(3);
    if (!comp.empty()) {
      int mn[2];
      for (int k = 0; k < 2; k++) {
        char c = comp[k];
        if (c >= 'X' && c <= 'Z') mn[k] = c - 'X';
        else if (c >= '1' && c <= '3') mn[k] = c - '1';
        else return fail(l, "invalid component " + lhs);
      }
      M = mn[0]; N = mn[1];
    }
    if (M >= 0) {
      comps.push_back({l, M, N, rhs});
      continue;
    }
    // NAME = number (SVTensor.cc:250-270)
    char *end;
    std::string v = trim(rhs);
    double cv = std::strtod(v.c_str(), &end);
    if (v.empty() || *end != 0) return fail(l, "invalid constant value");
    if (lhs.empty() || !(std::isalpha((unsigned char)lhs[0]) || lhs[0] == '_')) return fail(l, "syntax error");
    t->const_names.push_back(lhs);
    t->const_values.push_back(cplx(cv, 0.0));
  }
  for (const Component &c : comps) {
    std::string rhs = c.rhs, err;
    if (!replace_mps(rhs, *t, db, err)) return fail(c.line, err);
    Parser P(rhs, t->nodes, t->const_names, true);
    P.extra = &kSvtVars;
    int root = P.expr();
    P.skip();
    if (root >= 0 && P.p != rhs.size()) P.fail("junk after expression");
    if (!P.err.empty()) return fail(c.line, P.err + " in " + trim(rhs));
    // Eps1..Eps3 (the MP_ materials, variables 7-9 of kSvtVars) beyond the
    // materials named so far
    int undefined = uses_material_beyond(t->nodes, root, (int)t->mps.size());
    if (undefined) return fail(c.line, "Eps" + std::to_string(undefined) + " is not defined");
    t->root[c.M][c.N] = root;
    t->position = t->position || uses_position(t->nodes, root);
  }
  out = t;
  return BG_OK;
}

bool svtensor_position_dependent(const SVTensorFn &t) { return t.position; }

// Postfix program of the subtree at id: w, the constants and Eps1-3 become
// constants of the program (their values at this frequency), x, y, z, r,
// Theta and Phi stay variables.
namespace {
struct ExprEmitter {
  const SVTensorFn &t;
  cplx w, eps[3];
  DevExpr *out;
  int nop = 0, ncon = 0, depth = 0, maxdepth = 0;
  std::string err;
  void op(int code, int arg) {
    if (nop >= BG_EXPR_MAXOPS) { err = "too long"; return; }
    out->op[nop++] = code << 16 | arg;
  }
  void con(cplx v) {
    if (ncon >= BG_EXPR_MAXCON) { err = "too many constants"; return; }
    out->con[2 * ncon] = v.real();
    out->con[2 * ncon + 1] = v.imag();
    op(0, ncon++);
  }
  void push() { maxdepth = std::max(maxdepth, ++depth); }
  void emit(int id) {
    if (!err.empty()) return;
    const ExprNode &n = t.nodes[id];
    switch (n.kind) {
      case ExprNode::NUM: con(n.value); push(); return;
      case ExprNode::VAR:
        if (n.var == 0) con(w);
        else if (n.var > 0) con(t.const_values[n.var - 1]);
        else if (-n.var - 1 < 6) op(1, -n.var - 1);
        else con(eps[-n.var - 1 - 6]);
        push();
        return;
      case ExprNode::NEG: emit(n.a); op(2, 0); return;
      case ExprNode::FUN: emit(n.a); op(8, n.fun); return;
      default: break;
    }
    emit(n.a);
    emit(n.b);
    int code = n.kind == ExprNode::ADD ? 3 : n.kind == ExprNode::SUB ? 4 : n.kind == ExprNode::MUL ? 5
             : n.kind == ExprNode::DIV ? 6 : 7;
    op(code, 0);
    depth--;
  }
};
}  // namespace

int svtensor_compile(const SVTensorFn &t, double wr, double wi, DevExpr *out) {
  const double kFreqUnit = 3.0e14;
  ExprEmitter E{t, cplx(wr * kFreqUnit, wi * kFreqUnit), {cplx(1.0, 0.0), cplx(1.0, 0.0), cplx(1.0, 0.0)}, out};
  for (size_t k = 0; k < 3 && k < t.mps.size(); k++) {
    double e[2];
    matprop_eps(*t.mps[k], wr, wi, e);
    E.eps[k] = cplx(e[0], e[1]);
  }
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) {
      const int c = 3 * a + b;
      out->start[c] = E.nop;
      E.depth = 0;
      if (t.root[a][b] >= 0) E.emit(t.root[a][b]);
      out->len[c] = E.nop - out->start[c];
    }
  if (E.err.empty() && E.maxdepth > BG_EXPR_STACK) E.err = "nested too deeply";
  if (!E.err.empty()) {
    set_error("SVTENSOR %s: expression %s for the device (at most %d operations, %d constants, depth %d)",
              t.file.c_str(), E.err.c_str(), BG_EXPR_MAXOPS, BG_EXPR_MAXCON, BG_EXPR_STACK);
    return BG_ERR_ARG;
  }
  return BG_OK;
}

void svtensor_eval(const SVTensorFn &t, double wr, double wi, const double *x, double Q[18]) {
  const double kFreqUnit = 3.0e14;
  cplx v[9];
  v[0] = x[0]; v[1] = x[1]; v[2] = x[2];
  v[3] = std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  v[4] = std::atan2(std::sqrt(x[0] * x[0] + x[1] * x[1]), x[2]);
  v[5] = std::atan2(x[1], x[0]);
  for (size_t k = 0; k < 3; k++) {
    double e[2] = {1.0, 0.0};
    if (k < t.mps.size()) matprop_eps(*t.mps[k], wr, wi, e);
    v[6 + k] = cplx(e[0], e[1]);
  }
  cplx w(wr * kFreqUnit, wi * kFreqUnit), q[3][3];
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) {
      q[a][b] = (a == b) ? cplx(1.0, 0.0) : cplx(0.0, 0.0);
      if (t.root[a][b] >= 0) q[a][b] = eval(t.nodes, t.root[a][b], w, t.const_values, v);
    }
  for (int a = 0; a < 3; a++) {
    int b = (a + 1) % 3;
    cplx avg = 0.5 * (q[a][b] + q[b][a]);
    q[a][b] = q[b][a] = avg;
  }
  if (t.root[0][0] >= 0) {
    if (t.root[1][1] < 0) q[1][1] = q[0][0];
    if (t.root[2][2] < 0) q[2][2] = q[0][0];
  }
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) {
      Q[2 * (3 * a + b)] = q[a][b].real();
      Q[2 * (3 * a + b) + 1] = q[a][b].imag();
    }
}

}  // namespace bg
