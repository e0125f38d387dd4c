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
// Mu(w) is accepted and ignored (the VIE path is non-magnetic).  Expressions
// use + - * / ^ (right-associative), unary signs, parentheses, numbers with
// exponents, the constants i, pi and e, and the functions exp, log, sqrt,
// sin, cos, tan, sinh, cosh, tanh, asin, acos, atan, abs.
#include <cctype>
#include <cmath>
#include <complex>
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
                               "asin", "acos", "atan", "abs"};
static const int kNumFuncs = (int)(sizeof kFuncs / sizeof kFuncs[0]);

struct MatPropFn {
  std::string name;
  std::vector<std::string> const_names;
  std::vector<cplx> const_values;
  std::vector<ExprNode> nodes;
  int eps_root = -1;
};

namespace {

struct Parser {
  const std::string &s;
  size_t p = 0;
  std::vector<ExprNode> &nodes;
  const std::vector<std::string> &names;  // constants visible to this expression
  bool allow_w;
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

cplx eval(const std::vector<ExprNode> &nodes, int id, cplx w, const std::vector<cplx> &consts) {
  const ExprNode &n = nodes[id];
  switch (n.kind) {
    case ExprNode::NUM: return n.value;
    case ExprNode::VAR: return n.var == 0 ? w : consts[n.var - 1];
    case ExprNode::NEG: return cplx(0.0, 0.0) - eval(nodes, n.a, w, consts);   // -(4) is (-4, +0): sqrt(-4) = 2i
    case ExprNode::ADD: return eval(nodes, n.a, w, consts) + eval(nodes, n.b, w, consts);
    case ExprNode::SUB: return eval(nodes, n.a, w, consts) - eval(nodes, n.b, w, consts);
    case ExprNode::MUL: return eval(nodes, n.a, w, consts) * eval(nodes, n.b, w, consts);
    case ExprNode::DIV: return eval(nodes, n.a, w, consts) / eval(nodes, n.b, w, consts);
    case ExprNode::POW: {
      cplx x = eval(nodes, n.a, w, consts), y = eval(nodes, n.b, w, consts);
      // integer powers by repeated multiplication (wp^2 is then exact)
      if (y.imag() == 0.0 && y.real() == std::floor(y.real()) && std::fabs(y.real()) <= 64.0)
        return ipow(x, (long)y.real());
      return std::pow(x, y);
    }
    case ExprNode::FUN: {
      cplx x = eval(nodes, n.a, w, consts);
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
        default: return cplx(std::abs(x), 0.0);
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


}  // namespace bg
