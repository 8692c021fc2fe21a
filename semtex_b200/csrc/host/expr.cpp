#include "expr.hpp"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <stdexcept>

namespace stx {

namespace {

struct Default {
  const char* name;
  double value;
};

// femlib/defaults.h:10-96 (names and values of the reference defaults).
const Default kDefaults[] = {
    {"E", 2.71828182845904523536},  {"DEG", 57.29577951308232087721},
    {"PI", 3.14159265358979323844}, {"TWOPI", 6.28318530717958647688},
    {"EULER", 0.57721566490153286061}, {"GOLDEN", 1.61803398874989484820},
    {"t", 0.0}, {"D_T", 0.01}, {"TOL_REL", 1.0e-8}, {"TOL_ABS", 1.0e-8},
    {"TOL_POS", 1.0e-5}, {"z", 0.0}, {"BETA", 1.0}, {"LAMBDA2", 0.0},
    {"KINVIS", 1.0}, {"REFVIS", 1.0}, {"RHO", 1.0}, {"GRAVITY", 9.81},
    {"T_REF", 288.15}, {"PRANDTL", 0.72}, {"C_SMAG", 0.1}, {"LAMBDA_M", 2.0},
    {"FFX", 0.0}, {"FFY", 0.0}, {"FFZ", 0.0}, {"FFC", 0.0},
    {"X_SHIFT", 0.0}, {"Y_SHIFT", 0.0}, {"X_SCALE", 1.0}, {"Y_SCALE", 1.0},
    {"SVV_MN", -1}, {"SVV_EPSN", 0.0}, {"SVV_MZ", -1}, {"SVV_EPSZ", 0.0},
    {"UODelta", 0.05}, {"ITERATIVE", 0}, {"TBCS", 0}, {"CYLINDRICAL", 0},
    {"VERBOSE", 0}, {"CHKPOINT", 1}, {"AVERAGE", 0}, {"SPAWN", 0},
    {"N_PHASE", 0}, {"RANSEED", 0}, {"IO_FLD", 500}, {"IO_HIS", 10},
    {"IO_CFL", 50}, {"IO_MDL", 50}, {"IO_WSS", 0}, {"N_P", 5}, {"N_TIME", 2},
    {"N_STEP", 1}, {"N_Z", 1}, {"I_PROC", 0}, {"N_PROC", 1},
    {"STEP_MAX", 500}, {"NR_MAX", 20}, {"ADVECTION", 1},
};

double heav(double x) { return x >= 0.0 ? 1.0 : 0.0; }
double sgn(double x) { return (x > 0.0) - (x < 0.0); }

struct Parser {
  const std::string& s;
  size_t i = 0;
  std::map<std::string, double>& tab;
  const std::map<std::string, double>* vars;

  Parser(const std::string& src, std::map<std::string, double>& t,
         const std::map<std::string, double>* v)
      : s(src), tab(t), vars(v) {}

  void ws() {
    while (i < s.size() && std::isspace(static_cast<unsigned char>(s[i]))) ++i;
  }
  bool eat(char c) {
    ws();
    if (i < s.size() && s[i] == c) {
      ++i;
      return true;
    }
    return false;
  }
  [[noreturn]] void fail(const char* what) const {
    throw std::runtime_error(std::string("expression error (") + what + ") in: " + s);
  }

  double expr() {
    double v = term();
    for (;;) {
      if (eat('+')) v += term();
      else if (eat('-')) v -= term();
      else return v;
    }
  }
  double term() {
    double v = unary();
    for (;;) {
      if (eat('*')) {
        v *= unary();
      } else if (eat('/')) {
        double d = unary();
        if (d == 0.0) {
          std::fprintf(stderr, "yyparse: division by zero\n");
          v = 0.0;
        } else {
          v /= d;
        }
      } else if (eat('%')) {
        v = std::fmod(v, unary());
      } else {
        return v;
      }
    }
  }
  double unary() {
    if (eat('-')) return -unary();
    if (eat('+')) return unary();
    return power();
  }
  double power() {
    double a = atom();
    ws();
    if (i < s.size() && (s[i] == '^' || s[i] == '&' || s[i] == '~')) {
      char op = s[i++];
      double b = unary();  // right-associative
      if (op == '^') return std::pow(a, b);
      if (op == '&') return std::hypot(a, b);
      return std::atan2(a, b);
    }
    return a;
  }
  double call(const std::string& name, const std::vector<double>& a) {
    auto need = [&](size_t n) {
      if (a.size() != n) fail("wrong number of arguments");
    };
    if (name == "cos") { need(1); return std::cos(a[0]); }
    if (name == "sin") { need(1); return std::sin(a[0]); }
    if (name == "tan") { need(1); return std::tan(a[0]); }
    if (name == "exp") { need(1); return std::exp(a[0]); }
    if (name == "sinh") { need(1); return std::sinh(a[0]); }
    if (name == "cosh") { need(1); return std::cosh(a[0]); }
    if (name == "tanh") { need(1); return std::tanh(a[0]); }
    if (name == "erf") { need(1); return std::erf(a[0]); }
    if (name == "erfc") { need(1); return std::erfc(a[0]); }
    if (name == "int") { need(1); return std::rint(a[0]); }
    if (name == "abs") { need(1); return std::fabs(a[0]); }
    if (name == "floor") { need(1); return std::floor(a[0]); }
    if (name == "ceil") { need(1); return std::ceil(a[0]); }
    if (name == "acos") { need(1); return std::acos(a[0]); }
    if (name == "asin") { need(1); return std::asin(a[0]); }
    if (name == "atan") { need(1); return std::atan(a[0]); }
    if (name == "acosh") { need(1); return std::acosh(a[0]); }
    if (name == "asinh") { need(1); return std::asinh(a[0]); }
    if (name == "atanh") { need(1); return std::atanh(a[0]); }
    if (name == "log") { need(1); return std::log(a[0]); }
    if (name == "log10") { need(1); return std::log10(a[0]); }
    if (name == "sqrt") { need(1); return std::sqrt(a[0]); }
    if (name == "heav") { need(1); return heav(a[0]); }
    if (name == "sgn") { need(1); return sgn(a[0]); }
    if (name == "j0") { need(1); return ::j0(a[0]); }
    if (name == "j1") { need(1); return ::j1(a[0]); }
    if (name == "y0") { need(1); return ::y0(a[0]); }
    if (name == "y1") { need(1); return ::y1(a[0]); }
    if (name == "gamma") { need(1); return std::tgamma(a[0]); }
    if (name == "lgamma") { need(1); return std::lgamma(a[0]); }
    if (name == "jn") { need(2); return ::jn(static_cast<int>(a[0]), a[1]); }
    if (name == "yn") { need(2); return ::yn(static_cast<int>(a[0]), a[1]); }
    if (name == "rad") { need(2); return std::hypot(a[0], a[1]); }
    if (name == "ang") { need(2); return std::atan2(a[1], a[0]); }
    if (name == "step") { need(2); return a[0] >= a[1] ? 1.0 : 0.0; }
    fail(("unknown function " + name).c_str());
  }
  double lookup(const std::string& name) {
    if (vars) {
      auto it = vars->find(name);
      if (it != vars->end()) return it->second;
    }
    auto it = tab.find(name);
    if (it == tab.end()) {
      std::fprintf(stderr, "yyparse: undefined variable %s\n", name.c_str());
      return 0.0;
    }
    return it->second;
  }
  double atom() {
    ws();
    if (i >= s.size()) fail("unexpected end");
    char c = s[i];
    if (c == '(') {
      ++i;
      double v = expr();
      if (!eat(')')) fail("missing )");
      return v;
    }
    if (std::isdigit(static_cast<unsigned char>(c)) || c == '.') {
      size_t used = 0;
      double v = std::stod(s.substr(i), &used);
      i += used;
      return v;
    }
    if (std::isalpha(static_cast<unsigned char>(c)) || c == '_') {
      size_t j = i;
      while (j < s.size() &&
             (std::isalnum(static_cast<unsigned char>(s[j])) || s[j] == '_'))
        ++j;
      std::string name = s.substr(i, j - i);
      i = j;
      ws();
      if (i < s.size() && s[i] == '(') {
        ++i;
        std::vector<double> args;
        if (!eat(')')) {
          do {
            args.push_back(expr());
          } while (eat(','));
          if (!eat(')')) fail("missing ) after arguments");
        }
        return call(name, args);
      }
      if (i < s.size() && s[i] == '=' && (i + 1 >= s.size() || s[i + 1] != '=')) {
        ++i;
        double v = expr();
        tab[name] = v;
        return v;
      }
      return lookup(name);
    }
    fail("unexpected character");
  }
};

// The same grammar as Parser, emitting a postfix program instead of a
// value.  Operations whose operands are all constants are folded.
struct Compiler {
  const std::string& s;
  size_t i = 0;
  const std::map<std::string, double>& tab;
  ExprProgram prog;
  int sp = 0;

  Compiler(const std::string& src, const std::map<std::string, double>& t) : s(src), tab(t) {}

  void ws() {
    while (i < s.size() && std::isspace(static_cast<unsigned char>(s[i]))) ++i;
  }
  bool eat(char c) {
    ws();
    if (i < s.size() && s[i] == c) {
      ++i;
      return true;
    }
    return false;
  }
  [[noreturn]] void fail(const char* what) const {
    throw std::runtime_error(std::string("expression error (") + what + ") in: " + s);
  }
  bool last_const(int k) const {  // the k-th op from the end is a constant
    const int n = static_cast<int>(prog.ops.size());
    return n >= k && prog.ops[n - k].code == kExConst;
  }
  void push(int code, int fn = 0, double val = 0.0) {
    if (static_cast<int>(prog.ops.size()) >= kExprMaxOps) fail("program too long");
    prog.ops.push_back(ExprOp{code, fn, val});
  }
  void value(int code, double val = 0.0) {
    push(code, 0, val);
    if (++sp > kExprStack) fail("expression nested too deeply");
    prog.depth = std::max(prog.depth, sp);
  }
  void binary(int code) {
    if (last_const(1) && last_const(2)) {
      const double b = prog.ops.back().val;
      prog.ops.pop_back();
      prog.ops.back().val = expr_binary(code, prog.ops.back().val, b);
    } else {
      push(code);
    }
    --sp;
  }
  void fn2(int fn) {
    if (last_const(1) && last_const(2)) {
      const double b = prog.ops.back().val;
      prog.ops.pop_back();
      prog.ops.back().val = expr_fn2(fn, prog.ops.back().val, b);
    } else {
      push(kExFn2, fn);
    }
    --sp;
  }
  void fn1(int fn) {
    if (last_const(1)) prog.ops.back().val = expr_fn1(fn, prog.ops.back().val);
    else push(kExFn1, fn);
  }
  void negate() {
    if (last_const(1)) prog.ops.back().val = -prog.ops.back().val;
    else push(kExNeg);
  }

  void expr() {
    term();
    for (;;) {
      if (eat('+')) {
        term();
        binary(kExAdd);
      } else if (eat('-')) {
        term();
        binary(kExSub);
      } else {
        return;
      }
    }
  }
  void term() {
    unary();
    for (;;) {
      if (eat('*')) {
        unary();
        binary(kExMul);
      } else if (eat('/')) {
        unary();
        binary(kExDiv);
      } else if (eat('%')) {
        unary();
        binary(kExMod);
      } else {
        return;
      }
    }
  }
  void unary() {
    if (eat('-')) {
      unary();
      negate();
      return;
    }
    if (eat('+')) {
      unary();
      return;
    }
    power();
  }
  void power() {
    atom();
    ws();
    if (i < s.size() && (s[i] == '^' || s[i] == '&' || s[i] == '~')) {
      const char op = s[i++];
      unary();  // right-associative
      binary(op == '^' ? kExPow : op == '&' ? kExHypot : kExAtan2);
    }
  }
  void call(const std::string& name, int nargs) {
    static const std::map<std::string, int> one = {
        {"cos", kFnCos},     {"sin", kFnSin},     {"tan", kFnTan},     {"exp", kFnExp},
        {"sinh", kFnSinh},   {"cosh", kFnCosh},   {"tanh", kFnTanh},   {"erf", kFnErf},
        {"erfc", kFnErfc},   {"int", kFnInt},     {"abs", kFnAbs},     {"floor", kFnFloor},
        {"ceil", kFnCeil},   {"acos", kFnAcos},   {"asin", kFnAsin},   {"atan", kFnAtan},
        {"acosh", kFnAcosh}, {"asinh", kFnAsinh}, {"atanh", kFnAtanh}, {"log", kFnLog},
        {"log10", kFnLog10}, {"sqrt", kFnSqrt},   {"heav", kFnHeav},   {"sgn", kFnSgn},
        {"j0", kFnJ0},       {"j1", kFnJ1},       {"y0", kFnY0},       {"y1", kFnY1},
        {"gamma", kFnGamma}, {"lgamma", kFnLgamma}};
    static const std::map<std::string, int> two = {
        {"jn", kFnJn}, {"yn", kFnYn}, {"rad", kFnRad}, {"ang", kFnAng}, {"step", kFnStep}};
    auto a = one.find(name);
    if (a != one.end()) {
      if (nargs != 1) fail("wrong number of arguments");
      fn1(a->second);
      return;
    }
    auto b = two.find(name);
    if (b != two.end()) {
      if (nargs != 2) fail("wrong number of arguments");
      fn2(b->second);
      return;
    }
    fail(("unknown function " + name).c_str());
  }
  void atom() {
    ws();
    if (i >= s.size()) fail("unexpected end");
    const char c = s[i];
    if (c == '(') {
      ++i;
      expr();
      if (!eat(')')) fail("missing )");
      return;
    }
    if (std::isdigit(static_cast<unsigned char>(c)) || c == '.') {
      size_t used = 0;
      const double v = std::stod(s.substr(i), &used);
      i += used;
      value(kExConst, v);
      return;
    }
    if (std::isalpha(static_cast<unsigned char>(c)) || c == '_') {
      size_t j = i;
      while (j < s.size() && (std::isalnum(static_cast<unsigned char>(s[j])) || s[j] == '_')) ++j;
      const std::string name = s.substr(i, j - i);
      i = j;
      ws();
      if (i < s.size() && s[i] == '(') {
        ++i;
        int nargs = 0;
        if (!eat(')')) {
          do {
            expr();
            ++nargs;
          } while (eat(','));
          if (!eat(')')) fail("missing ) after arguments");
        }
        call(name, nargs);
        return;
      }
      if (i < s.size() && s[i] == '=' && (i + 1 >= s.size() || s[i + 1] != '='))
        fail("assignment inside a compiled expression");
      if (name == "x" || name == "y" || name == "z") {
        prog.uses_xyz = true;
        value(name == "x" ? kExX : name == "y" ? kExY : kExZ);
      } else if (name == "t") {
        prog.uses_t = true;
        value(kExT);
      } else {
        auto it = tab.find(name);
        if (it == tab.end()) std::fprintf(stderr, "yyparse: undefined variable %s\n", name.c_str());
        value(kExConst, it == tab.end() ? 0.0 : it->second);
      }
      return;
    }
    fail("unexpected character");
  }
};

}  // namespace

ExprProgram TokenTable::compile(const std::string& e) const {
  Compiler c(e, table_);
  c.expr();
  c.ws();
  if (c.i != e.size()) c.fail("trailing characters");
  if (c.sp != 1) c.fail("malformed expression");
  return c.prog;
}

TokenTable::TokenTable() {
  for (const auto& d : kDefaults) table_[d.name] = d.value;
}

double TokenTable::eval(const std::string& e,
                        const std::map<std::string, double>* vars) const {
  auto& tab = const_cast<std::map<std::string, double>&>(table_);
  Parser p(e, tab, vars);
  double v = p.expr();
  p.ws();
  if (p.i != e.size()) p.fail("trailing characters");
  return v;
}

void TokenTable::assign(const std::string& line) {
  Parser p(line, table_, nullptr);
  p.expr();
}

double TokenTable::value(const std::string& name) const {
  auto it = table_.find(name);
  if (it == table_.end()) return eval(name);
  return it->second;
}

int TokenTable::ivalue(const std::string& name) const {
  return static_cast<int>(std::lround(value(name)));
}

}  // namespace stx
