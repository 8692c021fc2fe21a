// Token table and expression interpreter for FEML sessions.
//
// Restates the grammar and built-ins of the reference's yacc parser
// (femlib/initial.y:138-249) and its default token table
// (femlib/defaults.h:10-96) as a recursive-descent evaluator:
//
//   expr   := term (('+'|'-') term)*
//   term   := unary (('*'|'/'|'%') unary)*
//   unary  := '-' unary | power
//   power  := atom (('^'|'&'|'~') unary)?      right-associative, binds
//                                               tighter than unary minus
//   atom   := NUMBER | NAME | NAME '(' args ')' | '(' expr ')' | NAME '=' expr
//
// '^' is pow, '&' is hypot, '~' is atan2, '%' is fmod; division by zero
// yields 0 with a warning, as in the reference.
#pragma once

#include <map>
#include <string>
#include <vector>

#include "../kernels/exprprog.hpp"

namespace stx {

// A compiled expression (see exprprog.hpp): the postfix program, the
// deepest operand stack it needs and which of x, y, z, t it reads.
struct ExprProgram {
  std::vector<ExprOp> ops;
  int depth = 0;
  bool uses_xyz = false;
  bool uses_t = false;
  bool constant() const { return !uses_xyz && !uses_t; }
  double run(double x, double y, double z, double t) const {
    return expr_run(ops.data(), static_cast<int>(ops.size()), x, y, z, t);
  }
};

class TokenTable {
 public:
  TokenTable();
  // Evaluate an expression; `vars` overrides table entries (x, y, z, t ...).
  double eval(const std::string& expr,
              const std::map<std::string, double>* vars = nullptr) const;
  // The expression as a program of the free variables x, y, z, t; other
  // names take their current table values.  Assignments inside the
  // expression are not accepted, nor programs longer than kExprMaxOps or
  // deeper than kExprStack (std::runtime_error).
  ExprProgram compile(const std::string& expr) const;
  // "NAME = expr" assignment (FEML <TOKENS> line).
  void assign(const std::string& line);
  double value(const std::string& name) const;
  int ivalue(const std::string& name) const;
  void set(const std::string& name, double v) { table_[name] = v; }
  bool has(const std::string& name) const { return table_.count(name) != 0; }

 private:
  std::map<std::string, double> table_;
};

}  // namespace stx
