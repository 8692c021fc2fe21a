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

namespace stx {

class TokenTable {
 public:
  TokenTable();
  // Evaluate an expression; `vars` overrides table entries (x, y, z, t ...).
  double eval(const std::string& expr,
              const std::map<std::string, double>* vars = nullptr) const;
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
