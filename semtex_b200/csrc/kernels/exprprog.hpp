// Session expressions compiled for evaluation at every node on the device.
//
// The reference evaluates a function of x, y, z, t at every node by running
// its yacc interpreter once per node (AuxField::operator= (const char*),
// src/auxfield.cpp:198-220, femlib/initial.y:138-249); a forcing term that
// depends on time does so every step (dns/fieldforce.cpp:475-489).  Here the
// expression is parsed once (TokenTable::compile) into a postfix program of
// ExprOp and run by expr_run, the same code on the host and on the device:
// token names other than x, y, z, t are looked up when the program is made.
// Operators and built-ins are those of the interpreter: '^' pow, '&' hypot,
// '~' atan2, '%' fmod, division by zero gives 0.
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define STX_HD __host__ __device__
#else
#define STX_HD
#endif

namespace stx {

enum ExprCode : int {
  kExConst,
  kExX,
  kExY,
  kExZ,
  kExT,
  kExNeg,
  kExAdd,
  kExSub,
  kExMul,
  kExDiv,
  kExMod,
  kExPow,
  kExHypot,
  kExAtan2,
  kExFn1,  // fn: one-argument built-in (ExprFn1)
  kExFn2,  // fn: two-argument built-in (ExprFn2)
};

enum ExprFn1 : int {
  kFnCos, kFnSin, kFnTan, kFnExp, kFnSinh, kFnCosh, kFnTanh, kFnErf, kFnErfc, kFnInt, kFnAbs,
  kFnFloor, kFnCeil, kFnAcos, kFnAsin, kFnAtan, kFnAcosh, kFnAsinh, kFnAtanh, kFnLog, kFnLog10,
  kFnSqrt, kFnHeav, kFnSgn, kFnJ0, kFnJ1, kFnY0, kFnY1, kFnGamma, kFnLgamma,
};

enum ExprFn2 : int { kFnJn, kFnYn, kFnRad, kFnAng, kFnStep };

struct ExprOp {
  int code;
  int fn;
  double val;
};

constexpr int kExprMaxOps = 512;  // longest program accepted
constexpr int kExprStack = 24;    // deepest operand stack accepted

STX_HD inline double expr_fn1(int fn, double a) {
  switch (fn) {
    case kFnCos: return cos(a);
    case kFnSin: return sin(a);
    case kFnTan: return tan(a);
    case kFnExp: return exp(a);
    case kFnSinh: return sinh(a);
    case kFnCosh: return cosh(a);
    case kFnTanh: return tanh(a);
    case kFnErf: return erf(a);
    case kFnErfc: return erfc(a);
    case kFnInt: return rint(a);
    case kFnAbs: return fabs(a);
    case kFnFloor: return floor(a);
    case kFnCeil: return ceil(a);
    case kFnAcos: return acos(a);
    case kFnAsin: return asin(a);
    case kFnAtan: return atan(a);
    case kFnAcosh: return acosh(a);
    case kFnAsinh: return asinh(a);
    case kFnAtanh: return atanh(a);
    case kFnLog: return log(a);
    case kFnLog10: return log10(a);
    case kFnSqrt: return sqrt(a);
    case kFnHeav: return a >= 0.0 ? 1.0 : 0.0;
    case kFnSgn: return static_cast<double>((a > 0.0) - (a < 0.0));
    case kFnJ0: return j0(a);
    case kFnJ1: return j1(a);
    case kFnY0: return y0(a);
    case kFnY1: return y1(a);
    case kFnGamma: return tgamma(a);
    case kFnLgamma: return lgamma(a);
    default: return 0.0;
  }
}

STX_HD inline double expr_fn2(int fn, double a, double b) {
  switch (fn) {
    case kFnJn: return jn(static_cast<int>(a), b);
    case kFnYn: return yn(static_cast<int>(a), b);
    case kFnRad: return hypot(a, b);
    case kFnAng: return atan2(b, a);
    case kFnStep: return a >= b ? 1.0 : 0.0;
    default: return 0.0;
  }
}

// Binary operator `code` on (a, b).
STX_HD inline double expr_binary(int code, double a, double b) {
  switch (code) {
    case kExAdd: return a + b;
    case kExSub: return a - b;
    case kExMul: return a * b;
    case kExDiv: return b == 0.0 ? 0.0 : a / b;
    case kExMod: return fmod(a, b);
    case kExPow: return pow(a, b);
    case kExHypot: return hypot(a, b);
    case kExAtan2: return atan2(a, b);
    default: return 0.0;
  }
}

// Value of the program at (x, y, z, t).  Programs are checked when made
// (TokenTable::compile): at most kExprStack operands are ever live.
STX_HD inline double expr_run(const ExprOp* ops, int n, double x, double y, double z, double t) {
  double s[kExprStack];
  int sp = 0;
  for (int i = 0; i < n; ++i) {
    const ExprOp o = ops[i];
    switch (o.code) {
      case kExConst: s[sp++] = o.val; break;
      case kExX: s[sp++] = x; break;
      case kExY: s[sp++] = y; break;
      case kExZ: s[sp++] = z; break;
      case kExT: s[sp++] = t; break;
      case kExNeg: s[sp - 1] = -s[sp - 1]; break;
      case kExFn1: s[sp - 1] = expr_fn1(o.fn, s[sp - 1]); break;
      case kExFn2: --sp; s[sp - 1] = expr_fn2(o.fn, s[sp - 1], s[sp]); break;
      default: --sp; s[sp - 1] = expr_binary(o.code, s[sp - 1], s[sp]); break;
    }
  }
  return sp ? s[sp - 1] : 0.0;
}

}  // namespace stx
