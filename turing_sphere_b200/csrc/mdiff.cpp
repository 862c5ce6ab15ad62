// Symbolic differentiation of lowered .m expressions (the adjoint's building
// block): d e / d x for x a variable (grid or spectral value) or a model
// parameter slot.  Derived scalars (functions of the parameters, e.g.
// vs = b/(a+b)^2) are differentiated through by the chain rule; constants
// fold as the derivative is built, so the emitted code stays small.
#include <cmath>
#include <stdexcept>

#include "mlang.h"

namespace tsm {

namespace {

ExprP mk(Expr::Kind k) {
  auto e = std::make_shared<Expr>();
  e->kind = k;
  return e;
}

ExprP lit(double v) {
  auto e = mk(Expr::Lit);
  e->value = v;
  e->exact = true;
  return e;
}

bool is_lit(const ExprP &e, double v) {
  return (e->kind == Expr::Lit || e->kind == Expr::Fill) && e->value == v;
}
bool is_const(const ExprP &e) { return e->kind == Expr::Lit || e->kind == Expr::Fill; }

ExprP bin(const std::string &op, ExprP a, ExprP b) {
  if (is_const(a) && is_const(b)) {
    const double x = a->value, y = b->value;
    if (op == "+") return lit(x + y);
    if (op == "-") return lit(x - y);
    if (op == "*") return lit(x * y);
    if (op == "/" && y != 0) return lit(x / y);
  }
  if (op == "+") {
    if (is_lit(a, 0)) return b;
    if (is_lit(b, 0)) return a;
  } else if (op == "-") {
    if (is_lit(b, 0)) return a;
  } else if (op == "*") {
    if (is_lit(a, 0) || is_lit(b, 0)) return lit(0);
    if (is_lit(a, 1)) return b;
    if (is_lit(b, 1)) return a;
  } else if (op == "/") {
    if (is_lit(a, 0)) return lit(0);
    if (is_lit(b, 1)) return a;
  }
  auto e = mk(Expr::Binary);
  e->op = op;
  e->args = {a, b};
  return e;
}

ExprP neg(ExprP a) {
  if (is_const(a)) return lit(-a->value);
  if (a->kind == Expr::Unary) return a->args[0];
  auto e = mk(Expr::Unary);
  e->op = "-";
  e->args = {a};
  return e;
}

ExprP call(const std::string &fn, std::vector<ExprP> args) {
  auto e = mk(Expr::Call);
  e->fn = fn;
  e->args = std::move(args);
  return e;
}

ExprP powi(ExprP a, int k) {
  if (k == 0) return lit(1);
  if (k == 1) return a;
  auto e = mk(Expr::PowI);
  e->k = k;
  e->args = {a};
  return e;
}

ExprP add(ExprP a, ExprP b) { return bin("+", a, b); }
ExprP sub(ExprP a, ExprP b) { return bin("-", a, b); }
ExprP mul(ExprP a, ExprP b) { return bin("*", a, b); }
ExprP dvd(ExprP a, ExprP b) { return bin("/", a, b); }

}  // namespace

ExprP differentiate(const Function &f, const ExprP &e, const Wrt &w) {
  switch (e->kind) {
    case Expr::Lit:
    case Expr::Fill:
      return lit(0);
    case Expr::Param:
      return lit(w.kind == Wrt::Param && w.index == e->index ? 1 : 0);
    case Expr::Scalar:
      if (w.kind != Wrt::Param) return lit(0);
      return differentiate(f, f.scalars.at(e->index).expr, w);
    case Expr::Var:
      return lit(w.kind == Wrt::Var && w.index == e->index ? 1 : 0);
    case Expr::Unary:
      return neg(differentiate(f, e->args[0], w));
    case Expr::Binary: {
      const ExprP &a = e->args[0], &b = e->args[1];
      const ExprP da = differentiate(f, a, w), db = differentiate(f, b, w);
      if (e->op == "+") return add(da, db);
      if (e->op == "-") return sub(da, db);
      if (e->op == "*") return add(mul(da, b), mul(a, db));
      if (e->op == "/") return sub(dvd(da, b), mul(dvd(a, b), dvd(db, b)));
      throw CompileError{"cannot differentiate operator '" + e->op + "'"};
    }
    case Expr::PowI: {
      const ExprP &a = e->args[0];
      const ExprP da = differentiate(f, a, w);
      if (is_lit(da, 0)) return lit(0);
      const int k = e->k;
      // d a^k = k a^(k-1) da; for k < 0 written as k a^k / a (|k - 1| may exceed 8)
      const ExprP g = k > 0 ? powi(a, k - 1) : dvd(e, a);
      return mul(mul(lit(k), g), da);
    }
    case Expr::Call: {
      const std::string &fn = e->fn;
      if (fn == "max" || fn == "min") {
        const ExprP da = differentiate(f, e->args[0], w), db = differentiate(f, e->args[1], w);
        if (is_lit(da, 0) && is_lit(db, 0)) return lit(0);
        // the derivative of the selected argument (ties take the first)
        return fn == "max" ? call("__ge_sel", {e->args[0], e->args[1], da, db})
                           : call("__ge_sel", {e->args[1], e->args[0], da, db});
      }
      if (fn == "atan2") {
        const ExprP &y = e->args[0], &x = e->args[1];
        const ExprP dy = differentiate(f, y, w), dx = differentiate(f, x, w);
        if (is_lit(dy, 0) && is_lit(dx, 0)) return lit(0);
        return dvd(sub(mul(x, dy), mul(y, dx)), add(mul(x, x), mul(y, y)));
      }
      const ExprP &a = e->args[0];
      const ExprP da = differentiate(f, a, w);
      if (is_lit(da, 0)) return lit(0);
      if (fn == "ceil" || fn == "floor" || fn == "round" || fn == "sign") return lit(0);
      ExprP g;
      if (fn == "abs") g = call("sign", {a});
      else if (fn == "exp") g = e;
      else if (fn == "log") g = dvd(lit(1), a);
      else if (fn == "log2") g = dvd(lit(1.0 / std::log(2.0)), a);
      else if (fn == "sqrt") g = dvd(lit(0.5), e);
      else if (fn == "sin") g = call("cos", {a});
      else if (fn == "cos") g = neg(call("sin", {a}));
      else if (fn == "tan") g = add(lit(1), powi(e, 2));
      else if (fn == "sinh") g = call("cosh", {a});
      else if (fn == "cosh") g = call("sinh", {a});
      else if (fn == "tanh") g = sub(lit(1), powi(e, 2));
      else if (fn == "asin") g = dvd(lit(1), call("sqrt", {sub(lit(1), powi(a, 2))}));
      else if (fn == "acos") g = neg(dvd(lit(1), call("sqrt", {sub(lit(1), powi(a, 2))})));
      else if (fn == "atan") g = dvd(lit(1), add(lit(1), powi(a, 2)));
      else throw CompileError{"cannot differentiate '" + fn + "'"};
      return mul(g, da);
    }
  }
  return lit(0);
}

bool is_zero(const ExprP &e) { return is_lit(e, 0); }

}  // namespace tsm
