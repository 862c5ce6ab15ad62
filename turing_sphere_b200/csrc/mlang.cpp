// .m front end: lexer, parser and specialisation (see mlang.h).
#include "mlang.h"

#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <set>
#include <sstream>

namespace tsm {

namespace {

// ------------------------------------------------------------------ lexer

struct Tok {
  enum Kind { Ident, Number, Op, Newline, Eof } kind;
  std::string text;
  double num = 0;
  long start = 0, end = 0;
};

[[noreturn]] void fail(const std::string &msg, long start = -1, long end = -1) {
  throw CompileError{msg, start, end, ""};
}

std::vector<Tok> lex(const std::string &s) {
  std::vector<Tok> out;
  const long n = (long)s.size();
  long i = 0;
  auto prev_allows_transpose = [&]() {
    if (out.empty()) return false;
    const Tok &t = out.back();
    if (t.kind == Tok::Ident || t.kind == Tok::Number) return true;
    return t.kind == Tok::Op && (t.text == ")" || t.text == "]" || t.text == "'" || t.text == ".'");
  };
  auto line_is = [&](long pos, const char *what) {
    // true if the line starting at pos is (whitespace) what (whitespace)
    long j = pos;
    while (j < n && (s[j] == ' ' || s[j] == '\t')) j++;
    const long w = (long)strlen(what);
    if (s.compare(j, w, what) != 0) return false;
    j += w;
    while (j < n && (s[j] == ' ' || s[j] == '\t' || s[j] == '\r')) j++;
    return j >= n || s[j] == '\n';
  };
  while (i < n) {
    const char c = s[i];
    if (c == ' ' || c == '\t' || c == '\r') {
      i++;
      continue;
    }
    if (c == '%') {
      // block comment: a line holding only "%{" up to a line holding only "%}"
      const long ls = s.rfind('\n', i == 0 ? 0 : i - 1);
      const long line_start = (ls == (long)std::string::npos || i == 0) ? 0 : ls + 1;
      if (i + 1 < n && s[i + 1] == '{' && line_is(line_start, "%{")) {
        long j = s.find('\n', i);
        int depth = 1;
        while (j != (long)std::string::npos && j < n) {
          const long next = j + 1;
          if (line_is(next, "%{")) depth++;
          if (line_is(next, "%}")) {
            if (--depth == 0) {
              j = s.find('\n', next);
              break;
            }
          }
          j = s.find('\n', next);
        }
        if (depth != 0) fail("unterminated block comment", i, n);
        i = (j == (long)std::string::npos) ? n : j;
        continue;
      }
      while (i < n && s[i] != '\n') i++;
      continue;
    }
    if (c == '\n') {
      out.push_back({Tok::Newline, "\n", 0, i, i + 1});
      i++;
      continue;
    }
    if (c == '.' && i + 2 < n && s[i + 1] == '.' && s[i + 2] == '.') {
      // continuation: the rest of the line is ignored
      while (i < n && s[i] != '\n') i++;
      if (i < n) i++;
      continue;
    }
    if (std::isdigit((unsigned char)c) || (c == '.' && i + 1 < n && std::isdigit((unsigned char)s[i + 1]))) {
      long j = i;
      while (j < n && std::isdigit((unsigned char)s[j])) j++;
      if (j < n && s[j] == '.' && !(j + 1 < n && (s[j + 1] == '*' || s[j + 1] == '/' ||
                                                  s[j + 1] == '^' || s[j + 1] == '\\' ||
                                                  s[j + 1] == '\''))) {
        j++;
        while (j < n && std::isdigit((unsigned char)s[j])) j++;
      }
      if (j < n && (s[j] == 'e' || s[j] == 'E')) {
        long k = j + 1;
        if (k < n && (s[k] == '+' || s[k] == '-')) k++;
        if (k < n && std::isdigit((unsigned char)s[k])) {
          j = k;
          while (j < n && std::isdigit((unsigned char)s[j])) j++;
        }
      }
      Tok t{Tok::Number, s.substr(i, j - i), 0, i, j};
      t.num = std::strtod(t.text.c_str(), nullptr);
      if (j < n && (std::isalpha((unsigned char)s[j]) || s[j] == '_'))
        fail("malformed number '" + s.substr(i, j - i + 1) + "'", i, j + 1);
      out.push_back(t);
      i = j;
      continue;
    }
    if (std::isalpha((unsigned char)c)) {
      long j = i;
      while (j < n && (std::isalnum((unsigned char)s[j]) || s[j] == '_')) j++;
      out.push_back({Tok::Ident, s.substr(i, j - i), 0, i, j});
      i = j;
      continue;
    }
    if (c == '\'' && !prev_allows_transpose()) {
      long j = i + 1;
      while (j < n && s[j] != '\'' && s[j] != '\n') j++;
      fail("character arrays are not supported in a model", i, j + 1);
    }
    if (c == '"') fail("strings are not supported in a model", i, i + 1);
    static const char *ops[] = {".*", "./", ".^", ".\\", ".'", "==", "~=", "<=", ">=", "&&", "||",
                                "+",  "-",  "*",  "/",   "^",  "\\", "'",  "<",  ">",  "&",  "|",
                                "~",  "!",  "=",  "(",   ")",  "[",  "]",  "{",  "}",  ",",  ";",
                                ":",  "@",  "."};
    bool matched = false;
    for (const char *op : ops) {
      const long w = (long)strlen(op);
      if (s.compare(i, w, op) == 0) {
        out.push_back({Tok::Op, op, 0, i, i + w});
        i += w;
        matched = true;
        break;
      }
    }
    if (!matched) fail(std::string("unexpected character '") + c + "'", i, i + 1);
  }
  out.push_back({Tok::Eof, "", 0, n, n});
  return out;
}

// ----------------------------------------------------------------- parser

const std::set<std::string> kUnsupportedKeywords = {
    "if", "elseif", "else", "for", "while", "switch", "case", "otherwise", "try", "catch",
    "break", "continue", "global", "persistent", "parfor", "do", "until", "classdef"};

struct Parser {
  std::vector<Tok> t;
  size_t p = 0;

  const Tok &cur() const { return t[p]; }
  bool is_op(const char *o) const { return cur().kind == Tok::Op && cur().text == o; }
  bool is_ident(const char *w) const { return cur().kind == Tok::Ident && cur().text == w; }
  void expect_op(const char *o) {
    if (!is_op(o))
      fail(std::string("expected '") + o + "' but found '" + describe_tok() + "'", cur().start,
           cur().end);
    p++;
  }
  std::string describe_tok() const {
    return cur().kind == Tok::Eof ? "end of file" : cur().kind == Tok::Newline ? "end of line" : cur().text;
  }
  void skip_newlines() {
    while (cur().kind == Tok::Newline || is_op(";") || is_op(",")) p++;
  }

  std::vector<AstFunction> file() {
    std::vector<AstFunction> fns;
    skip_newlines();
    while (cur().kind != Tok::Eof) {
      if (!is_ident("function"))
        fail("a model file may contain only function definitions (found '" + describe_tok() + "')",
             cur().start, cur().end);
      fns.push_back(function());
      skip_newlines();
    }
    return fns;
  }

  std::string ident(const char *what) {
    if (cur().kind != Tok::Ident)
      fail(std::string("expected ") + what + " but found '" + describe_tok() + "'", cur().start,
           cur().end);
    return t[p++].text;
  }

  AstFunction function() {
    AstFunction f;
    f.start = cur().start;
    p++;  // 'function'
    // [outs] = name(args) | out = name(args) | name(args)
    if (is_op("[")) {
      p++;
      while (!is_op("]")) {
        f.outputs.push_back(ident("an output name"));
        if (is_op(",")) p++;
      }
      p++;
      expect_op("=");
      f.name = ident("a function name");
    } else {
      const std::string first = ident("a function name");
      if (is_op("=")) {
        p++;
        f.outputs.push_back(first);
        f.name = ident("a function name");
      } else {
        f.name = first;
      }
    }
    if (is_op("(")) {
      p++;
      while (!is_op(")")) {
        if (is_op("~")) fail("ignored arguments (~) are not supported", cur().start, cur().end);
        f.params.push_back(ident("an argument name"));
        if (is_op(",")) p++;
        else if (!is_op(")"))
          fail("expected ',' or ')' in the argument list", cur().start, cur().end);
      }
      p++;
    }
    // body
    while (true) {
      skip_newlines();
      if (cur().kind == Tok::Eof || is_ident("function")) break;
      if (is_ident("end")) {
        p++;
        break;
      }
      if (is_ident("return")) {
        p++;
        continue;
      }
      if (cur().kind == Tok::Ident && kUnsupportedKeywords.count(cur().text))
        fail("'" + cur().text + "' is not supported in a model function: only assignments are",
             cur().start, cur().end);
      f.body.push_back(assignment());
    }
    f.end = t[p > 0 ? p - 1 : 0].end;
    return f;
  }

  AstAssign assignment() {
    AstAssign a;
    a.start = cur().start;
    if (is_op("["))
      fail("multiple assignment is not supported: assign one value per statement", cur().start,
           cur().end);
    if (cur().kind != Tok::Ident)
      fail("expected an assignment but found '" + describe_tok() + "'", cur().start, cur().end);
    a.lhs = t[p++].text;
    if (is_op("(") || is_op("{"))
      fail("indexed assignment is not supported: assign whole arrays", cur().start, cur().end);
    if (!is_op("=")) {
      fail("expected '=' after '" + a.lhs + "' (a model function may only contain assignments)",
           cur().start, cur().end);
    }
    p++;
    a.rhs = expr();
    a.end = a.rhs->end;
    if (!(cur().kind == Tok::Newline || cur().kind == Tok::Eof || is_op(";") || is_op(",")))
      fail("unexpected '" + describe_tok() + "' after the expression", cur().start, cur().end);
    return a;
  }

  std::unique_ptr<Ast> node(Ast::Kind k, long s, long e) {
    auto a = std::make_unique<Ast>();
    a->kind = k;
    a->start = s;
    a->end = e;
    return a;
  }

  std::unique_ptr<Ast> binary(const std::string &op, std::unique_ptr<Ast> l, std::unique_ptr<Ast> r) {
    auto a = node(Ast::Binary, l->start, r->end);
    a->op = op;
    a->args.push_back(std::move(l));
    a->args.push_back(std::move(r));
    return a;
  }

  std::unique_ptr<Ast> expr() {
    auto l = mult();
    while (is_op("+") || is_op("-")) {
      const std::string op = t[p++].text;
      l = binary(op, std::move(l), mult());
    }
    if (is_op("==") || is_op("~=") || is_op("<") || is_op(">") || is_op("<=") || is_op(">=") ||
        is_op("&") || is_op("|") || is_op("&&") || is_op("||") || is_op(":"))
      fail("operator '" + cur().text + "' is not supported in a model", cur().start, cur().end);
    return l;
  }

  std::unique_ptr<Ast> mult() {
    auto l = unary();
    while (is_op("*") || is_op("/") || is_op(".*") || is_op("./") || is_op("\\") || is_op(".\\")) {
      const std::string op = t[p].text;
      if (op == "\\" || op == ".\\")
        fail("left division is not supported", cur().start, cur().end);
      p++;
      l = binary(op, std::move(l), unary());
    }
    return l;
  }

  std::unique_ptr<Ast> unary() {
    if (is_op("-") || is_op("+")) {
      const long s = cur().start;
      const std::string op = t[p++].text;
      auto x = unary();
      auto a = node(Ast::Unary, s, x->end);
      a->op = op;
      a->args.push_back(std::move(x));
      return a;
    }
    if (is_op("~") || is_op("!")) fail("logical not is not supported", cur().start, cur().end);
    return power();
  }

  std::unique_ptr<Ast> power() {
    auto l = postfix();
    while (is_op("^") || is_op(".^")) {
      const std::string op = t[p++].text;
      l = binary(op, std::move(l), power_operand());
    }
    return l;
  }

  std::unique_ptr<Ast> power_operand() {
    if (is_op("-") || is_op("+")) {
      const long s = cur().start;
      const std::string op = t[p++].text;
      auto x = power_operand();
      auto a = node(Ast::Unary, s, x->end);
      a->op = op;
      a->args.push_back(std::move(x));
      return a;
    }
    return postfix();
  }

  std::unique_ptr<Ast> postfix() {
    auto x = primary();
    if (is_op("'") || is_op(".'")) fail("transpose is not supported", cur().start, cur().end);
    return x;
  }

  std::unique_ptr<Ast> primary() {
    const Tok &k = cur();
    if (k.kind == Tok::Number) {
      auto a = node(Ast::Num, k.start, k.end);
      a->num = k.num;
      p++;
      return a;
    }
    if (k.kind == Tok::Ident) {
      if (kUnsupportedKeywords.count(k.text) || k.text == "end" || k.text == "function")
        fail("unexpected keyword '" + k.text + "' in an expression", k.start, k.end);
      const std::string name = k.text;
      const long s = k.start;
      p++;
      if (is_op("(")) {
        p++;
        auto a = node(Ast::Call, s, s);
        a->name = name;
        while (!is_op(")")) {
          if (is_op(":")) fail("':' is not supported", cur().start, cur().end);
          a->args.push_back(expr());
          if (is_op(",")) p++;
          else if (!is_op(")"))
            fail("expected ',' or ')' in the argument list", cur().start, cur().end);
        }
        a->end = cur().end;
        p++;
        return a;
      }
      if (is_op("{")) fail("cell arrays are not supported", cur().start, cur().end);
      auto a = node(Ast::Ident, s, k.end);
      a->name = name;
      return a;
    }
    if (is_op("(")) {
      p++;
      auto e = expr();
      expect_op(")");
      return e;
    }
    if (is_op("[")) fail("array literals are not supported; use ones/zeros", k.start, k.end);
    if (is_op("@")) fail("function handles are not supported", k.start, k.end);
    fail("unexpected '" + describe_tok() + "' in an expression", k.start, k.end);
  }
};

// ----------------------------------------------------------- specialisation

const std::map<std::string, int> kElementwise = {
    {"abs", 1},  {"acos", 1}, {"asin", 1}, {"atan", 1}, {"atan2", 2}, {"ceil", 1}, {"cos", 1},
    {"cosh", 1}, {"exp", 1},  {"floor", 1}, {"log", 1}, {"log2", 1},  {"max", 2},  {"min", 2},
    {"round", 1}, {"sign", 1}, {"sin", 1}, {"sinh", 1}, {"sqrt", 1},  {"tan", 1},  {"tanh", 1}};

double fold_call(const std::string &fn, double a, double b) {
  if (fn == "abs") return std::fabs(a);
  if (fn == "acos") return std::acos(a);
  if (fn == "asin") return std::asin(a);
  if (fn == "atan") return std::atan(a);
  if (fn == "atan2") return std::atan2(a, b);
  if (fn == "ceil") return std::ceil(a);
  if (fn == "cos") return std::cos(a);
  if (fn == "cosh") return std::cosh(a);
  if (fn == "exp") return std::exp(a);
  if (fn == "floor") return std::floor(a);
  if (fn == "log") return std::log(a);
  if (fn == "log2") return std::log2(a);
  if (fn == "max") return std::fmax(a, b);
  if (fn == "min") return std::fmin(a, b);
  if (fn == "round") return std::nearbyint(a);  // ties to even, as WGSL round (wgsl.ts:64)
  if (fn == "sign") return (a > 0) - (a < 0);
  if (fn == "sin") return std::sin(a);
  if (fn == "sinh") return std::sinh(a);
  if (fn == "sqrt") return std::sqrt(a);
  if (fn == "tan") return std::tan(a);
  return std::tanh(a);
}

const char *dom_name(Dom d, const Grid &g, char *buf, size_t cap) {
  if (d == Dom::Grid) snprintf(buf, cap, "%ldx1", g.npts);
  else if (d == Dom::Spec) snprintf(buf, cap, "2x%ld", g.nlm);
  else snprintf(buf, cap, "1x1");
  return buf;
}

struct Lowerer {
  const std::vector<AstFunction> &file;
  const std::map<std::string, Binding> &bindings;
  const std::vector<std::string> &model_params;
  Grid g;
  Function f;
  // name -> value: Var id, runtime scalar (Scalar id / Param slot) or exact
  struct Val {
    enum K { V, Exact, ParamS, ScalarS } k;
    int id = -1;
    double value = 0;
  };
  std::map<std::string, Val> env;
  int ntemp = 0;

  ExprP mk(Expr::Kind k, const Ast &a) {
    auto e = std::make_shared<Expr>();
    e->kind = k;
    e->start = a.start;
    e->end = a.end;
    return e;
  }

  ExprP lit(double v, const Ast &a) {
    auto e = mk(Expr::Lit, a);
    e->value = v;
    e->exact = true;
    return e;
  }

  int new_var(const std::string &name, Dom d, bool temp) {
    f.vars.push_back(Var{name, d, temp, -1});
    return (int)f.vars.size() - 1;
  }

  ExprP var_ref(int id, const Ast &a) {
    auto e = mk(Expr::Var, a);
    e->index = id;
    e->dom = f.vars[id].dom;
    return e;
  }

  // make `e` available as a Var (hoisting a temporary statement if needed)
  int as_var(ExprP e, const Ast &a) {
    if (e->kind == Expr::Var) return e->index;
    if (e->dom == Dom::Scalar)
      fail("the transforms take an array argument, not a scalar", a.start, a.end);
    const int v = new_var("t" + std::to_string(++ntemp), e->dom, true);
    Stmt s;
    s.kind = Stmt::Elementwise;
    s.out = v;
    s.expr = e;
    s.start = a.start;
    s.end = a.end;
    f.body.push_back(s);
    return v;
  }

  Dom join(Dom a, Dom b, const Ast &at) {
    if (a == Dom::Scalar) return b;
    if (b == Dom::Scalar) return a;
    if (a != b) {
      char b1[64], b2[64];
      fail(std::string("implicit expansion is not supported: an operand is ") +
               dom_name(a, g, b1, 64) + " and the other " + dom_name(b, g, b2, 64) +
               " (the GPU kernel walks one index across every operand)",
           at.start, at.end);
    }
    return a;
  }

  ExprP lower(const Ast &a) {
    switch (a.kind) {
      case Ast::Num:
        return lit(a.num, a);
      case Ast::Ident: {
        auto it = env.find(a.name);
        if (it == env.end()) {
          if (a.name == "pi") return lit(M_PI, a);
          if (a.name == "Inf" || a.name == "inf" || a.name == "NaN" || a.name == "nan")
            fail("non-finite constants cannot be emitted", a.start, a.end);
          if (a.name == "synth" || a.name == "analys" || a.name == "numel" || a.name == "ones" ||
              a.name == "zeros" || kElementwise.count(a.name))
            return lower_call(a);  // called without parentheses
          fail("undefined function or variable '" + a.name + "'", a.start, a.end);
        }
        const Val &v = it->second;
        if (v.k == Val::V) return var_ref(v.id, a);
        if (v.k == Val::Exact) return lit(v.value, a);
        auto e = mk(v.k == Val::ParamS ? Expr::Param : Expr::Scalar, a);
        e->index = v.id;
        return e;
      }
      case Ast::Unary: {
        auto x = lower(*a.args[0]);
        if (a.op == "+") return x;
        if (x->exact) return lit(-x->value, a);
        auto e = mk(Expr::Unary, a);
        e->op = "-";
        e->dom = x->dom;
        e->args.push_back(x);
        return e;
      }
      case Ast::Binary:
        return lower_binary(a);
      case Ast::Call:
        return lower_call(a);
    }
    fail("unsupported expression", a.start, a.end);
  }

  ExprP lower_binary(const Ast &a) {
    auto l = lower(*a.args[0]);
    auto r = lower(*a.args[1]);
    const std::string &op = a.op;
    if (op == "^" || op == ".^") {
      if (!r->exact)
        fail("'.^' needs a literal integer exponent in [-8, 8] (got a runtime value); a negative "
             "base makes a general pow() undefined",
             a.start, a.end);
      const double k = r->value;
      if (k != std::floor(k) || std::fabs(k) > 8) {
        char buf[200];
        snprintf(buf, sizeof buf,
                 "'.^' needs a literal integer exponent in [-8, 8] (got %g); a negative base "
                 "makes a general pow() undefined",
                 k);
        fail(buf, a.start, a.end);
      }
      if (l->exact) return lit(std::pow(l->value, k), a);
      if (k == 0) return lit(1.0, a);
      auto e = mk(Expr::PowI, a);
      e->k = (int)k;
      e->dom = l->dom;
      e->args.push_back(l);
      return e;
    }
    std::string o;
    if (op == "+" || op == "-") o = op;
    else if (op == ".*" || op == "*") o = "*";
    else if (op == "./" || op == "/") o = "/";
    else fail("operator '" + op + "' is not supported", a.start, a.end);
    if ((op == "*" || op == "/") && l->dom != Dom::Scalar && r->dom != Dom::Scalar)
      fail(std::string("matrix '") + op + "' is not supported; use the element-wise form ('." + op +
               "')",
           a.start, a.end);
    const Dom d = join(l->dom, r->dom, a);
    if (l->exact && r->exact) {
      const double x = l->value, y = r->value;
      return lit(o == "+" ? x + y : o == "-" ? x - y : o == "*" ? x * y : x / y, a);
    }
    auto e = mk(Expr::Binary, a);
    e->op = o;
    e->dom = d;
    e->args.push_back(l);
    e->args.push_back(r);
    return e;
  }

  long exact_int(const ExprP &e, const Ast &a, const char *what) {
    if (!e->exact || e->value != std::floor(e->value) || e->value < 0)
      fail(std::string(what) + " needs compile-time non-negative integer sizes", a.start, a.end);
    return (long)e->value;
  }

  ExprP lower_call(const Ast &a) {
    const std::string &fn = a.name;
    if (env.count(fn) && a.kind == Ast::Call)
      fail("indexing '" + fn + "' is not supported: the GPU kernels work on whole arrays", a.start,
           a.end);
    std::vector<ExprP> args;
    if (a.kind == Ast::Call)
      for (auto &x : a.args) args.push_back(lower(*x));
    if (fn == "synth" || fn == "analys") {
      if (args.size() != 1)
        fail(fn + " takes exactly one argument, got " + std::to_string(args.size()), a.start, a.end);
      const Dom want = fn == "synth" ? Dom::Spec : Dom::Grid;
      if (args[0]->dom != want) {
        char b1[64], b2[64];
        fail(fn + " requires a " + dom_name(want, g, b1, 64) + " array, got " +
                 dom_name(args[0]->dom, g, b2, 64),
             a.start, a.end);
      }
      const int in = as_var(args[0], a);
      const Dom outd = fn == "synth" ? Dom::Grid : Dom::Spec;
      const int out = new_var("t" + std::to_string(++ntemp), outd, true);
      Stmt s;
      s.kind = fn == "synth" ? Stmt::Synth : Stmt::Analys;
      s.out = out;
      s.arg = in;
      s.start = a.start;
      s.end = a.end;
      f.body.push_back(s);
      return var_ref(out, a);
    }
    if (fn == "numel") {
      if (args.size() != 1) fail("numel takes one argument", a.start, a.end);
      const Dom d = args[0]->dom;
      return lit(d == Dom::Grid ? (double)g.npts : d == Dom::Spec ? 2.0 * g.nlm : 1.0, a);
    }
    if (fn == "ones" || fn == "zeros") {
      long r = 1, c = 1;
      if (args.size() == 1) r = c = exact_int(args[0], a, fn.c_str());
      else if (args.size() == 2) {
        r = exact_int(args[0], a, fn.c_str());
        c = exact_int(args[1], a, fn.c_str());
      } else if (!args.empty())
        fail(fn + " takes at most two size arguments", a.start, a.end);
      const double v = fn == "ones" ? 1.0 : 0.0;
      if (r == 1 && c == 1) return lit(v, a);
      Dom d;
      if (r == g.npts && c == 1) d = Dom::Grid;
      else if (r == 2 && c == g.nlm) d = Dom::Spec;
      else {
        char buf[256];
        snprintf(buf, sizeof buf,
                 "%s(%ld, %ld): only grid (%ldx1) and spectral (2x%ld) arrays are supported",
                 fn.c_str(), r, c, g.npts, g.nlm);
        fail(buf, a.start, a.end);
      }
      auto e = mk(Expr::Fill, a);
      e->value = v;
      e->dom = d;
      return e;
    }
    auto it = kElementwise.find(fn);
    if (it == kElementwise.end()) {
      for (const auto &d : file)
        if (d.name == fn)
          fail("'" + fn + "' is a function defined in this model. Only init and step are compiled "
               "— inline its body into the caller.",
               a.start, a.end);
      fail("'" + fn + "' cannot be evaluated element-wise on the GPU", a.start, a.end);
    }
    if ((int)args.size() != it->second)
      fail(fn + " takes " + std::to_string(it->second) + " argument(s)", a.start, a.end);
    bool all_exact = true;
    Dom d = Dom::Scalar;
    for (auto &x : args) {
      all_exact = all_exact && x->exact;
      d = join(d, x->dom, a);
    }
    if (all_exact) return lit(fold_call(fn, args[0]->value, args.size() > 1 ? args[1]->value : 0), a);
    auto e = mk(Expr::Call, a);
    e->fn = fn;
    e->dom = d;
    e->args = args;
    return e;
  }

  void run(const AstFunction &decl, int nargout) {
    f.name = decl.name;
    if ((int)decl.outputs.size() < nargout)
      fail("'" + decl.name + "' must return " + std::to_string(nargout) + " value" +
               (nargout == 1 ? "" : "s") + ", but declares " + std::to_string(decl.outputs.size()),
           decl.start, decl.end);
    for (size_t i = 0; i < decl.params.size(); i++) {
      const std::string &pn = decl.params[i];
      auto b = bindings.find(pn);
      if (b == bindings.end()) {
        std::string offered;
        for (auto &kv : bindings) offered += (offered.empty() ? "" : ", ") + kv.first;
        fail("'" + decl.name + "' takes an argument named '" + pn +
                 "', which this app does not provide. Available: " + offered + ".",
             decl.start, decl.end);
      }
      f.param_names.push_back(pn);
      f.param_bindings.push_back(b->second);
      f.param_vars.push_back(-1);
      f.param_slot.push_back(-1);
      Val v;
      if (b->second.kind == Binding::Tensor) {
        const int id = new_var(pn, b->second.dom, false);
        f.vars[id].param_index = (int)i;
        f.param_vars.back() = id;
        v.k = Val::V;
        v.id = id;
      } else if (b->second.kind == Binding::Const) {
        v.k = Val::Exact;
        v.value = b->second.value;
      } else {
        int slot = -1;
        for (size_t k = 0; k < model_params.size(); k++)
          if (model_params[k] == pn) slot = (int)k;
        if (slot < 0) fail("parameter '" + pn + "' is not in the model's parameter list");
        f.param_slot.back() = slot;
        v.k = Val::ParamS;
        v.id = slot;
      }
      env[pn] = v;
    }
    for (const auto &st : decl.body) {
      auto e = lower(*st.rhs);
      Val v;
      if (e->dom == Dom::Scalar) {
        if (e->exact) {
          v.k = Val::Exact;
          v.value = e->value;
        } else {
          f.scalars.push_back(DerivedScalar{st.lhs, e});
          v.k = Val::ScalarS;
          v.id = (int)f.scalars.size() - 1;
        }
      } else if (e->kind == Expr::Var && f.vars[e->index].temp && !f.body.empty() &&
                 f.body.back().out == e->index && f.body.back().kind != Stmt::Elementwise) {
        // `X = synth(Y)` / `X = analys(Y)`: the call's result takes the name
        f.vars[e->index].name = st.lhs;
        f.vars[e->index].temp = false;
        f.body.back().start = st.start;
        f.body.back().end = st.end;
        v.k = Val::V;
        v.id = e->index;
      } else {
        const int id = new_var(st.lhs, e->dom, false);
        Stmt s;
        s.kind = Stmt::Elementwise;
        s.out = id;
        s.expr = e;
        s.start = st.start;
        s.end = st.end;
        f.body.push_back(s);
        v.k = Val::V;
        v.id = id;
      }
      env[st.lhs] = v;
    }
    for (int i = 0; i < nargout; i++) {
      const std::string &on = decl.outputs[i];
      auto it = env.find(on);
      if (it == env.end())
        fail("'" + decl.name + "' declares the output '" + on + "' but never assigns it",
             decl.start, decl.end);
      if (it->second.k != Val::V)
        fail("output '" + on + "' of '" + decl.name + "' must be an array", decl.start, decl.end);
      f.output_names.push_back(on);
      f.output_vars.push_back(it->second.id);
    }
    for (auto &s : f.body) {
      const Var &o = f.vars[s.out];
      if (s.kind == Stmt::Synth) s.label = o.name + " = synth(" + f.vars[s.arg].name + ")";
      else if (s.kind == Stmt::Analys) s.label = o.name + " = analys(" + f.vars[s.arg].name + ")";
      else
        s.label = o.name + " = <" +
                  std::to_string(o.dom == Dom::Grid ? g.npts : 2 * g.nlm) +
                  " elements, element-wise>";
    }
  }
};

}  // namespace

std::vector<AstFunction> parse_model(const std::string &src) {
  Parser ps;
  ps.t = lex(src);
  return ps.file();
}

Function specialize(const std::vector<AstFunction> &file, const std::string &name,
                    const std::map<std::string, Binding> &bindings,
                    const std::vector<std::string> &model_params, int nargout, const Grid &g) {
  const AstFunction *decl = nullptr;
  for (const auto &d : file)
    if (d.name == name) decl = &d;
  if (!decl) {
    std::string defined;
    for (const auto &d : file) defined += (defined.empty() ? "'" : ", '") + d.name + "'";
    throw CompileError{"the model must define a function named '" + name + "'" +
                           (defined.empty() ? " (it defines no functions)"
                                            : " (it defines " + defined + ")"),
                       -1, -1, name};
  }
  Lowerer L{file, bindings, model_params, g, {}, {}, 0};
  try {
    L.run(*decl, nargout);
  } catch (CompileError &e) {
    e.fn = name;
    throw;
  }
  return L.f;
}

int count_kernels(const Function &f) {
  int n = 0;
  for (const auto &s : f.body) n += s.kind == Stmt::Elementwise;
  return n;
}

std::string describe(const Function &f) {
  std::ostringstream o;
  for (const auto &s : f.body) {
    const char *k = s.kind == Stmt::Synth ? "synth  " : s.kind == Stmt::Analys ? "analys " : "kernel ";
    o << k << " " << s.label << "\n";
  }
  return o.str();
}

}  // namespace tsm
