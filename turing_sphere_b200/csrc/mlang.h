// The .m model language: the subset of MATLAB the reference's models use,
// parsed, specialised for one grid and lowered to typed statements.
//
// This stands in for the numbl front end the reference drives
// (src/mgpu/compile.ts:83-190): parse the file, specialise `init`/`step` for
// the host's argument bindings, and fold single-use temporaries back into
// their consumer so that one element-wise source line is one statement
// (inlinePass).  The type rules of the external transforms are those of
// src/mgpu/externals.ts:39-95: synth: 2 x nlm -> npts x 1, analys: the reverse.
#pragma once

#include <map>
#include <memory>
#include <string>
#include <vector>

namespace tsm {

struct CompileError {
  std::string message;
  long start = -1, end = -1;  // byte offsets into the model source
  std::string fn;             // model function being compiled
};

// ------------------------------------------------------------------ AST
struct Ast {
  enum Kind { Num, Ident, Binary, Unary, Call } kind;
  double num = 0;
  std::string name;  // Ident / Call
  std::string op;    // Binary: + - .* ./ * / .^ ^ ; Unary: - +
  std::vector<std::unique_ptr<Ast>> args;
  long start = 0, end = 0;
};

struct AstAssign {
  std::string lhs;
  std::unique_ptr<Ast> rhs;
  long start = 0, end = 0;
};

struct AstFunction {
  std::string name;
  std::vector<std::string> params, outputs;
  std::vector<AstAssign> body;
  long start = 0, end = 0;
};

std::vector<AstFunction> parse_model(const std::string &src);

// ----------------------------------------------------------------- types
// Scalars are exact (a compile-time value) or runtime (a parameter or a
// value derived from parameters).  Arrays are grid fields (npts x 1) or
// spectral fields (2 x nlm); other shapes are rejected.
enum class Dom { Scalar, Grid, Spec };

struct Binding {
  enum Kind { Tensor, Param, Const } kind;
  Dom dom = Dom::Scalar;  // Tensor: Grid or Spec
  double value = 0;       // Const
};

// ---------------------------------------------------------------- lowered IR
struct Expr {
  enum Kind { Lit, Param, Scalar, Var, Binary, Unary, Call, PowI, Fill } kind;
  double value = 0;    // Lit; Fill (ones/zeros) value
  int index = -1;      // Param slot, Scalar id, Var id
  std::string op;      // Binary: + - * / ; Unary: -
  std::string fn;      // Call: builtin name
  int k = 0;           // PowI exponent, |k| <= 8
  std::vector<std::shared_ptr<Expr>> args;
  Dom dom = Dom::Scalar;
  bool exact = false;  // scalar known at compile time
  long start = 0, end = 0;
};
using ExprP = std::shared_ptr<Expr>;

struct Var {
  std::string name;  // source name, or a generated temporary name
  Dom dom;
  bool temp = false;
  int param_index = -1;  // >= 0: bound to the function's argument of this index
};

struct Stmt {
  enum Kind { Elementwise, Synth, Analys } kind;
  int out = -1;   // Var id
  int arg = -1;   // Synth/Analys input Var id
  ExprP expr;     // Elementwise
  long start = 0, end = 0;
  std::string label;
};

struct DerivedScalar {
  std::string name;
  ExprP expr;
};

struct Function {
  std::string name;
  std::vector<std::string> param_names;   // declared arguments
  std::vector<Binding> param_bindings;
  std::vector<int> param_vars;            // Var id per tensor argument (-1 otherwise)
  std::vector<int> param_slot;            // model-parameter index per Param argument (-1)
  std::vector<std::string> output_names;
  std::vector<int> output_vars;           // Var id holding each requested output
  std::vector<Var> vars;
  std::vector<Stmt> body;
  std::vector<DerivedScalar> scalars;
};

struct Grid {
  long npts, nlm;
};

// Specialise `name` for the bindings.  `model_params` fixes the slot of every
// parameter name (the model's parameter list); nargout = outputs requested.
Function specialize(const std::vector<AstFunction> &file, const std::string &name,
                    const std::map<std::string, Binding> &bindings,
                    const std::vector<std::string> &model_params, int nargout, const Grid &g);

std::string describe(const Function &f);
int count_kernels(const Function &f);

// Symbolic derivative d e / d w (mdiff.cpp): w is a variable or a model
// parameter slot; derived scalars are differentiated through.  The result
// may call "__ge_sel"(a, b, x, y) = a >= b ? x : y (max/min).
struct Wrt {
  enum Kind { Var, Param } kind;
  int index;
};
ExprP differentiate(const Function &f, const ExprP &e, const Wrt &w);
bool is_zero(const ExprP &e);

}  // namespace tsm
