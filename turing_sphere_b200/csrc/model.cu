// Compiled .m models: scheduling into fused launches, CUDA-C generation,
// NVRTC compilation for sm_100a, and execution.
//
// The reference turns every element-wise statement into one WGSL kernel and
// every synth/analys into two dispatches, round-tripping each grid field
// through memory (src/mgpu/plan.ts:287-478, src/mgpu/wgsl.ts:321-372).  Here
// a function is cut into phases:
//   LegSynth   the Legendre synthesis of every spectral value the phase reads
//   Phase      one generated kernel per latitude block: synthesis FFTs, the
//              phase's grid statements (the reaction) at every point, and the
//              analysis FFTs of the values passed to analys
//   LegAnalys  the Legendre analysis, with the spectral statements that
//              consume its results (the IMEX update) as its epilogue
//   SpecEW     spectral statements that depend on no analysis in flight
// Grid values stay on chip; only displayed fields and values a later phase
// reads are written out.  State outputs go to a second buffer per state and
// the two swap after the run (the feedback copies of plan.ts:256-281).
#include <nvrtc.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <set>
#include <sstream>

#include "kernel_sources.h"
#include "mlang.h"
#include "runtime.h"

#define TS_TC_FIELDS 64  // fields per tensor-core CTA (kernels/leg_tc.cuh)

using tsm::Dom;

namespace {

struct HostBuf {
  Dom dom;
  long count = 0;       // floats per instance
  bool shared = false;  // one copy for all instances (stride 0)
  bool state = false;
  float *cur = nullptr, *next = nullptr;
};

// where a value lives
struct Ref {
  enum K { None, Cur, Next, Plan } k = None;
  std::string host;
  int pbuf = -1;
};

struct Stage {
  enum Kind { SpecEW, LegSynth, Phase, LegAnalys } kind;
  std::string expr;  // kernel name expression (NVRTC)
  cudaKernel_t kern = nullptr;
  std::vector<Ref> in, out;
  int nsyn = 0, nana = 0;
  int lb = 0, F = 1, K = 1, W = 1, per_cta = 1;
  int threads = 0;    // phase: threads per CTA (two-phase FFT: P*R, lb = R rows)
  bool wimg = false;  // tensor-core plan: the phase writes the W image itself
  size_t smem = 0;
  // SpecEW: the variant that takes four consecutive coefficients per thread
  // (float4 loads and stores; used when every array and stride allows it)
  std::string expr_v4;
  cudaKernel_t kern_v4 = nullptr;
  std::string label;  // one line, for describe()
  std::string src;    // generated CUDA of this stage
};

struct Program {
  tsm::Function fn;
  std::vector<Stage> stages;
  std::vector<std::string> feedback;             // per output: state name or ""
  std::map<std::string, Ref> value_ref;           // readable values after a run
  std::map<std::string, std::string> lazy_views;  // view -> state it is synth() of
  std::vector<long> pcount;                       // plan buffer sizes (per instance)
  std::vector<float *> pbuf;
  std::set<std::string> swaps;                    // states this program recomputes
  int nsyn_max = 0, nana_max = 0;
};

long dom_count(Dom d, ts_plan p) {
  return d == Dom::Grid ? (long)p->nlat * p->nphi : 2 * p->nlm;
}

// ------------------------------------------------------------- code emitters

std::string flit(double v) {
  if (!std::isfinite(v)) throw tsm::CompileError{"cannot emit a non-finite literal"};
  const float f = (float)v;
  if (!std::isfinite(f)) throw tsm::CompileError{"literal out of float range"};
  char buf[64];
  snprintf(buf, sizeof buf, "%.9g", (double)f);
  std::string s = buf;
  if (s.find_first_of(".en") == std::string::npos) s += ".0";
  return s + "f";
}

const std::map<std::string, std::string> kCudaFn = {
    {"abs", "fabsf"},   {"acos", "acosf"},   {"asin", "asinf"}, {"atan", "atanf"},
    {"atan2", "atan2f"}, {"ceil", "ceilf"},  {"cos", "cosf"},   {"cosh", "coshf"},
    {"exp", "expf"},    {"floor", "floorf"}, {"log", "logf"},   {"log2", "log2f"},
    {"max", "fmaxf"},   {"min", "fminf"},    {"round", "rintf"}, {"sign", "ts_sign"},
    {"sin", "sinf"},    {"sinh", "sinhf"},   {"sqrt", "sqrtf"}, {"tan", "tanf"},
    {"tanh", "tanhf"}, {"__ge_sel", "ts_ge_sel"}};

struct Emitter {
  const tsm::Function &f;
  std::map<int, std::string> name;  // var id -> C expression

  std::string e(const tsm::ExprP &x) {
    switch (x->kind) {
      case tsm::Expr::Lit: return flit(x->value);
      case tsm::Expr::Fill: return flit(x->value);
      case tsm::Expr::Param: return "prm[" + std::to_string(x->index) + "]";
      case tsm::Expr::Scalar: return "s" + std::to_string(x->index);
      case tsm::Expr::Var: {
        auto it = name.find(x->index);
        if (it == name.end())
          throw tsm::CompileError{"internal: value '" + f.vars[x->index].name + "' not bound"};
        return it->second;
      }
      case tsm::Expr::Binary: return "(" + e(x->args[0]) + " " + x->op + " " + e(x->args[1]) + ")";
      case tsm::Expr::Unary: return "(-" + e(x->args[0]) + ")";
      case tsm::Expr::PowI: {
        const int k = x->k < 0 ? -x->k : x->k;
        const std::string b = "ts_pow_i" + std::to_string(k) + "(" + e(x->args[0]) + ")";
        return x->k < 0 ? "(1.0f / " + b + ")" : b;
      }
      case tsm::Expr::Call: {
        std::string s = kCudaFn.at(x->fn) + "(";
        for (size_t i = 0; i < x->args.size(); i++) s += (i ? ", " : "") + e(x->args[i]);
        return s + ")";
      }
    }
    return "0.0f";
  }

  // derived scalars, in definition order (they only read params and earlier scalars)
  std::string scalars() {
    std::string s;
    for (size_t i = 0; i < f.scalars.size(); i++)
      s += "  const float s" + std::to_string(i) + " = " + e(f.scalars[i].expr) + ";\n";
    return s;
  }
};

void collect_vars(const tsm::ExprP &x, std::set<int> &out) {
  if (x->kind == tsm::Expr::Var) out.insert(x->index);
  for (auto &a : x->args) collect_vars(a, out);
}

std::vector<int> stmt_inputs(const tsm::Stmt &s) {
  if (s.kind != tsm::Stmt::Elementwise) return {s.arg};
  std::set<int> v;
  collect_vars(s.expr, v);
  return std::vector<int>(v.begin(), v.end());
}

}  // namespace

// The step's adjoint: per statement of `step` a generated forward ("tape")
// and reverse kernel (element-wise statements) or the transform adjoints
// (synth / analys); every value of the step has a tape buffer and, unless it
// is a constant (lam, noise), a cotangent buffer, [instance][count].
struct AdjStmt {
  int stmt = -1;
  std::string fwd_name, rev_name;
  cudaKernel_t fwd = nullptr, rev = nullptr;
  std::vector<int> in;       // value inputs, in the order of TsAdjIO::in
  std::vector<int> dvars;    // inputs that receive cotangents (TsAdjIO::gin)
};
struct Adjoint {
  bool ready = false;
  cudaLibrary_t lib = nullptr;
  std::vector<AdjStmt> st;
  std::vector<float *> val, bar;  // per value of the step function
  std::vector<long> count;        // floats per instance
  std::vector<long> stride;       // per-instance stride of val (0 = shared)
  std::vector<bool> constant;     // no cotangent (lam, noise)
  std::vector<int> state_in, state_out;
  double *pbar = nullptr;         // [instance][nparams]
  float *tmp = nullptr;           // transform-adjoint output
  std::vector<float *> owned;
};

struct ts_model_s {
  ts_ctx ctx = nullptr;
  ts_plan plan = nullptr;
  int batch = 1;
  std::vector<std::string> state, view, params;
  std::map<std::string, HostBuf> host;
  Program prog[2];  // init, step
  float *d_prm = nullptr;
  std::vector<float> h_prm;
  ts_dbuf fm, gm, stash, qimg, wimg;
  cudaLibrary_t lib = nullptr;
  int last_ran = 0, stashed_ran = 0;
  std::string source;
  std::vector<float *> owned;
  // step graphs: one or two steps captured on the context stream, keyed by
  // the state buffers they were captured with (the ping-pong parity)
  struct StepGraph {
    std::vector<float *> key;
    int nsteps;
    cudaGraphExec_t exec;
  };
  std::vector<StepGraph> graphs;
  bool use_graphs = true;
  int eager_left = 2;  // steps run eagerly first: every lazily grown buffer exists after them
  Adjoint adj;
};

namespace {

// ------------------------------------------------------------------ scheduler

void schedule(ts_model m, Program &P, bool is_step) {
  const tsm::Function &f = P.fn;
  ts_plan p = m->plan;
  const int nv = (int)f.vars.size();
  std::vector<Ref> ref(nv);
  std::vector<bool> avail(nv, false);
  // consumers of every var (statement indices), and whether it is an output
  std::vector<std::vector<int>> users(nv);
  for (size_t i = 0; i < f.body.size(); i++)
    for (int v : stmt_inputs(f.body[i])) users[v].push_back((int)i);
  std::vector<int> output_of(nv, -1);
  for (size_t o = 0; o < f.output_vars.size(); o++) output_of[f.output_vars[o]] = (int)o;

  for (int v = 0; v < nv; v++)
    if (f.vars[v].param_index >= 0) {
      ref[v] = Ref{Ref::Cur, f.vars[v].name, -1};
      avail[v] = true;
    }
  // outputs that feed a state go to that state's second buffer
  P.feedback.assign(f.output_vars.size(), "");
  for (size_t o = 0; o < f.output_vars.size() && o < m->state.size(); o++) {
    const int v = f.output_vars[o];
    const std::string &st = m->state[o];
    P.feedback[o] = st;
    if (f.vars[v].dom != Dom::Spec)
      throw tsm::CompileError{"'" + f.output_names[o] + "' is a grid field and cannot feed the "
                              "spectral state '" + st + "'", -1, -1, f.name};
    if (f.vars[v].param_index >= 0) {
      if (f.vars[v].name != st)
        throw tsm::CompileError{"output '" + f.output_names[o] + "' passes an argument through "
                                "to state '" + st + "'; assign it instead", -1, -1, f.name};
      continue;  // identity feedback: the state is unchanged
    }
    ref[v] = Ref{Ref::Next, st, -1};
    P.swaps.insert(st);
  }
  // lazily evaluated views: v = synth(S) of a state input S that this
  // program advances.  The step may use v itself (a reaction term); the
  // displayed field is only computed when it is read, from the state the
  // last step started from (the second buffer of S's pair)
  std::set<int> lazy;
  if (is_step) {
    for (size_t o = m->state.size(); o < f.output_vars.size(); o++) {
      const int v = f.output_vars[o];
      for (const auto &s : f.body)
        if (s.kind == tsm::Stmt::Synth && s.out == v && f.vars[s.arg].param_index >= 0) {
          const std::string &src = f.vars[s.arg].name;
          bool is_state = std::find(m->state.begin(), m->state.end(), src) != m->state.end();
          if (is_state) {
            lazy.insert(v);
            P.lazy_views[f.output_names[o]] = src;
          }
        }
    }
  }
  auto plan_buf = [&](int v) {
    P.pcount.push_back(dom_count(f.vars[v].dom, p));
    return Ref{Ref::Plan, "", (int)P.pcount.size() - 1};
  };
  auto materialize = [&](int v) {
    if (ref[v].k == Ref::None) ref[v] = plan_buf(v);
  };

  std::vector<bool> done(f.body.size(), false);
  auto all_done = [&]() { return std::all_of(done.begin(), done.end(), [](bool b) { return b; }); };
  int tag = 0;
  const std::string ptag = is_step ? "s" : "i";
  while (!all_done()) {
    bool progress = false;
    // (A) spectral statements ready now
    {
      std::vector<int> grp;
      std::set<int> local;
      for (size_t i = 0; i < f.body.size(); i++) {
        const auto &s = f.body[i];
        if (done[i] || s.kind != tsm::Stmt::Elementwise || f.vars[s.out].dom != Dom::Spec) continue;
        bool ok = true;
        for (int v : stmt_inputs(s)) ok = ok && (avail[v] || local.count(v));
        if (ok) {
          grp.push_back((int)i);
          local.insert(s.out);
        }
      }
      if (!grp.empty()) {
        Stage st;
        st.kind = Stage::SpecEW;
        std::set<int> ins;
        for (int i : grp)
          for (int v : stmt_inputs(f.body[i]))
            if (!local.count(v)) ins.insert(v);
        for (int v : ins) st.in.push_back(ref[v]);
        std::set<int> grp_set(grp.begin(), grp.end());
        std::vector<int> outs;
        for (int i : grp) {
          const int v = f.body[i].out;
          bool needed = output_of[v] >= 0;
          for (int u : users[v]) needed = needed || !grp_set.count(u);
          if (needed) {
            materialize(v);
            outs.push_back(v);
            st.out.push_back(ref[v]);
          }
          done[i] = true;
        }
        for (int v : outs) avail[v] = true;
        // generated kernel
        Emitter em{f, {}};
        const std::string kn = "ts_specew_" + ptag + std::to_string(tag++);
        std::ostringstream src;
        src << "extern \"C\" __global__ void __launch_bounds__(256) " << kn
            << "(TsSpecIO io) {\n"
            << "  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;\n"
            << "  if (idx >= io.n) return;\n  const long inst = blockIdx.y;\n"
            << "  const float *prm = io.prm + inst * io.nprm;\n"
            << em.scalars();
        int k = 0;
        for (int v : ins) {
          em.name[v] = "v" + std::to_string(v);
          src << "  const float v" << v << " = io.sin[" << k << "][inst * io.sin_stride[" << k
              << "] + idx];\n";
          k++;
        }
        for (int i : grp) {
          const auto &s = f.body[i];
          src << "  const float v" << s.out << " = " << em.e(s.expr) << ";  // "
              << f.vars[s.out].name << "\n";
          em.name[s.out] = "v" + std::to_string(s.out);
        }
        for (size_t o = 0; o < outs.size(); o++)
          src << "  io.sout[" << o << "][inst * io.sout_stride[" << o << "] + idx] = v" << outs[o]
              << ";\n";
        src << "}\n";
        // the same statements on four consecutive coefficients per thread
        {
          Emitter ev{f, {}};
          src << "extern \"C\" __global__ void __launch_bounds__(256) " << kn << "_v4"
              << "(TsSpecIO io) {\n"
              << "  const long i4 = ((long)blockIdx.x * blockDim.x + threadIdx.x) * 4;\n"
              << "  if (i4 >= io.n) return;\n  const long inst = blockIdx.y;\n"
              << "  const float *prm = io.prm + inst * io.nprm;\n"
              << ev.scalars();
          int kk = 0;
          for (int v : ins) {
            src << "  const float4 x" << kk << " = *reinterpret_cast<const float4 *>(io.sin[" << kk
                << "] + inst * io.sin_stride[" << kk << "] + i4);\n";
            src << "  const float a" << kk << "[4] = {x" << kk << ".x, x" << kk << ".y, x" << kk
                << ".z, x" << kk << ".w};\n";
            kk++;
          }
          for (size_t o = 0; o < outs.size(); o++) src << "  float r" << o << "[4];\n";
          src << "#pragma unroll\n  for (int u = 0; u < 4; u++) {\n";
          kk = 0;
          for (int v : ins) {
            ev.name[v] = "v" + std::to_string(v);
            src << "    const float v" << v << " = a" << kk << "[u];\n";
            kk++;
          }
          for (int i : grp) {
            const auto &s2 = f.body[i];
            src << "    const float v" << s2.out << " = " << ev.e(s2.expr) << ";\n";
            ev.name[s2.out] = "v" + std::to_string(s2.out);
          }
          for (size_t o = 0; o < outs.size(); o++)
            src << "    r" << o << "[u] = v" << outs[o] << ";\n";
          src << "  }\n";
          for (size_t o = 0; o < outs.size(); o++)
            src << "  *reinterpret_cast<float4 *>(io.sout[" << o << "] + inst * io.sout_stride[" << o
                << "] + i4) = make_float4(r" << o << "[0], r" << o << "[1], r" << o << "[2], r" << o
                << "[3]);\n";
          src << "}\n";
          st.expr_v4 = kn + "_v4";
        }
        st.expr = kn;
        st.label = "kernel  " + std::to_string(grp.size()) + " spectral statement(s)";
        st.src = src.str();
        P.stages.push_back(st);
        progress = true;
        continue;
      }
    }
    // (B) a grid phase
    std::vector<int> S, G, A;
    std::set<int> local;
    for (size_t i = 0; i < f.body.size(); i++) {
      const auto &s = f.body[i];
      if (!done[i] && s.kind == tsm::Stmt::Synth && avail[s.arg]) {
        S.push_back((int)i);
        local.insert(s.out);
      }
    }
    for (size_t i = 0; i < f.body.size(); i++) {
      const auto &s = f.body[i];
      if (done[i] || s.kind != tsm::Stmt::Elementwise || f.vars[s.out].dom != Dom::Grid) continue;
      bool ok = true;
      for (int v : stmt_inputs(s)) ok = ok && (avail[v] || local.count(v));
      if (ok) {
        G.push_back((int)i);
        local.insert(s.out);
      }
    }
    for (size_t i = 0; i < f.body.size(); i++) {
      const auto &s = f.body[i];
      if (!done[i] && s.kind == tsm::Stmt::Analys && (avail[s.arg] || local.count(s.arg)))
        A.push_back((int)i);
    }
    if (S.empty() && G.empty() && A.empty()) {
      if (!progress)
        throw tsm::CompileError{"internal: statements could not be scheduled", -1, -1, f.name};
      continue;
    }
    std::set<int> phase(S.begin(), S.end());
    phase.insert(G.begin(), G.end());
    phase.insert(A.begin(), A.end());
    // grid inputs already in buffers
    std::set<int> gin;
    for (int i : G)
      for (int v : stmt_inputs(f.body[i]))
        if (!local.count(v)) gin.insert(v);
    for (int i : A)
      if (!local.count(f.body[i].arg)) gin.insert(f.body[i].arg);
    // grid values computed here that must reach memory
    std::vector<int> gout;
    for (int v : local) {
      if (lazy.count(v)) continue;
      bool needed = output_of[v] >= 0;
      for (int u : users[v]) needed = needed || !phase.count(u);
      if (needed) {
        materialize(v);
        gout.push_back(v);
      }
    }
    if ((int)gin.size() > TS_MAXIO || (int)gout.size() > TS_MAXIO || (int)S.size() > TS_MAXIO)
      throw tsm::CompileError{"too many grid fields in one phase (limit 8)", -1, -1, f.name};
    if (!S.empty()) {
      Stage st;
      st.kind = Stage::LegSynth;
      for (int i : S) st.in.push_back(ref[f.body[i].arg]);
      st.nsyn = (int)S.size();
      st.label = "legsyn  " + std::to_string(S.size()) + " field(s)";
      P.stages.push_back(st);
    }
    {
      Stage st;
      st.kind = Stage::Phase;
      st.nsyn = (int)S.size();
      st.nana = (int)A.size();
      for (int v : gin) st.in.push_back(ref[v]);
      for (int v : gout) st.out.push_back(ref[v]);
      Emitter em{f, {}};
      const std::string pn = "TsProg_" + ptag + std::to_string(tag++);
      std::ostringstream src;
      src << "struct " << pn << " {\n  static constexpr int NSYN = " << S.size()
          << ", NGIN = " << gin.size() << ", NANA = " << A.size() << ", NGOUT = " << gout.size()
          << ";\n  static __device__ __forceinline__ void eval(const float *in, float *out, "
             "const float *prm) {\n"
          << em.scalars();
      for (size_t k = 0; k < S.size(); k++) {
        const int v = f.body[S[k]].out;
        src << "    const float v" << v << " = in[" << k << "];  // " << f.vars[v].name << "\n";
        em.name[v] = "v" + std::to_string(v);
      }
      int k = (int)S.size();
      for (int v : gin) {
        src << "    const float v" << v << " = in[" << k++ << "];  // " << f.vars[v].name << "\n";
        em.name[v] = "v" + std::to_string(v);
      }
      for (int i : G) {
        const auto &s = f.body[i];
        src << "    const float v" << s.out << " = " << em.e(s.expr) << ";  // "
            << f.vars[s.out].name << "\n";
        em.name[s.out] = "v" + std::to_string(s.out);
      }
      for (size_t a = 0; a < A.size(); a++)
        src << "    out[" << a << "] = " << em.name.at(f.body[A[a]].arg) << ";\n";
      for (size_t o = 0; o < gout.size(); o++)
        src << "    out[" << A.size() + o << "] = " << em.name.at(gout[o]) << ";\n";
      src << "  }\n};\n";
      // two-phase FFT when the row length has a shape and the row blocks fit
      int fP = 0, fQ = 0, fR = 0;
      const int nb = std::max<int>({(int)S.size(), (int)A.size(), 1});
      if (ts_f2_phase_shape(p, &fP, &fQ)) fR = ts_f2_phase_rows(p, nb, m->batch, &st.smem);
      const bool tcw = p->precision != TS_PREC_FP32 && fR && !A.empty();
      if (fR) {
        st.expr = "ts_f2_phase<" + pn + ", " + std::to_string(fP) + ", " + std::to_string(fQ) +
                  ", " + std::to_string(fR) + ", " + (tcw ? "true" : "false") + ">";
        st.lb = fR;
        st.threads = fP * fR;
      } else {
        st.expr = "ts_fourier_phase<" + pn + ">";
      }
      st.wimg = tcw;
      if (tcw) st.per_cta = (int)A.size() * (TS_TC_FIELDS / (int)A.size());
      st.label = "phase   " + std::to_string(S.size()) + " synth, " + std::to_string(G.size()) +
                 " grid statement(s), " + std::to_string(A.size()) + " analys";
      st.src = src.str();
      P.stages.push_back(st);
      P.nsyn_max = std::max(P.nsyn_max, (int)S.size());
      P.nana_max = std::max(P.nana_max, (int)A.size());
    }
    for (int i : phase) done[i] = true;
    for (int v : gout) avail[v] = true;
    if (A.empty()) continue;
    // (C) analysis with the spectral statements that consume it as epilogue
    std::set<int> aouts;
    for (int i : A) aouts.insert(f.body[i].out);
    std::vector<int> E;
    std::set<int> elocal = aouts;
    // On tensor-core plans each epilogue thread walks every instance of its
    // 64-field block for one coefficient; with many instances that loop of
    // dependent state loads is latency-bound, so the analysis only stores and
    // the spectral statements run as a coalesced element-wise stage (A).
    const bool fuse_epi = p->precision == TS_PREC_FP32 || m->batch * (long)A.size() <= 16;
    for (size_t i = 0; i < f.body.size() && fuse_epi; i++) {
      const auto &s = f.body[i];
      if (done[i] || s.kind != tsm::Stmt::Elementwise || f.vars[s.out].dom != Dom::Spec) continue;
      bool ok = true, uses_a = false;
      for (int v : stmt_inputs(s)) {
        ok = ok && (avail[v] || elocal.count(v));
        uses_a = uses_a || elocal.count(v);
      }
      if (ok && uses_a) {
        E.push_back((int)i);
        elocal.insert(s.out);
      }
    }
    std::set<int> eset(E.begin(), E.end());
    std::set<int> sin;
    for (int i : E)
      for (int v : stmt_inputs(f.body[i]))
        if (!elocal.count(v)) sin.insert(v);
    std::vector<int> sout;
    for (int v : elocal) {
      bool needed = output_of[v] >= 0;
      for (int u : users[v]) needed = needed || !eset.count(u);
      if (needed) {
        materialize(v);
        sout.push_back(v);
      }
    }
    if ((int)sin.size() > TS_MAXIO || (int)sout.size() > TS_MAXIO)
      throw tsm::CompileError{"too many spectral fields in one epilogue (limit 8)", -1, -1, f.name};
    Stage st;
    st.kind = Stage::LegAnalys;
    st.nana = (int)A.size();
    st.wimg = P.stages.back().kind == Stage::Phase && P.stages.back().wimg;
    for (int v : sin) st.in.push_back(ref[v]);
    for (int v : sout) st.out.push_back(ref[v]);
    const bool tc = p->precision != TS_PREC_FP32;
    if (tc) {
      st.per_cta = st.nana * (TS_TC_FIELDS / st.nana);  // whole instances per 64-field block
      if (st.per_cta == 0)
        throw tsm::CompileError{"too many analys outputs per instance for the tensor-core path",
                                -1, -1, f.name};
    } else {
      ts_analys_shape(p, m->batch * st.nana, st.nana, &st.F, &st.K, &st.W, &st.per_cta);
    }
    Emitter em{f, {}};
    const std::string en = "TsEpi_" + ptag + std::to_string(tag++);
    std::ostringstream src;
    // The state inputs of 8 instances are loaded before any of their stores:
    // the loads then overlap instead of each waiting out the previous store
    // (the restrict-qualified locals tell the compiler that they do not alias).
    const int NA = (int)A.size();
    src << "struct " << en << " {\n  TsSpecIO io;\n"
        << "  __device__ __forceinline__ void operator()(long lm, int comp, const float *vals, "
           "int f0, int nf, int F) const {\n"
        << "    const long idx = 2 * lm + comp;\n"
        << "    const int ni = nf / " << NA << ";\n";
    for (size_t k = 0; k < sin.size(); k++)
      src << "    const float *__restrict__ in" << k << " = io.sin[" << k << "];\n";
    for (size_t o = 0; o < sout.size(); o++)
      src << "    float *__restrict__ out" << o << " = io.sout[" << o << "];\n";
    src << "    for (int i0 = 0; i0 < ni; i0 += 8) {\n";
    for (size_t k = 0; k < sin.size(); k++) src << "      float ld" << k << "[8];\n";
    src << "#pragma unroll\n      for (int u = 0; u < 8; u++) {\n"
        << "        if (i0 + u >= ni) break;\n"
        << "        const long inst = f0 / " << NA << " + i0 + u;\n";
    for (size_t k = 0; k < sin.size(); k++)
      src << "        ld" << k << "[u] = in" << k << "[inst * io.sin_stride[" << k << "] + idx];\n";
    src << "      }\n#pragma unroll\n      for (int u = 0; u < 8; u++) {\n"
        << "        if (i0 + u >= ni) break;\n"
        << "        const int i = i0 + u;\n"
        << "        const long inst = f0 / " << NA << " + i;\n"
        << "        const float *__restrict__ prm = io.prm + inst * io.nprm;\n";
    {
      std::istringstream sc(em.scalars());
      std::string line;
      while (std::getline(sc, line)) src << "      " << line << "\n";
    }
    for (size_t a = 0; a < A.size(); a++) {
      const int v = f.body[A[a]].out;
      src << "        const float v" << v << " = vals[i * " << NA << " + " << a << "];  // "
          << f.vars[v].name << "\n";
      em.name[v] = "v" + std::to_string(v);
    }
    int k = 0;
    for (int v : sin) {
      src << "        const float v" << v << " = ld" << k << "[u];  // " << f.vars[v].name << "\n";
      em.name[v] = "v" + std::to_string(v);
      k++;
    }
    for (int i : E) {
      const auto &s = f.body[i];
      src << "        const float v" << s.out << " = " << em.e(s.expr) << ";  // "
          << f.vars[s.out].name << "\n";
      em.name[s.out] = "v" + std::to_string(s.out);
    }
    for (size_t o = 0; o < sout.size(); o++)
      src << "        out" << o << "[inst * io.sout_stride[" << o << "] + idx] = v" << sout[o]
          << ";\n";
    src << "      }\n    }\n  }\n};\n";
    st.expr = tc ? "ts_leg_analys_tc<" + en + ">"
                 : "ts_leg_analys_f32<" + std::to_string(st.F) + ", " + std::to_string(st.K) +
                       ", 2, " + en + ">";
    st.label = "legana  " + std::to_string(A.size()) + " field(s), " + std::to_string(E.size()) +
               " spectral statement(s) fused";
    st.src = src.str();
    P.stages.push_back(st);
    for (int i : E) done[i] = true;
    for (int v : sout) avail[v] = true;
  }
  for (int o = 0; o < (int)f.output_vars.size(); o++) {
    const int v = f.output_vars[o];
    if (lazy.count(v)) continue;
    if (ref[v].k == Ref::None) materialize(v);
    P.value_ref[f.output_names[o]] = ref[v];
  }
  // every named (non-temporary) value that reached memory is readable
  for (int v = 0; v < nv; v++)
    if (!f.vars[v].temp && ref[v].k != Ref::None && !P.value_ref.count(f.vars[v].name))
      P.value_ref[f.vars[v].name] = ref[v];
  // reads happen after the run, when each state's second buffer has been
  // swapped in: a value written to `next` is then in `cur`
  for (auto &kv : P.value_ref)
    if (kv.second.k == Ref::Next) kv.second.k = Ref::Cur;
}

std::string stage_source(const Stage &s) { return s.src; }
std::string stage_title(const Stage &s) { return s.label; }

// --------------------------------------------------------------------- NVRTC

// NVRTC: the generated stages plus the kernel headers -> an sm_100a cubin,
// and the lowered name of every template instantiation.
std::vector<char> nvrtc_cubin(const std::string &code, const std::vector<std::string> &exprs,
                              std::map<std::string, std::string> &lowered);

std::vector<char> build_cubin(ts_model m, std::map<std::string, std::string> &lowered) {
  std::ostringstream src;
  src << "#include \"ts_common.cuh\"\n#include \"fft2.cuh\"\n#include \"fourier.cuh\"\n#include \"leg_f32.cuh\"\n"
      << "#include \"leg_tc.cuh\"\n";
  for (auto &P : m->prog)
    for (auto &s : P.stages) src << stage_source(s);
  std::vector<std::string> exprs;
  for (auto &P : m->prog)
    for (auto &s : P.stages)
      if (!s.expr.empty() && s.expr.find('<') != std::string::npos) exprs.push_back(s.expr);
  return nvrtc_cubin(src.str(), exprs, lowered);
}

// NVRTC: source (with the embedded kernel headers) -> an sm_100a cubin, and
// the lowered name of every template-instantiation expression
std::vector<char> nvrtc_cubin(const std::string &code, const std::vector<std::string> &exprs,
                              std::map<std::string, std::string> &lowered) {
  nvrtcProgram prog;
  auto nv = [&](nvrtcResult r, const char *what) {
    if (r != NVRTC_SUCCESS)
      ts_throw(TS_ERR_COMPILE, std::string(what) + ": " + nvrtcGetErrorString(r));
  };
  nv(nvrtcCreateProgram(&prog, code.c_str(), "model.cu", ts_src_count, ts_src_texts, ts_src_names),
     "nvrtcCreateProgram");
  for (auto &e : exprs) nv(nvrtcAddNameExpression(prog, e.c_str()), "nvrtcAddNameExpression");
  const char *opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "-lineinfo",
                        "--device-as-default-execution-space"};
  const nvrtcResult rc = nvrtcCompileProgram(prog, 4, opts);
  if (rc != NVRTC_SUCCESS) {
    size_t n = 0;
    nvrtcGetProgramLogSize(prog, &n);
    std::string log(n, '\0');
    nvrtcGetProgramLog(prog, &log[0]);
    nvrtcDestroyProgram(&prog);
    ts_throw(TS_ERR_COMPILE, "generated CUDA failed to compile:\n" + log + "\n--- source ---\n" + code);
  }
  size_t n = 0;
  nv(nvrtcGetCUBINSize(prog, &n), "nvrtcGetCUBINSize");
  std::vector<char> cubin(n);
  nv(nvrtcGetCUBIN(prog, cubin.data()), "nvrtcGetCUBIN");
  for (auto &e : exprs) {
    const char *ln = nullptr;
    nv(nvrtcGetLoweredName(prog, e.c_str(), &ln), "nvrtcGetLoweredName");
    lowered[e] = ln;
  }
  nvrtcDestroyProgram(&prog);
  return cubin;
}

void compile_kernels(ts_model m) {
  std::map<std::string, std::string> lowered;
  const std::vector<char> cubin = build_cubin(m, lowered);
  TS_CUDA(cudaLibraryLoadData(&m->lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
  for (auto &P : m->prog)
    for (auto &s : P.stages) {
      if (s.expr.empty()) continue;
      const std::string name = lowered.count(s.expr) ? lowered[s.expr] : s.expr;
      TS_CUDA(cudaLibraryGetKernel(&s.kern, m->lib, name.c_str()));
      if (!s.expr_v4.empty()) TS_CUDA(cudaLibraryGetKernel(&s.kern_v4, m->lib, s.expr_v4.c_str()));
      if (s.smem > 48 * 1024)
        TS_CUDA(cudaKernelSetAttributeForDevice(
            s.kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s.smem, m->ctx->device));
    }
}

// ------------------------------------------------------------------- runtime

float *resolve(ts_model m, Program &P, const Ref &r, long *stride) {
  if (r.k == Ref::Plan) {
    *stride = P.pcount[r.pbuf];
    return P.pbuf[r.pbuf];
  }
  HostBuf &h = m->host.at(r.host);
  *stride = h.shared ? 0 : h.count;
  return r.k == Ref::Next ? h.next : h.cur;
}

void fill_spec_io(ts_model m, Program &P, const Stage &s, TsSpecIO &io) {
  memset(&io, 0, sizeof io);
  for (size_t i = 0; i < s.in.size(); i++) io.sin[i] = resolve(m, P, s.in[i], &io.sin_stride[i]);
  for (size_t i = 0; i < s.out.size(); i++) io.sout[i] = resolve(m, P, s.out[i], &io.sout_stride[i]);
  io.prm = m->d_prm;
  io.nprm = (int)m->params.size();
  io.n = 2 * m->plan->nlm;
}

void run_program(ts_model m, Program &P, cudaStream_t st) {
  ts_plan p = m->plan;
  const long field = (long)(p->mmax + 1) * p->nlat;
  float2 *fm = (float2 *)m->fm.p, *gm = (float2 *)m->gm.p;
  const int B = m->batch;
  for (auto &s : P.stages) {
    switch (s.kind) {
      case Stage::LegSynth: {
        TsFields q{};
        for (size_t i = 0; i < s.in.size(); i++) {
          long stride;
          q.base[i] = (const float2 *)resolve(m, P, s.in[i], &stride);
          q.inst_stride[i] = stride / 2;
        }
        q.nper = s.nsyn;
        if (p->precision != TS_PREC_FP32)
          ts_launch_leg_synth_tc(p, q, fm, field, B * s.nsyn, st, &m->qimg);
        else
          ts_launch_leg_synth_fields(p, q, fm, field, B * s.nsyn, st);
        break;
      }
      case Stage::Phase: {
        TsPhaseIO io;
        memset(&io, 0, sizeof io);
        io.fm = fm;
        io.gm = gm;
        io.field = field;
        for (size_t i = 0; i < s.in.size(); i++) io.gin[i] = resolve(m, P, s.in[i], &io.gin_stride[i]);
        for (size_t i = 0; i < s.out.size(); i++)
          io.gout[i] = resolve(m, P, s.out[i], &io.gout_stride[i]);
        io.prm = m->d_prm;
        io.nprm = (int)m->params.size();
        io.nh = p->nh;
        if (s.wimg) {
          io.wimg = (char *)m->wimg.p;
          io.w_fpb = s.per_cta;
          io.w_nfb = (B * s.nana + s.per_cta - 1) / s.per_cta;
          io.w_nlc = (p->nh + 31) / 32;
          io.wq = p->d_wq;
          io.w_kmin = ts_tc_w_kmin(p);
        }
        TsFftTab ft = p->fft;
        void *args[] = {&ft, &io};
        if (s.threads) {  // two-phase FFT: R rows (R/2 latitude pairs) per CTA
          const int per = s.wimg ? s.lb / 2 : s.lb;
          dim3 grid(((s.wimg ? p->nh : p->nlat) + per - 1) / per, B);
          TS_CUDA(cudaLaunchKernel((const void *)s.kern, grid, dim3(s.threads), args, s.smem, st));
        } else {
          dim3 grid((p->nlat + s.lb - 1) / s.lb, B);
          TS_CUDA(cudaLaunchKernel((const void *)s.kern, grid, dim3(32 * s.lb), args, s.smem, st));
        }
        break;
      }
      case Stage::LegAnalys: {
        // the epilogue functor is a TsSpecIO (first and only member)
        TsSpecIO epi;
        fill_spec_io(m, P, s, epi);
        TsLegTab leg = p->leg;
        const float2 *g = gm;
        long gs = field;
        int nfields = B * s.nana;
        int per_cta = s.per_cta;
        if (p->precision != TS_PREC_FP32) {
          TsTcTab tc = ts_tc_tab(p);
          int S = ts_tc_analys_stages(p);
          int nmax = ts_tc_analys_nmax(p);
          int ntile = ts_tc_ntile(p);
          int w_nfb = (nfields + per_cta - 1) / per_cta;
          if (!s.wimg)  // the phase wrote G: fold it into the W image first
            ts_launch_wimage(p, gm, field, nfields, per_cta, (char *)m->wimg.p, st);
          const char *wimg = (const char *)m->wimg.p;
          void *args[] = {&leg, &tc, &wimg, &w_nfb, &epi, &nfields, &per_cta, &S, &nmax, &ntile};
          const int ctas = ts_tc_ctas(p, (long)(p->mmax + 1) * 2 * ntile * w_nfb);
          TS_CUDA(cudaLaunchKernel((const void *)s.kern, dim3(ctas), dim3(TS_TC_THREADS), args, s.smem, st));
        } else {
          const int nfb = (nfields + per_cta - 1) / per_cta;
          int lchunk = ts_analys_lchunk(p, nfb);
          void *args[] = {&leg, &g, &gs, &epi, &nfields, &per_cta, &lchunk};
          dim3 grid(p->mmax + 1, nfb, lchunk ? (p->lmax + lchunk) / lchunk : 1);
          TS_CUDA(cudaLaunchKernel((const void *)s.kern, grid, dim3(32 * s.W), args, s.smem, st));
        }
        break;
      }
      case Stage::SpecEW: {
        TsSpecIO io;
        fill_spec_io(m, P, s, io);
        void *args[] = {&io};
        // four coefficients per thread when every array start and stride is
        // a multiple of four floats (16-byte loads and stores)
        bool v4 = s.kern_v4 && io.n % 4 == 0;
        for (size_t i = 0; i < s.in.size() && v4; i++)
          v4 = io.sin_stride[i] % 4 == 0 && (reinterpret_cast<uintptr_t>(io.sin[i]) & 15) == 0;
        for (size_t i = 0; i < s.out.size() && v4; i++)
          v4 = io.sout_stride[i] % 4 == 0 && (reinterpret_cast<uintptr_t>(io.sout[i]) & 15) == 0;
        if (v4) {
          dim3 grid((unsigned)((io.n / 4 + 255) / 256), B);
          TS_CUDA(cudaLaunchKernel((const void *)s.kern_v4, grid, dim3(256), args, 0, st));
        } else {
          dim3 grid((unsigned)((2 * p->nlm + 255) / 256), B);
          TS_CUDA(cudaLaunchKernel((const void *)s.kern, grid, dim3(256), args, 0, st));
        }
        break;
      }
    }
  }
  for (auto &name : P.swaps) {
    HostBuf &h = m->host.at(name);
    std::swap(h.cur, h.next);
  }
}

void finish_shapes(ts_model m) {
  ts_plan p = m->plan;
  for (auto &P : m->prog)
    for (auto &s : P.stages) {
      if (s.kind == Stage::Phase) {
        const int nrows = s.nsyn + s.nana + 1;
        if (!s.threads) s.lb = ts_fourier_lb(p, m->batch, nrows, &s.smem);
      } else if (s.kind == Stage::LegAnalys) {
        s.smem = p->precision != TS_PREC_FP32 ? ts_tc_analys_smem(p) : ts_analys_smem(p, s.F, s.W);
      }
    }
}

// ------------------------------------------------------------- step graphs

void drop_graphs(ts_model m) {
  for (auto &g : m->graphs) cudaGraphExecDestroy(g.exec);
  m->graphs.clear();
}

// Graphs need a stream that can be captured and is not being captured by
// the caller already (a caller's capture records the eager launches).
bool graphs_usable(ts_model m) {
  if (!m->use_graphs) return false;
  cudaStream_t st = m->ctx->stream;
  if (st == nullptr || st == cudaStreamLegacy || st == cudaStreamPerThread) return false;
  cudaStreamCaptureStatus cs;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) return false;
  return cs == cudaStreamCaptureStatusNone;
}

std::vector<float *> state_key(ts_model m) {
  std::vector<float *> k;
  for (auto &name : m->prog[1].swaps) k.push_back(m->host.at(name).cur);
  return k;
}

void swap_states(ts_model m, int nsteps) {
  for (int i = 0; i < nsteps; i++)
    for (auto &name : m->prog[1].swaps) {
      HostBuf &h = m->host.at(name);
      std::swap(h.cur, h.next);
    }
}

// nsteps steps as one graph launch; the graph for the current state
// buffers is captured on first use.  Any capture failure turns graphs off
// for the model and runs the steps eagerly.
void run_steps_graphed(ts_model m, int nsteps) {
  cudaStream_t st = m->ctx->stream;
  const std::vector<float *> key = state_key(m);
  for (auto &g : m->graphs)
    if (g.nsteps == nsteps && g.key == key) {
      TS_CUDA(cudaGraphLaunch(g.exec, st));
      swap_states(m, nsteps);
      return;
    }
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool ok = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  if (ok) {
    int ran = 0;
    try {
      for (; ran < nsteps; ran++) run_program(m, m->prog[1], st);
    } catch (const ts_exc &) {
      ok = false;
    }
    const bool ended = cudaStreamEndCapture(st, &graph) == cudaSuccess;
    ok = ok && ended && graph;
    if (!ok) swap_states(m, ran);  // undo the host-side swaps of the failed capture
  }
  if (ok) ok = cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
  if (graph) cudaGraphDestroy(graph);
  if (!ok) {
    (void)cudaGetLastError();
    m->use_graphs = false;
    drop_graphs(m);
    for (int i = 0; i < nsteps; i++) run_program(m, m->prog[1], st);
    return;
  }
  m->graphs.push_back({key, nsteps, exec});
  TS_CUDA(cudaGraphLaunch(exec, st));
}

float *dalloc(long n);

// ------------------------------------------------------------------- adjoint
//
// Reverse mode over the step function, statement by statement:
//   out = e(x..., params):  xbar += de/dx * outbar,  pbar += sum de/dp * outbar
//   out = synth(x):         xbar += S^T outbar = c * analys(outbar / w)
//   out = analys(x):        xbar += A^T outbar = w * synth(outbar / c)
// with the derivatives of e generated symbolically (mdiff.cpp).  The
// forward values come from an unfused replay of the step (the tape);
// forward_backward checkpoints the state every K steps and replays each
// segment from its checkpoint.

std::string adj_source(ts_model m) {
  Adjoint &A = m->adj;
  const tsm::Function &f = m->prog[1].fn;
  const int nprm = std::max<int>((int)m->params.size(), 1);
  std::ostringstream src;
  src << "#include \"ts_common.cuh\"\n";
  for (auto &as : A.st) {
    const tsm::Stmt &s = f.body[as.stmt];
    if (s.kind != tsm::Stmt::Elementwise) continue;
    Emitter em{f, {}};
    for (size_t k = 0; k < as.in.size(); k++) em.name[as.in[k]] = "x" + std::to_string(k);
    std::ostringstream loads;
    for (size_t k = 0; k < as.in.size(); k++)
      loads << "    const float x" << k << " = io.in[" << k << "][inst * io.in_stride[" << k
            << "] + idx];\n";
    // forward
    src << "extern \"C\" __global__ void __launch_bounds__(256) " << as.fwd_name
        << "(TsAdjIO io) {\n  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;\n"
        << "  if (idx >= io.n) return;\n  const long inst = blockIdx.y;\n"
        << "  const float *prm = io.prm + inst * io.nprm;\n  (void)prm;\n"
        << em.scalars() << loads.str()
        << "  io.out[inst * io.out_stride + idx] = " << em.e(s.expr) << ";\n}\n";
    // reverse
    std::vector<std::pair<int, std::string>> dp;  // parameter slot, derivative
    for (int j = 0; j < (int)m->params.size(); j++) {
      const tsm::ExprP d = tsm::differentiate(f, s.expr, tsm::Wrt{tsm::Wrt::Param, j});
      if (!tsm::is_zero(d)) dp.push_back({j, em.e(d)});
    }
    src << "extern \"C\" __global__ void __launch_bounds__(256) " << as.rev_name
        << "(TsAdjIO io) {\n  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;\n"
        << "  const bool live = idx < io.n;\n  const long inst = blockIdx.y;\n"
        << "  const float *prm = io.prm + inst * io.nprm;\n  (void)prm;\n" << em.scalars();
    if (!dp.empty()) src << "  float gp[" << dp.size() << "] = {};\n";
    src << "  if (live) {\n" << loads.str()
        << "    const float gb = io.gout[inst * io.gout_stride + idx];\n";
    for (size_t k = 0; k < as.dvars.size(); k++) {
      const tsm::ExprP d = tsm::differentiate(f, s.expr, tsm::Wrt{tsm::Wrt::Var, as.dvars[k]});
      src << "    io.gin[" << k << "][inst * io.gin_stride[" << k << "] + idx] += (" << em.e(d)
          << ") * gb;\n";
    }
    for (size_t j = 0; j < dp.size(); j++) src << "    gp[" << j << "] = (" << dp[j].second << ") * gb;\n";
    src << "  }\n";
    if (!dp.empty()) {
      src << "  __shared__ float red[8];\n"
          << "  for (int j = 0; j < " << dp.size() << "; j++) {\n"
          << "    float v = gp[j];\n"
          << "    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);\n"
          << "    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;\n"
          << "    __syncthreads();\n"
          << "    if (threadIdx.x == 0) {\n"
          << "      float t = 0.f;\n"
          << "      for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];\n"
          << "      const int slot[" << dp.size() << "] = {";
      for (size_t j = 0; j < dp.size(); j++) src << (j ? ", " : "") << dp[j].first;
      src << "};\n"
          << "      atomicAdd(io.pbar + inst * " << nprm << " + slot[j], (double)t);\n"
          << "    }\n    __syncthreads();\n  }\n";
    }
    src << "}\n";
  }
  return src.str();
}

float *adj_alloc(Adjoint &A, long n) {
  float *q = dalloc(std::max<long>(n, 1));
  A.owned.push_back(q);
  return q;
}

// the adjoint's statement list and value classes (no device work)
void adj_structure(ts_model m) {
  Adjoint &A = m->adj;
  const tsm::Function &f = m->prog[1].fn;
  ts_plan p = m->plan;
  const int nv = (int)f.vars.size();
  const long npts = (long)p->nlat * p->nphi, nspec = 2 * p->nlm;
  A.st.clear();
  A.val.assign(nv, nullptr);
  A.bar.assign(nv, nullptr);
  A.count.assign(nv, 0);
  A.stride.assign(nv, 0);
  A.constant.assign(nv, false);
  for (int v = 0; v < nv; v++) {
    const Dom d = f.vars[v].dom;
    if (d == Dom::Scalar) continue;
    A.count[v] = d == Dom::Grid ? npts : nspec;
    A.stride[v] = A.count[v];
    const int pi = f.vars[v].param_index;
    if (pi >= 0) {
      const std::string &name = f.param_names[pi];
      A.constant[v] = std::find(m->state.begin(), m->state.end(), name) == m->state.end();
    }
  }
  A.state_in.assign(m->state.size(), -1);
  A.state_out.assign(m->state.size(), -1);
  for (size_t s = 0; s < m->state.size(); s++) {
    for (size_t i = 0; i < f.param_names.size(); i++)
      if (f.param_names[i] == m->state[s]) A.state_in[s] = f.param_vars[i];
    if (s < f.output_vars.size()) A.state_out[s] = f.output_vars[s];
    TS_REQUIRE(A.state_in[s] >= 0 && A.state_out[s] >= 0, TS_ERR_UNSUPPORTED,
               "adjoint: step must take and return every state");
  }
  int tag = 0;
  for (size_t i = 0; i < f.body.size(); i++) {
    const tsm::Stmt &s = f.body[i];
    AdjStmt as;
    as.stmt = (int)i;
    if (s.kind == tsm::Stmt::Elementwise) {
      as.in = stmt_inputs(s);
      TS_REQUIRE(as.in.size() <= TS_MAXIO, TS_ERR_UNSUPPORTED,
                 "adjoint: more than 8 values in one statement");
      for (int v : as.in)
        if (!A.constant[v]) as.dvars.push_back(v);
      as.fwd_name = "ts_adj_f" + std::to_string(tag);
      as.rev_name = "ts_adj_r" + std::to_string(tag++);
    }
    A.st.push_back(as);
  }
}

// build (once) the adjoint program of the step function: buffers, kernels
void adj_prepare(ts_model m) {
  Adjoint &A = m->adj;
  if (A.ready) return;
  adj_structure(m);
  const tsm::Function &f = m->prog[1].fn;
  const int B = m->batch, nv = (int)f.vars.size();
  for (int v = 0; v < nv; v++) {
    if (A.count[v] == 0) continue;
    const int pi = f.vars[v].param_index;
    if (A.constant[v]) {  // lam, noise: host-owned
      HostBuf &h = m->host.at(f.param_names[pi]);
      A.val[v] = h.cur;
      A.stride[v] = h.shared ? 0 : h.count;
      continue;
    }
    if (pi < 0) A.val[v] = adj_alloc(A, A.count[v] * B);  // states: bound per replayed step
    A.bar[v] = adj_alloc(A, A.count[v] * B);
  }
  const long npts = (long)m->plan->nlat * m->plan->nphi, nspec = 2 * m->plan->nlm;
  A.tmp = adj_alloc(A, std::max(npts, nspec) * B);
  TS_CUDA(cudaMalloc(&A.pbar, sizeof(double) * std::max<size_t>(m->params.size(), 1) * B));
  std::map<std::string, std::string> lowered;
  const std::vector<char> cubin = nvrtc_cubin(adj_source(m), {}, lowered);
  TS_CUDA(cudaLibraryLoadData(&A.lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
  for (auto &as : A.st)
    if (!as.fwd_name.empty()) {
      TS_CUDA(cudaLibraryGetKernel(&as.fwd, A.lib, as.fwd_name.c_str()));
      TS_CUDA(cudaLibraryGetKernel(&as.rev, A.lib, as.rev_name.c_str()));
    }
  A.ready = true;
}

void adj_free(Adjoint &A) {
  for (float *q : A.owned) cudaFree(q);
  A.owned.clear();
  if (A.pbar) cudaFree(A.pbar);
  A.pbar = nullptr;
  if (A.lib) cudaLibraryUnload(A.lib);
  A.lib = nullptr;
  A.ready = false;
}

TsAdjIO adj_io(ts_model m, const AdjStmt &as) {
  Adjoint &A = m->adj;
  const tsm::Stmt &s = m->prog[1].fn.body[as.stmt];
  TsAdjIO io;
  memset(&io, 0, sizeof io);
  for (size_t k = 0; k < as.in.size(); k++) {
    io.in[k] = A.val[as.in[k]];
    io.in_stride[k] = A.stride[as.in[k]];
  }
  io.out = A.val[s.out];
  io.out_stride = A.stride[s.out];
  io.gout = A.bar[s.out];
  io.gout_stride = A.count[s.out];
  for (size_t k = 0; k < as.dvars.size(); k++) {
    io.gin[k] = A.bar[as.dvars[k]];
    io.gin_stride[k] = A.count[as.dvars[k]];
  }
  io.prm = m->d_prm;
  io.nprm = std::max<int>((int)m->params.size(), 1);
  io.pbar = A.pbar;
  io.n = A.count[s.out];
  return io;
}

__global__ void ts_k_axpy(float *y, const float *x, long n) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x, step = (long)gridDim.x * blockDim.x;
  if ((n & 3) == 0 && ((reinterpret_cast<unsigned long long>(y) |
                        reinterpret_cast<unsigned long long>(x)) & 15) == 0) {
    float4 *y4 = reinterpret_cast<float4 *>(y);
    const float4 *x4 = reinterpret_cast<const float4 *>(x);
    for (long i = t; i < (n >> 2); i += step) {
      float4 a = y4[i];
      const float4 b = x4[i];
      a.x += b.x;
      a.y += b.y;
      a.z += b.z;
      a.w += b.w;
      y4[i] = a;
    }
  } else {
    for (long i = t; i < n; i += step) y[i] += x[i];
  }
}

void axpy(float *y, const float *x, long n, cudaStream_t st) {
  const int blocks = (int)std::min<long>((n + 255) / 256, 148L * 8);
  ts_k_axpy<<<blocks, 256, 0, st>>>(y, x, n);
  TS_CUDA(cudaGetLastError());
}

// the step's values from the states at `states[s]` ([instance][2 nlm] each)
void adj_tape(ts_model m, const std::vector<const float *> &states, cudaStream_t st) {
  Adjoint &A = m->adj;
  const tsm::Function &f = m->prog[1].fn;
  const int B = m->batch;
  for (size_t s = 0; s < states.size(); s++) A.val[A.state_in[s]] = const_cast<float *>(states[s]);
  for (auto &as : A.st) {
    const tsm::Stmt &s = f.body[as.stmt];
    if (s.kind == tsm::Stmt::Elementwise) {
      TsAdjIO io = adj_io(m, as);
      void *args[] = {&io};
      dim3 grid((unsigned)((io.n + 255) / 256), B);
      TS_CUDA(cudaLaunchKernel((const void *)as.fwd, grid, dim3(256), args, 0, st));
    } else if (s.kind == tsm::Stmt::Synth) {
      ts_synth_dev(m->plan, A.val[s.arg], A.val[s.out], B, st);
    } else {
      ts_analys_dev(m->plan, A.val[s.arg], A.val[s.out], B, st);
    }
  }
}

// one reverse step: lam[s] (cotangent of the step's output state s) in,
// cotangent of its input state s out (in place); parameter gradients add up
void adj_reverse(ts_model m, const std::vector<float *> &lam, cudaStream_t st) {
  Adjoint &A = m->adj;
  const tsm::Function &f = m->prog[1].fn;
  const int B = m->batch;
  for (size_t v = 0; v < A.bar.size(); v++)
    if (A.bar[v]) TS_CUDA(cudaMemsetAsync(A.bar[v], 0, sizeof(float) * A.count[v] * B, st));
  for (size_t s = 0; s < lam.size(); s++) axpy(A.bar[A.state_out[s]], lam[s], A.count[A.state_out[s]] * B, st);
  for (auto it = A.st.rbegin(); it != A.st.rend(); ++it) {
    const tsm::Stmt &s = f.body[it->stmt];
    if (s.kind == tsm::Stmt::Elementwise) {
      if (it->dvars.empty() && m->params.empty()) continue;
      TsAdjIO io = adj_io(m, *it);
      void *args[] = {&io};
      dim3 grid((unsigned)((io.n + 255) / 256), B);
      TS_CUDA(cudaLaunchKernel((const void *)it->rev, grid, dim3(256), args, 0, st));
    } else if (!A.constant[s.arg]) {
      if (s.kind == tsm::Stmt::Synth)
        ts_synth_adjoint(m->plan, A.bar[s.out], A.tmp, B, st);
      else
        ts_analys_adjoint(m->plan, A.bar[s.out], A.tmp, B, st);
      axpy(A.bar[s.arg], A.tmp, A.count[s.arg] * B, st);
    }
  }
  for (size_t s = 0; s < lam.size(); s++)
    TS_CUDA(cudaMemcpyAsync(lam[s], A.bar[A.state_in[s]], sizeof(float) * A.count[A.state_in[s]] * B,
                            cudaMemcpyDeviceToDevice, st));
}

void free_model(ts_model m) {
  adj_free(m->adj);
  drop_graphs(m);
  for (auto &kv : m->host) {
    if (kv.second.cur) cudaFree(kv.second.cur);
    if (kv.second.next) cudaFree(kv.second.next);
  }
  for (auto &P : m->prog)
    for (float *b : P.pbuf)
      if (b) cudaFree(b);
  if (m->d_prm) cudaFree(m->d_prm);
  m->fm.release();
  m->gm.release();
  m->stash.release();
  m->qimg.release();
  m->wimg.release();
  if (m->lib) cudaLibraryUnload(m->lib);
}

// device memory released at scope exit
struct DevMem {
  void *p = nullptr;
  explicit DevMem(size_t bytes) { TS_CUDA(cudaMalloc(&p, std::max<size_t>(bytes, 16))); }
  ~DevMem() {
    if (p) cudaFree(p);
  }
  DevMem(const DevMem &) = delete;
  DevMem &operator=(const DevMem &) = delete;
};

float *dalloc(long n) {
  float *p = nullptr;
  TS_CUDA(cudaMalloc(&p, sizeof(float) * std::max<long>(n, 1)));
  TS_CUDA(cudaMemset(p, 0, sizeof(float) * std::max<long>(n, 1)));
  return p;
}

void check_finite_params(std::vector<float> &v) {
  for (float &x : v)
    if (!std::isfinite(x)) x = 0.0f;  // plan.ts:414-416: non-finite values become 0
}

// Laplace-Beltrami eigenvalues l(l+1), duplicated over re/im (model.ts:46-56)
std::vector<float> eigenvalues(ts_plan p) {
  std::vector<float> lam(2 * p->nlm);
  for (int mm = 0; mm <= p->mmax; mm++)
    for (int l = mm; l <= p->lmax; l++) {
      const long i = ts_lm_index(p->lmax, l, mm);
      lam[2 * i] = lam[2 * i + 1] = (float)l * (l + 1);
    }
  return lam;
}

// which program's buffer holds `name` now (GpuModel.#locate, model.ts:243-252)
bool locate(ts_model m, const std::string &name, float **ptr, long *count, long *stride,
            std::string *lazy_state) {
  const int first = m->last_ran, second = 1 - m->last_ran;
  for (int which : {first, second}) {
    Program &P = m->prog[which];
    auto lz = P.lazy_views.find(name);
    if (lz != P.lazy_views.end()) {
      *lazy_state = lz->second;
      *ptr = nullptr;
      *count = (long)m->plan->nlat * m->plan->nphi;
      *stride = *count;
      return true;
    }
    auto it = P.value_ref.find(name);
    if (it != P.value_ref.end()) {
      *ptr = resolve(m, P, it->second, stride);
      *count = it->second.k == Ref::Plan ? P.pcount[it->second.pbuf]
                                          : m->host.at(it->second.host).count;
      lazy_state->clear();
      return true;
    }
  }
  auto h = m->host.find(name);
  if (h != m->host.end()) {
    *ptr = h->second.cur;
    *count = h->second.count;
    *stride = h->second.shared ? 0 : h->second.count;
    lazy_state->clear();
    return true;
  }
  return false;
}

// parse, specialise init/step and schedule them; fills `err` on rejection
void front_end(ts_model m, int nstate, int nview, ts_compile_error *err) {
  ts_plan plan = m->plan;
  const long npts = (long)plan->nlat * plan->nphi, nlm = plan->nlm;
  // the bindings a .m may name (model.ts:116-125)
  std::map<std::string, tsm::Binding> b;
  b["lam"] = {tsm::Binding::Tensor, Dom::Spec, 0};
  b["noise"] = {tsm::Binding::Tensor, Dom::Grid, 0};
  b["npts"] = {tsm::Binding::Const, Dom::Scalar, (double)npts};
  b["nlm"] = {tsm::Binding::Const, Dom::Scalar, (double)nlm};
  for (auto &s : m->state) b[s] = {tsm::Binding::Tensor, Dom::Spec, 0};
  for (auto &s : m->params) b[s] = {tsm::Binding::Param, Dom::Scalar, 0};
  const tsm::Grid g{npts, nlm};
  try {
    const auto file = tsm::parse_model(m->source);
    const int nargout = nstate + nview;
    m->prog[0].fn = tsm::specialize(file, "init", b, m->params, nargout, g);
    m->prog[1].fn = tsm::specialize(file, "step", b, m->params, nargout, g);
    schedule(m, m->prog[0], false);
    schedule(m, m->prog[1], true);
  } catch (const tsm::CompileError &ce) {
    if (err) {
      err->start = ce.start;
      err->end = ce.end;
      snprintf(err->fn, sizeof err->fn, "%s", ce.fn.c_str());
      snprintf(err->message, sizeof err->message, "%s", ce.message.c_str());
    }
    ts_throw(TS_ERR_COMPILE, ce.message);
  }
}

std::string describe_program(const Program &P) {
  std::string s = tsm::describe(P.fn);
  for (size_t o = 0; o < P.feedback.size(); o++)
    if (!P.feedback[o].empty()) s += "copy    " + P.fn.output_names[o] + " -> " + P.feedback[o] + "\n";
  s += "-- launches --\n";
  for (const auto &st : P.stages) s += stage_title(st) + "\n";
  return s;
}

}  // namespace

// ===================================================================== C ABI

extern "C" {

int ts_model_compile(ts_plan plan, const char *source, const char *const *state, int nstate,
                     const char *const *view, int nview, const char *const *params, int nparams,
                     int batch, ts_model *out, ts_compile_error *err) {
  ts_ctx ctx = plan ? plan->ctx : nullptr;
  ts_model m = nullptr;
  if (err) memset(err, 0, sizeof(*err));
  try {
    TS_REQUIRE(plan && source && out, TS_ERR_INVALID, "null argument");
    TS_REQUIRE(nstate >= 1 && nstate <= TS_MAXIO && nview >= 0 && nparams >= 0, TS_ERR_INVALID,
               "bad state/view/param counts");
    TS_REQUIRE(batch >= 1 && batch <= 65535, TS_ERR_INVALID, "batch must be in [1, 65535]");
    TS_REQUIRE(plan->fourier == TS_FOURIER_FFT, TS_ERR_UNSUPPORTED,
               "models need an FFT grid: nphi = 2^a 3^b (the fused phase kernel runs the FFT)");
    ts_device_guard dev_guard_(ctx->device);
    m = new ts_model_s();
    m->ctx = ctx;
    m->plan = plan;
    m->batch = batch;
    m->source = source;
    for (int i = 0; i < nstate; i++) m->state.push_back(state[i]);
    for (int i = 0; i < nview; i++) m->view.push_back(view[i]);
    for (int i = 0; i < nparams; i++) m->params.push_back(params[i]);
    front_end(m, nstate, nview, err);
    finish_shapes(m);
    compile_kernels(m);
    const long npts = (long)plan->nlat * plan->nphi, nlm = plan->nlm;
        // host-owned buffers: state (two each), eigenvalues (shared), noise
    for (auto &s : m->state) {
      HostBuf h{Dom::Spec, 2 * nlm, false, true, dalloc(2 * nlm * batch), dalloc(2 * nlm * batch)};
      m->host[s] = h;
    }
    m->host["lam"] = HostBuf{Dom::Spec, 2 * nlm, true, false, dalloc(2 * nlm), nullptr};
    m->host["noise"] = HostBuf{Dom::Grid, npts, false, false, dalloc(npts * batch), nullptr};
    const auto lam = eigenvalues(plan);
    TS_CUDA(cudaMemcpy(m->host["lam"].cur, lam.data(), sizeof(float) * lam.size(),
                       cudaMemcpyHostToDevice));
    for (auto &P : m->prog)
      for (long c : P.pcount) P.pbuf.push_back(dalloc(c * batch));
    const long field = (long)(plan->mmax + 1) * plan->nlat;
    const int nsyn = std::max({m->prog[0].nsyn_max, m->prog[1].nsyn_max, 1});
    const int nana = std::max({m->prog[0].nana_max, m->prog[1].nana_max, 1});
    m->fm.ensure(sizeof(float2) * field * nsyn * batch);
    m->gm.ensure(sizeof(float2) * field * nana * batch);
    if (plan->precision != TS_PREC_FP32) {
      size_t wb = 0;
      for (auto &P : m->prog)
        for (auto &st : P.stages)
          if (st.kind == Stage::LegAnalys)
            wb = std::max(wb, ts_tc_wimg_bytes(plan, batch * st.nana, st.per_cta));
      m->wimg.ensure(std::max<size_t>(wb, 16));
      TS_CUDA(cudaMemset(m->wimg.p, 0, m->wimg.cap));
      m->qimg.ensure(ts_tc_qimg_bytes(plan, batch * nsyn));
      TS_CUDA(cudaMemset(m->qimg.p, 0, m->qimg.cap));
    }
    m->stash.ensure(sizeof(float) * 2 * nlm * batch * nstate);
    m->h_prm.assign((size_t)std::max(nparams, 1) * batch, 0.0f);
    m->d_prm = dalloc((long)m->h_prm.size());
    *out = m;
    return TS_OK;
  } catch (const ts_exc &e) {
    if (err && err->message[0] == 0) snprintf(err->message, sizeof err->message, "%s", e.msg.c_str());
    if (m) {
      free_model(m);
      delete m;
    }
    ts_set_error(ctx, e.msg);
    return e.code;
  }
}

int ts_model_destroy(ts_model m) {
  if (!m) return TS_ERR_INVALID;
  ts_device_guard dev_guard_(m->ctx->device, true);
  cudaStreamSynchronize(m->ctx->stream);
  free_model(m);
  delete m;
  return TS_OK;
}

#define TSM_BEGIN(m)                                   \
  ts_ctx ctx = m ? m->ctx : nullptr;                   \
  try {                                                \
    TS_REQUIRE(m != nullptr, TS_ERR_INVALID, "null model"); \
    ts_device_guard dev_guard_(ctx->device);
#define TSM_END                                         \
  }                                                     \
  catch (const ts_exc &e) {                             \
    ts_set_error(ctx, e.msg);                           \
    return e.code;                                      \
  }                                                     \
  return TS_OK;

int ts_model_set_params(ts_model m, const float *values, int n) {
  TSM_BEGIN(m)
  TS_REQUIRE(n == (int)m->params.size(), TS_ERR_SIZE, "set_params: expected one value per parameter");
  const int np = std::max(n, 1);
  for (int i = 0; i < m->batch; i++)
    for (int k = 0; k < n; k++) m->h_prm[(size_t)i * np + k] = values[k];
  check_finite_params(m->h_prm);
  TS_CUDA(cudaMemcpyAsync(m->d_prm, m->h_prm.data(), sizeof(float) * m->h_prm.size(),
                          cudaMemcpyHostToDevice, ctx->stream));
  TS_CUDA(cudaStreamSynchronize(ctx->stream));
  TSM_END
}

int ts_model_set_params_batched(ts_model m, const float *values, int batch, int n) {
  TSM_BEGIN(m)
  TS_REQUIRE(n == (int)m->params.size() && batch == m->batch, TS_ERR_SIZE,
             "set_params_batched: expected batch x nparams values");
  if (n > 0) std::copy(values, values + (size_t)batch * n, m->h_prm.begin());
  check_finite_params(m->h_prm);
  TS_CUDA(cudaMemcpyAsync(m->d_prm, m->h_prm.data(), sizeof(float) * m->h_prm.size(),
                          cudaMemcpyHostToDevice, ctx->stream));
  TS_CUDA(cudaStreamSynchronize(ctx->stream));
  TSM_END
}

int ts_model_upload(ts_model m, const char *name, const float *data, long n) {
  TSM_BEGIN(m)
  TS_REQUIRE(name && data, TS_ERR_INVALID, "null argument");
  auto it = m->host.find(name);
  if (it == m->host.end()) ts_throw(TS_ERR_NOT_FOUND, std::string("upload: no buffer named '") + name + "'");
  HostBuf &h = it->second;
  const long total = h.shared ? h.count : h.count * m->batch;
  if (n != h.count && n != total) {
    char buf[200];
    snprintf(buf, sizeof buf, "upload '%s': expected %ld elements, got %ld", name, total, n);
    ts_throw(TS_ERR_SIZE, buf);
  }
  if (n == total) {
    TS_CUDA(cudaMemcpyAsync(h.cur, data, sizeof(float) * n, cudaMemcpyHostToDevice, ctx->stream));
  } else {  // one instance's worth: the same values for every instance
    for (int i = 0; i < m->batch; i++)
      TS_CUDA(cudaMemcpyAsync(h.cur + (long)i * h.count, data, sizeof(float) * n,
                              cudaMemcpyHostToDevice, ctx->stream));
  }
  TS_CUDA(cudaStreamSynchronize(ctx->stream));
  TSM_END
}

int ts_model_init(ts_model m, const float *noise, long n) {
  TSM_BEGIN(m)
  if (noise) {
    const int rc = ts_model_upload(m, "noise", noise, n);
    if (rc != TS_OK) return rc;
  }
  run_program(m, m->prog[0], ctx->stream);
  m->last_ran = 0;
  TSM_END
}

namespace {
// nsteps steps: eager warm-up steps, then captured graphs
void advance(ts_model m, int nsteps) {
  int done = 0;
  for (; done < nsteps && (m->eager_left > 0 || !graphs_usable(m)); done++) {
    run_program(m, m->prog[1], m->ctx->stream);
    if (m->eager_left > 0) m->eager_left--;
  }
  while (nsteps - done >= 2) {
    run_steps_graphed(m, 2);
    done += 2;
  }
  if (done < nsteps) run_steps_graphed(m, 1);
  if (nsteps > 0) m->last_ran = 1;
}
}  // namespace

int ts_model_step(ts_model m, int nsteps) {
  TSM_BEGIN(m)
  TS_REQUIRE(nsteps >= 0, TS_ERR_INVALID, "nsteps must be >= 0");
  advance(m, nsteps);
  TSM_END
}

// ------------------------------------------------------------ model groups
//
// Several models (ragged batches: instances at different lmax, each group
// its own plan) advance together: every step runs each model's kernels on
// its own branch stream, forked from and joined to the context stream by
// events, captured into one CUDA graph per step pair and replayed, so the
// models' kernels overlap on the GPU.

struct ts_group_s {
  std::vector<ts_model> models;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> done;
  cudaEvent_t fork = nullptr;
  struct G {
    std::vector<float *> key;
    int nsteps;
    cudaGraphExec_t exec;
  };
  std::vector<G> graphs;
  int eager_left = 2;
  bool use_graphs = true;
};

namespace {

std::vector<float *> group_key(ts_group g) {
  std::vector<float *> k;
  for (ts_model m : g->models) {
    auto mk = state_key(m);
    k.insert(k.end(), mk.begin(), mk.end());
  }
  return k;
}

// one step of every model, forked from / joined to the context stream
void group_launch(ts_group g) {
  cudaStream_t s0 = g->models[0]->ctx->stream;
  TS_CUDA(cudaEventRecord(g->fork, s0));
  for (size_t i = 0; i < g->models.size(); i++) {
    TS_CUDA(cudaStreamWaitEvent(g->streams[i], g->fork, 0));
    run_program(g->models[i], g->models[i]->prog[1], g->streams[i]);
    TS_CUDA(cudaEventRecord(g->done[i], g->streams[i]));
  }
  for (size_t i = 0; i < g->models.size(); i++) TS_CUDA(cudaStreamWaitEvent(s0, g->done[i], 0));
}

void group_swap(ts_group g, int nsteps) {
  for (ts_model m : g->models) swap_states(m, nsteps);
}

void group_steps(ts_group g, int nsteps) {
  cudaStream_t s0 = g->models[0]->ctx->stream;
  const std::vector<float *> key = group_key(g);
  for (auto &x : g->graphs)
    if (x.nsteps == nsteps && x.key == key) {
      TS_CUDA(cudaGraphLaunch(x.exec, s0));
      group_swap(g, nsteps);
      return;
    }
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool ok = cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  if (ok) {
    int ran = 0;
    try {
      for (; ran < nsteps; ran++) group_launch(g);
    } catch (const ts_exc &) {
      ok = false;
    }
    const bool ended = cudaStreamEndCapture(s0, &graph) == cudaSuccess;
    ok = ok && ended && graph;
    if (!ok) group_swap(g, ran);
  }
  if (ok) ok = cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
  if (graph) cudaGraphDestroy(graph);
  if (!ok) {
    (void)cudaGetLastError();
    g->use_graphs = false;
    for (int i = 0; i < nsteps; i++) group_launch(g);
    return;
  }
  g->graphs.push_back({key, nsteps, exec});
  TS_CUDA(cudaGraphLaunch(exec, s0));
}

}  // namespace

int ts_model_group_create(ts_model const *models, int n, ts_group *out) {
  ts_ctx ctx = (n > 0 && models && models[0]) ? models[0]->ctx : nullptr;
  ts_group g = nullptr;
  try {
    TS_REQUIRE(ctx && out && n >= 1, TS_ERR_INVALID, "need at least one model and an output");
    for (int i = 0; i < n; i++)
      TS_REQUIRE(models[i] && models[i]->ctx == ctx, TS_ERR_INVALID,
                 "group: every model must belong to the same context");
    ts_device_guard dev_guard_(ctx->device);
    g = new ts_group_s();
    g->models.assign(models, models + n);
    TS_CUDA(cudaEventCreateWithFlags(&g->fork, cudaEventDisableTiming));
    for (int i = 0; i < n; i++) {
      cudaStream_t st;
      cudaEvent_t ev;
      TS_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
      g->streams.push_back(st);
      TS_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      g->done.push_back(ev);
    }
    *out = g;
    return TS_OK;
  } catch (const ts_exc &e) {
    if (g) ts_model_group_destroy(g);
    ts_set_error(ctx, e.msg);
    return e.code;
  }
}

int ts_model_group_step(ts_group g, int nsteps) {
  ts_ctx ctx = g && !g->models.empty() ? g->models[0]->ctx : nullptr;
  try {
    TS_REQUIRE(g != nullptr && nsteps >= 0, TS_ERR_INVALID, "bad group or step count");
    ts_device_guard dev_guard_(ctx->device);
    const cudaStream_t s0 = ctx->stream;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    const bool capturable = g->use_graphs && s0 != nullptr && s0 != cudaStreamLegacy &&
                            s0 != cudaStreamPerThread &&
                            cudaStreamIsCapturing(s0, &cs) == cudaSuccess &&
                            cs == cudaStreamCaptureStatusNone;
    int done = 0;
    for (; done < nsteps && (g->eager_left > 0 || !capturable); done++) {
      group_launch(g);
      if (g->eager_left > 0) g->eager_left--;
    }
    while (nsteps - done >= 2) {
      group_steps(g, 2);
      done += 2;
    }
    if (done < nsteps) group_steps(g, 1);
    if (nsteps > 0)
      for (ts_model m : g->models) m->last_ran = 1;
    return TS_OK;
  } catch (const ts_exc &e) {
    ts_set_error(ctx, e.msg);
    return e.code;
  }
}

int ts_model_group_destroy(ts_group g) {
  if (!g) return TS_ERR_INVALID;
  ts_device_guard dev_guard_(g->models.empty() ? 0 : g->models[0]->ctx->device, true);
  if (!g->models.empty()) cudaStreamSynchronize(g->models[0]->ctx->stream);
  for (auto &x : g->graphs) cudaGraphExecDestroy(x.exec);
  for (cudaStream_t st : g->streams) cudaStreamDestroy(st);
  for (cudaEvent_t ev : g->done) cudaEventDestroy(ev);
  if (g->fork) cudaEventDestroy(g->fork);
  delete g;
  return TS_OK;
}

int ts_model_forward_backward(ts_model m, int nsteps, int every, const float *final_bar,
                              float *init_bar, double *param_bar) {
  TSM_BEGIN(m)
  TS_REQUIRE(nsteps >= 1 && every >= 1, TS_ERR_INVALID, "nsteps and every must be >= 1");
  TS_REQUIRE(final_bar && init_bar, TS_ERR_INVALID, "null argument");
  adj_prepare(m);
  Adjoint &A = m->adj;
  cudaStream_t st = ctx->stream;
  const int B = m->batch, ns = (int)m->state.size();
  const long sz = 2 * m->plan->nlm * (long)B;  // floats of one state, all instances
  const int nseg = (nsteps + every - 1) / every;
  // checkpoints [segment][state], segment states [step][state], cotangents [state]
  DevMem ck(sizeof(float) * sz * ns * nseg), seg(sizeof(float) * sz * ns * every),
      lamb(sizeof(float) * sz * ns);
  float *pck = (float *)ck.p, *pseg = (float *)seg.p, *plam = (float *)lamb.p;
  for (int i = 0; i < nsteps; i += every) {
    for (int s = 0; s < ns; s++)
      TS_CUDA(cudaMemcpyAsync(pck + ((long)(i / every) * ns + s) * sz, m->host.at(m->state[s]).cur,
                              sizeof(float) * sz, cudaMemcpyDeviceToDevice, st));
    advance(m, std::min(every, nsteps - i));
  }
  TS_CUDA(cudaMemcpyAsync(plam, final_bar, sizeof(float) * sz * ns, cudaMemcpyHostToDevice, st));
  TS_CUDA(cudaMemsetAsync(A.pbar, 0, sizeof(double) * std::max<size_t>(m->params.size(), 1) * B, st));
  std::vector<float *> lam(ns);
  for (int s = 0; s < ns; s++) lam[s] = plam + (long)s * sz;
  for (int g = nseg - 1; g >= 0; g--) {
    const int len = std::min(every, nsteps - g * every);
    TS_CUDA(cudaMemcpyAsync(pseg, pck + (long)g * ns * sz, sizeof(float) * sz * ns,
                            cudaMemcpyDeviceToDevice, st));
    auto states = [&](int j) {
      std::vector<const float *> v(ns);
      for (int s = 0; s < ns; s++) v[s] = pseg + ((long)j * ns + s) * sz;
      return v;
    };
    for (int j = 1; j < len; j++) {  // replay the segment: the state before every step
      adj_tape(m, states(j - 1), st);
      for (int s = 0; s < ns; s++)
        TS_CUDA(cudaMemcpyAsync(pseg + ((long)j * ns + s) * sz, A.val[A.state_out[s]],
                                sizeof(float) * sz, cudaMemcpyDeviceToDevice, st));
    }
    for (int j = len - 1; j >= 0; j--) {
      adj_tape(m, states(j), st);
      adj_reverse(m, lam, st);
    }
  }
  TS_CUDA(cudaMemcpyAsync(init_bar, plam, sizeof(float) * sz * ns, cudaMemcpyDeviceToHost, st));
  if (param_bar && !m->params.empty())
    TS_CUDA(cudaMemcpyAsync(param_bar, A.pbar, sizeof(double) * m->params.size() * B,
                            cudaMemcpyDeviceToHost, st));
  TS_CUDA(cudaStreamSynchronize(st));
  TS_CUDA(cudaGetLastError());
  TSM_END
}

int ts_model_set_graphs(ts_model m, int enable) {
  TSM_BEGIN(m)
  m->use_graphs = enable != 0;
  drop_graphs(m);
  TSM_END
}

int ts_model_read(ts_model m, const char *name, float *out, long n) {
  TSM_BEGIN(m)
  TS_REQUIRE(name && out, TS_ERR_INVALID, "null argument");
  float *ptr;
  long count, stride;
  std::string lazy;
  if (!locate(m, name, &ptr, &count, &stride, &lazy))
    ts_throw(TS_ERR_NOT_FOUND, std::string("read: the model has no value named '") + name + "'");
  const long total = count * m->batch;
  TS_REQUIRE(n == total || n == count, TS_ERR_SIZE,
             std::string("read '") + name + "': expected " + std::to_string(total) + " (or " +
                 std::to_string(count) + " for instance 0) elements");
  const int ninst = n == total ? m->batch : 1;
  ts_plan p = m->plan;
  if (!lazy.empty()) {
    // a displayed field computed on demand from the state it is synth() of
    HostBuf &h = m->host.at(lazy);
    const float *src = m->prog[1].swaps.count(lazy) ? h.next : h.cur;
    const long field = (long)(p->mmax + 1) * p->nlat;
    p->fm.ensure(sizeof(float2) * field * ninst);
    ts_launch_leg_synth(p, (const float2 *)src, p->nlm, (float2 *)p->fm.p, field, ninst, ctx->stream);
    float *tmp = nullptr;
    TS_CUDA(cudaMallocAsync(&tmp, sizeof(float) * count * ninst, ctx->stream));
    ts_launch_fourier_synth(p, (const float2 *)p->fm.p, field, tmp, count, ninst, ctx->stream);
    TS_CUDA(cudaMemcpyAsync(out, tmp, sizeof(float) * n, cudaMemcpyDeviceToHost, ctx->stream));
    TS_CUDA(cudaFreeAsync(tmp, ctx->stream));
  } else if (stride == 0 && ninst > 1) {
    for (int i = 0; i < ninst; i++)
      TS_CUDA(cudaMemcpyAsync(out + (long)i * count, ptr, sizeof(float) * count,
                              cudaMemcpyDeviceToHost, ctx->stream));
  } else {
    TS_CUDA(cudaMemcpyAsync(out, ptr, sizeof(float) * n, cudaMemcpyDeviceToHost, ctx->stream));
  }
  TS_CUDA(cudaStreamSynchronize(ctx->stream));
  // values computed by a tensor-core kernel that gave up a wait are incomplete
  ts_plan_take_timeout(p);
  TSM_END
}

int ts_model_value_ptr(ts_model m, const char *name, float **dev, long *count) {
  TSM_BEGIN(m)
  TS_REQUIRE(name && dev && count, TS_ERR_INVALID, "null argument");
  float *ptr;
  long stride;
  std::string lazy;
  if (!locate(m, name, &ptr, count, &stride, &lazy) || !lazy.empty())
    ts_throw(TS_ERR_NOT_FOUND, std::string("no device buffer holds '") + name + "'");
  *dev = ptr;
  TSM_END
}

int ts_model_snapshot(ts_model m) {
  TSM_BEGIN(m)
  const long n = 2 * m->plan->nlm * m->batch;
  long off = 0;
  for (auto &s : m->state) {
    TS_CUDA(cudaMemcpyAsync((float *)m->stash.p + off, m->host.at(s).cur, sizeof(float) * n,
                            cudaMemcpyDeviceToDevice, ctx->stream));
    off += n;
  }
  m->stashed_ran = m->last_ran;
  TSM_END
}

int ts_model_restore(ts_model m) {
  TSM_BEGIN(m)
  const long n = 2 * m->plan->nlm * m->batch;
  long off = 0;
  for (auto &s : m->state) {
    TS_CUDA(cudaMemcpyAsync(m->host.at(s).cur, (float *)m->stash.p + off, sizeof(float) * n,
                            cudaMemcpyDeviceToDevice, ctx->stream));
    off += n;
  }
  m->last_ran = m->stashed_ran;
  TSM_END
}

int ts_model_describe(ts_model m, int which, char *buf, size_t cap) {
  TSM_BEGIN(m)
  TS_REQUIRE(which == 0 || which == 1, TS_ERR_INVALID, "which: 0 = init, 1 = step");
  TS_REQUIRE(buf && cap > 0, TS_ERR_INVALID, "null buffer");
  snprintf(buf, cap, "%s", describe_program(m->prog[which]).c_str());
  TSM_END
}

int ts_model_source(ts_model m, char *buf, size_t cap) {
  TSM_BEGIN(m)
  TS_REQUIRE(buf && cap > 0, TS_ERR_INVALID, "null buffer");
  std::string s;
  for (auto &P : m->prog)
    for (auto &st : P.stages) s += stage_source(st);
  snprintf(buf, cap, "%s", s.c_str());
  TSM_END
}

namespace {
// CUDA kernel launches of one call of a program: on a tensor-core plan a
// Legendre synthesis stage is two (the operand relayout, then the tcgen05
// contraction)
int kernel_launches(ts_plan p, const Program &P) {
  int n = 0;
  for (auto &s : P.stages) n += s.kind == Stage::LegSynth && p->precision != TS_PREC_FP32 ? 2 : 1;
  return n;
}
}  // namespace

int ts_model_counts(ts_model m, int which, int *kernels, int *launches) {
  TSM_BEGIN(m)
  TS_REQUIRE(which == 0 || which == 1, TS_ERR_INVALID, "which: 0 = init, 1 = step");
  if (kernels) *kernels = tsm::count_kernels(m->prog[which].fn);
  if (launches) *launches = kernel_launches(m->plan, m->prog[which]);
  TSM_END
}

// Everything ts_model_compile does short of the GPU: parse, specialise,
// schedule, generate CUDA and compile it with NVRTC for sm_100a, on a grid
// described by its sizes.  Writes describe() of init and step (separated by a
// line "====") to `describe` and the kernel and launch counts of step.
int ts_model_check(int lmax, int mmax, int nlat, int nphi, const char *source,
                   const char *const *state, int nstate, const char *const *view, int nview,
                   const char *const *params, int nparams, int batch, int flags,
                   char *describe, size_t cap, int *kernels, int *launches,
                   ts_compile_error *err) {
  if (err) memset(err, 0, sizeof(*err));
  ts_ctx_s ctx;
  ctx.sm_count = 148;
  ctx.smem_optin = 232448;
  ts_plan_s plan;
  ts_model_s mod;
  try {
    TS_REQUIRE(source != nullptr, TS_ERR_INVALID, "null source");
    char why[256];
    if (ts_validate_config(lmax, mmax, nlat, nphi, why, sizeof why) != TS_OK)
      ts_throw(TS_ERR_INVALID, why);
    plan.ctx = &ctx;
    plan.lmax = lmax;
    plan.mmax = mmax;
    plan.nlat = nlat;
    plan.nphi = nphi;
    plan.nh = (nlat + 1) / 2;
    plan.nlm = ts_nlm_calc(lmax, mmax);
    plan.precision = flags & TS_PREC_MASK;
    plan.fft.nphi = nphi;
    plan.fft.H = nphi / 2;
    plan.fft.mmax = mmax;
    plan.fft.nlat = nlat;
    mod.ctx = &ctx;
    mod.plan = &plan;
    mod.batch = batch;
    mod.source = source;
    for (int i = 0; i < nstate; i++) mod.state.push_back(state[i]);
    for (int i = 0; i < nview; i++) mod.view.push_back(view[i]);
    for (int i = 0; i < nparams; i++) mod.params.push_back(params[i]);
    front_end(&mod, nstate, nview, err);
    finish_shapes(&mod);
    std::map<std::string, std::string> lowered;
    build_cubin(&mod, lowered);
    std::string adj_code;
    if (flags & TS_CHECK_ADJOINT) {
      adj_structure(&mod);
      adj_code = adj_source(&mod);
      nvrtc_cubin(adj_code, {}, lowered);
    }
    if (describe && cap && (flags & TS_CHECK_SOURCE)) {
      std::string code;
      for (auto &P : mod.prog)
        for (auto &st : P.stages) code += stage_source(st);
      snprintf(describe, cap, "%s%s", code.c_str(), adj_code.c_str());
    } else if (describe && cap) {
      snprintf(describe, cap, "%s====\n%s", describe_program(mod.prog[0]).c_str(),
               describe_program(mod.prog[1]).c_str());
    }
    if (kernels) *kernels = tsm::count_kernels(mod.prog[1].fn);
    if (launches) *launches = kernel_launches(&plan, mod.prog[1]);
    return TS_OK;
  } catch (const ts_exc &e) {
    if (err && err->message[0] == 0) snprintf(err->message, sizeof err->message, "%s", e.msg.c_str());
    ts_set_error(nullptr, e.msg);
    return e.code;
  }
}

}  // extern "C"
