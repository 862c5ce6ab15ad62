/*
 * turing_sht.h — C ABI of libturing_sht.so, the B200 (sm_100a) implementation
 * of turing-sphere's spherical-harmonic transforms and IMEX model step.
 *
 * This is the drop-in boundary for the reference's WebGPU path: a host
 * binding (the TypeScript side through N-API/koffi, or Python through ctypes)
 * calls these functions where the reference installs a WebGPU device
 * (scripts/nodeWebGpu.ts:18-65) and drives ShtPlan (src/sht/sht.ts),
 * ModelPlan (src/mgpu/plan.ts) and GpuModel (src/mgpu/model.ts).
 *
 * Rules of the ABI:
 *   - plain C types only: pointers, sizes, ints, floats; opaque handles;
 *   - every function returns a status (TS_OK = 0, negative = error) and never
 *     throws; ts_last_error(ctx) returns the message of the last failure on
 *     that context;
 *   - `_dev` entry points take device pointers and a cudaStream_t passed as
 *     void* (NULL = the context's stream) and return without synchronising;
 *     the others take caller-owned HOST arrays and block until done;
 *   - device arrays of the transforms must be 8-byte aligned (coefficient
 *     pairs and grid rows are accessed as float2): other pointers are refused
 *     with TS_ERR_INVALID before anything runs;
 *   - every call makes the context's device current for its duration and
 *     gives the calling thread back the CUDA context it had on entry;
 *   - one host thread per context.
 *
 * Layouts (src/sht/layout.ts:1-16): spectral arrays are float pairs
 * [re, im] per coefficient in m-major order lm(l,m) = m(lmax+1) - m(m-1)/2 +
 * (l-m), length 2*nlm per field; spatial arrays are float[nlat*nphi] per
 * field, spat[ilat*nphi + iphi], ilat north to south.  A batch of B fields is
 * B such arrays back to back.
 */
#ifndef TURING_SHT_H
#define TURING_SHT_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ts_ctx_s *ts_ctx;
typedef struct ts_plan_s *ts_plan;
typedef struct ts_model_s *ts_model;
typedef struct ts_group_s *ts_group;

enum ts_status {
  TS_OK = 0,
  TS_ERR_INVALID = -1,     /* bad argument or configuration */
  TS_ERR_CUDA = -2,        /* a CUDA runtime/driver call failed */
  TS_ERR_COMPILE = -3,     /* model source rejected (see ts_model_compile) */
  TS_ERR_NOT_FOUND = -4,   /* unknown name */
  TS_ERR_SIZE = -5,        /* length mismatch */
  TS_ERR_UNSUPPORTED = -6, /* valid request this build does not implement */
  TS_ERR_TIMEOUT = -7,     /* a bounded device-side wait gave up */
  TS_ERR_STATE = -8        /* call out of order (e.g. read before run) */
};

/* Plan flags (bitwise OR). */
enum ts_plan_flags {
  TS_PREC_FP32 = 0,        /* plain FP32 on-the-fly recurrence (default) */
  TS_PREC_TF32X3 = 1,      /* tcgen05 tensor-core Legendre, 3-pass split TF32 */
  TS_PREC_BF16X3 = 2,      /* tcgen05 tensor-core Legendre, 3-pass split BF16 */
  TS_PREC_MASK = 0xF,
  TS_CHECK_SOURCE = 0x100, /* ts_model_check: return the generated source */
  TS_CHECK_ADJOINT = 0x200, /* ts_model_check: also generate and compile the step's adjoint */
  TS_FOURIER_AUTO = 0,     /* mixed-radix FFT whenever nphi = 2^a 3^b, else DFT */
  TS_FOURIER_FFT = 0x10,   /* require the FFT (error if nphi has other factors) */
  TS_FOURIER_DFT = 0x20,   /* direct band-limited sum (sht.ts:241-289 semantics) */
  TS_FOURIER_MASK = 0x30,
  TS_PLAN_AUTOTUNE = 0x40  /* time the kernel shapes at plan creation, keep the fastest */
};

/* ------------------------------------------------------------ context
 * Replaces installWebGpu()/requestShtDevice() (scripts/nodeWebGpu.ts:18-65,
 * src/sht/sht.ts:495-513): one CUDA device and one stream. */
int ts_ctx_create(int device_ordinal, ts_ctx *out);
int ts_ctx_destroy(ts_ctx ctx);
const char *ts_last_error(ts_ctx ctx);
/* Use an external cudaStream_t (as void*) for this context's work; NULL
 * restores the context's own stream. */
int ts_ctx_set_stream(ts_ctx ctx, void *stream);
void *ts_ctx_stream(ts_ctx ctx);
/* GPU name into buf (describeAdapter, sht.ts:464-493). */
int ts_ctx_device_name(ts_ctx ctx, char *buf, size_t cap);
/* Wait for all work on the context's stream (GPUQueue.onSubmittedWorkDone,
 * session.ts:167-169). */
int ts_sync(ts_ctx ctx);

/* ------------------------------------------------------------- layout
 * src/sht/layout.ts:24-59. */
long ts_nlm_calc(int lmax, int mmax);
long ts_lm_index(int lmax, int l, int m);
/* 0 if valid, else TS_ERR_INVALID with the reason in buf (validateConfig). */
int ts_validate_config(int lmax, int mmax, int nlat, int nphi, char *buf, size_t cap);
void ts_grid_for_lmax(int lmax, int pdeg, int *nlat, int *nphi);

/* ------------------------------------------------------------ SHT plan
 * ShtPlan.create (sht.ts:166-183): validates the config, computes the
 * Gauss-Legendre nodes/weights and the recurrence coefficients in FP64 on the
 * GPU, and uploads FP32 tables.  flags: ts_plan_flags. */
int ts_sht_plan_create(ts_ctx ctx, int lmax, int mmax, int nlat, int nphi, int flags,
                       ts_plan *out);
int ts_sht_plan_destroy(ts_plan plan);

typedef struct ts_plan_info {
  int lmax, mmax, nlat, nphi;
  long nlm;
  int precision;  /* TS_PREC_* in use */
  int fourier;    /* TS_FOURIER_FFT or TS_FOURIER_DFT in use */
  int fft_stages; /* Stockham stages of the nphi/2-point FFT (0 for DFT) */
  int fft_radix[16];
  long table_bytes; /* tensor-core P tables in device memory (0 for FP32) */
  /* kernel shapes in use (chosen by TS_PLAN_AUTOTUNE, else the defaults) */
  int tc_lat_tile;   /* tensor-core synthesis: latitudes per tile (0 for FP32) */
  int tc_deg_tile;   /* tensor-core analysis: degrees per tile (0 for FP32) */
  int fft_p, fft_q;  /* two-phase FFT H = P*Q (0 when the Stockham/DFT kernels run) */
  int fft_rows;      /* grid rows per FFT CTA */
  int tuned;         /* 1 when the shapes were timed (TS_PLAN_AUTOTUNE) */
  /* tensor-core polar skip: synthesis tiles written as zeros, and synthesis
   * degree chunks plus analysis latitude chunks left out, because every
   * table value in them is below 1e-10 of the largest of their m (synthesis)
   * or tile (analysis) */
  int tc_skip_tiles, tc_skip_chunks;
} ts_plan_info;
int ts_sht_plan_info(ts_plan plan, ts_plan_info *info);

/* Synchronises the context's stream, then reports TS_ERR_TIMEOUT (and clears
 * the flag) if a tensor-core kernel of this plan gave up a bounded wait for its
 * MMAs since the last call; TS_OK otherwise. */
int ts_sht_plan_status(ts_plan plan);
/* Test hook for failure detection (no reference counterpart).  With
 * stall_copies != 0 the tensor-core kernels' copy warp issues no copies, so
 * every bounded wait of the kernel runs out after `wait_limit` polls (0 =
 * the default limit): the kernel records the error, frees its tensor memory
 * and returns, and ts_sht_plan_status reports TS_ERR_TIMEOUT once.  Nothing
 * faults or hangs; stall_copies = 0 restores normal operation.
 * TS_ERR_UNSUPPORTED on FP32 plans. */
int ts_sht_plan_test_stall(ts_plan plan, int stall_copies, unsigned wait_limit);

/* Nodes x_i = cos(theta_i) (decreasing) and Gauss weights w_i, f64, nlat each,
 * as computed on the GPU (ShtPlan.cosTheta / gaussWeights, sht.ts:120-125). */
int ts_sht_plan_nodes(ts_plan plan, double *cos_theta, double *weights);

/* Batched transforms on device pointers.  synth: qlm[B][2*nlm] ->
 * spat[B][nlat*nphi]; analys: the reverse.  The fm intermediate is plan-owned
 * scratch, grown on first use for a larger batch (encodeSynthInto /
 * encodeAnalysInto, sht.ts:326-353; the scratch is sht.ts:291-298's fmBuf). */
int ts_sht_synth_dev(ts_plan plan, const float *qlm, float *spat, int batch, void *stream);
int ts_sht_analys_dev(ts_plan plan, const float *spat, float *qlm, int batch, void *stream);

/* Allocation-free synthesis.  No counterpart in the reference: it exists for
 * callers that cannot let the library call cudaMalloc (hosts that own every
 * device allocation, or loops that must not stall on cudaMalloc's implicit
 * device synchronisation).  Same inputs, outputs and result as
 * ts_sht_synth_dev, but the Fourier intermediate lives in a fixed 16 MiB
 * array compiled into the library (held on every GPU that loads it until the
 * process exits), so the call allocates nothing.  A batch whose intermediate
 * exceeds 16 MiB ((mmax+1)*nlat*8 bytes per field) fails with TS_ERR_SIZE.
 * The first call on a device looks up the array's device address; make that
 * first call before any stream capture.  All calls share the one array: calls
 * that overlap on the GPU (different streams, no ordering) race.  It runs the
 * FP32 Legendre kernels whatever the plan's precision (the tensor-core path
 * needs an operand image the plan grows on demand). */
int ts_sht_synth_noalloc(ts_plan plan, const float *qlm, float *spat, int batch, void *stream);

/* Blocking transforms on host arrays (ShtPlan.synth / ShtPlan.analys,
 * sht.ts:414-461); they fail with TS_ERR_SIZE on a length mismatch.  A batch
 * moves in chunks of fields: one chunk's host->device copy, another's
 * transform and a third's device->host copy run at once (two copy streams
 * and the context's stream, ordered by events).  Page-locked host arrays
 * (cudaHostAlloc / cudaHostRegister) get the full overlap; pageable arrays
 * are correct but copied through the driver's staging.  Staging device
 * arrays are plan-owned and grown on first use. */
int ts_sht_synth(ts_plan plan, const float *qlm, long qlm_len, float *spat, long spat_len,
                 int batch);
int ts_sht_analys(ts_plan plan, const float *spat, long spat_len, float *qlm, long qlm_len,
                  int batch);
/* Round trips on host arrays: qlm_out = analys(synth(qlm_in)) per field, the
 * grid staying on the device.  The round trip of scripts/bench-sht.ts:190-217
 * (coefficients written to the device, encodeSynthInto + encodeAnalysInto,
 * the result copied to a readback buffer and mapped) as one blocking call,
 * pipelined over chunks of fields like ts_sht_synth. */
int ts_sht_roundtrip(ts_plan plan, const float *qlm_in, long in_len, float *qlm_out,
                     long out_len, int batch);

/* Single stages, for diagnostics (ShtPlan.encodeStage, sht.ts:362-401;
 * scripts/diagnose-sht.ts).  fm is [B][mmax+1][nlat] complex (2 floats). */
int ts_sht_leg_synth_dev(ts_plan plan, const float *qlm, float *fm, int batch, void *stream);
int ts_sht_fourier_synth_dev(ts_plan plan, const float *fm, float *spat, int batch,
                             void *stream);
int ts_sht_fourier_analys_dev(ts_plan plan, const float *spat, float *fm, int batch,
                              void *stream);
int ts_sht_leg_analys_dev(ts_plan plan, const float *fm, float *qlm, int batch, void *stream);

/* Adjoints of the transforms (no reference counterpart: the reference has
 * no differentiation).  With coefficients read as 2*nlm reals and the grid
 * as nlat*nphi reals, synth_adjoint applies S^T (grid cotangent -> spectral
 * cotangent) and analys_adjoint applies A^T (spectral -> grid), exactly the
 * transposes of ts_sht_synth_dev / ts_sht_analys_dev; the imaginary part of
 * m = 0 of a spectral cotangent is zero. */
int ts_sht_synth_adjoint_dev(ts_plan plan, const float *gbar, float *qbar, int batch,
                             void *stream);
int ts_sht_analys_adjoint_dev(ts_plan plan, const float *qbar, float *gbar, int batch,
                              void *stream);

/* The two stages of ts_sht_analys_dev on a tensor-core plan, for timing them
 * apart (no reference counterpart: the reference has one analysis path).  The
 * Fourier analysis writes the folded, weighted operand image of the
 * tensor-core Legendre analysis (ts_sht_wimage_bytes(plan, batch) bytes; the
 * caller zero-fills it once, the stage writes every entry that is not
 * padding); the Legendre stage reads it.  TS_ERR_UNSUPPORTED on an FP32 plan
 * or a row length without a two-phase FFT shape. */
size_t ts_sht_wimage_bytes(ts_plan plan, int batch);
int ts_sht_fourier_analys_w_dev(ts_plan plan, const float *spat, void *wimage, int batch,
                                void *stream);
int ts_sht_leg_analys_w_dev(ts_plan plan, const void *wimage, float *qlm, int batch,
                            void *stream);

/* --------------------------------------------------------------- models
 * A .m model (init/step functions, src/mgpu/model.ts:1-19) compiled for a
 * plan's grid: parsed and specialised (src/mgpu/compile.ts:83-190), every
 * element-wise statement emitted as CUDA C and compiled by NVRTC for sm_100a,
 * with the grid statements fused between the synthesis and analysis FFTs and
 * the spectral statements after an analysis fused into its Legendre epilogue.
 * The host bindings a .m may name are those of model.ts:116-125: lam
 * (l(l+1), 2 x nlm), noise (npts x 1), npts, nlm, the state names (2 x nlm)
 * and the parameter names (runtime scalars: changing one rewrites a small
 * buffer and recompiles nothing, compile.ts:34-40).  `batch` independent
 * instances advance together; each has its own state, noise and parameters. */
typedef struct ts_compile_error {
  long start, end; /* byte offsets into the source, -1 when unknown */
  char fn[64];     /* function being compiled ("init", "step") */
  char message[1024];
} ts_compile_error;

/* GpuModel.create (model.ts:103-163).  Returns TS_ERR_COMPILE with `err`
 * filled (ModelCompileError / UnsupportedOnGpu, errors.ts:14-31) when the
 * source is rejected. */
int ts_model_compile(ts_plan plan, const char *source, const char *const *state, int nstate,
                     const char *const *view, int nview, const char *const *params, int nparams,
                     int batch, ts_model *out, ts_compile_error *err);
int ts_model_destroy(ts_model model);

/* ModelPlan.setParams (plan.ts:410-420): values in the model's parameter
 * order, the same for every instance; non-finite values become 0. */
int ts_model_set_params(ts_model model, const float *values, int n);
/* Per-instance parameters: values[batch][n] (a parameter sweep). */
int ts_model_set_params_batched(ts_model model, const float *values, int batch, int n);

/* GpuModel.upload (plan.ts:77-86): a host-owned value (a state, noise, lam)
 * from host memory; n = one instance's length (copied to every instance) or
 * batch times it.  TS_ERR_NOT_FOUND for an unknown name, TS_ERR_SIZE for a
 * wrong length. */
int ts_model_upload(ts_model model, const char *name, const float *data, long n);

/* GpuModel.init (model.ts:180-186): upload the seeded perturbation (may be
 * NULL to keep the current one) and run `init`.  Asynchronous. */
int ts_model_init(ts_model model, const float *noise, long n);
/* GpuModel.step (model.ts:229-234): `nsteps` timesteps.  Asynchronous. */
int ts_model_step(ts_model model, int nsteps);
/* Steps run as CUDA graphs (no reference counterpart: the reference encodes
 * one command buffer per step, plan.ts:468-495).  After two eager warm-up
 * steps, pairs of steps (and a single step for an odd count) are captured on
 * the context stream once per state-buffer parity and replayed; a stream the
 * caller is capturing itself, or the legacy default stream, runs eagerly.
 * enable = 0 turns graphs off for this model (results are identical). */
int ts_model_set_graphs(ts_model model, int enable);

/* Model groups (no reference counterpart): ragged batches, e.g. instances
 * at lmax 63/127/255 each compiled as one model on its own plan, advance
 * together.  Each step runs every model's kernels on its own branch stream
 * forked from the context stream; after two eager steps, steps are captured
 * as one CUDA graph per state parity and replayed.  All models must share
 * the context; a model in a group is stepped through the group only. */
int ts_model_group_create(ts_model const *models, int n, ts_group *out);
int ts_model_group_step(ts_group group, int nsteps);
int ts_model_group_destroy(ts_group group);

/* Forward/backward pair of the adjoint (no reference counterpart; the
 * autograd.Function of this path).  Advances the model nsteps steps from its
 * current state, as ts_model_step does, keeping a checkpoint of the state
 * every `every` steps; then runs the hand-written adjoint of the step (the
 * transposed transforms, the symbolically differentiated element-wise
 * statements and the implicit diffusion solve) backwards, replaying each
 * segment from its checkpoint.  final_bar: dL/d(final state), host
 * [state][instance][2 nlm] in the model's state order; init_bar receives
 * dL/d(initial state) in the same layout; param_bar (may be NULL) receives
 * dL/d(parameters), host double [instance][nparams]. */
int ts_model_forward_backward(ts_model model, int nsteps, int every, const float *final_bar,
                              float *init_bar, double *param_bar);

/* GpuModel.read (model.ts:262-277): blocking read of a named value — from the
 * function that ran most recently, as #locate does (model.ts:243-252).
 * n = batch x length (all instances) or length (instance 0). */
int ts_model_read(ts_model model, const char *name, float *out, long n);
/* GpuModel.valueBuffer (model.ts:254-259): the device buffer of a named value
 * ([batch][count] floats; stride 0 for values shared by all instances). */
int ts_model_value_ptr(ts_model model, const char *name, float **dev, long *count);

/* snapshotState / restoreState (model.ts:195-223). */
int ts_model_snapshot(ts_model model);
int ts_model_restore(ts_model model);

/* GpuModel.describe (plan.ts:486-488): the statements each function compiled
 * to and the launches that run them; which = 0 (init) or 1 (step). */
int ts_model_describe(ts_model model, int which, char *buf, size_t cap);
/* The generated CUDA C of both functions. */
int ts_model_source(ts_model model, char *buf, size_t cap);
/* Element-wise statements (the reference's kernel count, the fusion guard of
 * test/modelChecks.ts:17-21) and CUDA kernel launches per call (on a
 * tensor-core plan a Legendre synthesis is two: the operand relayout and the
 * tcgen05 contraction). */
int ts_model_counts(ts_model model, int which, int *kernels, int *launches);

/* Everything ts_model_compile does short of the GPU — parse, specialise,
 * schedule, generate CUDA C and compile it with NVRTC for sm_100a — for a grid
 * given by its sizes (no context, no device).  `describe` receives the
 * describe() text of init and step separated by a "====" line; flags selects
 * the precision (TS_PREC_*) whose kernels are generated, optionally ORed
 * with TS_CHECK_SOURCE to receive the generated CUDA source of both programs
 * in `describe` instead of the stage list; `kernels` and `launches` are those
 * of step.  For host-side checks of a model source
 * (the editor's compile-on-type, src/editor/, and the tests). */
int ts_model_check(int lmax, int mmax, int nlat, int nphi, const char *source,
                   const char *const *state, int nstate, const char *const *view, int nview,
                   const char *const *params, int nparams, int batch, int flags,
                   char *describe, size_t cap, int *kernels, int *launches,
                   ts_compile_error *err);

/* Seeding (src/mgpu/noise.ts:15-51; bench-sht.ts:132-144): mulberry32 and
 * Box-Muller, bit-identical integer state to the reference's.  amp-scaled
 * normals per grid point, and a uniform [-1, 1) spectrum with m = 0 imaginary
 * parts zero. */
void ts_seeded_noise(long npts, double amp, unsigned seed, float *out);
void ts_seeded_spectrum(int lmax, int mmax, unsigned seed, float *qlm);

#ifdef __cplusplus
}
#endif

#endif /* TURING_SHT_H */
