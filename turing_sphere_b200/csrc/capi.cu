// C ABI entry points: context, layout helpers, SHT plans and transforms.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "runtime.h"

namespace {

int fail(ts_ctx ctx, const ts_exc &e) {
  ts_set_error(ctx, e.msg);
  return e.code;
}

#define TS_API_BEGIN try {
#define TS_API_END(ctx)                                           \
  }                                                               \
  catch (const ts_exc &e) {                                       \
    return fail(ctx, e);                                          \
  }                                                               \
  catch (const std::exception &e) {                               \
    return fail(ctx, ts_exc{TS_ERR_INVALID, e.what()});           \
  }                                                               \
  catch (...) {                                                   \
    return fail(ctx, ts_exc{TS_ERR_INVALID, "unknown exception"}); \
  }                                                               \
  return TS_OK;

thread_local std::string g_noctx_err;

std::string config_error(int lmax, int mmax, int nlat, int nphi) {
  char buf[256];
  if (lmax < 1) {
    snprintf(buf, sizeof buf, "lmax must be an integer >= 1 (got %d)", lmax);
    return buf;
  }
  if (mmax < 0 || mmax > lmax) {
    snprintf(buf, sizeof buf, "mmax must be an integer in [0, lmax] (got %d)", mmax);
    return buf;
  }
  if (nlat <= lmax) {
    snprintf(buf, sizeof buf,
             "nlat must be an integer > lmax for exact Gauss quadrature (got nlat=%d, lmax=%d)",
             nlat, lmax);
    return buf;
  }
  if (nphi < 2 * mmax + 1) {
    snprintf(buf, sizeof buf,
             "nphi must be an integer >= 2*mmax+1 to avoid aliasing (got nphi=%d, mmax=%d)", nphi,
             mmax);
    return buf;
  }
  return "";
}

// H = nphi/2 = 2^a 3^b -> Stockham radices (3s first, then 4s, one 2 if a odd)
bool fft_radices(int nphi, TsFftTab &ft) {
  if (nphi % 2) return false;
  int H = nphi / 2, a = 0, b = 0;
  while (H % 2 == 0) {
    H /= 2;
    a++;
  }
  while (H % 3 == 0) {
    H /= 3;
    b++;
  }
  if (H != 1) return false;
  int n = 0;
  for (int i = 0; i < b; i++) ft.radix[n++] = 3;
  for (int i = 0; i < a / 2; i++) ft.radix[n++] = 4;
  if (a & 1) ft.radix[n++] = 2;
  if (n > 16) return false;
  ft.nst = n;
  return true;
}

void plan_free(ts_plan p) {
  for (void *q : {(void *)p->d_x64, (void *)p->d_w64, (void *)p->d_ab64, (void *)p->d_amm64,
                  (void *)p->d_ct, (void *)p->d_st, (void *)p->d_wq, (void *)p->d_amm,
                  (void *)p->d_ab, (void *)p->d_tw})
    if (q) cudaFree(q);
  p->fm.release();
  p->stage_q.release();
  p->stage_q2.release();
  p->stage_s.release();
  p->adj_grid.release();
  p->adj_spec.release();
  ts_tc_free(p);
}

void check_batch(ts_plan p, const void *a, const void *b, int batch) {
  TS_REQUIRE(p != nullptr, TS_ERR_INVALID, "null plan");
  TS_REQUIRE(a != nullptr && b != nullptr, TS_ERR_INVALID, "null buffer");
  TS_REQUIRE(batch >= 1 && batch <= 65535, TS_ERR_INVALID, "batch must be in [1, 65535]");
  ts_require_aligned8(a, b);
}

long npts_of(ts_plan p) { return (long)p->nlat * p->nphi; }

}  // namespace

void ts_synth_dev(ts_plan p, const float *qlm, float *spat, int batch, cudaStream_t s) {
  const long fm_stride = (long)(p->mmax + 1) * p->nlat;
  p->fm.ensure(sizeof(float2) * fm_stride * batch);
  float2 *fm = (float2 *)p->fm.p;
  ts_launch_leg_synth(p, (const float2 *)qlm, p->nlm, fm, fm_stride, batch, s);
  ts_launch_fourier_synth(p, fm, fm_stride, spat, npts_of(p), batch, s);
}

void ts_analys_dev(ts_plan p, const float *spat, float *qlm, int batch, cudaStream_t s) {
  if (p->precision != TS_PREC_FP32) return ts_analys_tc_full(p, spat, npts_of(p), qlm, batch, s);
  const long fm_stride = (long)(p->mmax + 1) * p->nlat;
  p->fm.ensure(sizeof(float2) * fm_stride * batch);
  float2 *fm = (float2 *)p->fm.p;
  ts_launch_fourier_analys(p, spat, npts_of(p), fm, fm_stride, batch, s);
  ts_launch_leg_analys(p, fm, fm_stride, (float2 *)qlm, p->nlm, batch, s);
}

namespace {
void synth_dev(ts_plan p, const float *qlm, float *spat, int batch, cudaStream_t s) {
  ts_synth_dev(p, qlm, spat, batch, s);
}
void analys_dev(ts_plan p, const float *spat, float *qlm, int batch, cudaStream_t s) {
  ts_analys_dev(p, spat, qlm, batch, s);
}
}  // namespace

void ts_set_error(ts_ctx ctx, const std::string &msg) {
  if (ctx)
    ctx->err = msg;
  else
    g_noctx_err = msg;
}

void ts_plan_take_timeout(ts_plan p) {
  if (!ts_tc_check_error(p)) return;
  int zero = 0;
  TS_CUDA(cudaMemcpy(ts_tc_tab(p).err, &zero, sizeof(int), cudaMemcpyHostToDevice));
  ts_throw(TS_ERR_TIMEOUT, "a tensor-core kernel gave up a bounded wait: its results are incomplete");
}

cudaStream_t ts_pick_stream(ts_ctx ctx, void *stream) {
  return stream ? (cudaStream_t)stream : ctx->stream;
}

namespace {
using ts_ctx_get_fn = CUresult (*)(CUcontext *);
using ts_ctx_set_fn = CUresult (*)(CUcontext);
struct ts_ctx_fns {
  ts_ctx_get_fn get = nullptr;
  ts_ctx_set_fn set = nullptr;
};
// the driver's current-context calls, through the runtime's entry-point
// table (the library links the runtime only)
const ts_ctx_fns &ctx_fns() {
  static const ts_ctx_fns fns = [] {
    ts_ctx_fns f;
    void *g = nullptr, *s = nullptr;
    cudaDriverEntryPointQueryResult q1, q2;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &g, 12000, cudaEnableDefault, &q1) ==
            cudaSuccess &&
        q1 == cudaDriverEntryPointSuccess &&
        cudaGetDriverEntryPointByVersion("cuCtxSetCurrent", &s, 12000, cudaEnableDefault, &q2) ==
            cudaSuccess &&
        q2 == cudaDriverEntryPointSuccess) {
      f.get = (ts_ctx_get_fn)g;
      f.set = (ts_ctx_set_fn)s;
    }
    return f;
  }();
  return fns;
}
}  // namespace

namespace {
void check_host_batch(ts_plan p, const void *a, const void *b, int batch) {
  TS_REQUIRE(p != nullptr, TS_ERR_INVALID, "null plan");
  TS_REQUIRE(a != nullptr && b != nullptr, TS_ERR_INVALID, "null buffer");
  TS_REQUIRE(batch >= 1 && batch <= 65535, TS_ERR_INVALID, "batch must be in [1, 65535]");
}

void require_len(const char *name, long got, long want) {
  if (got == want) return;
  char buf[128];
  snprintf(buf, sizeof buf, "%s must have length %ld", name, want);
  ts_throw(TS_ERR_SIZE, buf);
}

// Fields per chunk of a host-array transform.  The pipeline ends one chunk's
// transform and device->host copy after the last host->device copy, while a
// chunk's transform has a fixed cost (tensor-core tiles of 64 fields) that
// the copies must hide.  Fields of 192 KB or more (lmax >= 255) go 24 at a
// time: on B200 (55 GB/s one way, 45 GB/s each way at once) the round trip
// of 256 fields at lmax 255 measured 1.68 ms in chunks of 24 against 1.83
// for 20, 1.84 for 28, 1.95 for 32 and 64, 2.07 for 16; 64 fields at lmax 511
// 2.20 ms in chunks of 20-24 against 2.35 for 16 and 3.10 for 64.  Smaller
// fields (lmax 63, 127: the fixed cost dominates) go a quarter of the batch
// at a time, a multiple of 16 fields with at most 64 MB of the larger host
// array, and a batch under 32 fields in one piece.  TS_HOST_CHUNK overrides it.
int host_chunk(int batch, long floats_per_field) {
  if (const char *e = getenv("TS_HOST_CHUNK")) {
    const int c = atoi(e);
    if (c > 0) return std::min(c, batch);
  }
  if (4 * floats_per_field >= (192L << 10)) return std::min(24, batch);
  if (batch < 32) return batch;
  long c = ((batch + 3) / 4 + 15) / 16 * 16;
  const long cap = std::max(16L, (64L << 20) / (4 * floats_per_field) / 16 * 16);
  return (int)std::min<long>(std::min(c, cap), batch);
}

void ensure_copy_streams(ts_ctx ctx, size_t nevents) {
  if (!ctx->copy_in) TS_CUDA(cudaStreamCreateWithFlags(&ctx->copy_in, cudaStreamNonBlocking));
  if (!ctx->copy_out) TS_CUDA(cudaStreamCreateWithFlags(&ctx->copy_out, cudaStreamNonBlocking));
  while (ctx->events.size() < nevents) {
    cudaEvent_t e;
    TS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ctx->events.push_back(e);
  }
}

// A blocking host-array transform as a pipeline over chunks of fields:
// chunk c's host->device copy (copy_in stream), its transform `fn` (the
// context's stream) and its device->host copy (copy_out stream) are ordered
// by events, so copies of one chunk overlap the transform of another and the
// two copy directions run at once.  `din`/`dout` are device staging arrays
// for the whole batch (each chunk has its own slice, so nothing is reused
// while in flight).  All host->device copies and transforms are enqueued
// before the first device->host copy: a pageable destination makes that copy
// block the host until its chunk is done, which then delays nothing else.
// Page-locked host arrays (cudaHostAlloc, cudaHostRegister) give the full
// overlap; pageable ones are copied through the driver's staging.  Returns
// when every copy has landed; on an error it waits for whatever was enqueued
// before rethrowing, so no copy still touches the caller's arrays.
template <class Fn>
void host_pipeline(ts_plan p, const float *in, long in_pf, float *din, float *out, long out_pf,
                   float *dout, int batch, int chunk, Fn fn) {
  ts_ctx ctx = p->ctx;
  const int nch = (batch + chunk - 1) / chunk;
  ensure_copy_streams(ctx, 2 * (size_t)nch + 1);
  cudaStream_t s = ctx->stream;
  try {
    // the staging arrays are idle once the work queued before this call is done
    TS_CUDA(cudaEventRecord(ctx->events[2 * nch], s));
    TS_CUDA(cudaStreamWaitEvent(ctx->copy_in, ctx->events[2 * nch], 0));
    for (int c = 0; c < nch; c++) {
      const long f0 = (long)c * chunk;
      const int nf = std::min<int>(chunk, batch - (int)f0);
      TS_CUDA(cudaMemcpyAsync(din + f0 * in_pf, in + f0 * in_pf, sizeof(float) * nf * in_pf,
                              cudaMemcpyHostToDevice, ctx->copy_in));
      TS_CUDA(cudaEventRecord(ctx->events[2 * c], ctx->copy_in));
      TS_CUDA(cudaStreamWaitEvent(s, ctx->events[2 * c], 0));
      fn(din + f0 * in_pf, dout + f0 * out_pf, nf, s);
      TS_CUDA(cudaEventRecord(ctx->events[2 * c + 1], s));
    }
    for (int c = 0; c < nch; c++) {
      const long f0 = (long)c * chunk;
      const int nf = std::min<int>(chunk, batch - (int)f0);
      TS_CUDA(cudaStreamWaitEvent(ctx->copy_out, ctx->events[2 * c + 1], 0));
      TS_CUDA(cudaMemcpyAsync(out + f0 * out_pf, dout + f0 * out_pf, sizeof(float) * nf * out_pf,
                              cudaMemcpyDeviceToHost, ctx->copy_out));
    }
    TS_CUDA(cudaStreamSynchronize(ctx->copy_out));
    TS_CUDA(cudaStreamSynchronize(s));
  } catch (...) {
    cudaStreamSynchronize(ctx->copy_in);
    cudaStreamSynchronize(s);
    cudaStreamSynchronize(ctx->copy_out);
    throw;
  }
}
}  // namespace

ts_device_guard::ts_device_guard(int device, bool nothrow) {
  const ts_ctx_fns &f = ctx_fns();
  CUcontext prev = nullptr;
  if (f.get && f.get(&prev) == CUDA_SUCCESS) {
    prev_ = (void *)prev;
    saved_ = true;
  }
  const cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) {
    ok_ = false;
    if (!nothrow) {
      saved_ = false;  // the destructor does not run when the constructor throws
      ts_throw(TS_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    }
  }
}

ts_device_guard::~ts_device_guard() {
  if (!saved_) return;
  const ts_ctx_fns &f = ctx_fns();
  CUcontext cur = nullptr;
  if (f.get(&cur) == CUDA_SUCCESS && cur != (CUcontext)prev_) f.set((CUcontext)prev_);
}

extern "C" {

// ------------------------------------------------------------------ context

int ts_ctx_create(int device_ordinal, ts_ctx *out) {
  ts_ctx ctx = nullptr;
  try {
    TS_REQUIRE(out != nullptr, TS_ERR_INVALID, "null output handle");
    int n = 0;
    TS_CUDA(cudaGetDeviceCount(&n));
    TS_REQUIRE(device_ordinal >= 0 && device_ordinal < n, TS_ERR_INVALID,
               "device ordinal out of range");
    ctx = new ts_ctx_s();
    ctx->device = device_ordinal;
    ts_device_guard dev_guard_(device_ordinal);
    cudaDeviceProp prop;
    TS_CUDA(cudaGetDeviceProperties(&prop, device_ordinal));
    ctx->sm_count = prop.multiProcessorCount;
    ctx->smem_optin = prop.sharedMemPerBlockOptin;
    ctx->name = prop.name;
    TS_CUDA(cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking));
    ctx->stream = ctx->own_stream;
    ts_kernel_attrs_once(ctx);
    *out = ctx;
    return TS_OK;
  } catch (const ts_exc &e) {
    g_noctx_err = e.msg;
    if (ctx) {
      if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
      delete ctx;
    }
    return e.code;
  }
}

int ts_ctx_destroy(ts_ctx ctx) {
  if (!ctx) return TS_ERR_INVALID;
  ts_device_guard dev_guard_(ctx->device, true);
  if (ctx->own_stream) {
    cudaStreamSynchronize(ctx->own_stream);
    cudaStreamDestroy(ctx->own_stream);
  }
  for (cudaStream_t st : {ctx->copy_in, ctx->copy_out})
    if (st) {
      cudaStreamSynchronize(st);
      cudaStreamDestroy(st);
    }
  for (cudaEvent_t e : ctx->events) cudaEventDestroy(e);
  delete ctx;
  return TS_OK;
}

const char *ts_last_error(ts_ctx ctx) { return ctx ? ctx->err.c_str() : g_noctx_err.c_str(); }

int ts_ctx_set_stream(ts_ctx ctx, void *stream) {
  if (!ctx) return TS_ERR_INVALID;
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
  return TS_OK;
}

void *ts_ctx_stream(ts_ctx ctx) { return ctx ? (void *)ctx->stream : nullptr; }

int ts_ctx_device_name(ts_ctx ctx, char *buf, size_t cap) {
  if (!ctx || !buf || cap == 0) return TS_ERR_INVALID;
  snprintf(buf, cap, "%s", ctx->name.c_str());
  return TS_OK;
}

int ts_sync(ts_ctx ctx) {
  TS_API_BEGIN
  TS_REQUIRE(ctx != nullptr, TS_ERR_INVALID, "null context");
  ts_device_guard dev_guard_(ctx->device);
  TS_CUDA(cudaStreamSynchronize(ctx->stream));
  TS_API_END(ctx)
}

// ------------------------------------------------------------------- layout

long ts_nlm_calc(int lmax, int mmax) {
  return (long)(mmax + 1) * (lmax + 1) - (long)mmax * (mmax + 1) / 2;
}

long ts_lm_index(int lmax, int l, int m) {
  return (long)m * (lmax + 1) - (long)m * (m - 1) / 2 + (l - m);
}

int ts_validate_config(int lmax, int mmax, int nlat, int nphi, char *buf, size_t cap) {
  const std::string e = config_error(lmax, mmax, nlat, nphi);
  if (buf && cap) snprintf(buf, cap, "%s", e.c_str());
  return e.empty() ? TS_OK : TS_ERR_INVALID;
}

void ts_grid_for_lmax(int lmax, int pdeg, int *nlat, int *nphi) {
  double minlat = ((double)(pdeg + 1) * lmax + 1) / 2.0;
  if (minlat < lmax + 1) minlat = lmax + 1;
  *nlat = 2 * (int)std::ceil(minlat / 2.0);
  int n = 1;
  while (n < (pdeg + 1) * lmax + 1) n *= 2;
  *nphi = n;
}

// --------------------------------------------------------------------- plan

int ts_sht_plan_create(ts_ctx ctx, int lmax, int mmax, int nlat, int nphi, int flags,
                       ts_plan *out) {
  ts_plan p = nullptr;
  try {
    TS_REQUIRE(ctx != nullptr, TS_ERR_INVALID, "null context");
    TS_REQUIRE(out != nullptr, TS_ERR_INVALID, "null output handle");
    const std::string e = config_error(lmax, mmax, nlat, nphi);
    TS_REQUIRE(e.empty(), TS_ERR_INVALID, e);
    ts_device_guard dev_guard_(ctx->device);
    p = new ts_plan_s();
    p->ctx = ctx;
    p->lmax = lmax;
    p->mmax = mmax;
    p->nlat = nlat;
    p->nphi = nphi;
    p->nh = (nlat + 1) / 2;
    p->nlm = ts_nlm_calc(lmax, mmax);
    p->precision = flags & TS_PREC_MASK;
    TS_REQUIRE(p->precision == TS_PREC_FP32 || p->precision == TS_PREC_TF32X3 ||
                   p->precision == TS_PREC_BF16X3,
               TS_ERR_INVALID, "unknown precision flag");
    p->fft.nphi = nphi;
    p->fft.H = nphi / 2;
    p->fft.mmax = mmax;
    p->fft.nlat = nlat;
    const int want = flags & TS_FOURIER_MASK;
    const bool fft_ok = fft_radices(nphi, p->fft);
    if (want == TS_FOURIER_FFT && !fft_ok) {
      char buf[160];
      snprintf(buf, sizeof buf, "fourier 'fft' requires nphi = 2^a 3^b with a >= 1 (nphi=%d)", nphi);
      ts_throw(TS_ERR_INVALID, buf);
    }
    p->fourier = (want == TS_FOURIER_DFT || !fft_ok) ? TS_FOURIER_DFT : TS_FOURIER_FFT;
    if (p->fourier == TS_FOURIER_DFT) p->fft.nst = 0;
    ts_init_tables(p);
    if (p->precision == TS_PREC_BF16X3)
      ts_throw(TS_ERR_UNSUPPORTED, "split-BF16 tensor-core Legendre is not built; use TF32x3");
    if (p->precision == TS_PREC_TF32X3) ts_tc_init(p);
    // TS_FFT_ALT=1 selects the FFT's second split where the row length has
    // one (what the autotuner may also choose)
    if (const char *e = getenv("TS_FFT_ALT")) p->fft_alt = atoi(e) != 0 && ts_f2_has_alt(p);
    if (flags & TS_PLAN_AUTOTUNE) ts_autotune(p);
    *out = p;
    return TS_OK;
  } catch (const ts_exc &e) {
    if (p) {
      plan_free(p);
      delete p;
    }
    ts_set_error(ctx, e.msg);
    return e.code;
  }
}

int ts_sht_plan_destroy(ts_plan p) {
  if (!p) return TS_ERR_INVALID;
  ts_device_guard dev_guard_(p->ctx->device, true);
  cudaStreamSynchronize(p->ctx->stream);
  plan_free(p);
  delete p;
  return TS_OK;
}

int ts_sht_plan_info(ts_plan p, ts_plan_info *info) {
  if (!p || !info) return TS_ERR_INVALID;
  memset(info, 0, sizeof(*info));
  info->lmax = p->lmax;
  info->mmax = p->mmax;
  info->nlat = p->nlat;
  info->nphi = p->nphi;
  info->nlm = p->nlm;
  info->precision = p->precision;
  info->fourier = p->fourier;
  info->fft_stages = p->fourier == TS_FOURIER_FFT ? p->fft.nst : 0;
  info->table_bytes = (long)ts_tc_bytes(p);
  for (int i = 0; i < info->fft_stages; i++) info->fft_radix[i] = p->fft.radix[i];
  if (p->tc) {
    const TsTcGeom g = ts_tc_geom(p);
    info->tc_lat_tile = g.NL;
    info->tc_deg_tile = g.LTL;
    ts_tc_skip_counts(p, &info->tc_skip_tiles, &info->tc_skip_chunks);
  }
  int P = 0, Q = 0;
  if (ts_f2_shape(p, &P, &Q)) {
    info->fft_p = P;
    info->fft_q = Q;
    info->fft_rows = ts_f2_rows(p);
  }
  info->tuned = p->tuned ? 1 : 0;
  return TS_OK;
}

int ts_sht_plan_test_stall(ts_plan p, int stall_copies, unsigned wait_limit) {
  ts_ctx ctx = p ? p->ctx : nullptr;
  TS_API_BEGIN
  TS_REQUIRE(p != nullptr, TS_ERR_INVALID, "null plan");
  TS_REQUIRE(p->tc != nullptr, TS_ERR_UNSUPPORTED, "FP32 plans have no bounded waits");
  ts_device_guard dev_guard_(ctx->device);
  TS_CUDA(cudaStreamSynchronize(ctx->stream));
  ts_tc_set_fault(p, stall_copies, wait_limit);
  TS_API_END(ctx)
}

int ts_sht_plan_status(ts_plan p) {
  ts_ctx ctx = p ? p->ctx : nullptr;
  TS_API_BEGIN
  TS_REQUIRE(p != nullptr, TS_ERR_INVALID, "null plan");
  ts_device_guard dev_guard_(ctx->device);
  TS_CUDA(cudaStreamSynchronize(ctx->stream));
  ts_plan_take_timeout(p);
  TS_API_END(ctx)
}

int ts_sht_plan_nodes(ts_plan p, double *cos_theta, double *weights) {
  if (!p) return TS_ERR_INVALID;
  if (cos_theta) memcpy(cos_theta, p->h_x.data(), sizeof(double) * p->nlat);
  if (weights) memcpy(weights, p->h_w.data(), sizeof(double) * p->nlat);
  return TS_OK;
}

// ---------------------------------------------------------------- transforms

int ts_sht_synth_dev(ts_plan p, const float *qlm, float *spat, int batch, void *stream) {
  ts_ctx ctx = p ? p->ctx : nullptr;
  TS_API_BEGIN
  check_batch(p, qlm, spat, batch);
  ts_device_guard dev_guard_(ctx->device);
  synth_dev(p, qlm, spat, batch, ts_pick_stream(ctx, stream));
  TS_API_END(ctx)
}

int ts_sht_analys_dev(ts_plan p, const float *spat, float *qlm, int batch, void *stream) {
  ts_ctx ctx = p ? p->ctx : nullptr;
  TS_API_BEGIN
  check_batch(p, spat, qlm, batch);
  ts_device_guard dev_guard_(ctx->device);
  analys_dev(p, spat, qlm, batch, ts_pick_stream(ctx, stream));
  TS_API_END(ctx)
}

int ts_sht_synth(ts_plan p, const float *qlm, long qlm_len, float *spat, long spat_len,
                 int batch) {
  ts_ctx ctx = p ? p->ctx : nullptr;
  TS_API_BEGIN
  check_host_batch(p, qlm, spat, batch);
  require_len("qlm", qlm_len, 2 * p->nlm * batch);
  require_len("spat", spat_len, npts_of(p) * batch);
  ts_device_guard dev_guard_(ctx->device);
  const int chunk = host_chunk(batch, std::max<long>(2 * p->nlm, npts_of(p)));
  p->stage_q.ensure(sizeof(float) * 2 * p->nlm * batch);
  p->stage_s.ensure(sizeof(float) * npts_of(p) * batch);
  host_pipeline(p, qlm, 2 * p->nlm, (float *)p->stage_q.p, spat, npts_of(p),
                (float *)p->stage_s.p, batch, chunk,
                [&](const float *din, float *dout, int nf, cudaStream_t s) {
                  synth_dev(p, din, dout, nf, s);
                });
  TS_API_END(ctx)
}

int ts_sht_analys(ts_plan p, const float *spat, long spat_len, float *qlm, long qlm_len,
                  int batch) {
  ts_ctx ctx = p ? p->ctx : nullptr;
  TS_API_BEGIN
  check_host_batch(p, spat, qlm, batch);
  require_len("spat", spat_len, npts_of(p) * batch);
  require_len("qlm", qlm_len, 2 * p->nlm * batch);
  ts_device_guard dev_guard_(ctx->device);
  const int chunk = host_chunk(batch, std::max<long>(2 * p->nlm, npts_of(p)));
  p->stage_s.ensure(sizeof(float) * npts_of(p) * batch);
  p->stage_q.ensure(sizeof(float) * 2 * p->nlm * batch);
  host_pipeline(p, spat, npts_of(p), (float *)p->stage_s.p, qlm, 2 * p->nlm,
                (float *)p->stage_q.p, batch, chunk,
                [&](const float *din, float *dout, int nf, cudaStream_t s) {
                  analys_dev(p, din, dout, nf, s);
                });
  TS_API_END(ctx)
}

int ts_sht_roundtrip(ts_plan p, const float *qlm_in, long in_len, float *qlm_out, long out_len,
                     int batch) {
  ts_ctx ctx = p ? p->ctx : nullptr;
  TS_API_BEGIN
  check_host_batch(p, qlm_in, qlm_out, batch);
  require_len("qlm_in", in_len, 2 * p->nlm * batch);
  require_len("qlm_out", out_len, 2 * p->nlm * batch);
  ts_device_guard dev_guard_(ctx->device);
  const int chunk = host_chunk(batch, 2 * p->nlm);
  p->stage_q.ensure(sizeof(float) * 2 * p->nlm * batch);
  p->stage_q2.ensure(sizeof(float) * 2 * p->nlm * batch);
  p->stage_s.ensure(sizeof(float) * npts_of(p) * chunk);
  float *grid = (float *)p->stage_s.p;
  host_pipeline(p, qlm_in, 2 * p->nlm, (float *)p->stage_q.p, qlm_out, 2 * p->nlm,
                (float *)p->stage_q2.p, batch, chunk,
                [&](const float *din, float *dout, int nf, cudaStream_t s) {
                  synth_dev(p, din, grid, nf, s);
                  analys_dev(p, grid, dout, nf, s);
                });
  TS_API_END(ctx)
}

int ts_sht_leg_synth_dev(ts_plan p, const float *qlm, float *fm, int batch, void *stream) {
  ts_ctx ctx = p ? p->ctx : nullptr;
  TS_API_BEGIN
  check_batch(p, qlm, fm, batch);
  ts_device_guard dev_guard_(ctx->device);
  ts_launch_leg_synth(p, (const float2 *)qlm, p->nlm, (float2 *)fm, (long)(p->mmax + 1) * p->nlat,
                      batch, ts_pick_stream(ctx, stream));
  TS_API_END(ctx)
}

int ts_sht_fourier_synth_dev(ts_plan p, const float *fm, float *spat, int batch, void *stream) {
  ts_ctx ctx = p ? p->ctx : nullptr;
  TS_API_BEGIN
  check_batch(p, fm, spat, batch);
  ts_device_guard dev_guard_(ctx->device);
  ts_launch_fourier_synth(p, (const float2 *)fm, (long)(p->mmax + 1) * p->nlat, spat, npts_of(p),
                          batch, ts_pick_stream(ctx, stream));
  TS_API_END(ctx)
}

int ts_sht_fourier_analys_dev(ts_plan p, const float *spat, float *fm, int batch, void *stream) {
  ts_ctx ctx = p ? p->ctx : nullptr;
  TS_API_BEGIN
  check_batch(p, spat, fm, batch);
  ts_device_guard dev_guard_(ctx->device);
  ts_launch_fourier_analys(p, spat, npts_of(p), (float2 *)fm, (long)(p->mmax + 1) * p->nlat,
                           batch, ts_pick_stream(ctx, stream));
  TS_API_END(ctx)
}

int ts_sht_leg_analys_dev(ts_plan p, const float *fm, float *qlm, int batch, void *stream) {
  ts_ctx ctx = p ? p->ctx : nullptr;
  TS_API_BEGIN
  check_batch(p, fm, qlm, batch);
  ts_device_guard dev_guard_(ctx->device);
  ts_launch_leg_analys(p, (const float2 *)fm, (long)(p->mmax + 1) * p->nlat, (float2 *)qlm,
                       p->nlm, batch, ts_pick_stream(ctx, stream));
  TS_API_END(ctx)
}

size_t ts_sht_wimage_bytes(ts_plan p, int batch) {
  if (!p || p->precision == TS_PREC_FP32 || batch < 1) return 0;
  return ts_tc_wimg_bytes(p, batch, TS_TC_FIELDS);
}

int ts_sht_fourier_analys_w_dev(ts_plan p, const float *spat, void *wimage, int batch,
                                void *stream) {
  ts_ctx ctx = p ? p->ctx : nullptr;
  TS_API_BEGIN
  check_batch(p, spat, wimage, batch);
  TS_REQUIRE(p->precision != TS_PREC_FP32, TS_ERR_UNSUPPORTED, "FP32 plans have no W image");
  ts_device_guard dev_guard_(ctx->device);
  TS_REQUIRE(ts_launch_fourier_analys_w(p, spat, npts_of(p), batch, TS_TC_FIELDS, (char *)wimage,
                                        ts_pick_stream(ctx, stream)),
             TS_ERR_UNSUPPORTED, "the plan's row length has no two-phase FFT shape");
  TS_API_END(ctx)
}

int ts_sht_leg_analys_w_dev(ts_plan p, const void *wimage, float *qlm, int batch, void *stream) {
  ts_ctx ctx = p ? p->ctx : nullptr;
  TS_API_BEGIN
  check_batch(p, wimage, qlm, batch);
  TS_REQUIRE(p->precision != TS_PREC_FP32, TS_ERR_UNSUPPORTED, "FP32 plans have no W image");
  ts_device_guard dev_guard_(ctx->device);
  ts_launch_analys_tc_img(p, (const char *)wimage, batch, (float2 *)qlm, p->nlm,
                          ts_pick_stream(ctx, stream));
  TS_API_END(ctx)
}

}  // extern "C"

// ----------------------------------------------------------------- seeding
// mulberry32 uniform deviates and Box-Muller normals with a spare (the
// generators of src/mgpu/noise.ts:15-51): integer state, then one division
// by 2^32, so any faithful implementation draws the same sequence.
namespace {
struct Mulberry {
  uint32_t s;
  bool have = false;
  double spare = 0;
  double uniform() {
    s += 0x6d2b79f5u;
    uint32_t t = s;
    t = (t ^ (t >> 15)) * (t | 1u);
    t ^= t + (t ^ (t >> 7)) * (t | 61u);
    return (double)(t ^ (t >> 14)) / 4294967296.0;
  }
  double normal() {
    if (have) {
      have = false;
      return spare;
    }
    double u = 0;
    while (u == 0) u = uniform();
    const double r = std::sqrt(-2.0 * std::log(u));
    const double th = 2.0 * M_PI * uniform();
    spare = r * std::sin(th);
    have = true;
    return r * std::cos(th);
  }
};
}  // namespace

extern "C" void ts_seeded_noise(long npts, double amp, unsigned seed, float *out) {
  Mulberry g{seed};
  for (long i = 0; i < npts; i++) out[i] = (float)(amp * g.normal());
}

extern "C" void ts_seeded_spectrum(int lmax, int mmax, unsigned seed, float *qlm) {
  Mulberry g{seed};
  long lm = 0;
  for (int m = 0; m <= mmax; m++)
    for (int l = m; l <= lmax; l++, lm++) {
      qlm[2 * lm] = (float)(2.0 * g.uniform() - 1.0);
      const float im = (float)(2.0 * g.uniform() - 1.0);
      qlm[2 * lm + 1] = m == 0 ? 0.0f : im;
    }
}
