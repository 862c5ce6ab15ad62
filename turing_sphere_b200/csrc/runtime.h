// Internal runtime types of libturing_sht.so (not part of the C ABI).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/turing_sht.h"
#include "kernels/ts_common.cuh"

struct ts_exc {
  int code;
  std::string msg;
};

[[noreturn]] inline void ts_throw(int code, const std::string &msg) { throw ts_exc{code, msg}; }

#define TS_CUDA(call)                                                                \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess)                                                           \
      ts_throw(TS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));     \
  } while (0)

#define TS_REQUIRE(cond, code, msg) \
  do {                              \
    if (!(cond)) ts_throw(code, msg); \
  } while (0)

// Device arrays of the transforms hold complex pairs and grid rows that the
// kernels read and write as float2 (8 bytes); a float pointer that is only
// 4-byte aligned is refused before any launch.
inline void ts_require_aligned8(const void *a, const void *b) {
  TS_REQUIRE(((reinterpret_cast<unsigned long long>(a) | reinterpret_cast<unsigned long long>(b)) &
              7) == 0,
             TS_ERR_INVALID,
             "device arrays must be 8-byte aligned (coefficient pairs and grid rows are read "
             "as float2)");
}

// Makes `device` current for the lifetime of the guard (one C-ABI call) and
// then gives the calling thread back the CUDA context it had before the call,
// including none: a caller working on another device, or one that never
// touched CUDA, finds its thread as it left it.  The saved context is read
// and restored through the driver (cuCtxGetCurrent / cuCtxSetCurrent, looked
// up once through the runtime), so restoring never creates a primary context
// on a device the caller did not use.  `nothrow` guards (destroy calls) report
// a failed cudaSetDevice by leaving ok() false instead of throwing.
class ts_device_guard {
 public:
  explicit ts_device_guard(int device, bool nothrow = false);
  ~ts_device_guard();
  bool ok() const { return ok_; }
  ts_device_guard(const ts_device_guard &) = delete;
  ts_device_guard &operator=(const ts_device_guard &) = delete;

 private:
  void *prev_ = nullptr;  // CUcontext current on entry (may be null)
  bool saved_ = false, ok_ = true;
};

struct ts_ctx_s {
  int device = 0;
  int sm_count = 0;
  size_t smem_optin = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  // host-array transforms: copy streams (host->device, device->host) and a
  // pool of ordering events, created on first use
  cudaStream_t copy_in = nullptr, copy_out = nullptr;
  std::vector<cudaEvent_t> events;
  std::string err;
  std::string name;
};

// Device buffer with grow-on-demand capacity (bytes).
struct ts_dbuf {
  void *p = nullptr;
  size_t cap = 0;
  void ensure(size_t bytes) {
    if (bytes <= cap) return;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    TS_CUDA(cudaMalloc(&p, bytes));
    cap = bytes;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

struct ts_plan_s {
  ts_ctx ctx = nullptr;
  int lmax = 0, mmax = 0, nlat = 0, nphi = 0, nh = 0;
  long nlm = 0;
  int precision = TS_PREC_FP32;
  int fourier = TS_FOURIER_FFT;
  // FP64 nodes/weights as computed on the GPU, host copies
  std::vector<double> h_x, h_w;
  // device tables
  double *d_x64 = nullptr, *d_w64 = nullptr, *d_ab64 = nullptr, *d_amm64 = nullptr;
  float *d_ct = nullptr, *d_st = nullptr, *d_wq = nullptr, *d_amm = nullptr;
  float2 *d_ab = nullptr, *d_tw = nullptr;
  TsLegTab leg{};
  TsFftTab fft{};
  // scratch: fm intermediate, host-call staging, adjoint scalings
  ts_dbuf fm, stage_q, stage_s, stage_q2, adj_grid, adj_spec;
  // tensor-core tables (precision != FP32)
  void *tc = nullptr;
  // kernel shapes: 0 = default (or TS_TC_NL / TS_TC_LTL); set by the autotuner
  int tune_nl = 0, tune_ltl = 0, fft_rows = 0;
  // the FFT's second P*Q split (TS_F2_ALT_SHAPES) instead of the default one
  bool fft_alt = false;
  bool tuned = false;
};

// whole transforms on device buffers (capi.cu) and their adjoints (adjoint.cu)
void ts_synth_dev(ts_plan p, const float *qlm, float *spat, int batch, cudaStream_t s);
void ts_analys_dev(ts_plan p, const float *spat, float *qlm, int batch, cudaStream_t s);
void ts_synth_adjoint(ts_plan p, const float *gbar, float *qbar, int nf, cudaStream_t s);
void ts_analys_adjoint(ts_plan p, const float *qbar, float *gbar, int nf, cudaStream_t s);

// autotune.cu: time the candidate kernel shapes of a plan, keep the fastest
void ts_autotune(ts_plan p);
// rows per two-phase FFT CTA in use (0 when the plan's rows have no shape)
int ts_f2_rows(ts_plan p);

cudaStream_t ts_pick_stream(ts_ctx ctx, void *stream);
void ts_set_error(ts_ctx ctx, const std::string &msg);

// launchers (sht_kernels.cu)
void ts_launch_leg_synth(ts_plan p, const float2 *q, long q_stride, float2 *fm, long fm_stride,
                         int nfields, cudaStream_t s);
void ts_launch_leg_analys(ts_plan p, const float2 *g, long g_stride, float2 *q, long q_stride,
                          int nfields, cudaStream_t s);
void ts_launch_fourier_synth(ts_plan p, const float2 *fm, long fm_stride, float *spat,
                             long spat_stride, int nfields, cudaStream_t s);
void ts_launch_fourier_analys(ts_plan p, const float *spat, long spat_stride, float2 *g,
                              long g_stride, int nfields, cudaStream_t s);
void ts_launch_leg_synth_fields(ts_plan p, const TsFields &q, float2 *fm, long fm_stride,
                                int nfields, cudaStream_t s);
// the FP32 on-the-fly recurrence whatever the plan's precision (allocates nothing)
void ts_launch_leg_synth_plain(ts_plan p, const TsFields &q, float2 *fm, long fm_stride,
                               int nfields, cudaStream_t s);
// analysis launch shape: fields per CTA F (template), latitudes per thread K,
// warps W; groups = fields handled per CTA (a multiple of `per_inst`)
void ts_analys_shape(ts_plan p, int nfields, int per_inst, int *F, int *K, int *W, int *per_cta);
size_t ts_analys_smem(ts_plan p, int F, int W);
int ts_analys_lchunk(ts_plan p, int nfb);
// rows per Fourier CTA for a kernel holding `nrows` rows per warp
int ts_fourier_lb(ts_plan p, int nblocks_y, int nrows, size_t *smem);
// warp-register FFT: R1 = H/32 (0 = not applicable) and rows per CTA
// two-phase FFT (kernels/fft2.cuh): the plan's shape H = P*Q (false: none,
// the Stockham kernels run), its shared memory, and the rows of a phase CTA
bool ts_f2_shape(ts_plan p, int *P, int *Q);
// the split of the fused grid phase (always the default), and whether the
// plan's row length has a second split for the standalone FFTs
bool ts_f2_phase_shape(ts_plan p, int *P, int *Q);
bool ts_f2_has_alt(ts_plan p);
size_t ts_f2_bytes(int P, int Q, int R, int nb);
int ts_f2_phase_rows(ts_plan p, int nb, int batch, size_t *smem);
// raise a kernel's dynamic shared-memory limit on `device` (once per size)
void ts_allow_smem(const void *fn, int device, size_t bytes);
void ts_init_tables(ts_plan p);
// tensor-core tables and kernels (sht_tc.cu)
struct TsTcTab;
void ts_tc_init(ts_plan p);
void ts_tc_free(ts_plan p);
const TsTcTab &ts_tc_tab(ts_plan p);
int ts_tc_ntile(ts_plan p);
size_t ts_tc_bytes(ts_plan p);
size_t ts_tc_synth_smem(ts_plan p);
size_t ts_tc_analys_smem(ts_plan p);
int ts_tc_synth_stages(ts_plan p);
int ts_tc_analys_stages(ts_plan p);
int ts_tc_analys_nmax(ts_plan p);
struct TsTcGeom {
  int NL, nLT, LTL, ntile;
};
TsTcGeom ts_tc_geom(ts_plan p);
void ts_tc_set_fault(ts_plan p, int stall_copies, unsigned wait_limit);
// tiles / chunks the tensor-core polar skip drops
void ts_tc_skip_counts(ts_plan p, int *tiles, int *chunks);
// per (32-latitude chunk, parity): the order m from which the W image's chunk
// is never read (null: every chunk is read)
const int *ts_tc_w_kmin(ts_plan p);
int ts_tc_ctas(ts_plan p, long ntiles);
// TC synthesis: fields -> q image (qbuf, or the plan's) -> fm
void ts_launch_leg_synth_tc(ts_plan p, const TsFields &q, float2 *fm, long fm_stride, int nfields,
                            cudaStream_t s, ts_dbuf *qbuf = nullptr);
// TC analysis from G in the gm layout (stage-level)
void ts_launch_leg_analys_tc(ts_plan p, const float2 *g, long g_stride, float2 *q, long q_stride,
                             int nfields, cudaStream_t s);
// TC analysis from the grid: spat -> w image -> q
#ifndef TS_TC_FIELDS
#define TS_TC_FIELDS 64  // fields per tensor-core block (kernels/leg_tc.cuh)
#endif
#ifndef TS_TC_THREADS
#define TS_TC_THREADS 448  // threads of a tensor-core Legendre CTA (kernels/leg_tc.cuh)
#endif
void ts_launch_analys_tc_img(ts_plan p, const char *wimg, int nf, float2 *out, long os,
                             cudaStream_t s);
void ts_analys_tc_full(ts_plan p, const float *spat, long spat_stride, float *qlm, int nfields,
                       cudaStream_t s);
size_t ts_tc_qimg_bytes(ts_plan p, int nfields);
size_t ts_tc_wimg_bytes(ts_plan p, int nfields, int fpb);
void ts_launch_wimage(ts_plan p, const float2 *g, long gs, int nf, int fpb, char *img,
                      cudaStream_t s);
// spat -> w image with the paired register FFT; false when the grid does not allow it
bool ts_launch_fourier_analys_w(ts_plan p, const float *spat, long ss, int nf, int fpb,
                                char *wimg, cudaStream_t s);
// north/south pairs per CTA of the paired Fourier kernels, and their shared memory
int ts_tc_check_error(ts_plan p);
// after a synchronisation: TS_ERR_TIMEOUT (once; the flag is cleared) when a
// tensor-core kernel of the plan gave up a bounded wait since the last check
void ts_plan_take_timeout(ts_plan p);
void ts_kernel_attrs_once(ts_ctx ctx);
