// Allocation-free synthesis: ts_sht_synth_noalloc.
//
// Some callers cannot let a library call cudaMalloc: hosts that own every
// device allocation themselves (a plugin inside a memory-capped process, a
// pool-managed runtime), and latency-critical loops, because cudaMalloc may
// synchronise the whole device.  ts_sht_synth_dev grows the plan's Fourier
// intermediate with cudaMalloc the first time it sees a larger batch; this
// entry point instead takes that intermediate from a fixed array compiled
// into the library, so it allocates nothing.
//
// The array is a file-scope __device__ variable of TS_NOALLOC_SCRATCH_BYTES
// (16 MiB): every GPU that loads the library holds it until the process exits.
// Host code cannot use the symbol's name as a device address (on the host it
// names a stand-in object), so the device address is looked up once per
// device with cudaGetSymbolAddress, with that device current, and passed to
// the kernels.
#include <cstring>
#include <mutex>

#include "runtime.h"

#define TS_NOALLOC_SCRATCH_BYTES (16u << 20)
#define TS_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) float2 ts_noalloc_fm[TS_NOALLOC_SCRATCH_BYTES / sizeof(float2)];

namespace {

std::mutex g_noalloc_mu;
float2 *g_noalloc_ptr[TS_NOALLOC_MAX_DEVICES] = {};

// Device address of ts_noalloc_fm on the current device (set-up on first use).
float2 *noalloc_scratch(int device) {
  TS_REQUIRE(device >= 0 && device < TS_NOALLOC_MAX_DEVICES, TS_ERR_INVALID,
             "device ordinal out of range for the allocation-free entry point");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[device]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, ts_noalloc_fm);
    if (e != cudaSuccess)
      ts_throw(TS_ERR_CUDA,
               std::string("cudaGetSymbolAddress(ts_noalloc_fm): ") + cudaGetErrorString(e));
    g_noalloc_ptr[device] = static_cast<float2 *>(p);
  }
  return g_noalloc_ptr[device];
}

}  // namespace

extern "C" int ts_sht_synth_noalloc(ts_plan p, const float *qlm, float *spat, int batch,
                                    void *stream) {
  ts_ctx ctx = p ? p->ctx : nullptr;
  try {
    TS_REQUIRE(p != nullptr, TS_ERR_INVALID, "null plan");
    TS_REQUIRE(qlm != nullptr && spat != nullptr, TS_ERR_INVALID, "null buffer");
    TS_REQUIRE(batch >= 1 && batch <= 65535, TS_ERR_INVALID, "batch must be in [1, 65535]");
    ts_require_aligned8(qlm, spat);
    const long fm_stride = (long)(p->mmax + 1) * p->nlat;
    const size_t need = sizeof(float2) * (size_t)fm_stride * (size_t)batch;
    if (need > TS_NOALLOC_SCRATCH_BYTES) {
      char buf[256];
      snprintf(buf, sizeof buf,
               "ts_sht_synth_noalloc: batch %d at lmax %d needs %zu bytes of scratch, above the "
               "fixed %u-byte limit (use at most %ld fields per call)",
               batch, p->lmax, need, TS_NOALLOC_SCRATCH_BYTES,
               (long)(TS_NOALLOC_SCRATCH_BYTES / (sizeof(float2) * (size_t)fm_stride)));
      ts_throw(TS_ERR_SIZE, buf);
    }
    ts_device_guard dev_guard_(ctx->device);
    float2 *fm = noalloc_scratch(ctx->device);
    // The Legendre stage writes every (field, m, latitude) entry the Fourier
    // stage then reads, so nothing left in the array by an earlier call is used.
    cudaStream_t s = ts_pick_stream(ctx, stream);
    // The FP32 Legendre kernels read the coefficients as they are; the
    // tensor-core path would first relayout them into a plan-owned operand
    // image grown on demand, so this entry point always takes the FP32 path.
    TsFields qf{};
    qf.base[0] = (const float2 *)qlm;
    qf.inst_stride[0] = p->nlm;
    qf.nper = 1;
    ts_launch_leg_synth_plain(p, qf, fm, fm_stride, batch, s);
    ts_launch_fourier_synth(p, fm, fm_stride, spat, (long)p->nlat * p->nphi, batch, s);
    return TS_OK;
  } catch (const ts_exc &e) {
    ts_set_error(ctx, e.msg);
    return e.code;
  }
}
