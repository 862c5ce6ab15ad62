// Adjoints (transposes) of the spherical-harmonic transforms.
//
// With the coefficient vector read as 2*nlm reals (re, im of every lm) and
// the grid as nlat*nphi reals, the transforms of this library are the
// matrices
//   synth:  g = S q,   S[(i,j), (lm,re)] =  c_m P_lm(x_i) cos(m phi_j),
//                      S[(i,j), (lm,im)] = -c_m P_lm(x_i) sin(m phi_j),
//   analys: q = A g,   A[(lm,re), (i,j)] =  w_i P_lm(x_i) cos(m phi_j),
//                      A[(lm,im), (i,j)] = -w_i P_lm(x_i) sin(m phi_j),
// with c_0 = 1, c_m = 2 for m > 0 (a real field from its m >= 0 half) and
// w_i the Gauss weight times 2 pi/nphi.  Hence
//   S^T = diag(c) A diag(1/w),   A^T = diag(w) S diag(1/c),
// so each adjoint is the other forward transform between two diagonal
// scalings, on the same (FP32 or tensor-core) kernels.  The imaginary part
// of m = 0 is neither read by the synthesis nor produced by the analysis;
// the adjoints give it zero.
#include "runtime.h"

namespace {

// grid[f][lat][phi] *= w(lat) (mul) or /= w(lat); w is stored for the
// northern half and mirrored.  grid = (nlat, fields): one row per CTA, its
// weight read once, 16-byte accesses when the row allows them.
__global__ void ts_k_scale_grid(float *out, const float *in, const float *__restrict__ wq,
                                int nlat, int nphi, int nh, int mul) {
  const int lat = blockIdx.x;
  const int h = lat < nh ? lat : nlat - 1 - lat;
  const float w = wq[h];
  const long off = ((long)blockIdx.y * nlat + lat) * nphi;
  const float *src = in + off;
  float *dst = out + off;
  if ((nphi & 3) == 0 && ((reinterpret_cast<unsigned long long>(src) |
                           reinterpret_cast<unsigned long long>(dst)) & 15) == 0) {
    const float4 *s4 = reinterpret_cast<const float4 *>(src);
    float4 *d4 = reinterpret_cast<float4 *>(dst);
    for (int i = threadIdx.x; i < (nphi >> 2); i += blockDim.x) {
      float4 v = s4[i];
      if (mul) {
        v.x *= w; v.y *= w; v.z *= w; v.w *= w;
      } else {
        v.x /= w; v.y /= w; v.z /= w; v.w /= w;
      }
      d4[i] = v;
    }
  } else {
    for (int i = threadIdx.x; i < nphi; i += blockDim.x) dst[i] = mul ? src[i] * w : src[i] / w;
  }
}

// spec[f][lm] (complex) *= c_m (mul) or /= c_m; imaginary part of m = 0 -> 0
__global__ void ts_k_scale_spec(float2 *out, const float2 *in, int lmax, int mmax, long nlm,
                                int mul) {
  const int m = blockIdx.y;
  const long f = blockIdx.z;
  const long base = ts_lm_base(lmax, m);
  const float c = m == 0 ? 1.f : (mul ? 2.f : 0.5f);
  for (int l = m + blockIdx.x * blockDim.x + threadIdx.x; l <= lmax; l += gridDim.x * blockDim.x) {
    const long i = f * nlm + base + (l - m);
    float2 v = in[i];
    v.x *= c;
    v.y = m == 0 ? 0.f : v.y * c;
    out[i] = v;
  }
}

void scale_grid(ts_plan p, float *out, const float *in, int nf, bool mul, cudaStream_t s) {
  dim3 grid(p->nlat, nf);
  ts_k_scale_grid<<<grid, 256, 0, s>>>(out, in, p->d_wq, p->nlat, p->nphi, p->nh, mul ? 1 : 0);
  TS_CUDA(cudaGetLastError());
}

void scale_spec(ts_plan p, float *out, const float *in, int nf, bool mul, cudaStream_t s) {
  dim3 grid((p->lmax + 1 + 127) / 128, p->mmax + 1, nf);
  ts_k_scale_spec<<<grid, 128, 0, s>>>((float2 *)out, (const float2 *)in, p->lmax, p->mmax,
                                       p->nlm, mul ? 1 : 0);
  TS_CUDA(cudaGetLastError());
}

}  // namespace

// qbar = S^T gbar = c * analys(gbar / w); gbar is left unchanged
void ts_synth_adjoint(ts_plan p, const float *gbar, float *qbar, int nf, cudaStream_t s) {
  p->adj_grid.ensure(sizeof(float) * (size_t)p->nlat * p->nphi * nf);
  float *tmp = (float *)p->adj_grid.p;
  scale_grid(p, tmp, gbar, nf, false, s);
  ts_analys_dev(p, tmp, qbar, nf, s);
  scale_spec(p, qbar, qbar, nf, true, s);
}

// gbar = A^T qbar = w * synth(qbar / c); qbar is left unchanged
void ts_analys_adjoint(ts_plan p, const float *qbar, float *gbar, int nf, cudaStream_t s) {
  p->adj_spec.ensure(sizeof(float2) * (size_t)p->nlm * nf);
  float *tmp = (float *)p->adj_spec.p;
  scale_spec(p, tmp, qbar, nf, false, s);
  ts_synth_dev(p, tmp, gbar, nf, s);
  scale_grid(p, gbar, gbar, nf, true, s);
}

extern "C" {

int ts_sht_synth_adjoint_dev(ts_plan p, const float *gbar, float *qbar, int batch, void *stream) {
  ts_ctx ctx = p ? p->ctx : nullptr;
  try {
    TS_REQUIRE(p != nullptr, TS_ERR_INVALID, "null plan");
    TS_REQUIRE(gbar != nullptr && qbar != nullptr, TS_ERR_INVALID, "null buffer");
    TS_REQUIRE(batch >= 1 && batch <= 65535, TS_ERR_INVALID, "batch must be in [1, 65535]");
    ts_require_aligned8(gbar, qbar);
    ts_device_guard dev_guard_(ctx->device);
    ts_synth_adjoint(p, gbar, qbar, batch, ts_pick_stream(ctx, stream));
    return TS_OK;
  } catch (const ts_exc &e) {
    ts_set_error(ctx, e.msg);
    return e.code;
  }
}

int ts_sht_analys_adjoint_dev(ts_plan p, const float *qbar, float *gbar, int batch, void *stream) {
  ts_ctx ctx = p ? p->ctx : nullptr;
  try {
    TS_REQUIRE(p != nullptr, TS_ERR_INVALID, "null plan");
    TS_REQUIRE(gbar != nullptr && qbar != nullptr, TS_ERR_INVALID, "null buffer");
    TS_REQUIRE(batch >= 1 && batch <= 65535, TS_ERR_INVALID, "batch must be in [1, 65535]");
    ts_require_aligned8(gbar, qbar);
    ts_device_guard dev_guard_(ctx->device);
    ts_analys_adjoint(p, qbar, gbar, batch, ts_pick_stream(ctx, stream));
    return TS_OK;
  } catch (const ts_exc &e) {
    ts_set_error(ctx, e.msg);
    return e.code;
  }
}

}  // extern "C"
