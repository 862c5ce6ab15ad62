// Plan tables (FP64 on the GPU) and launchers of the plain FP32 transform
// kernels.
#include <cmath>
#include <map>
#include <mutex>
#include <type_traits>

#include "kernels/fft2.cuh"
#include "kernels/fourier.cuh"
#include "kernels/leg_f32.cuh"
#include "runtime.h"

// ------------------------------------------------------------ FP64 tables

// Gauss-Legendre nodes x_i = cos(theta_i) (decreasing) and weights, one
// thread per node pair: Newton's method on P_n from the Tricomi-type start
// cos(pi (i + 3/4) / (n + 1/2)), P_n and P_{n-1} by the Bonnet recurrence,
// w = 2 / ((1 - x^2) P_n'(x)^2).  (gauss.ts:11-51 of the reference uses the
// same start, stopping rule and one polishing step.)
__global__ void ts_k_gauss_f64(int n, double *x, double *w) {
  const int half = (n + 1) >> 1;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= half) return;
  double z = cos(M_PI * (i + 0.75) / (n + 0.5));
  double dp = 0.0;
  auto legendre = [n](double zz, double &pn, double &pnm1) {
    double p1 = 1.0, p2 = 0.0;
    for (int j = 1; j <= n; j++) {
      const double p3 = p2;
      p2 = p1;
      p1 = ((2.0 * j - 1.0) * zz * p2 - (j - 1.0) * p3) / j;
    }
    pn = p1;
    pnm1 = p2;
  };
  for (int it = 0; it < 100; it++) {
    double pn, pm;
    legendre(z, pn, pm);
    dp = n * (z * pn - pm) / (z * z - 1.0);
    const double dz = pn / dp;
    z -= dz;
    if (fabs(dz) < 1e-15 * fabs(z) + 1e-300) {
      legendre(z, pn, pm);
      dp = n * (z * pn - pm) / (z * z - 1.0);
      z -= pn / dp;
      break;
    }
  }
  const double wi = 2.0 / ((1.0 - z * z) * dp * dp);
  x[i] = z;
  x[n - 1 - i] = -z;
  w[i] = wi;
  w[n - 1 - i] = wi;
  if ((n & 1) && i == half - 1) x[i] = 0.0;
}

// Recurrence coefficients of the orthonormal associated Legendre functions
// with the Condon-Shortley phase (coeffs.ts:28-56):
//   a_{m+1}^m = sqrt(2m+3),
//   a_l^m = sqrt((2l+1)(2l-1) / ((l+m)(l-m))),
//   b_l^m = -sqrt((2l+1)/(2l-3) (l-1+m)(l-1-m) / ((l+m)(l-m))),
//   amm_m = (-1)^m sqrt(prod_{k<=m} (2k+1)/(2k) / (4 pi)).
// grid.x = m, threads over l.
__global__ void ts_k_legendre_coeffs_f64(int lmax, int mmax, double *ab, double *amm) {
  const int m = blockIdx.x;
  const long base = (long)m * (lmax + 1) - ((long)m * (m - 1)) / 2;
  for (int l = m + threadIdx.x; l <= lmax; l += blockDim.x) {
    double a = 0.0, b = 0.0;
    if (l == m + 1) {
      a = sqrt(2.0 * m + 3.0);
    } else if (l >= m + 2) {
      const double t1 = (double)(l + m) * (l - m);
      const double t2 = (double)(l - 1 + m) * (l - 1 - m);
      a = sqrt((2.0 * l + 1.0) * (2.0 * l - 1.0) / t1);
      b = -sqrt((2.0 * l + 1.0) / (2.0 * l - 3.0) * (t2 / t1));
    }
    ab[2 * (base + l - m)] = a;
    ab[2 * (base + l - m) + 1] = b;
  }
  if (m == 0 && threadIdx.x == 0) {
    double t = 1.0 / (4.0 * M_PI);
    amm[0] = sqrt(t);
    for (int k = 1; k <= mmax; k++) {
      t *= (2.0 * k + 1.0) / (2.0 * k);
      amm[k] = (k & 1) ? -sqrt(t) : sqrt(t);
    }
  }
}

// FP32 working tables from the FP64 ones.
__global__ void ts_k_tables_f32(int nlat, int nh, int nphi, long nlm, int mmax, const double *x,
                                const double *w, const double *ab, const double *amm, float *ct,
                                float *st, float *wq, float2 *ab32, float *amm32) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nh) {
    ct[i] = (float)x[i];
    st[i] = (float)sqrt(1.0 - x[i] * x[i]);
    wq[i] = (float)(w[i] * (2.0 * M_PI / nphi));
  }
  if (i < nlm) ab32[i] = make_float2((float)ab[2 * i], (float)ab[2 * i + 1]);
  if (i <= mmax) amm32[i] = (float)amm[i];
}

void ts_init_tables(ts_plan p) {
  cudaStream_t s = p->ctx->stream;
  const int nlat = p->nlat, nh = p->nh;
  TS_CUDA(cudaMalloc(&p->d_x64, sizeof(double) * nlat));
  TS_CUDA(cudaMalloc(&p->d_w64, sizeof(double) * nlat));
  TS_CUDA(cudaMalloc(&p->d_ab64, sizeof(double) * 2 * p->nlm));
  TS_CUDA(cudaMalloc(&p->d_amm64, sizeof(double) * (p->mmax + 1)));
  TS_CUDA(cudaMalloc(&p->d_ct, sizeof(float) * nh));
  TS_CUDA(cudaMalloc(&p->d_st, sizeof(float) * nh));
  TS_CUDA(cudaMalloc(&p->d_wq, sizeof(float) * nh));
  TS_CUDA(cudaMalloc(&p->d_amm, sizeof(float) * (p->mmax + 1)));
  TS_CUDA(cudaMalloc(&p->d_ab, sizeof(float2) * p->nlm));
  TS_CUDA(cudaMalloc(&p->d_tw, sizeof(float2) * p->nphi));

  const int half = (nlat + 1) / 2;
  ts_k_gauss_f64<<<(half + 63) / 64, 64, 0, s>>>(nlat, p->d_x64, p->d_w64);
  TS_CUDA(cudaGetLastError());
  ts_k_legendre_coeffs_f64<<<p->mmax + 1, 128, 0, s>>>(p->lmax, p->mmax, p->d_ab64, p->d_amm64);
  TS_CUDA(cudaGetLastError());
  const long n = std::max<long>(std::max<long>(nh, p->nlm), p->mmax + 1);
  ts_k_tables_f32<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(
      nlat, nh, p->nphi, p->nlm, p->mmax, p->d_x64, p->d_w64, p->d_ab64, p->d_amm64, p->d_ct,
      p->d_st, p->d_wq, p->d_ab, p->d_amm);
  TS_CUDA(cudaGetLastError());

  // twiddles e^{2 pi i k / nphi}: computed on the host in f64, as the
  // reference does (sht.ts:200-205), then rounded to float
  std::vector<float2> tw(p->nphi);
  for (int k = 0; k < p->nphi; k++) {
    const double a = 2.0 * M_PI * k / p->nphi;
    tw[k] = make_float2((float)std::cos(a), (float)std::sin(a));
  }
  TS_CUDA(cudaMemcpyAsync(p->d_tw, tw.data(), sizeof(float2) * p->nphi, cudaMemcpyHostToDevice, s));
  p->h_x.resize(nlat);
  p->h_w.resize(nlat);
  TS_CUDA(cudaMemcpyAsync(p->h_x.data(), p->d_x64, sizeof(double) * nlat, cudaMemcpyDeviceToHost, s));
  TS_CUDA(cudaMemcpyAsync(p->h_w.data(), p->d_w64, sizeof(double) * nlat, cudaMemcpyDeviceToHost, s));
  TS_CUDA(cudaStreamSynchronize(s));

  p->leg.ct = p->d_ct;
  p->leg.st = p->d_st;
  p->leg.wq = p->d_wq;
  p->leg.ab = p->d_ab;
  p->leg.amm = p->d_amm;
  p->leg.lmax = p->lmax;
  p->leg.mmax = p->mmax;
  p->leg.nlat = p->nlat;
  p->leg.nh = p->nh;
  p->fft.tw = p->d_tw;
}

// ------------------------------------------------------------- DFT stage
//
// Direct band-limited sums, for grids whose nphi has prime factors other
// than 2 and 3 (sht.ts:169-179 falls back the same way; fourier.ts:241-289).
__global__ void ts_k_dft_synth(TsFftTab ft, const float2 *__restrict__ fm, long fm_stride,
                               float *__restrict__ spat, long spat_stride) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int lat = blockIdx.y;
  const long f = blockIdx.z;
  if (j >= ft.nphi) return;
  const float2 *src = fm + f * fm_stride + lat;
  float v = src[0].x;
  int idx = 0;
  for (int m = 1; m <= ft.mmax; m++) {
    idx += j;
    if (idx >= ft.nphi) idx -= ft.nphi;
    const float2 c = src[(long)m * ft.nlat];
    const float2 w = ft.tw[idx];
    v += 2.0f * (c.x * w.x - c.y * w.y);
  }
  spat[f * spat_stride + (long)lat * ft.nphi + j] = v;
}

__global__ void ts_k_dft_analys(TsFftTab ft, const float *__restrict__ spat, long spat_stride,
                                float2 *__restrict__ g, long g_stride) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const int lat = blockIdx.y;
  const long f = blockIdx.z;
  if (m > ft.mmax) return;
  const float *row = spat + f * spat_stride + (long)lat * ft.nphi;
  float2 acc = make_float2(0.f, 0.f);
  int idx = 0;
  for (int j = 0; j < ft.nphi; j++) {
    const float2 w = ft.tw[idx];
    acc.x += row[j] * w.x;
    acc.y -= row[j] * w.y;
    idx += m;
    if (idx >= ft.nphi) idx -= ft.nphi;
  }
  g[f * g_stride + (long)m * ft.nlat + lat] = acc;
}

// ------------------------------------------------------------- launchers

namespace {

template <int F>
void leg_synth_t(ts_plan p, const float2 *q, long qs, float2 *fm, long fs, int nf, cudaStream_t s) {
  const int bd = p->nh >= 128 ? 64 : 32;
  dim3 grid((p->nh + bd - 1) / bd, p->mmax + 1, (nf + F - 1) / F);
  const size_t smem = sizeof(float2) * (size_t)(p->lmax + 1) * (1 + F);
  TsFields qf{};
  qf.base[0] = q;
  qf.inst_stride[0] = qs;
  qf.nper = 1;
  ts_leg_synth_f32<F><<<grid, bd, smem, s>>>(p->leg, qf, fm, fs, nf);
  TS_CUDA(cudaGetLastError());
}

template <int F, int K>
void leg_analys_t(ts_plan p, int W, const float2 *g, long gs, float2 *q, long qs, int nf,
                  cudaStream_t s) {
  constexpr int P = 2;
  constexpr int N = 4 * P * F;
  const int nfb = (nf + F - 1) / F;
  const int lchunk = ts_analys_lchunk(p, nfb);
  dim3 grid(p->mmax + 1, nfb, lchunk ? (p->lmax + lchunk) / lchunk : 1);
  const size_t smem = sizeof(float2) * (p->lmax + 1) + sizeof(float) * (size_t)(W * N + N);
  TsAnalysStore epi{q, qs};
  ts_leg_analys_f32<F, K, P, TsAnalysStore><<<grid, 32 * W, smem, s>>>(p->leg, g, gs, epi, nf, F,
                                                                       lchunk);
  TS_CUDA(cudaGetLastError());
}

template <int F>
void leg_analys_f(ts_plan p, int K, int W, const float2 *g, long gs, float2 *q, long qs, int nf,
                  cudaStream_t s) {
  switch (K) {
    case 1: return leg_analys_t<F, 1>(p, W, g, gs, q, qs, nf, s);
    case 2: return leg_analys_t<F, 2>(p, W, g, gs, q, qs, nf, s);
    case 3: return leg_analys_t<F, 3>(p, W, g, gs, q, qs, nf, s);
    case 4: return leg_analys_t<F, 4>(p, W, g, gs, q, qs, nf, s);
    case 6: return leg_analys_t<F, 6>(p, W, g, gs, q, qs, nf, s);
    default: return leg_analys_t<F, 8>(p, W, g, gs, q, qs, nf, s);
  }
}

// latitudes per thread (K) and warps (W) for the analysis.  The warp
// reduction costs about 2 operations per reduced value against K*4 useful
// FMAs, so K is taken as large as possible (up to 8) with the least idle
// lanes; more CTAs, not more warps per CTA, supply the parallelism.
void pick_kw(int nh, int &K, int &W) {
  // smaller K first: K = 3, W = 2 at nh = 192 holds 12 fields x latitudes in
  // registers instead of 24 and runs the lmax-255 analysis in 745 us instead
  // of 915 (K = 6, W = 1: one warp per CTA, 11 % of the warp slots active)
  static const int Ks[] = {4, 3, 2, 8, 6, 1};
  int best = 1 << 30;
  K = 8;
  W = 8;
  for (int k : Ks)
    for (int w = 1; w <= 8; w++) {
      const int cap = 32 * w * k;
      if (cap < nh) continue;
      const int waste = cap - nh;
      // prefer less waste; accept up to 1/8 idle lanes for a larger K
      if (waste * 8 <= cap && waste < best + 32 * k / 4) {
        if (best == (1 << 30) || waste < best) {
          best = waste;
          K = k;
          W = w;
        }
      }
      break;
    }
  if (best == (1 << 30)) {  // tiny grids: one warp, one latitude per lane
    K = 1;
    W = (nh + 31) / 32;
  }
}

// rows (warps) per Fourier CTA: as many as shared memory allows, fewer when
// the grid would otherwise leave SMs idle
int pick_lb(ts_plan p, int nfields, int nbuf, size_t *smem_out) {
  const TsFftTab &ft = p->fft;
  const size_t cap = p->ctx->smem_optin;
  int lb = 8;
  for (; lb > 1; lb >>= 1) {
    const size_t smem = sizeof(float2) * ((size_t)ft.nphi + (size_t)(ft.mmax + 1) * lb +
                                          (size_t)lb * nbuf * ft.H);
    const long ctas = (long)nfields * ((p->nlat + lb - 1) / lb);
    if (smem <= cap && ctas >= 2L * p->ctx->sm_count) break;
  }
  *smem_out = sizeof(float2) * ((size_t)ft.nphi + (size_t)(ft.mmax + 1) * lb + (size_t)lb * nbuf * ft.H);
  TS_REQUIRE(*smem_out <= cap, TS_ERR_UNSUPPORTED, "grid too large for the shared-memory FFT");
  return lb;
}

}  // namespace

void ts_kernel_attrs_once(ts_ctx ctx) {
  // cudaFuncSetAttribute acts on the current device's copy of a kernel, so
  // the limits are raised per (device, kernel): a context on a second GPU of
  // the process gets its own (ts_allow_smem keys its record by device).
  const size_t cap = ctx->smem_optin;
  const int dev = ctx->device;
  ts_allow_smem((const void *)ts_leg_synth_f32<1>, dev, cap);
  ts_allow_smem((const void *)ts_leg_synth_f32<2>, dev, cap);
  ts_allow_smem((const void *)ts_leg_synth_f32<4>, dev, cap);
  ts_allow_smem((const void *)ts_leg_synth_f32<8>, dev, cap);
  ts_allow_smem((const void *)ts_fourier_synth, dev, cap);
  ts_allow_smem((const void *)ts_fourier_analys, dev, cap);
}

void ts_launch_leg_synth_fields(ts_plan p, const TsFields &q, float2 *fm, long fs, int nf,
                                cudaStream_t s) {
  if (p->precision != TS_PREC_FP32) return ts_launch_leg_synth_tc(p, q, fm, fs, nf, s);
  ts_launch_leg_synth_plain(p, q, fm, fs, nf, s);
}

void ts_launch_leg_synth_plain(ts_plan p, const TsFields &q, float2 *fm, long fs, int nf,
                               cudaStream_t s) {
  const int bd = p->nh >= 128 ? 64 : 32;
  auto go = [&](auto Fc) {
    constexpr int F = decltype(Fc)::value;
    dim3 grid((p->nh + bd - 1) / bd, p->mmax + 1, (nf + F - 1) / F);
    const size_t smem = sizeof(float2) * (size_t)(p->lmax + 1) * (1 + F);
    ts_leg_synth_f32<F><<<grid, bd, smem, s>>>(p->leg, q, fm, fs, nf);
    TS_CUDA(cudaGetLastError());
  };
  if (nf >= 8) return go(std::integral_constant<int, 8>());
  if (nf >= 4) return go(std::integral_constant<int, 4>());
  if (nf >= 2) return go(std::integral_constant<int, 2>());
  return go(std::integral_constant<int, 1>());
}

void ts_analys_shape(ts_plan p, int nfields, int per_inst, int *F, int *K, int *W, int *per_cta) {
  pick_kw(p->nh, *K, *W);
  int f = 4;
  while (f > 1 && *K * f > 24) f >>= 1;
  while (f < per_inst) f <<= 1;  // a CTA holds at least one whole instance
  int groups = f / per_inst;
  if (nfields < f) {
    f = 1;
    while (f < nfields) f <<= 1;
    groups = (f / per_inst) > 0 ? f / per_inst : 1;
  }
  *F = f;
  *per_cta = groups * per_inst;
}

// degrees per FP32-analysis CTA: 0 (all of one m) unless the grid of
// (mmax+1) x nfb CTAs would leave SMs idle; then chunks of a multiple of 4
// degrees so that about two CTAs per SM exist
int ts_analys_lchunk(ts_plan p, int nfb) {
  const long ctas = (long)(p->mmax + 1) * nfb;
  if (ctas >= p->ctx->sm_count) return 0;
  const long want = (2L * p->ctx->sm_count + ctas - 1) / ctas;  // chunks per m
  int len = (int)((p->lmax + 1 + want - 1) / want);
  len = std::max(8, (len + 3) & ~3);
  return len >= p->lmax + 1 ? 0 : len;
}

size_t ts_analys_smem(ts_plan p, int F, int W) {
  const int N = 4 * 2 * F;
  return sizeof(float2) * (p->lmax + 1) + sizeof(float) * (size_t)(W * N + N);
}

int ts_fourier_lb(ts_plan p, int nblocks_y, int nrows, size_t *smem) {
  return pick_lb(p, nblocks_y, nrows, smem);
}

void ts_launch_leg_synth(ts_plan p, const float2 *q, long qs, float2 *fm, long fs, int nf,
                         cudaStream_t s) {
  if (p->precision != TS_PREC_FP32) {
    TsFields qf{};
    qf.base[0] = q;
    qf.inst_stride[0] = qs;
    qf.nper = 1;
    return ts_launch_leg_synth_tc(p, qf, fm, fs, nf, s);
  }
  if (nf >= 8) return leg_synth_t<8>(p, q, qs, fm, fs, nf, s);
  if (nf >= 4) return leg_synth_t<4>(p, q, qs, fm, fs, nf, s);
  if (nf >= 2) return leg_synth_t<2>(p, q, qs, fm, fs, nf, s);
  return leg_synth_t<1>(p, q, qs, fm, fs, nf, s);
}

void ts_launch_leg_analys(ts_plan p, const float2 *g, long gs, float2 *q, long qs, int nf,
                          cudaStream_t s) {
  if (p->precision != TS_PREC_FP32) return ts_launch_leg_analys_tc(p, g, gs, q, qs, nf, s);
  int K, W;
  pick_kw(p->nh, K, W);
  // registers hold K*F complex pairs of weighted inputs: keep K*F <= 24
  int F = nf >= 4 ? 4 : (nf >= 2 ? 2 : 1);
  while (F > 1 && K * F > 24) F >>= 1;
  if (F == 4) return leg_analys_f<4>(p, K, W, g, gs, q, qs, nf, s);
  if (F == 2) return leg_analys_f<2>(p, K, W, g, gs, q, qs, nf, s);
  return leg_analys_f<1>(p, K, W, g, gs, q, qs, nf, s);
}

// Two-phase FFT shapes: H = P*Q with P, Q in-register DFT lengths, and the
// two row counts R of a transform CTA (P*R threads) the kernels are built
// for: X(H, P, Q, R_small, R_default)
#define TS_F2_SHAPES(X) \
  X(32, 8, 4, 8, 16)    \
  X(48, 8, 6, 8, 16)    \
  X(64, 8, 8, 8, 16)    \
  X(96, 12, 8, 8, 16)   \
  X(128, 16, 8, 8, 16)  \
  X(192, 16, 12, 8, 16) \
  X(256, 16, 16, 8, 16) \
  X(384, 24, 16, 8, 16) \
  X(512, 32, 16, 8, 16) \
  X(768, 32, 24, 8, 16) \
  X(1024, 32, 32, 8, 16) \
  X(1536, 48, 32, 4, 8)

// The second split the autotuner tries for the grids of the transform
// workloads (nphi = 192, 384, 768, 1536): a longer DFT in the second phase,
// fewer rows in flight per thread block.  The fused grid phase always runs
// the default split (its registers hold every species' P points).
#define TS_F2_ALT_SHAPES(X) \
  X(96, 16, 6, 8, 16)       \
  X(192, 24, 8, 8, 16)      \
  X(384, 32, 12, 8, 16)     \
  X(768, 48, 16, 4, 8)

bool ts_f2_has_alt(ts_plan p) {
  if (p->fourier != TS_FOURIER_FFT) return false;
  switch (p->fft.H) {
#define TS_F2_CASE(h, pp, qq, rlo, rhi) \
  case h:                               \
    return true;
    TS_F2_ALT_SHAPES(TS_F2_CASE)
#undef TS_F2_CASE
    default:
      return false;
  }
}

bool ts_f2_phase_shape(ts_plan p, int *P, int *Q) {
  if (p->fourier != TS_FOURIER_FFT) return false;
  switch (p->fft.H) {
#define TS_F2_CASE(h, pp, qq, rlo, rhi) \
  case h:                               \
    *P = pp;                            \
    *Q = qq;                            \
    return true;
    TS_F2_SHAPES(TS_F2_CASE)
#undef TS_F2_CASE
    default:
      return false;
  }
}

bool ts_f2_shape(ts_plan p, int *P, int *Q) {
  if (p->fourier != TS_FOURIER_FFT) return false;
  if (p->fft_alt) switch (p->fft.H) {
#define TS_F2_CASE(h, pp, qq, rlo, rhi) \
  case h:                               \
    *P = pp;                            \
    *Q = qq;                            \
    return true;
      TS_F2_ALT_SHAPES(TS_F2_CASE)
#undef TS_F2_CASE
      default:
        break;
    }
  switch (p->fft.H) {
#define TS_F2_CASE(h, pp, qq, rlo, rhi) \
  case h:                               \
    *P = pp;                            \
    *Q = qq;                            \
    return true;
    TS_F2_SHAPES(TS_F2_CASE)
#undef TS_F2_CASE
    default:
      return false;
  }
}

size_t ts_f2_bytes(int P, int Q, int R, int nb) {
  const int H = P * Q, RP = (H + Q) | 1;
  return sizeof(float2) * ((size_t)Q * (P + 1) + (size_t)nb * R * RP);
}

// rows per phase CTA with nb row blocks: the largest of 16, 8, 4 that fits
// and still gives every SM a CTA for `batch` instances (0: none fits)
int ts_f2_phase_rows(ts_plan p, int nb, int batch, size_t *smem) {
  int P, Q;
  if (!ts_f2_phase_shape(p, &P, &Q)) return 0;
  const size_t cap = p->ctx->smem_optin;
  int want = 0;  // TS_PHASE_ROWS (16, 8 or 4) tunes it, like the reference's SHT_* knobs
  if (const char *e = getenv("TS_PHASE_ROWS")) want = atoi(e);
  // fewer rows per CTA while the grid would leave SMs idle (a small batch)
  int chosen = 0;
  for (int R : {16, 8, 4}) {
    if (want && R != want) continue;
    const size_t b = ts_f2_bytes(P, Q, R, nb);
    if (P * R > 1024 || b > cap) continue;
    chosen = R;
    *smem = b;
    if (want || (long)batch * ((p->nlat + R - 1) / R) >= p->ctx->sm_count) break;
  }
  return chosen;
}

void ts_allow_smem(const void *fn, int device, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void *>, size_t> done;
  std::lock_guard<std::mutex> lock(mu);
  size_t &have = done[{device, fn}];
  if (have >= bytes) return;
  TS_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  have = bytes;
}

namespace {
template <int P, int Q, int R>
void f2_synth(ts_plan p, const float2 *fm, long fs, float *spat, long ss, int nf, cudaStream_t s) {
  const size_t smem = ts_f2_bytes(P, Q, R, 1);
  ts_allow_smem((const void *)ts_f2_synth<P, Q, R>, p->ctx->device, smem);
  dim3 grid((p->nlat + R - 1) / R, nf);
  ts_f2_synth<P, Q, R><<<grid, P * R, smem, s>>>(p->fft, fm, fs, spat, ss);
  TS_CUDA(cudaGetLastError());
}
template <int P, int Q, int R>
void f2_analys(ts_plan p, const float *spat, long ss, float2 *g, long gs, int nf, cudaStream_t s) {
  const size_t smem = ts_f2_bytes(P, Q, R, 1);
  ts_allow_smem((const void *)ts_f2_analys<P, Q, R>, p->ctx->device, smem);
  dim3 grid((p->nlat + R - 1) / R, nf);
  ts_f2_analys<P, Q, R><<<grid, P * R, smem, s>>>(p->fft, spat, ss, g, gs);
  TS_CUDA(cudaGetLastError());
}
template <int P, int Q, int R>
void f2_analys_w(ts_plan p, const float *spat, long ss, int nf, int fpb, char *wimg,
                 cudaStream_t s) {
  const size_t smem = ts_f2_bytes(P, Q, R, 1);
  ts_allow_smem((const void *)ts_f2_analys_w<P, Q, R>, p->ctx->device, smem);
  const int nlc = (p->nh + 31) / 32;
  dim3 grid((p->nh + R / 2 - 1) / (R / 2), nf);
  ts_f2_analys_w<P, Q, R><<<grid, P * R, smem, s>>>(p->fft, spat, ss, p->d_wq, wimg,
                                                    (nf + fpb - 1) / fpb, fpb, nlc, p->nh,
                                                    ts_tc_w_kmin(p));
  TS_CUDA(cudaGetLastError());
}
}  // namespace

namespace {
// rows of a standalone FFT CTA: the tuned choice, else the default unless a
// small batch would leave SMs idle
int pick_rows(ts_plan p, int nf, int rlo, int rhi) {
  if (p->fft_rows) return p->fft_rows == rlo ? rlo : rhi;
  return (long)nf * ((p->nlat + rhi - 1) / rhi) < p->ctx->sm_count ? rlo : rhi;
}
}  // namespace

int ts_f2_rows(ts_plan p) {
  if (p->fourier != TS_FOURIER_FFT) return 0;
  if (p->fft_alt) switch (p->fft.H) {
#define TS_F2_CASE(h, pp, qq, rlo, rhi) \
  case h:                               \
    return p->fft_rows == rlo ? rlo : rhi;
      TS_F2_ALT_SHAPES(TS_F2_CASE)
#undef TS_F2_CASE
      default:
        break;
    }
  switch (p->fft.H) {
#define TS_F2_CASE(h, pp, qq, rlo, rhi) \
  case h:                               \
    return p->fft_rows == rlo ? rlo : rhi;
    TS_F2_SHAPES(TS_F2_CASE)
#undef TS_F2_CASE
    default:
      return 0;
  }
}

bool ts_launch_fourier_analys_w(ts_plan p, const float *spat, long ss, int nf, int fpb,
                                char *wimg, cudaStream_t s) {
  if (p->fourier != TS_FOURIER_FFT) return false;
#define TS_F2_CASE(h, pp, qq, rlo, rhi)                                     \
  case h:                                                                   \
    if (pick_rows(p, nf, rlo, rhi) == rlo)                                  \
      f2_analys_w<pp, qq, rlo>(p, spat, ss, nf, fpb, wimg, s);              \
    else                                                                    \
      f2_analys_w<pp, qq, rhi>(p, spat, ss, nf, fpb, wimg, s);              \
    return true;
  if (p->fft_alt) switch (p->fft.H) {
      TS_F2_ALT_SHAPES(TS_F2_CASE)
      default:
        break;
    }
  switch (p->fft.H) {
    TS_F2_SHAPES(TS_F2_CASE)
#undef TS_F2_CASE
    default:
      return false;
  }
}

void ts_launch_fourier_synth(ts_plan p, const float2 *fm, long fs, float *spat, long ss, int nf,
                             cudaStream_t s) {
  if (p->fourier == TS_FOURIER_FFT) {
#define TS_F2_CASE(h, pp, qq, rlo, rhi)                                         \
  case h:                                                                       \
    return pick_rows(p, nf, rlo, rhi) == rlo ? f2_synth<pp, qq, rlo>(p, fm, fs, spat, ss, nf, s) \
                              : f2_synth<pp, qq, rhi>(p, fm, fs, spat, ss, nf, s);
    if (p->fft_alt) switch (p->fft.H) {
        TS_F2_ALT_SHAPES(TS_F2_CASE)
        default:
          break;
      }
    switch (p->fft.H) {
      TS_F2_SHAPES(TS_F2_CASE)
#undef TS_F2_CASE
      default:
        break;
    }
  }
  if (p->fourier == TS_FOURIER_DFT) {
    dim3 grid((p->nphi + 63) / 64, p->nlat, nf);
    ts_k_dft_synth<<<grid, 64, 0, s>>>(p->fft, fm, fs, spat, ss);
    TS_CUDA(cudaGetLastError());
    return;
  }
  size_t smem;
  const int lb = pick_lb(p, nf, 2, &smem);
  dim3 grid((p->nlat + lb - 1) / lb, nf);
  ts_fourier_synth<<<grid, 32 * lb, smem, s>>>(p->fft, fm, fs, spat, ss);
  TS_CUDA(cudaGetLastError());
}

void ts_launch_fourier_analys(ts_plan p, const float *spat, long ss, float2 *g, long gs, int nf,
                              cudaStream_t s) {
  if (p->fourier == TS_FOURIER_FFT) {
#define TS_F2_CASE(h, pp, qq, rlo, rhi)                                        \
  case h:                                                                      \
    return pick_rows(p, nf, rlo, rhi) == rlo ? f2_analys<pp, qq, rlo>(p, spat, ss, g, gs, nf, s) \
                              : f2_analys<pp, qq, rhi>(p, spat, ss, g, gs, nf, s);
    if (p->fft_alt) switch (p->fft.H) {
        TS_F2_ALT_SHAPES(TS_F2_CASE)
        default:
          break;
      }
    switch (p->fft.H) {
      TS_F2_SHAPES(TS_F2_CASE)
#undef TS_F2_CASE
      default:
        break;
    }
  }
  if (p->fourier == TS_FOURIER_DFT) {
    dim3 grid((p->mmax + 1 + 63) / 64, p->nlat, nf);
    ts_k_dft_analys<<<grid, 64, 0, s>>>(p->fft, spat, ss, g, gs);
    TS_CUDA(cudaGetLastError());
    return;
  }
  size_t smem;
  const int lb = pick_lb(p, nf, 2, &smem);
  dim3 grid((p->nlat + lb - 1) / lb, nf);
  ts_fourier_analys<<<grid, 32 * lb, smem, s>>>(p->fft, spat, ss, g, gs);
  TS_CUDA(cudaGetLastError());
}
