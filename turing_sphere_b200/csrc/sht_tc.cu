// Tensor-core Legendre tables (FP64 on the GPU) and launchers.
#include <cmath>
#include <vector>

#include "kernels/leg_f32.cuh"
#include "kernels/leg_tc.cuh"
#include "runtime.h"

namespace {

// x rounded to 11 significant bits, ties away from zero (cvt.rna.tf32)
__device__ double ts_round_tf32(double x) {
  if (x == 0.0) return 0.0;
  int e;
  const double mnt = frexp(x, &e);
  return ldexp(round(ldexp(mnt, 11)), e - 11);
}

// One thread per (m, northern latitude): the orthonormal associated Legendre
// functions of every l by the three-term recurrence in FP64, the running
// pair renormalised by 2^500 whenever it leaves [2^-500, 2^500] so that
// sin(theta)^m cannot underflow before the recurrence has grown it back.
// Each value is split into TF32 hi + lo and written into both MMA images.
__global__ void ts_k_tc_tables(int lmax, int mmax, int nh, const double *x, const double *ab,
                               const double *amm, TsTcTab tc, char *synth, char *anal) {
  const int m = blockIdx.y;
  const int lat = blockIdx.x * blockDim.x + threadIdx.x;
  if (lat >= nh) return;
  const double ct = x[lat];
  const double st = sqrt(1.0 - ct * ct);
  const long base = (long)m * (lmax + 1) - ((long)m * (m - 1)) / 2;
  const int kp0 = ts_kpar(lmax, m, 0), kp1 = ts_kpar(lmax, m, 1);
  const int nch0 = (kp0 + TS_TC_KCH - 1) / TS_TC_KCH;
  (void)kp1;
  const int NL = tc.NL;
  const long sblk = 2L * NL * 128;

  auto emit = [&](int l, double y, int e) {
    double P = e < -1100 ? 0.0 : ldexp(y, e);
    if (fabs(P) < 1e-30) P = 0.0;
    const double hi = ts_round_tf32(P);
    const double lo = ts_round_tf32(P - hi);
    const int j = (l - m) >> 1, par = (l - m) & 1;
    // synthesis image: [par][chunk][lat tile][hi|lo][NL x 32]
    {
      const int cc = j / TS_TC_KCH, k = j % TS_TC_KCH;
      const int lt = lat / NL, r = lat % NL;
      const long off = tc.synth_off[m] + (long)((par ? nch0 : 0) + cc) * tc.nLT * sblk + lt * sblk;
      *reinterpret_cast<float *>(synth + off + ts_swz(r, k)) = (float)hi;
      *reinterpret_cast<float *>(synth + off + (long)NL * 128 + ts_swz(r, k)) = (float)lo;
    }
    // analysis image: [par][l tile][lat chunk][hi|lo][N x 32]
    {
      const int ltile = j / tc.LTL, jj = j % tc.LTL;
      const int N = ts_round16(ts_atile_count(lmax, m, par, ltile, tc.LTL));
      const int c = lat / TS_TC_KCH, k = lat % TS_TC_KCH;
      const long off = ts_atile_offset(tc, lmax, m, par, ltile) + (long)c * 2 * N * 128;
      *reinterpret_cast<float *>(anal + off + ts_swz(jj, k)) = (float)hi;
      *reinterpret_cast<float *>(anal + off + (long)N * 128 + ts_swz(jj, k)) = (float)lo;
    }
  };

  double y = 1.0;
  int e = 0;
  for (int i = 0; i < m; i++) {
    y *= st;
    if (y < 0x1p-500) {
      y *= 0x1p500;
      e -= 500;
    }
  }
  double y0 = y * amm[m];
  emit(m, y0, e);
  if (m == lmax) return;
  double y1 = ab[2 * (base + 1)] * ct * y0;
  emit(m + 1, y1, e);
  for (int l = m + 2; l <= lmax; l++) {
    const long lm = base + (l - m);
    const double y2 = ab[2 * lm] * ct * y1 + ab[2 * lm + 1] * y0;
    y0 = y1;
    y1 = y2;
    if (fabs(y1) > 0x1p500) {
      y0 *= 0x1p-500;
      y1 *= 0x1p-500;
      e += 500;
    }
    emit(l, y1, e);
  }
}

int kpar_h(int lmax, int m, int par) { return (lmax - m + 1 + 1 - par) / 2; }

}  // namespace

struct ts_tc_tables {
  char *synth = nullptr, *anal = nullptr;
  long *synth_off = nullptr, *anal_off = nullptr;
  int *err = nullptr;
  TsTcTab tab{};
  size_t bytes = 0;
  int ntile = 1;  // analysis l tiles per parity (grid.z = 2*ntile)
};

void ts_tc_init(ts_plan p) {
  auto *t = new ts_tc_tables();
  p->tc = t;
  const int nh = p->nh;
  int NL = ((nh + 15) / 16) * 16;
  if (NL > 192) NL = 192;
  const int nLT = (nh + NL - 1) / NL;
  const int LTL = 256;
  const int nLC = (nh + TS_TC_KCH - 1) / TS_TC_KCH;
  std::vector<long> soff(p->mmax + 2), aoff(p->mmax + 2);
  long s = 0, a = 0;
  for (int m = 0; m <= p->mmax; m++) {
    soff[m] = s;
    aoff[m] = a;
    int nch = 0;
    for (int par = 0; par < 2; par++) {
      const int kp = kpar_h(p->lmax, m, par);
      nch += (kp + TS_TC_KCH - 1) / TS_TC_KCH;
      for (int lt0 = 0; lt0 < kp; lt0 += LTL) {
        const int cnt = std::min(kp, lt0 + LTL) - lt0;
        a += (long)nLC * 2 * (((cnt + 15) / 16) * 16) * 128;
      }
    }
    s += (long)nch * nLT * 2 * NL * 128;
  }
  soff[p->mmax + 1] = s;
  aoff[p->mmax + 1] = a;
  t->ntile = (kpar_h(p->lmax, 0, 0) + LTL - 1) / LTL;
  TS_CUDA(cudaMalloc(&t->synth, s));
  TS_CUDA(cudaMalloc(&t->anal, a));
  TS_CUDA(cudaMemset(t->synth, 0, s));
  TS_CUDA(cudaMemset(t->anal, 0, a));
  TS_CUDA(cudaMalloc(&t->synth_off, sizeof(long) * soff.size()));
  TS_CUDA(cudaMalloc(&t->anal_off, sizeof(long) * aoff.size()));
  TS_CUDA(cudaMalloc(&t->err, sizeof(int)));
  TS_CUDA(cudaMemset(t->err, 0, sizeof(int)));
  TS_CUDA(cudaMemcpy(t->synth_off, soff.data(), sizeof(long) * soff.size(), cudaMemcpyHostToDevice));
  TS_CUDA(cudaMemcpy(t->anal_off, aoff.data(), sizeof(long) * aoff.size(), cudaMemcpyHostToDevice));
  t->bytes = s + a;
  TsTcTab &tc = t->tab;
  tc.synth = t->synth;
  tc.synth_off = t->synth_off;
  tc.anal = t->anal;
  tc.anal_off = t->anal_off;
  tc.NL = NL;
  tc.nLT = nLT;
  tc.LTL = LTL;
  tc.nLC = nLC;
  tc.err = t->err;
  dim3 grid((nh + 63) / 64, p->mmax + 1);
  ts_k_tc_tables<<<grid, 64, 0, p->ctx->stream>>>(p->lmax, p->mmax, nh, p->d_x64, p->d_ab64,
                                                  p->d_amm64, tc, t->synth, t->anal);
  TS_CUDA(cudaGetLastError());
  TS_CUDA(cudaStreamSynchronize(p->ctx->stream));
}

void ts_tc_free(ts_plan p) {
  auto *t = static_cast<ts_tc_tables *>(p->tc);
  if (!t) return;
  for (void *q : {(void *)t->synth, (void *)t->anal, (void *)t->synth_off, (void *)t->anal_off,
                  (void *)t->err})
    if (q) cudaFree(q);
  delete t;
  p->tc = nullptr;
}

const TsTcTab &ts_tc_tab(ts_plan p) { return static_cast<ts_tc_tables *>(p->tc)->tab; }
int ts_tc_ntile(ts_plan p) { return static_cast<ts_tc_tables *>(p->tc)->ntile; }
size_t ts_tc_bytes(ts_plan p) { return p->tc ? static_cast<ts_tc_tables *>(p->tc)->bytes : 0; }

// pipeline depth and shared memory of the two kernels
namespace {
const size_t kSmemBudget = 227 * 1024 - 2048;
int synth_stages(ts_plan p) {
  const size_t stage = 2 * 16384 + 2 * (size_t)ts_tc_tab(p).NL * 128;
  return (int)std::min<size_t>(TS_TC_MAXSTAGE, kSmemBudget / stage);
}
int analys_N(ts_plan p) { return std::min(256, ((kpar_h(p->lmax, 0, 0) + 15) / 16) * 16); }
}  // namespace

int ts_tc_synth_stages(ts_plan p) { return synth_stages(p); }
int ts_tc_analys_stages(ts_plan p) {
  // the planner's dry run has no tables: derive from the grid alone
  const size_t stage = 2 * 16384 + 2 * (size_t)analys_N(p) * 128;
  return (int)std::min<size_t>(TS_TC_MAXSTAGE, kSmemBudget / stage);
}

size_t ts_tc_synth_smem(ts_plan p) {
  const size_t stage = 2 * 16384 + 2 * (size_t)ts_tc_tab(p).NL * 128;
  return synth_stages(p) * stage + 1024 + sizeof(TsTcPipe);
}

size_t ts_tc_analys_smem(ts_plan p) {
  const int N = analys_N(p);
  const size_t stage = 2 * 16384 + 2 * (size_t)N * 128;
  return std::max(ts_tc_analys_stages(p) * stage, (size_t)N * 2 * TS_TC_FIELDS * 4) + 1024 +
         sizeof(TsTcPipe);
}

void ts_launch_leg_synth_tc(ts_plan p, const TsFields &q, float2 *fm, long fs, int nf,
                            cudaStream_t s) {
  static bool attr = false;
  if (!attr) {
    TS_CUDA(cudaFuncSetAttribute(ts_leg_synth_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)p->ctx->smem_optin));
    attr = true;
  }
  const TsTcTab &tc = ts_tc_tab(p);
  dim3 grid((nf + TS_TC_FIELDS - 1) / TS_TC_FIELDS, p->mmax + 1, tc.nLT);
  ts_leg_synth_tc<<<grid, TS_TC_THREADS, ts_tc_synth_smem(p), s>>>(p->leg, tc, q, fm, fs, nf,
                                                                    synth_stages(p));
  TS_CUDA(cudaGetLastError());
}

void ts_launch_leg_analys_tc(ts_plan p, const float2 *g, long gs, float2 *out, long os, int nf,
                             cudaStream_t s) {
  static bool attr = false;
  if (!attr) {
    TS_CUDA(cudaFuncSetAttribute(ts_leg_analys_tc<TsAnalysStore>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)p->ctx->smem_optin));
    attr = true;
  }
  const TsTcTab &tc = ts_tc_tab(p);
  dim3 grid((nf + TS_TC_FIELDS - 1) / TS_TC_FIELDS, p->mmax + 1, 2 * ts_tc_ntile(p));
  TsAnalysStore epi{out, os};
  ts_leg_analys_tc<TsAnalysStore><<<grid, TS_TC_THREADS, ts_tc_analys_smem(p), s>>>(
      p->leg, tc, g, gs, epi, nf, TS_TC_FIELDS, ts_tc_analys_stages(p));
  TS_CUDA(cudaGetLastError());
}

int ts_tc_check_error(ts_plan p) {
  if (!p->tc) return 0;
  int h = 0;
  TS_CUDA(cudaMemcpy(&h, ts_tc_tab(p).err, sizeof(int), cudaMemcpyDeviceToHost));
  return h;
}
