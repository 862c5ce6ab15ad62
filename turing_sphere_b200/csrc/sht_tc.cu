// Tensor-core Legendre tables (FP64 on the GPU) and launchers.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstring>
#include <cstdlib>
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

// Tile geometry of the tensor-core kernels, from the plan's sizes alone (so
// the model compiler can size shared memory without the tables).  TS_TC_NL
// (the synthesis latitude tile, a multiple of 16 <= 96: two accumulator
// buffers of 2*NL columns and two 64-column operand slots fit in the 512
// TMEM columns) and TS_TC_LTL (the analysis degree tile, a multiple of
// 16 <= 128: two 128-column accumulator buffers and four operand slots) tune
// it, like the reference's SHT_* knobs (src/sht/sht.ts:47-56).
TsTcGeom ts_tc_geom(ts_plan p) {
  TsTcGeom g;
  int nl_cap = 96;
  if (p->tune_nl > 0)
    nl_cap = std::max(16, std::min(96, p->tune_nl & ~15));
  else if (const char *e = getenv("TS_TC_NL"))
    nl_cap = std::max(16, std::min(96, atoi(e) & ~15));
  g.NL = std::min(nl_cap, ((p->nh + 15) / 16) * 16);
  g.nLT = (p->nh + g.NL - 1) / g.NL;
  g.LTL = 128;
  if (p->tune_ltl > 0)
    g.LTL = std::max(16, std::min(128, p->tune_ltl & ~15));
  else if (const char *e = getenv("TS_TC_LTL"))
    g.LTL = std::max(16, std::min(128, atoi(e) & ~15));
  g.ntile = (kpar_h(p->lmax, 0, 0) + g.LTL - 1) / g.LTL;
  return g;
}

// max |value| over the first n[b] floats at img + off[b] (the hi halves of
// table blocks); one CTA per block
__global__ void ts_k_block_absmax(const char *img, const long *off, const int *n, int nb,
                                  float *out) {
  __shared__ float red[8];
  const int b = blockIdx.x;
  if (b >= nb) return;
  const float *v = reinterpret_cast<const float *>(img + off[b]);
  float mx = 0.f;
  for (int i = threadIdx.x; i < n[b]; i += blockDim.x) mx = fmaxf(mx, fabsf(v[i]));
  for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) mx = fmaxf(mx, red[w]);
    out[b] = fmaxf(red[0], mx);
  }
}

// Relative size below which a table value is dropped by the polar skip: the
// dropped terms are then ~10^3 below the FP32 rounding of the kept ones.
constexpr double kPolarSkip = 1e-10;

struct ts_tc_tables {
  char *synth = nullptr, *anal = nullptr;
  long *synth_off = nullptr, *anal_off = nullptr;
  int *err = nullptr;
  int *chunk_prefix = nullptr, *chunk_m = nullptr, *chunk_pc = nullptr;
  unsigned char *syn_zero = nullptr, *syn_cs = nullptr;
  int *ana_c0 = nullptr;
  int *w_kmin = nullptr;  // per (latitude chunk, parity): the m from which it is never read
  // synthesis tiles, synthesis degree chunks and analysis latitude chunks the polar skip drops
  int skip_syn = 0, skip_syn_chunks = 0, skip_ana = 0;
  ts_dbuf qimg, wimg, gscratch;  // operand images and a G scratch of the standalone transforms
  TsTcTab tab{};
  size_t bytes = 0;
  int ntile = 1;  // analysis l tiles per parity (grid.z = 2*ntile)
};

// Polar skip (the associated Legendre functions of high m vanish to many
// digits near the poles): find the synthesis tiles and the leading analysis
// latitude chunks whose table values are all below kPolarSkip times the
// largest value of their m (synthesis) or of their tile (analysis), from the
// tables themselves, and give the kernels the skip lists.
void tc_polar_skip(ts_plan p, ts_tc_tables *t, const std::vector<long> &soff,
                   const std::vector<long> &aoff, int nLC) {
  if (const char *e = getenv("TS_TC_POLAR_SKIP"))
    if (e[0] == '0') return;
  const TsTcGeom gm = ts_tc_geom(p);
  const int NL = gm.NL, nLT = gm.nLT, LTL = gm.LTL, M = p->mmax + 1;
  // synthesis blocks (m, chunk, lt): hi half = NL rows x 32 floats
  std::vector<long> off;
  std::vector<int> n;
  std::vector<int> sblk_m, sblk_lt;
  for (int m = 0; m < M; m++) {
    int nch = 0;
    for (int par = 0; par < 2; par++) nch += (kpar_h(p->lmax, m, par) + TS_TC_KCH - 1) / TS_TC_KCH;
    for (int ch = 0; ch < nch; ch++)
      for (int lt = 0; lt < nLT; lt++) {
        off.push_back(soff[m] + ((long)ch * nLT + lt) * 2 * NL * 128);
        n.push_back(NL * 32);
        sblk_m.push_back(m);
        sblk_lt.push_back(lt);
      }
  }
  const size_t nsyn = off.size();
  // analysis blocks (m, par, ltile, c): hi half = N rows x 32 floats
  std::vector<int> ablk_tile;  // (2 m + par) ntile + ltile
  for (int m = 0; m < M; m++) {
    long a = aoff[m];
    for (int par = 0; par < 2; par++) {
      const int kp = kpar_h(p->lmax, m, par);
      for (int lt = 0, lo = 0; lo < kp; lt++, lo += LTL) {
        const int N = ((std::min(kp, lo + LTL) - lo + 15) / 16) * 16;
        for (int c = 0; c < nLC; c++) {
          off.push_back(a + (long)c * 2 * N * 128);
          n.push_back(N * 32);
          ablk_tile.push_back((2 * m + par) * t->ntile + lt);
        }
        a += (long)nLC * 2 * N * 128;
      }
    }
  }
  const size_t nb = off.size();
  long *d_off = nullptr;
  int *d_n = nullptr;
  float *d_mx = nullptr;
  TS_CUDA(cudaMalloc(&d_off, sizeof(long) * nb));
  TS_CUDA(cudaMalloc(&d_n, sizeof(int) * nb));
  TS_CUDA(cudaMalloc(&d_mx, sizeof(float) * nb));
  TS_CUDA(cudaMemcpy(d_off, off.data(), sizeof(long) * nb, cudaMemcpyHostToDevice));
  TS_CUDA(cudaMemcpy(d_n, n.data(), sizeof(int) * nb, cudaMemcpyHostToDevice));
  if (nsyn)
    ts_k_block_absmax<<<(unsigned)nsyn, 256, 0, p->ctx->stream>>>(t->synth, d_off, d_n, (int)nsyn,
                                                                  d_mx);
  if (nb > nsyn)
    ts_k_block_absmax<<<(unsigned)(nb - nsyn), 256, 0, p->ctx->stream>>>(
        t->anal, d_off + nsyn, d_n + nsyn, (int)(nb - nsyn), d_mx + nsyn);
  std::vector<float> mx(nb);
  TS_CUDA(cudaGetLastError());
  TS_CUDA(cudaMemcpyAsync(mx.data(), d_mx, sizeof(float) * nb, cudaMemcpyDeviceToHost,
                          p->ctx->stream));
  TS_CUDA(cudaStreamSynchronize(p->ctx->stream));
  cudaFree(d_off);
  cudaFree(d_n);
  cudaFree(d_mx);
  // synthesis: tile (m, lt) is dropped when all its blocks are negligible
  std::vector<double> mmax_m(M, 0.0), tmax(M * nLT, 0.0);
  for (size_t b = 0; b < nsyn; b++) {
    mmax_m[sblk_m[b]] = std::max(mmax_m[sblk_m[b]], (double)mx[b]);
    double &tm = tmax[sblk_m[b] * nLT + sblk_lt[b]];
    tm = std::max(tm, (double)mx[b]);
  }
  // leading degree-chunk pairs of each tile, both parities negligible; at
  // least one chunk of each parity stays (it initialises the accumulator)
  std::vector<unsigned char> csk(M * nLT, 0);
  {
    size_t b = 0;
    for (int m = 0; m < M; m++) {
      const int n0 = (kpar_h(p->lmax, m, 0) + TS_TC_KCH - 1) / TS_TC_KCH;
      const int n1 = (kpar_h(p->lmax, m, 1) + TS_TC_KCH - 1) / TS_TC_KCH;
      const size_t mb = b;  // block (ch, lt) of m at mb + ch nLT + lt
      b += (size_t)(n0 + n1) * nLT;
      if (n1 == 0) continue;
      const int cap = std::min(std::min(n0, n1) - 1, 255);
      for (int lt = 0; lt < nLT; lt++) {
        int c = 0;
        while (c < cap && mx[mb + (size_t)c * nLT + lt] < kPolarSkip * mmax_m[m] &&
               mx[mb + (size_t)(n0 + c) * nLT + lt] < kPolarSkip * mmax_m[m])
          c++;
        csk[m * nLT + lt] = (unsigned char)c;
      }
    }
  }
  std::vector<unsigned char> zero(M * nLT, 0);
  for (int m = 0; m < M; m++)
    for (int lt = 0; lt < nLT; lt++)
      if (mmax_m[m] > 0 && tmax[m * nLT + lt] < kPolarSkip * mmax_m[m]) {
        zero[m * nLT + lt] = 1;
        t->skip_syn++;
      }
  // analysis: leading chunks of a tile below the threshold of the tile's max
  const int ntiles = 2 * M * t->ntile;
  std::vector<double> amax(ntiles, 0.0);
  for (size_t b = nsyn; b < nb; b++)
    amax[ablk_tile[b - nsyn]] = std::max(amax[ablk_tile[b - nsyn]], (double)mx[b]);
  std::vector<int> c0(ntiles, 0);
  std::vector<int> seen(ntiles, 0);
  for (size_t b = nsyn; b < nb; b++) {  // blocks of a tile come in chunk order
    const int tl = ablk_tile[b - nsyn];
    if (seen[tl]) continue;
    if (mx[b] < kPolarSkip * amax[tl])
      c0[tl]++;
    else
      seen[tl] = 1;
  }
  for (int tl = 0; tl < ntiles; tl++) t->skip_ana += c0[tl];
  std::vector<int> wc0(2 * M, nLC);
  for (int tl = 0; tl < ntiles; tl++) {
    const int mp = tl / t->ntile;  // 2 m + parity
    // tiles without degrees (cnt 0) read nothing; the others bound it
    const int m = mp / 2, par = mp % 2, lt = tl % t->ntile;
    if (lt * LTL < kpar_h(p->lmax, m, par)) wc0[mp] = std::min(wc0[mp], c0[tl]);
  }
  // per (chunk, parity): the smallest m0 such that no tile of any m >= m0
  // reads the chunk (the W writers leave those blocks out)
  std::vector<int> kmin(2 * nLC, M);
  for (int par = 0; par < 2; par++)
    for (int ch = 0; ch < nLC; ch++) {
      int m0 = M;
      while (m0 > 0 && ch < wc0[2 * (m0 - 1) + par]) m0--;
      kmin[2 * ch + par] = m0;
    }
  TS_CUDA(cudaMalloc(&t->w_kmin, sizeof(int) * kmin.size()));
  TS_CUDA(cudaMemcpy(t->w_kmin, kmin.data(), sizeof(int) * kmin.size(), cudaMemcpyHostToDevice));
  for (int i = 0; i < M * nLT; i++)
    if (!zero[i]) t->skip_syn_chunks += 2 * csk[i];
  TS_CUDA(cudaMalloc(&t->syn_cs, csk.size()));
  TS_CUDA(cudaMemcpy(t->syn_cs, csk.data(), csk.size(), cudaMemcpyHostToDevice));
  t->tab.syn_cs = t->syn_cs;
  TS_CUDA(cudaMalloc(&t->syn_zero, zero.size()));
  TS_CUDA(cudaMalloc(&t->ana_c0, sizeof(int) * c0.size()));
  TS_CUDA(cudaMemcpy(t->syn_zero, zero.data(), zero.size(), cudaMemcpyHostToDevice));
  TS_CUDA(cudaMemcpy(t->ana_c0, c0.data(), sizeof(int) * c0.size(), cudaMemcpyHostToDevice));
  t->tab.syn_zero = t->syn_zero;
  t->tab.ana_c0 = t->ana_c0;
}

void ts_tc_init(ts_plan p) {
  auto *t = new ts_tc_tables();
  p->tc = t;
  const int nh = p->nh;
  const TsTcGeom gm = ts_tc_geom(p);
  const int NL = gm.NL, nLT = gm.nLT, LTL = gm.LTL;
  const int nLC = (nh + TS_TC_KCH - 1) / TS_TC_KCH;
  std::vector<long> soff(p->mmax + 2), aoff(p->mmax + 2);
  std::vector<int> cpre(p->mmax + 2), cm, cpc;
  long s = 0, a = 0;
  for (int m = 0; m <= p->mmax; m++) {
    soff[m] = s;
    aoff[m] = a;
    cpre[m] = (int)cm.size();
    int nch = 0;
    for (int par = 0; par < 2; par++) {
      const int kp = kpar_h(p->lmax, m, par);
      const int nc = (kp + TS_TC_KCH - 1) / TS_TC_KCH;
      for (int c = 0; c < nc; c++) {
        cm.push_back(m);
        cpc.push_back((par << 16) | c);
      }
      nch += nc;
      for (int lt0 = 0; lt0 < kp; lt0 += LTL) {
        const int cnt = std::min(kp, lt0 + LTL) - lt0;
        a += (long)nLC * 2 * (((cnt + 15) / 16) * 16) * 128;
      }
    }
    s += (long)nch * nLT * 2 * NL * 128;
  }
  soff[p->mmax + 1] = s;
  aoff[p->mmax + 1] = a;
  cpre[p->mmax + 1] = (int)cm.size();
  TS_CUDA(cudaMalloc(&t->chunk_prefix, sizeof(int) * cpre.size()));
  TS_CUDA(cudaMalloc(&t->chunk_m, sizeof(int) * cm.size()));
  TS_CUDA(cudaMalloc(&t->chunk_pc, sizeof(int) * cpc.size()));
  TS_CUDA(cudaMemcpy(t->chunk_prefix, cpre.data(), sizeof(int) * cpre.size(), cudaMemcpyHostToDevice));
  TS_CUDA(cudaMemcpy(t->chunk_m, cm.data(), sizeof(int) * cm.size(), cudaMemcpyHostToDevice));
  TS_CUDA(cudaMemcpy(t->chunk_pc, cpc.data(), sizeof(int) * cpc.size(), cudaMemcpyHostToDevice));
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
  tc.chunk_prefix = t->chunk_prefix;
  tc.chunk_m = t->chunk_m;
  tc.chunk_pc = t->chunk_pc;
  tc.nchunks = (int)cm.size();
  tc.ntile = t->ntile;
  tc.syn_zero = nullptr;
  tc.syn_cs = nullptr;
  tc.ana_c0 = nullptr;
  dim3 grid((nh + 63) / 64, p->mmax + 1);
  ts_k_tc_tables<<<grid, 64, 0, p->ctx->stream>>>(p->lmax, p->mmax, nh, p->d_x64, p->d_ab64,
                                                  p->d_amm64, tc, t->synth, t->anal);
  TS_CUDA(cudaGetLastError());
  TS_CUDA(cudaStreamSynchronize(p->ctx->stream));
  tc_polar_skip(p, t, soff, aoff, nLC);
}

void ts_tc_free(ts_plan p) {
  auto *t = static_cast<ts_tc_tables *>(p->tc);
  if (!t) return;
  for (void *q : {(void *)t->synth, (void *)t->anal, (void *)t->synth_off, (void *)t->anal_off,
                  (void *)t->err, (void *)t->chunk_prefix, (void *)t->chunk_m, (void *)t->chunk_pc,
                  (void *)t->syn_zero, (void *)t->syn_cs, (void *)t->ana_c0, (void *)t->w_kmin})
    if (q) cudaFree(q);
  t->qimg.release();
  t->wimg.release();
  t->gscratch.release();
  delete t;
  p->tc = nullptr;
}

const TsTcTab &ts_tc_tab(ts_plan p) { return static_cast<ts_tc_tables *>(p->tc)->tab; }

void ts_tc_set_fault(ts_plan p, int stall_copies, unsigned wait_limit) {
  TsTcTab &t = static_cast<ts_tc_tables *>(p->tc)->tab;
  t.stall_copies = stall_copies;
  t.wait_limit = wait_limit;
}
const int *ts_tc_w_kmin(ts_plan p) {
  const auto *t = static_cast<ts_tc_tables *>(p->tc);
  return t ? t->w_kmin : nullptr;
}

void ts_tc_skip_counts(ts_plan p, int *tiles, int *chunks) {
  const auto *t = static_cast<ts_tc_tables *>(p->tc);
  *tiles = t ? t->skip_syn : 0;
  *chunks = t ? t->skip_ana + t->skip_syn_chunks : 0;
}
int ts_tc_ntile(ts_plan p) { return static_cast<ts_tc_tables *>(p->tc)->ntile; }
size_t ts_tc_bytes(ts_plan p) { return p->tc ? static_cast<ts_tc_tables *>(p->tc)->bytes : 0; }

// pipeline depth and shared memory of the two persistent kernels
namespace {
const size_t kSmemBudget = 227 * 1024 - 2048;
size_t synth_stage(ts_plan p) { return TS_TC_STAGE_A + 2 * (size_t)ts_tc_geom(p).NL * 128; }
int synth_stages(ts_plan p) {
  return (int)std::min<size_t>(TS_TC_MAXSTAGE,
                               (kSmemBudget - 2 * TS_TC_SYN_NSTG * TS_TC_SYN_STAGING) / synth_stage(p));
}
int analys_N(ts_plan p) { return std::min(ts_tc_geom(p).LTL, ((kpar_h(p->lmax, 0, 0) + 15) / 16) * 16); }
size_t analys_stage(ts_plan p) { return TS_TC_STAGE_A + 2 * (size_t)analys_N(p) * 128; }
size_t analys_staging(ts_plan p) {
  return 2 * (size_t)std::min(analys_N(p), TS_TC_ANA_COLS) * 2 * TS_TC_ANA_ROW * 4;
}
}  // namespace

int ts_tc_synth_stages(ts_plan p) { return synth_stages(p); }
int ts_tc_analys_stages(ts_plan p) {
  return (int)std::min<size_t>(TS_TC_MAXSTAGE, (kSmemBudget - analys_staging(p)) / analys_stage(p));
}
int ts_tc_analys_nmax(ts_plan p) { return analys_N(p); }

size_t ts_tc_synth_smem(ts_plan p) {
  return synth_stages(p) * synth_stage(p) + 2 * TS_TC_SYN_NSTG * TS_TC_SYN_STAGING + 1024 +
         sizeof(TsTcPipe);
}

size_t ts_tc_analys_smem(ts_plan p) {
  return ts_tc_analys_stages(p) * analys_stage(p) + analys_staging(p) + 1024 + sizeof(TsTcPipe);
}

int ts_tc_ctas(ts_plan p, long ntiles) {
  return (int)std::max<long>(1, std::min<long>(p->ctx->sm_count, ntiles));
}

// ---------------------------------------------------------- operand images

namespace {

// Q (fields) -> raw fp32 synthesis image; grid = (nchunks, q_nfb), block =
// 256: warp -> 8 fields, lane -> k (coalesced 128-byte image rows).  The CTA
// of a parity-0 chunk also writes the parity-1 chunk of the same k range
// (degrees m + 2j and m + 2j + 1 are adjacent, one 16-byte load when
// aligned); parity-1 CTAs leave at once.  A thread issues the loads of all
// its 8 fields before its first store, so 8 loads per thread are in flight.
__global__ void ts_k_qimage(TsLegTab t, TsTcTab tc, TsFields q, int nfields, char *img,
                            int nfb) {
  constexpr int NF = TS_TC_FIELDS / 8;  // fields per thread
  const int c = blockIdx.x, fb = blockIdx.y;
  const int pc = tc.chunk_pc[c];
  if (pc >> 16) return;  // parity-1 chunks are written with their parity-0 partner
  const int m = tc.chunk_m[c], cc = pc & 0xffff;
  const int kp0 = ts_kpar(t.lmax, m, 0), kp1 = ts_kpar(t.lmax, m, 1);
  const int n0 = (kp0 + TS_TC_KCH - 1) / TS_TC_KCH, n1 = (kp1 + TS_TC_KCH - 1) / TS_TC_KCH;
  const long base = ts_lm_base(t.lmax, m);
  char *blk0 = img + ((long)c * nfb + fb) * 16384;
  const bool has1 = cc < n1;
  char *blk1 = img + ((long)(tc.chunk_prefix[m] + n0 + cc) * nfb + fb) * 16384;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int j = cc * TS_TC_KCH + lane;
  const bool v0 = j < kp0, v1 = j < kp1;
  float2 a[NF], b[NF];
#pragma unroll
  for (int i = 0; i < NF; i++) {
    const int f = fb * TS_TC_FIELDS + warp + 8 * i;
    a[i] = b[i] = make_float2(0.f, 0.f);
    if (f < nfields && v0) {
      // degrees l = m + 2j (parity 0) and m + 2j + 1 (parity 1) are adjacent
      const float2 *src = ts_field(q, f) + base + 2 * j;
      if (v1 && (reinterpret_cast<unsigned long long>(src) & 15) == 0) {
        const float4 x = __ldg(reinterpret_cast<const float4 *>(src));
        a[i] = make_float2(x.x, x.y);
        b[i] = make_float2(x.z, x.w);
      } else {
        a[i] = __ldg(src);
        if (v1) b[i] = __ldg(src + 1);
      }
    }
  }
#pragma unroll
  for (int i = 0; i < NF; i++) {
    const int fl = warp + 8 * i;
    *reinterpret_cast<float *>(blk0 + ts_swz_img(2 * fl, lane)) = a[i].x;
    *reinterpret_cast<float *>(blk0 + ts_swz_img(2 * fl + 1, lane)) = a[i].y;
    if (has1) {
      *reinterpret_cast<float *>(blk1 + ts_swz_img(2 * fl, lane)) = b[i].x;
      *reinterpret_cast<float *>(blk1 + ts_swz_img(2 * fl + 1, lane)) = b[i].y;
    }
  }
}

// G[field][m][lat] -> raw fp32 W image (the fold the Fourier analysis does
// itself when it can: see ts_f2_analys_w).  grid = (nLC, nfb*2, mmax+1),
// block = 256: warp -> 8 fields, lane -> latitude of the chunk
__global__ void ts_k_wimage(TsLegTab t, const float2 *g, long gs, int nfields, int fpb, int nfb,
                            int nlc, char *img) {
  const int c = blockIdx.x, fb = blockIdx.y >> 1, par = blockIdx.y & 1, m = blockIdx.z;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int lat = c * TS_TC_KCH + lane;
  const bool live = lat < t.nh;
  const float w = live ? t.wq[lat] : 0.f;
  const int south = t.nlat - 1 - lat;
  char *blk = img + ((((long)m * nfb + fb) * 2 + par) * nlc + c) * 16384;
  constexpr int NF = TS_TC_FIELDS / 8;  // fields per thread, loaded before any store
  float2 gn[NF], gsv[NF];
#pragma unroll
  for (int i = 0; i < NF; i++) {
    const int fl = warp + 8 * i, f = fb * fpb + fl;
    gn[i] = gsv[i] = make_float2(0.f, 0.f);
    if (live && fl < fpb && f < nfields) {
      const float2 *src = g + (long)f * gs + (long)m * t.nlat;
      gn[i] = __ldg(src + lat);
      if (south != lat) gsv[i] = __ldg(src + south);
    }
  }
#pragma unroll
  for (int i = 0; i < NF; i++) {
    const int fl = warp + 8 * i;
    const float a = par ? gn[i].x - gsv[i].x : gn[i].x + gsv[i].x;
    const float b = par ? gn[i].y - gsv[i].y : gn[i].y + gsv[i].y;
    *reinterpret_cast<float *>(blk + ts_swz_img(2 * fl, lane)) = a * w;
    *reinterpret_cast<float *>(blk + ts_swz_img(2 * fl + 1, lane)) = b * w;
  }
}

void ensure_zeroed(ts_dbuf &b, size_t bytes) {
  if (bytes <= b.cap) return;
  b.ensure(bytes);
  TS_CUDA(cudaMemset(b.p, 0, b.cap));
}

}  // namespace

size_t ts_tc_qimg_bytes(ts_plan p, int nfields) {
  const long nfb = (nfields + TS_TC_FIELDS - 1) / TS_TC_FIELDS;
  return (size_t)ts_tc_tab(p).nchunks * nfb * 16384;
}

size_t ts_tc_wimg_bytes(ts_plan p, int nfields, int fpb) {
  const long nfb = (nfields + fpb - 1) / fpb;
  return (size_t)(p->mmax + 1) * nfb * 2 * ts_tc_tab(p).nLC * 16384;
}

void ts_launch_qimage(ts_plan p, const TsFields &q, int nf, char *img, cudaStream_t s) {
  const int nfb = (nf + TS_TC_FIELDS - 1) / TS_TC_FIELDS;
  dim3 grid(ts_tc_tab(p).nchunks, nfb);
  ts_k_qimage<<<grid, 256, 0, s>>>(p->leg, ts_tc_tab(p), q, nf, img, nfb);
  TS_CUDA(cudaGetLastError());
}

void ts_launch_wimage(ts_plan p, const float2 *g, long gs, int nf, int fpb, char *img,
                      cudaStream_t s) {
  const int nfb = (nf + fpb - 1) / fpb;
  const int nlc = ts_tc_tab(p).nLC;
  dim3 grid(nlc, nfb * 2, p->mmax + 1);
  ts_k_wimage<<<grid, 256, 0, s>>>(p->leg, g, gs, nf, fpb, nfb, nlc, img);
  TS_CUDA(cudaGetLastError());
}

static_assert(sizeof(TsTmaDesc) == sizeof(CUtensorMap), "tensor map size");

namespace {
PFN_cuTensorMapEncodeTiled_v12000 tma_encoder() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }();
  return fn;
}

// fm[field][m][lat] (float2, field stride fs) as floats [field][m][2 nlat],
// box (16 latitudes x re,im = 32 floats, 1 m, 64 fields), 128-byte swizzle
bool fm_store_map(ts_plan p, TsTmaDesc *map, float2 *fm, long fs, int nf) {
  const auto encode = tma_encoder();
  if (!encode || (reinterpret_cast<uintptr_t>(fm) & 15) || (p->nlat & 1) || (fs & 1)) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)2 * p->nlat, (cuuint64_t)p->mmax + 1, (cuuint64_t)nf};
  const cuuint64_t strides[2] = {(cuuint64_t)p->nlat * 8, (cuuint64_t)fs * 8};
  const cuuint32_t box[3] = {32, 1, TS_TC_FIELDS};
  const cuuint32_t estr[3] = {1, 1, 1};
  return encode(reinterpret_cast<CUtensorMap *>(map), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, fm, dims,
                strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
}  // namespace

void ts_launch_synth_tc_img(ts_plan p, const char *qimg, int nf, float2 *fm, long fs,
                            cudaStream_t s) {
  TsTmaDesc map;
  memset(&map, 0, sizeof map);
  const int tma_ok = fm_store_map(p, &map, fm, fs, nf) ? 1 : 0;  // else plain stores
  ts_allow_smem((const void *)ts_leg_synth_tc, p->ctx->device, ts_tc_synth_smem(p));
  const TsTcTab &tc = ts_tc_tab(p);
  const int nfb = (nf + TS_TC_FIELDS - 1) / TS_TC_FIELDS;
  const int ctas = ts_tc_ctas(p, (long)(p->mmax + 1) * tc.nLT * nfb);
  ts_leg_synth_tc<<<ctas, TS_TC_THREADS, ts_tc_synth_smem(p), s>>>(p->leg, tc, qimg, nfb, fm, fs,
                                                                   nf, synth_stages(p), map, tma_ok);
  TS_CUDA(cudaGetLastError());
}

// fields -> q image (caller's buffer, or the plan's) -> fm
void ts_launch_leg_synth_tc(ts_plan p, const TsFields &q, float2 *fm, long fs, int nf,
                            cudaStream_t s, ts_dbuf *qbuf) {
  auto *t = static_cast<ts_tc_tables *>(p->tc);
  ts_dbuf &b = qbuf ? *qbuf : t->qimg;
  ensure_zeroed(b, ts_tc_qimg_bytes(p, nf));
  ts_launch_qimage(p, q, nf, (char *)b.p, s);
  ts_launch_synth_tc_img(p, (const char *)b.p, nf, fm, fs, s);
}

void ts_launch_analys_tc_img(ts_plan p, const char *wimg, int nf, float2 *out, long os,
                             cudaStream_t s) {
  ts_allow_smem((const void *)ts_leg_analys_tc<TsAnalysStore>, p->ctx->device,
                ts_tc_analys_smem(p));
  const int nfb = (nf + TS_TC_FIELDS - 1) / TS_TC_FIELDS;
  const int ntile = ts_tc_ntile(p);
  const int ctas = ts_tc_ctas(p, (long)(p->mmax + 1) * 2 * ntile * nfb);
  TsAnalysStore epi{out, os};
  ts_leg_analys_tc<TsAnalysStore><<<ctas, TS_TC_THREADS, ts_tc_analys_smem(p), s>>>(
      p->leg, ts_tc_tab(p), wimg, nfb, epi, nf, TS_TC_FIELDS, ts_tc_analys_stages(p),
      ts_tc_analys_nmax(p), ntile);
  TS_CUDA(cudaGetLastError());
}

// G (gm layout) -> w image -> q: the stage-level analysis of a TC plan
void ts_launch_leg_analys_tc(ts_plan p, const float2 *g, long gs, float2 *out, long os, int nf,
                             cudaStream_t s) {
  auto *t = static_cast<ts_tc_tables *>(p->tc);
  ensure_zeroed(t->wimg, ts_tc_wimg_bytes(p, nf, TS_TC_FIELDS));
  ts_launch_wimage(p, g, gs, nf, TS_TC_FIELDS, (char *)t->wimg.p, s);
  ts_launch_analys_tc_img(p, (const char *)t->wimg.p, nf, out, os, s);
}

// spat -> w image directly (register FFT over latitude pairs) when the grid
// allows it, else spat -> G scratch -> w image; then -> q
void ts_analys_tc_full(ts_plan p, const float *spat, long ss, float *qlm, int nf, cudaStream_t s) {
  auto *t = static_cast<ts_tc_tables *>(p->tc);
  ensure_zeroed(t->wimg, ts_tc_wimg_bytes(p, nf, TS_TC_FIELDS));
  if (!ts_launch_fourier_analys_w(p, spat, ss, nf, TS_TC_FIELDS, (char *)t->wimg.p, s)) {
    const long field = (long)(p->mmax + 1) * p->nlat;
    t->gscratch.ensure(sizeof(float2) * field * nf);
    ts_launch_fourier_analys(p, spat, ss, (float2 *)t->gscratch.p, field, nf, s);
    ts_launch_wimage(p, (const float2 *)t->gscratch.p, field, nf, TS_TC_FIELDS, (char *)t->wimg.p, s);
  }
  ts_launch_analys_tc_img(p, (const char *)t->wimg.p, nf, (float2 *)qlm, p->nlm, s);
}

int ts_tc_check_error(ts_plan p) {
  if (!p->tc) return 0;
  int h = 0;
  TS_CUDA(cudaMemcpy(&h, ts_tc_tab(p).err, sizeof(int), cudaMemcpyDeviceToHost));
  return h;
}
