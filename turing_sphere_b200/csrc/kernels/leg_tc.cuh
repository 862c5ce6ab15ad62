// Tensor-core Legendre stage: per-m dense contractions on tcgen05 with
// 3-pass split-TF32 products accumulated in FP32 in tensor memory.
//
// For one m and a block of 64 complex fields (128 real rows: row = 2f + re|im)
//   synthesis  D_par[row, lat] = sum_{l of parity par} Q[row, l] P_l(lat)
//              north = D_0 + D_1, south = D_0 - D_1      (parity fold)
//   analysis   D[row, l]       = sum_{lat} W_par[row, lat] P_l(lat)
//              W_0 = w (G_north + G_south), W_1 = w (G_north - G_south)
// P comes from tables computed in FP64 on the GPU and stored as TF32 hi/lo
// pairs, already in the shared-memory byte image the MMA reads (K-major,
// 128-byte swizzle), so a CTA streams them with plain 16-byte copies.  The
// data operand (Q or W) is split on the fly: hi = rna_tf32(x),
// lo = rna_tf32(x - hi); each k-step issues hi*hi + hi*lo + lo*hi.
//
// One elected thread issues the MMAs; tcgen05.commit signals an mbarrier per
// shared-memory stage (two stages).  Every wait is bounded: on timeout the
// kernel records an error flag, skips the epilogue, frees its tensor memory
// and returns.
#pragma once
#include "ts_common.cuh"

#define TS_TC_ROWS 128          // MMA M: 64 complex fields
#define TS_TC_FIELDS 64
#define TS_TC_KCH 32            // tf32 values per 128-byte swizzle row
#define TS_TC_WAIT_LIMIT (1u << 24)



// ------------------------------------------------------------ PTX helpers
TS_DEV unsigned ts_smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

TS_DEV float ts_rna_tf32(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

TS_DEV void ts_mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(ts_smem_u32(bar)), "r"(count)
               : "memory");
}

// Wait for the completion of the barrier phase of the given parity; gives up
// after `limit` polls and returns false.
TS_DEV bool ts_mbar_wait(unsigned long long *bar, unsigned parity, unsigned limit) {
  const unsigned addr = ts_smem_u32(bar);
  for (unsigned i = 0; i < limit; i++) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

TS_DEV void ts_tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
TS_DEV void ts_tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
TS_DEV void ts_fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (SBO), version 1 (sm_100).
TS_DEV unsigned long long ts_umma_desc(unsigned saddr) {
  unsigned long long d = 0;
  d |= (unsigned long long)((saddr >> 4) & 0x3FFF);
  d |= (unsigned long long)1 << 16;              // LBO (unused for swizzled K-major)
  d |= (unsigned long long)(1024 >> 4) << 32;    // SBO
  d |= (unsigned long long)1 << 46;              // version
  d |= (unsigned long long)2 << 61;              // SWIZZLE_128B
  return d;
}

// Instruction descriptor: D f32, A/B tf32, both K-major, M = 128, N = n.
TS_DEV unsigned ts_idesc_tf32(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((unsigned)(n >> 3) << 17) |
         ((unsigned)(TS_TC_ROWS >> 4) << 24);
}

TS_DEV void ts_mma_tf32(unsigned dtmem, unsigned long long adesc, unsigned long long bdesc,
                        unsigned idesc, unsigned accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      ::"r"(dtmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0),
      "r"(0));
}

TS_DEV void ts_mma_commit(unsigned long long *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   ts_smem_u32(bar))
               : "memory");
}

TS_DEV void ts_tmem_ld16(unsigned taddr, float (&v)[16]) {
  unsigned r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

TS_DEV unsigned ts_tmem_cols(int n) {
  unsigned c = 32;
  while (c < (unsigned)n) c <<= 1;
  return c;
}

// warp 0 allocates `ncols` columns of tensor memory; the base lands in *slot
TS_DEV void ts_tmem_alloc(unsigned *slot, unsigned ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   ts_smem_u32(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

TS_DEV void ts_tmem_free(unsigned base, unsigned ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols)
               : "memory");
}

// byte offset of element (row r, k) in a K-major 128B-swizzled tile whose
// rows are 32 tf32 values
TS_DEV int ts_swz(int r, int k) {
  return (r >> 3) * 1024 + (r & 7) * 128 + ((((k >> 2) ^ (r & 7))) << 4) + ((k & 3) << 2);
}

// 16-byte copy of `bytes` from global to shared by the whole CTA
TS_DEV void ts_copy16(char *dst, const char *src, int bytes) {
  const int4 *s = reinterpret_cast<const int4 *>(src);
  int4 *d = reinterpret_cast<int4 *>(dst);
  for (int i = threadIdx.x; i < (bytes >> 4); i += blockDim.x) d[i] = __ldg(s + i);
}

// ---------------------------------------------------------- table geometry
TS_DEV int ts_kpar(int lmax, int m, int par) {  // l of parity par: l = m + par + 2j
  const int K = lmax - m + 1;
  return (K + 1 - par) / 2;
}
TS_DEV int ts_round16(int n) { return (n + 15) & ~15; }

// analysis tile (par, ltile) of m: l count, N (rows of its image), byte offset
TS_DEV int ts_atile_count(int lmax, int m, int par, int ltile, int LTL) {
  const int kp = ts_kpar(lmax, m, par);
  const int lo = ltile * LTL, hi = min(kp, lo + LTL);
  return hi > lo ? hi - lo : 0;
}

TS_DEV long ts_atile_offset(const TsTcTab &tc, int lmax, int m, int par, int ltile) {
  long off = tc.anal_off[m];
  for (int p = 0; p <= par; p++) {
    const int nt = (ts_kpar(lmax, m, p) + tc.LTL - 1) / tc.LTL;
    for (int t = 0; t < nt; t++) {
      if (p == par && t == ltile) return off;
      const int n = ts_round16(ts_atile_count(lmax, m, p, t, tc.LTL));
      off += (long)tc.nLC * 2 * n * 128;
    }
  }
  return off;
}

// ----------------------------------------------------------------- synthesis
//
// grid = (ceil(nfields/64), mmax+1, nLT), block = 128.  Dynamic shared memory:
// 1024-aligned, max(2 stages x (2*NL*128 + 2*16384), 2*128*(NL+4)*4) + 64.
__global__ void __launch_bounds__(128, 1)
ts_leg_synth_tc(TsLegTab t, TsTcTab tc, TsFields q, float2 *__restrict__ fm, long fm_stride,
                int nfields) {
  extern __shared__ __align__(1024) char ts_smem_st[];
  char *smem = (char *)(((unsigned long long)ts_smem_st + 1023) & ~1023ull);
  const int fb = blockIdx.x, m = blockIdx.y, lt = blockIdx.z;
  const int NL = tc.NL;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long base = ts_lm_base(t.lmax, m);
  const int kp0 = ts_kpar(t.lmax, m, 0), kp1 = ts_kpar(t.lmax, m, 1);
  const int nch0 = (kp0 + TS_TC_KCH - 1) / TS_TC_KCH, nch1 = (kp1 + TS_TC_KCH - 1) / TS_TC_KCH;
  const int C = nch0 + nch1;
  const int bbytes = NL * 128;                     // one B image (hi or lo)
  const int stage = 2 * bbytes + 2 * 16384;        // B hi, B lo, A hi, A lo
  const int SP = NL + 1;  // staging row pitch (floats), odd: conflict-free
  const int stage_all = max(2 * stage, 2 * TS_TC_ROWS * SP * 4);
  unsigned long long *bars = reinterpret_cast<unsigned long long *>(smem + stage_all);
  unsigned *slot = reinterpret_cast<unsigned *>(smem + stage_all + 16);
  const unsigned ncols = ts_tmem_cols(2 * NL);

  if (tid == 0) {
    ts_mbar_init(&bars[0], 1);
    ts_mbar_init(&bars[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) ts_tmem_alloc(slot, ncols);
  ts_tc_fence_before();
  __syncthreads();
  ts_tc_fence_after();
  const unsigned tmem = *slot;
  const unsigned idesc = ts_idesc_tf32(NL);
  bool ok = true;

  for (int c = 0; c < C && ok; c++) {
    const int b = c & 1;
    char *sb = smem + b * stage;
    if (c >= 2) ok = ts_mbar_wait(&bars[b], ((c >> 1) - 1) & 1, TS_TC_WAIT_LIMIT);
    if (!__syncthreads_and(ok)) {
      ok = false;
      break;
    }
    const int par = c < nch0 ? 0 : 1;
    const int cc = par ? c - nch0 : c;
    // P image chunk (hi then lo), laid out exactly as the MMA reads it
    const long src = tc.synth_off[m] + (long)((par ? nch0 : 0) + cc) * tc.nLT * 2 * bbytes +
                     (long)lt * 2 * bbytes;
    ts_copy16(sb, tc.synth + src, 2 * bbytes);
    // Q chunk split into hi/lo: thread -> (field, 16 consecutive k)
    {
      const int fl = tid & 63, kh = tid >> 6;
      const int f = fb * TS_TC_FIELDS + fl;
      const float2 *qf = f < nfields ? ts_field(q, f) + base : nullptr;
      char *ahi = sb + 2 * bbytes, *alo = ahi + 16384;
#pragma unroll
      for (int k4 = 0; k4 < 4; k4++) {
        float re[4], im[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int j = cc * TS_TC_KCH + kh * 16 + k4 * 4 + u;
          float2 v = make_float2(0.f, 0.f);
          if (qf && j < (par ? kp1 : kp0)) v = qf[par + 2 * j];
          re[u] = v.x;
          im[u] = v.y;
        }
        const int k = kh * 16 + k4 * 4;
        float4 h, l;
        h = make_float4(ts_rna_tf32(re[0]), ts_rna_tf32(re[1]), ts_rna_tf32(re[2]), ts_rna_tf32(re[3]));
        l = make_float4(ts_rna_tf32(re[0] - h.x), ts_rna_tf32(re[1] - h.y), ts_rna_tf32(re[2] - h.z),
                        ts_rna_tf32(re[3] - h.w));
        *reinterpret_cast<float4 *>(ahi + ts_swz(2 * fl, k)) = h;
        *reinterpret_cast<float4 *>(alo + ts_swz(2 * fl, k)) = l;
        h = make_float4(ts_rna_tf32(im[0]), ts_rna_tf32(im[1]), ts_rna_tf32(im[2]), ts_rna_tf32(im[3]));
        l = make_float4(ts_rna_tf32(im[0] - h.x), ts_rna_tf32(im[1] - h.y), ts_rna_tf32(im[2] - h.z),
                        ts_rna_tf32(im[3] - h.w));
        *reinterpret_cast<float4 *>(ahi + ts_swz(2 * fl + 1, k)) = h;
        *reinterpret_cast<float4 *>(alo + ts_swz(2 * fl + 1, k)) = l;
      }
    }
    ts_fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      ts_tc_fence_after();
      const unsigned bhi = ts_smem_u32(sb), blo = bhi + bbytes;
      const unsigned ahi = bhi + 2 * bbytes, alo = ahi + 16384;
      const unsigned d = tmem + (unsigned)(par * NL);
#pragma unroll
      for (int kk = 0; kk < 4; kk++) {
        const unsigned acc = (cc > 0 || kk > 0) ? 1u : 0u;
        ts_mma_tf32(d, ts_umma_desc(ahi + kk * 32), ts_umma_desc(bhi + kk * 32), idesc, acc);
        ts_mma_tf32(d, ts_umma_desc(ahi + kk * 32), ts_umma_desc(blo + kk * 32), idesc, 1u);
        ts_mma_tf32(d, ts_umma_desc(alo + kk * 32), ts_umma_desc(bhi + kk * 32), idesc, 1u);
      }
      ts_mma_commit(&bars[b]);
    }
  }
  // all MMAs done once the last commit has landed
  if (ok && C > 0) ok = ts_mbar_wait(&bars[(C - 1) & 1], ((C - 1) >> 1) & 1, TS_TC_WAIT_LIMIT);
  ok = __syncthreads_and(ok);
  ts_tc_fence_after();
  if (ok) {
    // TMEM -> shared staging sE/sO[row][NL+4]
    float *sE = reinterpret_cast<float *>(smem);
    float *sO = sE + TS_TC_ROWS * SP;
    const int row = warp * 32 + lane;
    for (int c0 = 0; c0 < NL; c0 += 16) {
      float v[16];
      ts_tmem_ld16(tmem + ((unsigned)(warp * 32) << 16) + (unsigned)c0, v);
#pragma unroll
      for (int i = 0; i < 16; i++) sE[row * SP + c0 + i] = v[i];
      if (nch1 > 0) {
        ts_tmem_ld16(tmem + ((unsigned)(warp * 32) << 16) + (unsigned)(NL + c0), v);
#pragma unroll
        for (int i = 0; i < 16; i++) sO[row * SP + c0 + i] = v[i];
      } else {
#pragma unroll
        for (int i = 0; i < 16; i++) sO[row * SP + c0 + i] = 0.f;
      }
    }
    ts_tc_fence_before();
    __syncthreads();
    for (int idx = tid; idx < TS_TC_FIELDS * NL; idx += blockDim.x) {
      const int fl = idx / NL, j = idx - fl * NL;
      const int f = fb * TS_TC_FIELDS + fl;
      const int lat = lt * NL + j;
      if (f >= nfields || lat >= t.nh) continue;
      const float er = sE[(2 * fl) * SP + j], ei = sE[(2 * fl + 1) * SP + j];
      const float orr = sO[(2 * fl) * SP + j], oi = sO[(2 * fl + 1) * SP + j];
      float2 *dst = fm + (long)f * fm_stride + (long)m * t.nlat;
      dst[lat] = make_float2(er + orr, ei + oi);
      const int south = t.nlat - 1 - lat;
      if (south != lat) dst[south] = make_float2(er - orr, ei - oi);
    }
  } else if (tid == 0) {
    atomicExch(tc.err, 1);
  }
  ts_tc_fence_before();
  __syncthreads();
  if (warp == 0) ts_tmem_free(tmem, ncols);
}

// ------------------------------------------------------------------ analysis
//
// grid = (ceil(nfields/per_cta), mmax+1, 2*ntile), block = 128; z = par*ntile
// + ltile (empty tiles return at once).  per_cta <= 64 fields.  Dynamic
// shared memory: 1024-aligned, max(2 stages x (2*16384 + 2*N*128),
// N*2*64*4) + 64, N <= LTL.
template <class Epi>
__global__ void __launch_bounds__(128, 1)
ts_leg_analys_tc(TsLegTab t, TsTcTab tc, const float2 *__restrict__ g, long g_stride, Epi epi,
                 int nfields, int per_cta) {
  extern __shared__ __align__(1024) char ts_smem_at[];
  char *smem = (char *)(((unsigned long long)ts_smem_at + 1023) & ~1023ull);
  const int m = blockIdx.y;
  const int ntile = gridDim.z / 2;
  const int par = blockIdx.z / ntile, ltile = blockIdx.z - par * ntile;
  const int cnt = ts_atile_count(t.lmax, m, par, ltile, tc.LTL);
  if (cnt == 0) return;  // uniform for the CTA, before any barrier or allocation
  const int N = ts_round16(cnt);
  const int f0 = blockIdx.x * per_cta;
  const int nf = min(per_cta, nfields - f0);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long base = ts_lm_base(t.lmax, m);
  const int bbytes = N * 128;
  const int stage = 2 * 16384 + 2 * bbytes;  // A hi, A lo, B hi, B lo
  const int stage_all = max(2 * stage, N * 2 * TS_TC_FIELDS * 4);
  unsigned long long *bars = reinterpret_cast<unsigned long long *>(smem + stage_all);
  unsigned *slot = reinterpret_cast<unsigned *>(smem + stage_all + 16);
  const unsigned ncols = ts_tmem_cols(N);
  const long toff = ts_atile_offset(tc, t.lmax, m, par, ltile);
  const int C = tc.nLC;

  if (tid == 0) {
    ts_mbar_init(&bars[0], 1);
    ts_mbar_init(&bars[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) ts_tmem_alloc(slot, ncols);
  ts_tc_fence_before();
  __syncthreads();
  ts_tc_fence_after();
  const unsigned tmem = *slot;
  const unsigned idesc = ts_idesc_tf32(N);
  bool ok = true;

  for (int c = 0; c < C && ok; c++) {
    const int b = c & 1;
    char *sb = smem + b * stage;
    if (c >= 2) ok = ts_mbar_wait(&bars[b], ((c >> 1) - 1) & 1, TS_TC_WAIT_LIMIT);
    if (!__syncthreads_and(ok)) {
      ok = false;
      break;
    }
    ts_copy16(sb + 2 * 16384, tc.anal + toff + (long)c * 2 * bbytes, 2 * bbytes);
    // W chunk: thread -> (latitude k of the chunk, 16 fields)
    {
      const int k = tid & 31, fg = tid >> 5;
      const int lat = c * TS_TC_KCH + k;
      const bool live = lat < t.nh;
      const float w = live ? t.wq[lat] : 0.f;
      const int south = t.nlat - 1 - lat;
      char *ahi = sb, *alo = sb + 16384;
#pragma unroll 4
      for (int i = 0; i < 16; i++) {
        const int fl = fg * 16 + i;
        float2 gn = make_float2(0.f, 0.f), gs = make_float2(0.f, 0.f);
        if (live && fl < nf) {
          const float2 *src = g + (long)(f0 + fl) * g_stride + (long)m * t.nlat;
          gn = src[lat];
          if (south != lat) gs = src[south];
        }
        const float wr = par ? (gn.x - gs.x) * w : (gn.x + gs.x) * w;
        const float wi = par ? (gn.y - gs.y) * w : (gn.y + gs.y) * w;
        const float hr = ts_rna_tf32(wr), hi = ts_rna_tf32(wi);
        *reinterpret_cast<float *>(ahi + ts_swz(2 * fl, k)) = hr;
        *reinterpret_cast<float *>(alo + ts_swz(2 * fl, k)) = ts_rna_tf32(wr - hr);
        *reinterpret_cast<float *>(ahi + ts_swz(2 * fl + 1, k)) = hi;
        *reinterpret_cast<float *>(alo + ts_swz(2 * fl + 1, k)) = ts_rna_tf32(wi - hi);
      }
    }
    ts_fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      ts_tc_fence_after();
      const unsigned ahi = ts_smem_u32(sb), alo = ahi + 16384;
      const unsigned bhi = ahi + 2 * 16384, blo = bhi + bbytes;
#pragma unroll
      for (int kk = 0; kk < 4; kk++) {
        const unsigned acc = (c > 0 || kk > 0) ? 1u : 0u;
        ts_mma_tf32(tmem, ts_umma_desc(ahi + kk * 32), ts_umma_desc(bhi + kk * 32), idesc, acc);
        ts_mma_tf32(tmem, ts_umma_desc(ahi + kk * 32), ts_umma_desc(blo + kk * 32), idesc, 1u);
        ts_mma_tf32(tmem, ts_umma_desc(alo + kk * 32), ts_umma_desc(bhi + kk * 32), idesc, 1u);
      }
      ts_mma_commit(&bars[b]);
    }
  }
  if (ok && C > 0) ok = ts_mbar_wait(&bars[(C - 1) & 1], ((C - 1) >> 1) & 1, TS_TC_WAIT_LIMIT);
  ok = __syncthreads_and(ok);
  ts_tc_fence_after();
  if (ok) {
    // TMEM -> shared [j][comp][field], then the epilogue per (lm, comp)
    float *sD = reinterpret_cast<float *>(smem);
    const int row = warp * 32 + lane, fl = row >> 1, comp = row & 1;
    for (int c0 = 0; c0 < N; c0 += 16) {
      float v[16];
      ts_tmem_ld16(tmem + ((unsigned)(warp * 32) << 16) + (unsigned)c0, v);
#pragma unroll
      for (int i = 0; i < 16; i++) sD[((c0 + i) * 2 + comp) * TS_TC_FIELDS + fl] = v[i];
    }
    ts_tc_fence_before();
    __syncthreads();
    for (int idx = tid; idx < cnt * 2; idx += blockDim.x) {
      const int j = idx >> 1, cp = idx & 1;
      const int l = m + par + 2 * (ltile * tc.LTL + j);
      epi(base + (l - m), cp, sD + (j * 2 + cp) * TS_TC_FIELDS, f0, nf, TS_TC_FIELDS);
    }
  } else if (tid == 0) {
    atomicExch(tc.err, 1);
  }
  ts_tc_fence_before();
  __syncthreads();
  if (warp == 0) ts_tmem_free(tmem, ncols);
}
