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
// Warp roles (192 threads): warps 0-3 build the data operand of each stage
// and run the epilogue (they own TMEM lanes 0-127), warp 4 streams the table
// chunks with cp.async.bulk (expect-tx mbarrier), warp 5 issues the MMAs and
// commits each stage back to its producers.  Every wait is bounded: on
// timeout the kernel records an error flag, skips the epilogue, frees its
// tensor memory and returns.
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

TS_DEV void ts_mbar_arrive(unsigned long long *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(ts_smem_u32(bar)) : "memory");
}

TS_DEV void ts_mbar_arrive_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(ts_smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// global -> shared bulk copy (no multicast), completion counted on `bar`
TS_DEV void ts_bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          ts_smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(ts_smem_u32(bar))
      : "memory");
}

#define TS_TC_THREADS 192
#define TS_TC_MAXSTAGE 4

// Pipeline bookkeeping shared by both kernels: full[s] completes when the
// table bytes of stage s have landed and the 4 producer warps have arrived;
// empty[s] completes when the MMAs that read stage s are done; done[0] when
// all MMAs are.
struct TsTcPipe {
  unsigned long long full[TS_TC_MAXSTAGE], empty[TS_TC_MAXSTAGE], done;
  unsigned tmem;
  int bad;
};

TS_DEV void ts_tc_pipe_init(TsTcPipe *pp, int S) {
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; s++) {
      ts_mbar_init(&pp->full[s], 5);
      ts_mbar_init(&pp->empty[s], 1);
    }
    ts_mbar_init(&pp->done, 1);
    pp->bad = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
}

TS_DEV void ts_tc_flag(TsTcPipe *pp) { atomicExch(&pp->bad, 1); }

// ----------------------------------------------------------------- synthesis
//
// grid = (ceil(nfields/64), mmax+1, nLT), block = 192.  Stages (2*16384 bytes
// of data operand + 2*NL*128 bytes of table each) cycle through the k chunks
// of both parities, interleaved.  Dynamic shared memory: S*stage + 1024 +
// sizeof(TsTcPipe).
__global__ void __launch_bounds__(TS_TC_THREADS, 1)
ts_leg_synth_tc(TsLegTab t, TsTcTab tc, TsFields q, float2 *__restrict__ fm, long fm_stride,
                int nfields, int S) {
  extern __shared__ __align__(1024) char ts_smem_st[];
  char *smem = (char *)(((unsigned long long)ts_smem_st + 1023) & ~1023ull);
  const int fb = blockIdx.x, m = blockIdx.y, lt = blockIdx.z;
  const int NL = tc.NL;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long base = ts_lm_base(t.lmax, m);
  const int kp0 = ts_kpar(t.lmax, m, 0), kp1 = ts_kpar(t.lmax, m, 1);
  const int nch0 = (kp0 + TS_TC_KCH - 1) / TS_TC_KCH, nch1 = (kp1 + TS_TC_KCH - 1) / TS_TC_KCH;
  const int T = nch0 + nch1;
  const int bbytes = NL * 128;
  const int stage = 2 * 16384 + 2 * bbytes;  // A hi, A lo, B hi, B lo
  TsTcPipe *pp = reinterpret_cast<TsTcPipe *>(smem + S * stage);
  const unsigned ncols = ts_tmem_cols(2 * NL);
  // chunk t -> (parity, chunk of that parity): parities interleaved
  auto chunk = [&](int t_, int &par, int &cc) {
    const int both = 2 * min(nch0, nch1);
    if (t_ < both) {
      par = t_ & 1;
      cc = t_ >> 1;
    } else {
      par = nch0 > nch1 ? 0 : 1;
      cc = (t_ - both) + min(nch0, nch1);
    }
  };

  ts_tc_pipe_init(pp, S);
  if (warp == 0) ts_tmem_alloc(&pp->tmem, ncols);
  ts_tc_fence_before();
  __syncthreads();
  ts_tc_fence_after();
  const unsigned tmem = pp->tmem;

  if (warp < 4) {
    // ---- data operand producers: Q split into TF32 hi/lo, 16 k per thread
    const int fl = tid & 63, kh = tid >> 6;
    const int f = fb * TS_TC_FIELDS + fl;
    const float2 *qf = f < nfields ? ts_field(q, f) + base : nullptr;
    for (int t_ = 0; t_ < T; t_++) {
      const int s = t_ % S, use = t_ / S;
      int par, cc;
      chunk(t_, par, cc);
      float2 v[16];
      const int kp = par ? kp1 : kp0;
#pragma unroll
      for (int u = 0; u < 16; u++) {
        const int j = cc * TS_TC_KCH + kh * 16 + u;
        v[u] = (qf && j < kp) ? qf[par + 2 * j] : make_float2(0.f, 0.f);
      }
      if (use > 0 && !ts_mbar_wait(&pp->empty[s], (use - 1) & 1, TS_TC_WAIT_LIMIT)) {
        ts_tc_flag(pp);
        break;
      }
      char *ahi = smem + s * stage, *alo = ahi + 16384;
#pragma unroll
      for (int k4 = 0; k4 < 4; k4++) {
        const int k = kh * 16 + k4 * 4;
        float4 h, l;
        h = make_float4(ts_rna_tf32(v[4 * k4].x), ts_rna_tf32(v[4 * k4 + 1].x),
                        ts_rna_tf32(v[4 * k4 + 2].x), ts_rna_tf32(v[4 * k4 + 3].x));
        l = make_float4(ts_rna_tf32(v[4 * k4].x - h.x), ts_rna_tf32(v[4 * k4 + 1].x - h.y),
                        ts_rna_tf32(v[4 * k4 + 2].x - h.z), ts_rna_tf32(v[4 * k4 + 3].x - h.w));
        *reinterpret_cast<float4 *>(ahi + ts_swz(2 * fl, k)) = h;
        *reinterpret_cast<float4 *>(alo + ts_swz(2 * fl, k)) = l;
        h = make_float4(ts_rna_tf32(v[4 * k4].y), ts_rna_tf32(v[4 * k4 + 1].y),
                        ts_rna_tf32(v[4 * k4 + 2].y), ts_rna_tf32(v[4 * k4 + 3].y));
        l = make_float4(ts_rna_tf32(v[4 * k4].y - h.x), ts_rna_tf32(v[4 * k4 + 1].y - h.y),
                        ts_rna_tf32(v[4 * k4 + 2].y - h.z), ts_rna_tf32(v[4 * k4 + 3].y - h.w));
        *reinterpret_cast<float4 *>(ahi + ts_swz(2 * fl + 1, k)) = h;
        *reinterpret_cast<float4 *>(alo + ts_swz(2 * fl + 1, k)) = l;
      }
      ts_fence_proxy_async();
      __syncwarp();
      if (lane == 0) ts_mbar_arrive(&pp->full[s]);
    }
  } else if (warp == 4) {
    // ---- table stream
    if (lane == 0) {
      for (int t_ = 0; t_ < T; t_++) {
        const int s = t_ % S, use = t_ / S;
        int par, cc;
        chunk(t_, par, cc);
        if (use > 0 && !ts_mbar_wait(&pp->empty[s], (use - 1) & 1, TS_TC_WAIT_LIMIT)) {
          ts_tc_flag(pp);
          break;
        }
        const long src = tc.synth_off[m] + (long)((par ? nch0 : 0) + cc) * tc.nLT * 2 * bbytes +
                         (long)lt * 2 * bbytes;
        ts_mbar_arrive_tx(&pp->full[s], 2 * bbytes);
        ts_bulk_g2s(smem + s * stage + 2 * 16384, tc.synth + src, 2 * bbytes, &pp->full[s]);
      }
    }
  } else {
    // ---- MMA issue
    if (lane == 0) {
      const unsigned idesc = ts_idesc_tf32(NL);
      for (int t_ = 0; t_ < T; t_++) {
        const int s = t_ % S, use = t_ / S;
        int par, cc;
        chunk(t_, par, cc);
        if (!ts_mbar_wait(&pp->full[s], use & 1, TS_TC_WAIT_LIMIT)) {
          ts_tc_flag(pp);
          break;
        }
        ts_tc_fence_after();
        const unsigned ahi = ts_smem_u32(smem + s * stage), alo = ahi + 16384;
        const unsigned bhi = ahi + 2 * 16384, blo = bhi + bbytes;
        const unsigned d = tmem + (unsigned)(par * NL);
#pragma unroll
        for (int kk = 0; kk < 4; kk++) {
          const unsigned acc = (cc > 0 || kk > 0) ? 1u : 0u;
          ts_mma_tf32(d, ts_umma_desc(ahi + kk * 32), ts_umma_desc(bhi + kk * 32), idesc, acc);
          ts_mma_tf32(d, ts_umma_desc(ahi + kk * 32), ts_umma_desc(blo + kk * 32), idesc, 1u);
          ts_mma_tf32(d, ts_umma_desc(alo + kk * 32), ts_umma_desc(bhi + kk * 32), idesc, 1u);
        }
        ts_mma_commit(&pp->empty[s]);
      }
      ts_mma_commit(&pp->done);
    }
  }

  // ---- epilogue (warps 0-3 own TMEM lanes 0-127): rows 2f (re) and 2f+1 (im)
  // sit in adjacent lanes; each pair swaps halves so that every thread writes
  // 8 consecutive complex values, north and (mirrored) south
  if (warp < 4) {
    bool ok = ts_mbar_wait(&pp->done, 0, TS_TC_WAIT_LIMIT) && !pp->bad;
    ts_tc_fence_after();
    const int fl = (warp * 32 + lane) >> 1, comp = lane & 1;
    const int f = fb * TS_TC_FIELDS + fl;
    float2 *dst = fm + (long)f * fm_stride + (long)m * t.nlat;
    if (ok) {
      for (int c0 = 0; c0 < NL; c0 += 16) {
        float e[16], o[16];
        ts_tmem_ld16(tmem + ((unsigned)(warp * 32) << 16) + (unsigned)c0, e);
        if (nch1 > 0)
          ts_tmem_ld16(tmem + ((unsigned)(warp * 32) << 16) + (unsigned)(NL + c0), o);
        else
#pragma unroll
          for (int i = 0; i < 16; i++) o[i] = 0.f;
        // re-lane keeps columns 0-7 and takes the partner's im; im-lane 8-15
        float2 en[8], on[8];
#pragma unroll
        for (int i = 0; i < 8; i++) {
          const float se = __shfl_xor_sync(0xffffffffu, comp ? e[i] : e[8 + i], 1);
          const float so = __shfl_xor_sync(0xffffffffu, comp ? o[i] : o[8 + i], 1);
          en[i] = comp ? make_float2(se, e[8 + i]) : make_float2(e[i], se);
          on[i] = comp ? make_float2(so, o[8 + i]) : make_float2(o[i], so);
        }
        if (f < nfields) {
#pragma unroll
          for (int i = 0; i < 8; i++) {
            const int lat = lt * NL + c0 + comp * 8 + i;
            if (lat < t.nh) {
              dst[lat] = make_float2(en[i].x + on[i].x, en[i].y + on[i].y);
              const int south = t.nlat - 1 - lat;
              if (south != lat) dst[south] = make_float2(en[i].x - on[i].x, en[i].y - on[i].y);
            }
          }
        }
      }
    }
    if (!ok && tid == 0) atomicExch(tc.err, 1);
  }
  ts_tc_fence_before();
  __syncthreads();
  if (warp == 0) ts_tmem_free(tmem, ncols);
}

// ------------------------------------------------------------------ analysis
//
// grid = (ceil(nfields/per_cta), mmax+1, 2*ntile), block = 192; z = par*ntile
// + ltile (empty tiles return at once).  per_cta <= 64 fields.  Stages: 2*16384
// bytes of data operand + 2*N*128 bytes of table, over the latitude chunks.
// Dynamic shared memory: max(S*stage, N*2*64*4) + 1024 + sizeof(TsTcPipe).
template <class Epi>
__global__ void __launch_bounds__(TS_TC_THREADS, 1)
ts_leg_analys_tc(TsLegTab t, TsTcTab tc, const float2 *__restrict__ g, long g_stride, Epi epi,
                 int nfields, int per_cta, int S) {
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
  const int stage = 2 * 16384 + 2 * bbytes;
  const int region = max(S * stage, N * 2 * TS_TC_FIELDS * 4);
  TsTcPipe *pp = reinterpret_cast<TsTcPipe *>(smem + region);
  const unsigned ncols = ts_tmem_cols(N);
  const long toff = ts_atile_offset(tc, t.lmax, m, par, ltile);
  const int T = tc.nLC;

  ts_tc_pipe_init(pp, S);
  if (warp == 0) ts_tmem_alloc(&pp->tmem, ncols);
  ts_tc_fence_before();
  __syncthreads();
  ts_tc_fence_after();
  const unsigned tmem = pp->tmem;

  if (warp < 4) {
    // ---- data operand: W = w (G_north +- G_south), lane = latitude of the chunk
    const int k = lane, fg = warp;
    for (int c = 0; c < T; c++) {
      const int s = c % S, use = c / S;
      const int lat = c * TS_TC_KCH + k;
      const bool live = lat < t.nh;
      const float w = live ? t.wq[lat] : 0.f;
      const int south = t.nlat - 1 - lat;
      float2 gn[16], gs[16];
#pragma unroll
      for (int i = 0; i < 16; i++) {
        const int fl = fg * 16 + i;
        gn[i] = gs[i] = make_float2(0.f, 0.f);
        if (live && fl < nf) {
          const float2 *src = g + (long)(f0 + fl) * g_stride + (long)m * t.nlat;
          gn[i] = src[lat];
          if (south != lat) gs[i] = src[south];
        }
      }
      if (use > 0 && !ts_mbar_wait(&pp->empty[s], (use - 1) & 1, TS_TC_WAIT_LIMIT)) {
        ts_tc_flag(pp);
        break;
      }
      char *ahi = smem + s * stage, *alo = ahi + 16384;
#pragma unroll
      for (int i = 0; i < 16; i++) {
        const int fl = fg * 16 + i;
        const float wr = par ? (gn[i].x - gs[i].x) * w : (gn[i].x + gs[i].x) * w;
        const float wi = par ? (gn[i].y - gs[i].y) * w : (gn[i].y + gs[i].y) * w;
        const float hr = ts_rna_tf32(wr), hi = ts_rna_tf32(wi);
        *reinterpret_cast<float *>(ahi + ts_swz(2 * fl, k)) = hr;
        *reinterpret_cast<float *>(alo + ts_swz(2 * fl, k)) = ts_rna_tf32(wr - hr);
        *reinterpret_cast<float *>(ahi + ts_swz(2 * fl + 1, k)) = hi;
        *reinterpret_cast<float *>(alo + ts_swz(2 * fl + 1, k)) = ts_rna_tf32(wi - hi);
      }
      ts_fence_proxy_async();
      __syncwarp();
      if (lane == 0) ts_mbar_arrive(&pp->full[s]);
    }
  } else if (warp == 4) {
    if (lane == 0) {
      for (int c = 0; c < T; c++) {
        const int s = c % S, use = c / S;
        if (use > 0 && !ts_mbar_wait(&pp->empty[s], (use - 1) & 1, TS_TC_WAIT_LIMIT)) {
          ts_tc_flag(pp);
          break;
        }
        ts_mbar_arrive_tx(&pp->full[s], 2 * bbytes);
        ts_bulk_g2s(smem + s * stage + 2 * 16384, tc.anal + toff + (long)c * 2 * bbytes,
                    2 * bbytes, &pp->full[s]);
      }
    }
  } else {
    if (lane == 0) {
      const unsigned idesc = ts_idesc_tf32(N);
      for (int c = 0; c < T; c++) {
        const int s = c % S, use = c / S;
        if (!ts_mbar_wait(&pp->full[s], use & 1, TS_TC_WAIT_LIMIT)) {
          ts_tc_flag(pp);
          break;
        }
        ts_tc_fence_after();
        const unsigned ahi = ts_smem_u32(smem + s * stage), alo = ahi + 16384;
        const unsigned bhi = ahi + 2 * 16384, blo = bhi + bbytes;
#pragma unroll
        for (int kk = 0; kk < 4; kk++) {
          const unsigned acc = (c > 0 || kk > 0) ? 1u : 0u;
          ts_mma_tf32(tmem, ts_umma_desc(ahi + kk * 32), ts_umma_desc(bhi + kk * 32), idesc, acc);
          ts_mma_tf32(tmem, ts_umma_desc(ahi + kk * 32), ts_umma_desc(blo + kk * 32), idesc, 1u);
          ts_mma_tf32(tmem, ts_umma_desc(alo + kk * 32), ts_umma_desc(bhi + kk * 32), idesc, 1u);
        }
        ts_mma_commit(&pp->empty[s]);
      }
      ts_mma_commit(&pp->done);
    }
  }

  // ---- epilogue: TMEM -> shared [j][comp][field] -> Epi per (lm, comp)
  bool ok = true;
  if (warp < 4) {
    ok = ts_mbar_wait(&pp->done, 0, TS_TC_WAIT_LIMIT) && !pp->bad;
    ts_tc_fence_after();
    if (ok) {
      float *sD = reinterpret_cast<float *>(smem);
      const int row = warp * 32 + lane, fl = row >> 1, comp = row & 1;
      for (int c0 = 0; c0 < N; c0 += 16) {
        float v[16];
        ts_tmem_ld16(tmem + ((unsigned)(warp * 32) << 16) + (unsigned)c0, v);
#pragma unroll
        for (int i = 0; i < 16; i++) sD[((c0 + i) * 2 + comp) * TS_TC_FIELDS + fl] = v[i];
      }
    }
  }
  ts_tc_fence_before();
  ok = __syncthreads_and(ok || warp >= 4) && !pp->bad;
  if (ok) {
    const float *sD = reinterpret_cast<const float *>(smem);
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
