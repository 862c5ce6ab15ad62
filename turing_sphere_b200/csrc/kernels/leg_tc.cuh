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
// 128-byte swizzle), so a CTA streams them with plain bulk copies.  The
// data operand (Q or W) is split on the fly: hi = rna_tf32(x),
// lo = rna_tf32(x - hi); each k-step issues hi*hi + hi*lo + lo*hi.
//
// Both operands reach shared memory by cp.async.bulk: the P table from its
// precomputed image and the data operand from a raw-fp32 image of the same
// byte layout (TsTcImg; written by a relayout kernel for the synthesis and by
// the Fourier analysis itself for the analysis).  The split data operand then
// lives in tensor memory: the MMAs read A (hi, lo) from TMEM and only B (the
// table) from shared memory.  A stage then moves about 40% fewer
// shared-memory bytes (no A reads by the MMAs, no hi/lo stores by the split),
// and a ring slot needs 16 KB less, which buys a fourth slot and
// double-buffered epilogue staging.  The kernels are persistent
// (one CTA per SM walking tiles blockIdx.x + k*gridDim.x) with 448 threads in
// fixed roles: warps 0-3 split each data tile row by row (thread = row = TMEM
// lane) into rna-rounded TF32 hi and lo in an NA-slot TMEM operand ring, warp 4
// issues the copies (expect-tx mbarriers over an S-slot shared-memory ring),
// warp 5 issues the MMAs, warps 6-13 drain the accumulators.  Tensor memory
// holds two accumulator buffers, so the epilogue of tile i overlaps the MMAs
// of tile i+1, and both operand rings stream across tile boundaries.
// Every wait is bounded: on timeout the kernel records an error flag, waits
// (bounded) for its copies and MMAs in flight, frees its tensor memory and
// returns.
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
  {
    // a phase that has already completed (the usual case on the MMA thread's
    // path) is seen by the non-blocking test without the try_wait's latency
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
  }
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

// the same with A (128 lanes x 8 columns of tf32) read from tensor memory
TS_DEV void ts_mma_tf32_ta(unsigned dtmem, unsigned atmem, unsigned long long bdesc,
                           unsigned idesc, unsigned accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      ::"r"(dtmem), "r"(atmem), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0),
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

// 16 consecutive columns of this thread's TMEM lane (warp-collective; taddr
// is the warp's lane base plus the first column)
TS_DEV void ts_tmem_st16(unsigned taddr, const float (&v)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16};" ::"r"(taddr),
      "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
      "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
      "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])), "r"(__float_as_uint(v[8])),
      "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
      "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])),
      "r"(__float_as_uint(v[15]))
      : "memory");
}
TS_DEV void ts_tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

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

// An encoded tensor map (the driver's 128-byte CUtensorMap), passed by value
// as a __grid_constant__ kernel parameter.
struct __align__(64) TsTmaDesc {
  unsigned long long v[16];
};

// 3-D tile store of the shared-memory box at src to element coordinates
// (x, y, z); completion tracked by the issuing thread's bulk group
TS_DEV void ts_tma_store3(const TsTmaDesc *map, const void *src, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(
          reinterpret_cast<unsigned long long>(map)),
      "r"(x), "r"(y), "r"(z), "r"(ts_smem_u32(src))
      : "memory");
}
TS_DEV void ts_bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
TS_DEV void ts_bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// all but the most recent bulk group have finished reading shared memory
TS_DEV void ts_bulk_wait_read1() { asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); }
TS_DEV void ts_bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

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

#define TS_TC_THREADS 448  // 14 warps: split 0-3, copy 4, MMA 5, epilogue 6-13
#define TS_TC_MAXSTAGE 4
#define TS_TC_ASLOTS 4      // TMEM operand slots at most (64 columns each: hi | lo)
#define TS_TC_STAGE_A 16384 // shared-memory bytes of a stage's raw data tile

// Persistent pipeline state.  Shared-memory ring: full[s] the copies of slot
// s landed; empty[s] the MMAs that read its table are done.  TMEM operand
// ring: a_full[a] the 4 split warps stored a data tile's hi/lo in slot a;
// a_empty[a] the MMAs that read it are done.  Accumulators (two TMEM
// buffers): acc_full[b] the MMAs of a tile into buffer b are done;
// acc_empty[b] the epilogue warps have read it out.
struct TsTcPipe {
  unsigned long long full[TS_TC_MAXSTAGE], empty[TS_TC_MAXSTAGE];
  unsigned long long a_full[TS_TC_ASLOTS], a_empty[TS_TC_ASLOTS];
  unsigned long long acc_full[2], acc_empty[2];
  unsigned long long epi;    // the 4 epilogue warps' own barrier
  unsigned long long drain;  // the MMA warp's last commit before exit
  unsigned tmem;
  unsigned limit;            // polls of a bounded wait
  int bad;
  int epi_go[2];  // per accumulator buffer: the epilogue warps proceed (1) or leave (0)
};

// shared-memory staging of the epilogues: the synthesis keeps 64 field rows
// of [north|south][16 latitudes][re, im] (68 floats per row keeps rows
// 16-byte aligned); the analysis keeps [l][re|im] rows of 64 fields padded to
// 65 floats, so that lanes reading different rows hit different banks
#define TS_TC_SYN_ROW 64
#define TS_TC_SYN_STAGING (TS_TC_FIELDS * TS_TC_SYN_ROW * 4)  // one staging buffer: 16 KB
#define TS_TC_SYN_NSTG 2  // staging buffers per epilogue group, used in turn
// float index of value c (0..63) of field row fl in the synthesis staging of
// the plain-store path: 16-byte chunks XOR (fl mod 8), so the 16 rows a warp
// writes at once spread over 8 bank groups (a 64-float row pitch alone would
// put them all in one)
TS_DEV int ts_syn_stg(int fl, int c) {
  return fl * TS_TC_SYN_ROW + ((((c >> 2) ^ (fl & 7)) << 2) | (c & 3));
}
#define TS_TC_ANA_ROW (TS_TC_FIELDS + 1)
#define TS_TC_ANA_COLS 32  // accumulator columns an analysis group stages at a time

// The epilogue runs in two groups of 4 warps (warps 6-9 and 10-13; each
// group covers all 128 TMEM lanes) that take alternate column chunks of a
// tile.  ts_epi_bar(g) is group g's barrier (named barrier 1 + g),
// ts_epi_bar_all() the barrier of all 8 epilogue warps (named barrier 3).
// Every epilogue warp runs the same sequence of these (exits are decided
// uniformly, through TsTcPipe::epi_go), so none is left waiting.
TS_DEV int ts_epi_group(int warp) { return (warp - 6) >> 2; }
TS_DEV void ts_epi_bar(int g) {
  __syncwarp();
  if (g == 0)
    asm volatile("bar.sync 1, 128;" ::: "memory");
  else
    asm volatile("bar.sync 2, 128;" ::: "memory");
}
TS_DEV void ts_epi_bar_all() {
  __syncwarp();
  asm volatile("bar.sync 3, 256;" ::: "memory");
}

TS_DEV void ts_tc_pipe_init(TsTcPipe *pp, int S, const TsTcTab &tc) {
  if (threadIdx.x == 0) {
    pp->limit = tc.wait_limit ? tc.wait_limit : TS_TC_WAIT_LIMIT;
    for (int s = 0; s < S; s++) {
      ts_mbar_init(&pp->full[s], 1);
      ts_mbar_init(&pp->empty[s], 1);
    }
    for (int a = 0; a < TS_TC_ASLOTS; a++) {
      ts_mbar_init(&pp->a_full[a], 4);
      ts_mbar_init(&pp->a_empty[a], 1);
    }
    for (int b = 0; b < 2; b++) {
      ts_mbar_init(&pp->acc_full[b], 1);
      ts_mbar_init(&pp->acc_empty[b], 8);
    }
    ts_mbar_init(&pp->epi, 4);
    ts_mbar_init(&pp->drain, 1);
    pp->bad = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
}

TS_DEV bool ts_tc_bad(const TsTcPipe *pp) { return *reinterpret_cast<const volatile int *>(&pp->bad); }

TS_DEV void ts_tc_flag(TsTcPipe *pp) { atomicExch(&pp->bad, 1); }

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

// warps 0-3: row r (= tid, the TMEM lane of warp r/32) of the raw fp32 data
// tile at `tile` (K-major, 128-byte swizzle, 32 values) split into
// hi = rna_tf32(x) and lo = rna_tf32(x - hi), stored in TMEM columns
// [col, col + 32) and [col + 32, col + 64) of the lane; `taddr` is the warp's
// lane base plus col.  A warp reads each 16-byte chunk index of 32 rows: the
// swizzle spreads every 8 rows over 8 distinct bank groups.
TS_DEV void ts_tc_split_tmem(const char *tile, unsigned taddr, int r) {
  const char *row = tile + (r >> 3) * 1024 + (r & 7) * 128;
#pragma unroll
  for (int h = 0; h < 2; h++) {
    float hi[16], lo[16];
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const float4 x = *reinterpret_cast<const float4 *>(row + (((4 * h + c) ^ (r & 7)) << 4));
      hi[4 * c + 0] = ts_rna_tf32(x.x);
      hi[4 * c + 1] = ts_rna_tf32(x.y);
      hi[4 * c + 2] = ts_rna_tf32(x.z);
      hi[4 * c + 3] = ts_rna_tf32(x.w);
      lo[4 * c + 0] = ts_rna_tf32(x.x - hi[4 * c + 0]);
      lo[4 * c + 1] = ts_rna_tf32(x.y - hi[4 * c + 1]);
      lo[4 * c + 2] = ts_rna_tf32(x.z - hi[4 * c + 2]);
      lo[4 * c + 3] = ts_rna_tf32(x.w - hi[4 * c + 3]);
    }
    ts_tmem_st16(taddr + 16 * h, hi);
    ts_tmem_st16(taddr + 32 + 16 * h, lo);
  }
}

// A position in a ring of n slots walked in order: the slot of the current
// stage and the parity of that slot's current use (the uses of a slot
// alternate parity, and every slot flips once per round).  Counters instead
// of stage / n and stage % n keep integer division out of the roles' loops.
struct TsRing {
  int slot, n;
  unsigned phase;  // parity of the current use
  bool wrapped;    // past the first round: every slot has been used before
  TS_DEV explicit TsRing(int n_) : slot(0), n(n_), phase(0), wrapped(false) {}
  TS_DEV void next() {
    if (++slot == n) {
      slot = 0;
      phase ^= 1u;
      wrapped = true;
    }
  }
};

// MMA issue (one thread): per tile, wait until the epilogue has drained the
// accumulator buffer, then per stage wait for the split data tile in TMEM
// slot a (the split warps waited for the stage's copies, table included),
// issue the 3-pass products of its 4 k-steps and commit the shared-memory slot
// back to the copy warp and the TMEM slot back to the split warps; the tile's
// last commit signals the epilogue.  TMEM columns: accumulator buffer b at
// b * acc_cols, operand slot a at a_col0 + 64 a (hi, then lo).
template <class Sched>
TS_DEV void ts_tc_mma_role(char *smem, TsTcPipe *pp, int S, int NA, unsigned stage_bytes,
                           unsigned tmem, int acc_cols, unsigned a_col0, const Sched &sc) {
  const int ntiles = sc.ntiles();
  const unsigned smem0 = ts_smem_u32(smem) + TS_TC_STAGE_A;
  TsRing rs(S), ra(NA);
  int i = 0;
  for (int tile = blockIdx.x; tile < ntiles && !ts_tc_bad(pp); tile += gridDim.x, i++) {
    const int b = i & 1;
    if (i >= 2 && !ts_mbar_wait(&pp->acc_empty[b], ((i >> 1) - 1) & 1, pp->limit)) {
      ts_tc_flag(pp);
      return;
    }
    ts_tc_fence_after();
    const auto ti = sc.tile(tile);
    const int T = sc.stages(ti);
    const unsigned tb = sc.table_bytes(ti);
    const unsigned idesc = ts_idesc_tf32(sc.n(ti));
    const unsigned dbase = tmem + (unsigned)(b * acc_cols);
    for (int t_ = 0; t_ < T; t_++, rs.next(), ra.next()) {
      if (!ts_mbar_wait(&pp->a_full[ra.slot], ra.phase, pp->limit)) {
        ts_tc_flag(pp);
        return;
      }
      ts_tc_fence_after();
      // k-step kk reads the 32 bytes at kk * 32 of each 128-byte row: the
      // descriptor's start-address field (address >> 4) advances by 2
      const unsigned bhi = smem0 + (unsigned)rs.slot * stage_bytes;
      const unsigned long long dhi = ts_umma_desc(bhi), dlo = ts_umma_desc(bhi + tb / 2);
      const unsigned ahi = tmem + a_col0 + 64u * (unsigned)ra.slot, alo = ahi + 32;
      int dcol;
      bool init;
      sc.stage_acc(ti, t_, dcol, init);
      const unsigned d = dbase + (unsigned)dcol;
#pragma unroll
      for (int kk = 0; kk < 4; kk++) {
        const unsigned acc = (!init || kk > 0) ? 1u : 0u;
        ts_mma_tf32_ta(d, ahi + kk * 8, dhi + 2 * kk, idesc, acc);
        ts_mma_tf32_ta(d, ahi + kk * 8, dlo + 2 * kk, idesc, 1u);
        ts_mma_tf32_ta(d, alo + kk * 8, dhi + 2 * kk, idesc, 1u);
      }
      ts_mma_commit(&pp->empty[rs.slot]);
      ts_mma_commit(&pp->a_empty[ra.slot]);
    }
    ts_mma_commit(&pp->acc_full[b]);
  }
}

// Persistent schedule.  The CTA takes tiles blockIdx.x, blockIdx.x +
// gridDim.x, ...; `Sched` maps a tile to a descriptor (sc.tile: stage count,
// bases, skip offsets, computed once per tile) and, per stage, the data
// tile, the table chunk and the accumulator column; every role walks the
// same sequence, so ring slots and barrier phases stay in step.  Warps 0-3
// split data tiles into the TMEM operand ring (NA slots of 64 columns from
// a_col0), warp 4 copies, warp 5 issues MMAs, warps 6-13 drain the
// accumulators through `epilogue(tile, tmem_cols_of_buffer)`.  A
// shared-memory slot holds the raw data tile (TS_TC_STAGE_A bytes) and then
// the table's hi and lo images.
template <class Sched, class Epilogue>
TS_DEV void ts_tc_persistent(char *smem, TsTcPipe *pp, int S, int NA, unsigned stage_bytes,
                             unsigned tmem, int acc_cols, unsigned a_col0, const Sched &sc,
                             Epilogue epilogue) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ntiles = sc.ntiles();
  if (warp < 4) {
    TsRing rs(S), ra(NA);
    const unsigned lanebase = tmem + ((unsigned)(warp * 32) << 16) + a_col0;
    for (int tile = blockIdx.x; tile < ntiles && !ts_tc_bad(pp); tile += gridDim.x) {
      const int T = sc.stages(tile);
      for (int t_ = 0; t_ < T; t_++, rs.next(), ra.next()) {
        if (!ts_mbar_wait(&pp->full[rs.slot], rs.phase, pp->limit) ||
            (ra.wrapped && !ts_mbar_wait(&pp->a_empty[ra.slot], ra.phase ^ 1u, pp->limit))) {
          ts_tc_flag(pp);
          return;
        }
        ts_tc_fence_after();  // the stores follow the MMAs that read the slot before
        ts_tc_split_tmem(smem + rs.slot * stage_bytes, lanebase + 64u * (unsigned)ra.slot, tid);
        ts_tmem_wait_st();
        ts_tc_fence_before();
        __syncwarp();
        if (lane == 0) ts_mbar_arrive(&pp->a_full[ra.slot]);
      }
    }
  } else if (warp == 4) {
    if (lane == 0 && !sc.tc->stall_copies) {
      TsRing rs(S);
      int g = 0;  // stages issued
      for (int tile = blockIdx.x; tile < ntiles && !ts_tc_bad(pp); tile += gridDim.x) {
        const auto ti = sc.tile(tile);
        const int T = sc.stages(ti);
        const unsigned tb = sc.table_bytes(ti);
        int t_ = 0;
        for (; t_ < T; t_++, g++, rs.next()) {
          if (rs.wrapped && !ts_mbar_wait(&pp->empty[rs.slot], rs.phase ^ 1u, pp->limit)) {
            ts_tc_flag(pp);
            break;
          }
          char *st = smem + rs.slot * stage_bytes;
          ts_mbar_arrive_tx(&pp->full[rs.slot], TS_TC_STAGE_A + tb);
          ts_bulk_g2s(st, sc.a_src(ti, t_), TS_TC_STAGE_A, &pp->full[rs.slot]);
          ts_bulk_g2s(st + TS_TC_STAGE_A, sc.b_src(ti, t_), tb, &pp->full[rs.slot]);
        }
        if (t_ < T) break;
      }
      // no copy may still be landing in shared memory when the CTA exits:
      // wait (bounded) for the last use of every slot that was issued
      for (int s = 0; s < S && s < g; s++) {
        const unsigned last = (unsigned)((g - 1 - s) / S);
        if (!ts_mbar_wait(&pp->full[s], last & 1, pp->limit)) ts_tc_flag(pp);
      }
    }
  } else if (warp == 5) {
    if (lane == 0) {
      ts_tc_mma_role(smem, pp, S, NA, stage_bytes, tmem, acc_cols, a_col0, sc);
      // every MMA this thread issued has finished before TMEM is released
      ts_mma_commit(&pp->drain);
      if (!ts_mbar_wait(&pp->drain, 0, pp->limit)) ts_tc_flag(pp);
    }
  } else {
    // one thread waits for the accumulator and tells the other epilogue warps
    // whether to go on, so that they all take the same barriers
    int i = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, i++) {
      const int b = i & 1;
      if (warp == 6 && lane == 0) {
        const bool ok = ts_mbar_wait(&pp->acc_full[b], (i >> 1) & 1, pp->limit);
        if (!ok) ts_tc_flag(pp);
        pp->epi_go[b] = ok && !ts_tc_bad(pp);
      }
      ts_epi_bar_all();
      if (!*reinterpret_cast<volatile int *>(&pp->epi_go[b])) return;
      ts_tc_fence_after();
      epilogue(tile, tmem + (unsigned)(b * acc_cols));
      ts_tc_fence_before();
      __syncwarp();
      if (lane == 0) ts_mbar_arrive(&pp->acc_empty[b]);
    }
  }
}

// rows 32*(warp%4) .. of TMEM belong to epilogue warp `warp` (warps 6-13)
TS_DEV int ts_epi_row(int warp, int lane) { return (warp & 3) * 32 + lane; }

// ----------------------------------------------------------------- synthesis
struct TsSynthSched {
  const TsTcTab *tc;
  int lmax, mmax, nfb, NL, nLT;
  const char *qimg;
  // what the roles need of one tile, computed once per tile
  struct Tile {
    int n0, n1;   // degree chunks of parity 0 / 1
    int cs;       // leading chunk pairs left out by the polar skip
    int T;        // stages that run
    const char *q;  // Q image block of (chunk 0 of m, field block)
    const char *b;  // table block of (chunk 0 of m, latitude tile)
  };
  TS_DEV int ntiles() const { return (mmax + 1) * nLT * nfb; }
  TS_DEV void decode(int tile, int &m, int &lt, int &fb) const {
    m = tile / (nLT * nfb);
    const int r = tile - m * nLT * nfb;
    lt = r / nfb;
    fb = r - lt * nfb;
  }
  TS_DEV void nch(int m, int &n0, int &n1) const {
    n0 = (ts_kpar(lmax, m, 0) + TS_TC_KCH - 1) / TS_TC_KCH;
    n1 = (ts_kpar(lmax, m, 1) + TS_TC_KCH - 1) / TS_TC_KCH;
  }
  TS_DEV Tile tile(int tile) const {
    Tile ti;
    int m, lt, fb;
    decode(tile, m, lt, fb);
    nch(m, ti.n0, ti.n1);
    const int i = m * nLT + lt;
    ti.cs = tc->syn_cs ? tc->syn_cs[i] : 0;
    ti.T = (tc->syn_zero && tc->syn_zero[i]) ? 0 : ti.n0 + ti.n1 - 2 * ti.cs;
    ti.q = qimg + ((long)tc->chunk_prefix[m] * nfb + fb) * 16384;
    ti.b = tc->synth + tc->synth_off[m] + (long)lt * 2 * NL * 128;
    return ti;
  }
  // parity and chunk-of-parity of stage t_ (after the skipped pairs)
  TS_DEV void parcc(const Tile &ti, int t_, int &par, int &cc) const {
    const int t = t_ + 2 * ti.cs;
    const int mn = min(ti.n0, ti.n1), both = 2 * mn;
    if (t < both) {
      par = t & 1;
      cc = t >> 1;
    } else {
      par = ti.n0 > ti.n1 ? 0 : 1;
      cc = (t - both) + mn;
    }
  }
  TS_DEV int stages(const Tile &ti) const { return ti.T; }
  TS_DEV int stages(int t) const { return tile(t).T; }
  TS_DEV unsigned table_bytes(const Tile &) const { return 2u * NL * 128; }
  TS_DEV int n(const Tile &) const { return NL; }
  TS_DEV const char *a_src(const Tile &ti, int t_) const {
    int par, cc;
    parcc(ti, t_, par, cc);
    return ti.q + (long)((par ? ti.n0 : 0) + cc) * nfb * 16384;
  }
  TS_DEV const char *b_src(const Tile &ti, int t_) const {
    int par, cc;
    parcc(ti, t_, par, cc);
    return ti.b + (long)((par ? ti.n0 : 0) + cc) * nLT * 2 * NL * 128;
  }
  // accumulator column of stage t_ (its parity's half) and whether it starts
  // the accumulation
  TS_DEV void stage_acc(const Tile &ti, int t_, int &dcol, bool &first) const {
    int par, cc;
    parcc(ti, t_, par, cc);
    dcol = par * NL;
    first = cc == ti.cs;
  }
};

// grid = min(#SMs, tiles), block = 448, persistent.  Dynamic shared memory:
// S*(16384 + 2*NL*128) + 2*TS_TC_SYN_NSTG*TS_TC_SYN_STAGING + 1024 + sizeof(TsTcPipe).
// TMEM: two accumulator buffers of 2*NL columns, then (512 - 4*NL)/64 operand
// slots (NL <= 96: at least two).  With tma_ok, fmap maps fm as floats
// [field][m][2 nlat] with a (32, 1, 64) box in the 128-byte swizzle, and
// whole 16-latitude chunks leave through tensor stores (one thread per
// epilogue group issues them); other chunks, or tma_ok = 0, use plain stores.
__global__ void __launch_bounds__(TS_TC_THREADS, 1)
ts_leg_synth_tc(TsLegTab t, TsTcTab tc, const char *__restrict__ qimg, int q_nfb,
                float2 *__restrict__ fm, long fm_stride, int nfields, int S,
                const __grid_constant__ TsTmaDesc fmap, int tma_ok) {
  extern __shared__ __align__(1024) char ts_smem_st[];
  char *smem = (char *)(((unsigned long long)ts_smem_st + 1023) & ~1023ull);
  const int NL = tc.NL;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const unsigned stage = TS_TC_STAGE_A + 2 * NL * 128;
  const int NA = min(TS_TC_ASLOTS, (512 - 4 * NL) / 64);
  TsTcPipe *pp = reinterpret_cast<TsTcPipe *>(smem + S * stage +
                                               2 * TS_TC_SYN_NSTG * TS_TC_SYN_STAGING);
  const TsSynthSched sc{&tc, t.lmax, t.mmax, q_nfb, NL, tc.nLT, qimg};
  ts_tc_pipe_init(pp, S, tc);
  if (warp == 0) ts_tmem_alloc(&pp->tmem, 512);
  ts_tc_fence_before();
  __syncthreads();
  ts_tc_fence_after();
  const unsigned tmem = pp->tmem;

  // epilogue, per 16 latitudes: each thread (row 2f+re|im) puts north = E+O
  // and south = E-O of its component into the group's staging rows; whole
  // chunks then leave as two tensor stores (north box, mirrored south box),
  // a partial chunk as 16-byte runs of whole complex values written by the
  // 128 threads, north in latitude order and south mirrored
  const int grp = ts_epi_group(warp);
  // the group's staging buffers, used in turn: a chunk is staged while the
  // previous chunk's tensor stores still read the other buffer
  char *sE0 = smem + S * stage + (grp > 0 ? TS_TC_SYN_NSTG * TS_TC_SYN_STAGING : 0);
  int nstaged = 0;
  const bool elected = warp >= 6 && ((warp - 6) & 3) == 0 && lane == 0;  // one per epilogue group
  const bool vec = (t.nlat % 2 == 0) && (fm_stride % 2 == 0) &&
                   ((reinterpret_cast<unsigned long long>(fm) & 15) == 0);
  auto epilogue = [&](int tile, unsigned tbase) {
    int m, lt, fb, n0, n1;
    sc.decode(tile, m, lt, fb);
    sc.nch(m, n0, n1);
    const int et = ts_epi_row(warp, lane);  // 0..127 = TMEM lane = 2*field + comp
    const unsigned lanebase = tbase + ((unsigned)((warp & 3) * 32) << 16);
    const bool zero = sc.stages(tile) == 0;  // a polar tile: no MMAs ran
    for (int c0 = 16 * grp; c0 < NL; c0 += 32) {
      float e[16], o[16];
      if (zero) {
#pragma unroll
        for (int i = 0; i < 16; i++) e[i] = o[i] = 0.f;
      } else {
        ts_tmem_ld16(lanebase + (unsigned)c0, e);
        if (n1 > 0)
          ts_tmem_ld16(lanebase + (unsigned)(NL + c0), o);
        else
#pragma unroll
          for (int i = 0; i < 16; i++) o[i] = 0.f;
      }
      // the tensor stores that read this staging buffer (two chunks ago) are done
      float *sE = reinterpret_cast<float *>(sE0 + (nstaged & 1) * TS_TC_SYN_STAGING);
      nstaged++;
      if (elected) ts_bulk_wait_read1();
      ts_epi_bar(grp);
      const int lat0 = lt * NL + c0;
      if (tma_ok && lat0 + 16 <= t.nh) {
        // north box [64 fields][16 latitudes x re,im] and south box (its
        // latitudes mirrored, so in decreasing order of the north ones), both
        // in the 128-byte swizzle the tensor map writes from
        char *stN = reinterpret_cast<char *>(sE), *stS = stN + 8192;
        const int fl = et >> 1, comp = et & 1;
#pragma unroll
        for (int i = 0; i < 16; i++) {
          *reinterpret_cast<float *>(stN + ts_swz(fl, 2 * i + comp)) = e[i] + o[i];
          *reinterpret_cast<float *>(stS + ts_swz(fl, 2 * (15 - i) + comp)) = e[i] - o[i];
        }
        ts_fence_proxy_async();
        ts_epi_bar(grp);
        if (elected) {
          ts_tma_store3(&fmap, stN, 2 * lat0, m, fb * TS_TC_FIELDS);
          ts_tma_store3(&fmap, stS, 2 * (t.nlat - lat0 - 16), m, fb * TS_TC_FIELDS);
          ts_bulk_commit();
        }
        continue;
      }
#pragma unroll
      for (int i = 0; i < 16; i++) {
        sE[ts_syn_stg(et >> 1, 2 * i + (et & 1))] = e[i] + o[i];
        sE[ts_syn_stg(et >> 1, 32 + 2 * i + (et & 1))] = e[i] - o[i];
      }
      ts_epi_bar(grp);
#pragma unroll 2
      for (int k = 0; k < 8; k++) {
        const int q = et + 128 * k, seg = q >> 3, part = q & 7;
        const int fl = seg >> 1, ns = seg & 1;
        const float4 v = *reinterpret_cast<const float4 *>(sE + ts_syn_stg(fl, ns * 32 + part * 4));
        const int f = fb * TS_TC_FIELDS + fl;
        const int lat = lt * NL + c0 + 2 * part;
        if (f >= nfields || lat >= t.nh) continue;
        float2 *row = fm + (long)f * fm_stride + (long)m * t.nlat;
        const bool two = lat + 1 < t.nh;
        if (ns == 0) {
          if (vec && two) {
            *reinterpret_cast<float4 *>(row + lat) = v;
          } else {
            row[lat] = make_float2(v.x, v.y);
            if (two) row[lat + 1] = make_float2(v.z, v.w);
          }
        } else {
          const int s0 = t.nlat - 1 - lat, s1 = s0 - 1;  // south of lat, lat + 1
          if (vec && two) {
            *reinterpret_cast<float4 *>(row + s1) = make_float4(v.z, v.w, v.x, v.y);
          } else {
            if (s0 != lat) row[s0] = make_float2(v.x, v.y);
            if (two && s1 != lat + 1) row[s1] = make_float2(v.z, v.w);
          }
        }
      }
      ts_epi_bar(grp);
    }
  };
  ts_tc_persistent(smem, pp, S, NA, stage, tmem, 2 * NL, 4u * NL, sc, epilogue);
  if (elected) ts_bulk_wait_all();
  ts_tc_fence_before();
  __syncthreads();
  if (pp->bad && tid == 0) atomicExch(tc.err, 1);
  if (warp == 0) ts_tmem_free(tmem, 512);
}

// ------------------------------------------------------------------ analysis
struct TsAnalysSched {
  const TsTcTab *tc;
  int lmax, mmax, nfb, ntile;
  const char *wimg;
  struct Tile {
    int cnt;        // degrees of the tile
    int T;          // stages that run (latitude chunks after the polar skip)
    unsigned tb;    // table bytes per stage
    int n;          // MMA N
    const char *w;  // W image block of the first chunk that runs
    const char *b;  // table block of the first chunk that runs
  };
  TS_DEV int ntiles() const { return (mmax + 1) * 2 * ntile * nfb; }
  TS_DEV void decode(int tile, int &m, int &par, int &lt, int &fb) const {
    m = tile / (2 * ntile * nfb);
    int r = tile - m * 2 * ntile * nfb;
    fb = r % nfb;
    r /= nfb;
    par = r / ntile;
    lt = r - par * ntile;
  }
  TS_DEV int cnt(int tile) const {
    int m, par, lt, fb;
    decode(tile, m, par, lt, fb);
    return ts_atile_count(lmax, m, par, lt, tc->LTL);
  }
  TS_DEV Tile tile(int tile) const {
    Tile ti;
    int m, par, lt, fb;
    decode(tile, m, par, lt, fb);
    ti.cnt = ts_atile_count(lmax, m, par, lt, tc->LTL);
    // leading latitude chunks skipped (their table values are all negligible)
    const int c0 = tc->ana_c0 ? tc->ana_c0[(2 * m + par) * tc->ntile + lt] : 0;
    ti.T = ti.cnt > 0 ? tc->nLC - c0 : 0;
    ti.n = max(16, ts_round16(ti.cnt));
    ti.tb = 2u * ti.n * 128;
    ti.w = wimg + ((((long)m * nfb + fb) * 2 + par) * tc->nLC + c0) * 16384;
    ti.b = ti.T > 0 ? tc->anal + ts_atile_offset(*tc, lmax, m, par, lt) + (long)c0 * ti.tb
                    : tc->anal;
    return ti;
  }
  TS_DEV int stages(const Tile &ti) const { return ti.T; }
  TS_DEV int stages(int t) const { return tile(t).T; }
  TS_DEV int n(const Tile &ti) const { return ti.n; }
  TS_DEV unsigned table_bytes(const Tile &ti) const { return ti.tb; }
  TS_DEV const char *a_src(const Tile &ti, int c) const { return ti.w + (long)c * 16384; }
  TS_DEV const char *b_src(const Tile &ti, int c) const { return ti.b + (long)c * ti.tb; }
  TS_DEV void stage_acc(const Tile &, int c, int &dcol, bool &first) const {
    dcol = 0;
    first = c == 0;
  }
};

// grid = min(#SMs, tiles), block = 448, persistent.  Tiles with no l values
// have no stages; their epilogue does nothing; tiles whose latitude chunks
// the polar skip drops entirely write zeros.  Dynamic shared memory:
// S*(16384 + 2*Nmax*128) + 2*min(Nmax, TS_TC_ANA_COLS)*2*TS_TC_ANA_ROW*4 + 1024
// + sizeof(TsTcPipe).  TMEM: two accumulator buffers of 128 columns, then four
// operand slots of 64.
template <class Epi>
__global__ void __launch_bounds__(TS_TC_THREADS, 1)
ts_leg_analys_tc(TsLegTab t, TsTcTab tc, const char *__restrict__ wimg, int w_nfb, Epi epi,
                 int nfields, int per_cta, int S, int nmax, int ntile) {
  extern __shared__ __align__(1024) char ts_smem_at[];
  char *smem = (char *)(((unsigned long long)ts_smem_at + 1023) & ~1023ull);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const unsigned stage = TS_TC_STAGE_A + 2 * nmax * 128;
  const int grp = ts_epi_group(warp);
  const int ana_stg = min(nmax, TS_TC_ANA_COLS) * 2 * TS_TC_ANA_ROW * 4;  // bytes per group
  float *sD = reinterpret_cast<float *>(smem + S * stage + (grp > 0 ? ana_stg : 0));
  TsTcPipe *pp = reinterpret_cast<TsTcPipe *>(smem + S * stage + 2 * ana_stg);
  const TsAnalysSched sc{&tc, t.lmax, t.mmax, w_nfb, ntile, wimg};
  ts_tc_pipe_init(pp, S, tc);
  if (warp == 0) ts_tmem_alloc(&pp->tmem, 512);
  ts_tc_fence_before();
  __syncthreads();
  ts_tc_fence_after();
  const unsigned tmem = pp->tmem;

  // epilogue: TMEM -> shared [j][comp][field] -> Epi per (lm, comp)
  auto epilogue = [&](int tile, unsigned tbase) {
    const int cnt = sc.cnt(tile);
    if (cnt == 0) return;
    const bool zero = sc.stages(tile) == 0;  // every chunk skipped: no MMAs ran
    int m, par, lt, fb;
    sc.decode(tile, m, par, lt, fb);
    const int N = ts_round16(cnt);
    const int row = ts_epi_row(warp, lane), fl = row >> 1, comp = row & 1;
    const unsigned lanebase = tbase + ((unsigned)((warp & 3) * 32) << 16);
    const int f0 = fb * per_cta;
    const int nf = min(per_cta, nfields - f0);
    const long base = ts_lm_base(t.lmax, m);
    for (int h0 = TS_TC_ANA_COLS * grp; h0 < N; h0 += 2 * TS_TC_ANA_COLS) {
      const int hn = min(TS_TC_ANA_COLS, N - h0);
      ts_epi_bar(grp);  // the previous epi calls are done with sD
      for (int c0 = 0; c0 < hn; c0 += 16) {
        float v[16];
        if (zero) {
#pragma unroll
          for (int i = 0; i < 16; i++) v[i] = 0.f;
        } else {
          ts_tmem_ld16(lanebase + (unsigned)(h0 + c0), v);
        }
#pragma unroll
        for (int i = 0; i < 16; i++) sD[((c0 + i) * 2 + comp) * TS_TC_ANA_ROW + fl] = v[i];
      }
      ts_epi_bar(grp);
      const int jn = min(hn, cnt - h0);
      for (int idx = (warp & 3) * 32 + lane; idx < jn * 2; idx += 128) {
        const int jj = idx >> 1, cp = idx & 1;
        const int l = m + par + 2 * (lt * tc.LTL + h0 + jj);
        epi(base + (l - m), cp, sD + (jj * 2 + cp) * TS_TC_ANA_ROW, f0, nf, TS_TC_FIELDS);
      }
    }
  };
  ts_tc_persistent(smem, pp, S, TS_TC_ASLOTS, stage, tmem, 128, 256u, sc, epilogue);
  ts_tc_fence_before();
  __syncthreads();
  if (pp->bad && tid == 0) atomicExch(tc.err, 1);
  if (warp == 0) ts_tmem_free(tmem, 512);
}
